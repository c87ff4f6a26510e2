"""Handle life cycle and independence on the GPU: every RNG on every
persistent-kernel shape, cleanup and re-initialization of one handle with
another system, and two handles stepped alternately (the reference's
constant-memory box tables allow only one updater per process,
UpdaterGPUScBFM_AB_Type.cu:84-133; these handles carry their parameters in
kernel arguments).  All bit-exact against the oracle."""
import numpy as np
import pytest

import pscbfm_b200 as pb
from oracle import oracle
from pscbfm_b200 import systems

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape", [0, 1, 2, 6, 7, 8])
@pytest.mark.parametrize("rng", [pb.Rng.IntHash, pb.Rng.Philox])
def test_every_shape_with_every_rng(shape, rng):
    s = systems.add_crosslinks(systems.saw_chains(40, 24, box=(32, 32, 32), seed=101), 20)
    pb.r250_seed(5)
    st = pb.r250_get_state()
    u = pb.UpdaterGPUScBFM_AB_Type().setup(s, rng=rng, age=123, steps_between_sortings=41)
    u.setSweepShape(shape)
    o = oracle.Sweep(s, rng=int(rng), age=123, sort_every=41, threads=4)
    for nmcs in (30, 70):
        u.runSimulationOnGPU(nmcs)
        o.run(nmcs, st)
        assert np.array_equal(u.getAllMonomerPositions(), o.positions())


def test_cleanup_and_reinitialize_with_another_system():
    a = systems.saw_chains(30, 16, box=(32, 32, 32), seed=102)
    b = systems.star_comb(4, arm_len=16, side_every=4, side_len=4, box=(64, 64, 64), seed=103)
    u = pb.UpdaterGPUScBFM_AB_Type()
    for s in (a, b, a):
        pb.r250_seed(6)
        st = pb.r250_get_state()
        u.setup(s, rng=pb.Rng.Saru)
        o = oracle.Sweep(s, rng=2, threads=4)
        u.runSimulationOnGPU(60)
        o.run(60, st)
        assert np.array_equal(u.getAllMonomerPositions(), o.positions())
        u.cleanup()


def test_two_handles_stepped_alternately():
    a = systems.saw_chains(30, 16, box=(32, 32, 32), seed=104)
    b = systems.ordered_melt(32)
    pb.r250_seed(7)
    st = pb.r250_get_state()
    ua = pb.UpdaterGPUScBFM_AB_Type().setup(a, rng=pb.Rng.Saru)
    ub = pb.UpdaterGPUScBFM_AB_Type().setup(b, rng=pb.Rng.IntHash)
    oa = oracle.Sweep(a, rng=2, threads=4)
    ob = oracle.Sweep(b, rng=1, threads=4)
    for nmcs in (10, 25, 40):
        ua.runSimulationOnGPU(nmcs)
        oa.run(nmcs, st)          # both draw from the one process-wide R250, in call order
        ub.runSimulationOnGPU(nmcs)
        ob.run(nmcs, st)
        assert np.array_equal(ua.getAllMonomerPositions(), oa.positions())
        assert np.array_equal(ub.getAllMonomerPositions(), ob.positions())


def test_handles_of_different_sizes_share_the_kernels():
    """Two handles with the same generator use the same kernel functions,
    whose dynamic shared-memory limit is per function: a handle configured
    for a small system after one for a large system must not lower the
    limit below the large one's launches (it is only ever raised)."""
    big = systems.ordered_melt(64)
    small = systems.saw_chains(12, 8, box=(16, 16, 16), seed=105)
    pb.r250_seed(8)
    st = pb.r250_get_state()
    ub = pb.UpdaterGPUScBFM_AB_Type().setup(big, rng=pb.Rng.Saru)
    us = pb.UpdaterGPUScBFM_AB_Type().setup(small, rng=pb.Rng.Saru)
    assert ub.getLaunchInfo()["smem_bytes"] > us.getLaunchInfo()["smem_bytes"]
    ob = oracle.Sweep(big, rng=2, threads=4)
    osm = oracle.Sweep(small, rng=2, threads=4)
    for nmcs in (15, 30):
        ub.runSimulationOnGPU(nmcs)
        ob.run(nmcs, st)
        us.runSimulationOnGPU(nmcs)
        osm.run(nmcs, st)
        assert np.array_equal(ub.getAllMonomerPositions(), ob.positions())
        assert np.array_equal(us.getAllMonomerPositions(), osm.positions())
