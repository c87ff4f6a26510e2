"""Non-periodic (wall) boundaries.

The reference's check kernel (UpdaterGPUScBFM_AB_Type.cu:988-996) refuses a
move that would take a cube corner out of 0 .. L-2 along a non-periodic axis
(its unsigned coordinate types; it compares y and z with the x size, the
same test for cubic boxes).  CPU: the oracle keeps every corner inside the
walls and its lattice consistent.  GPU: the CUDA path against the oracle bit
for bit (all kernel shapes, mixed periodicity, non-cubic boxes), against the
reference's own build for cubic boxes with 8- and 16-bit coordinates, and
the set-up's refusal of a monomer outside the walls."""
import numpy as np
import pytest

import pscbfm_b200 as pb
from oracle import oracle
from pscbfm_b200 import systems


def _inside(pos, box, periodic):
    for a in range(3):
        if not periodic[a]:
            if pos[:, a].min() < 0 or pos[:, a].max() > box[a] - 2:
                return False
    return True


@pytest.mark.parametrize("periodic", [(False, False, False), (False, True, True), (True, False, True)])
def test_oracle_keeps_monomers_inside_the_walls(periodic):
    s = systems.open_box_chains(30, 16, box=(32, 32, 32), seed=81, periodic=periodic)
    sw = oracle.Sweep(s, rng=2, periodic=periodic, threads=4)
    st = oracle.r250_state(3)
    sw.run(400, st)
    p = sw.positions()
    assert _inside(p, s.box, periodic)
    # a wall really stops monomers: without it some cross the edge
    free = oracle.Sweep(s, rng=2, threads=4)
    free.run(400, oracle.r250_state(3))
    assert not _inside(free.positions(), s.box, periodic)


SHAPES = [-1, 0, 1, 2, 3, 4, 6, 7, 8]


@pytest.mark.gpu
@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("periodic,box", [((False, False, False), (32, 32, 32)), ((False, True, True), (32, 16, 64)),
                                          ((True, True, False), (16, 32, 32))])
def test_open_box_matches_oracle(periodic, box, shape):
    s = systems.open_box_chains(24, 12, box=box, seed=82, periodic=periodic)
    pb.r250_seed(55)
    st = pb.r250_get_state()
    u = pb.UpdaterGPUScBFM_AB_Type().setup(s, rng=pb.Rng.Saru, steps_between_sortings=37)
    if shape != -1:
        u.setSweepShape(shape)
    o = oracle.Sweep(s, rng=2, sort_every=37, periodic=periodic, threads=4)
    for nmcs in (25, 150):
        u.runSimulationOnGPU(nmcs)
        o.run(nmcs, st)
        assert np.array_equal(u.getAllMonomerPositions(), o.positions())
    assert _inside(u.getAllMonomerPositions(), s.box, periodic)
    assert np.array_equal(u.getLattice(), oracle.lattice_words(o.positions(), s.box))


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [1, 2])
def test_open_box_split_kernels_match_oracle(mode):
    periodic = (False, False, True)
    s = systems.open_box_chains(24, 12, box=(32, 32, 32), seed=83, periodic=periodic)
    pb.r250_seed(56)
    st = pb.r250_get_state()
    u = pb.UpdaterGPUScBFM_AB_Type()
    u.setLaunchMode(mode)
    u.setup(s, rng=pb.Rng.IntHash)
    o = oracle.Sweep(s, rng=1, periodic=periodic, threads=4)
    u.runSimulationOnGPU(120)
    o.run(120, st)
    assert np.array_equal(u.getAllMonomerPositions(), o.positions())


@pytest.mark.gpu
@pytest.mark.parametrize("ctype", [1, 2])
@pytest.mark.parametrize("periodic", [(False, False, False), (True, False, True)])
def test_open_box_matches_reference_build(periodic, ctype):
    if oracle.ref_gpu() is None:
        pytest.skip("reference build not present")
    s = systems.open_box_chains(30, 16, box=(32, 32, 32), seed=84, periodic=periodic)
    pb.r250_seed(57)
    st = pb.r250_get_state()
    st_ref = st.copy()
    u = pb.UpdaterGPUScBFM_AB_Type().setup(s, rng=pb.Rng.Saru)
    ref = oracle.RefUpdater(s, rng=2, ctype=ctype, periodic=periodic)
    for nmcs in (40, 160):
        u.runSimulationOnGPU(nmcs)
        ref.run(nmcs, st_ref)
        assert np.array_equal(u.getAllMonomerPositions(), ref.positions())


@pytest.mark.gpu
def test_monomer_outside_the_walls_is_refused():
    s = systems.open_box_chains(10, 8, box=(32, 32, 32), seed=85, periodic=(False, True, True))
    s.pos = s.pos.copy()
    s.pos[:, 0] += 32 - 2 - s.pos[:, 0].max() + 1      # push the highest corner onto L-1
    u = pb.UpdaterGPUScBFM_AB_Type()
    with pytest.raises(ValueError):
        u.setup(s, rng=pb.Rng.Saru)
