"""Bit-exact parity at the benchmark configurations.

Three implementations run the same system from the same R250 state: the
CUDA sweep through the C ABI, the CPU oracle, and -- where it was built --
the reference's own UpdaterGPUScBFM_AB_Type<T> compiled for sm_100a
(oracle/_ref).  After every call the positions (unfolded) and the occupation
lattice must be identical, bit for bit.  This is the reference's own
correctness idea (testCorrectness.sh:219-237 diffs a run against a stored
result), with the stored result replaced by live runs.

  * C2, the 4096 x 256 melt on 256^3, as benchmarked: 240 MCS with the age
    set so that the 5000-MCS spatial re-sort falls inside the run;
  * C1, 128 self-avoiding chains x 64 on 128^3: 1000 MCS (int32 reference);
  * solo systems of the batched-ensemble generator with edges 32, 64, 128;
  * the star-comb melt of C3 scaled to 128^3 (121,170 monomers, side chains
    on every 8th backbone monomer) with re-sorts inside the run.

The reference's 8-bit coordinates with a non-zero start age unfold some
positions with a wrong image count at set-up (its initialize runs
kernelTreatOverflows against an unwritten buffer, UpdaterGPUScBFM_AB_Type.cu
:2073-2077); its trajectory is unaffected, so such runs compare it modulo the
box.
"""
import os

import numpy as np
import pytest

import pscbfm_b200 as pb
from oracle import oracle
from pscbfm_b200 import systems

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 4


def _with_positions(s, pos):
    return systems.System(s.box, np.ascontiguousarray(pos, dtype=np.int32), s.deg, s.nbr, s.allowed, s.chains,
                          s.attributes, s.name)


def _melted(s, mcs, seed):
    """the system after `mcs` MCS of the CUDA sweep: a start with the
    acceptance rates of a melted state instead of the ordered set-up"""
    pb.r250_seed(seed)
    u = pb.UpdaterGPUScBFM_AB_Type().setup(s, rng=pb.Rng.Saru)
    u.runSimulationOnGPU(mcs)
    pos = u.getAllMonomerPositions()
    u.cleanup()
    return _with_positions(s, pos)


def three_way(s, calls, *, age=0, sort_every=5000, ctype=1, r250_seed=4242, ref_mod_box=False):
    """run `calls` (MCS per call) on the CUDA sweep, the oracle and the
    reference build from one R250 state; compare after every call"""
    pb.r250_seed(r250_seed)
    st_o = pb.r250_get_state()
    st_r = st_o.copy()
    u = pb.UpdaterGPUScBFM_AB_Type().setup(s, rng=pb.Rng.Saru, age=age, steps_between_sortings=sort_every)
    o = oracle.Sweep(s, rng=2, age=age, sort_every=sort_every, threads=THREADS)
    ref = None
    if oracle.ref_gpu() is not None:
        ref = oracle.RefUpdater(s, rng=2, age=age, sort_every=sort_every, ctype=ctype)
    box = np.array(s.box)
    for nmcs in calls:
        u.runSimulationOnGPU(nmcs)
        o.run(nmcs, st_o)
        got, want = u.getAllMonomerPositions(), o.positions()
        assert np.array_equal(got, want), f"{int((got != want).any(axis=1).sum())} monomers differ after {nmcs} MCS"
        assert np.array_equal(u.getLattice(), oracle.lattice_words(got, s.box))
        if ref is not None:
            ref.run(nmcs, st_r)
            r = ref.positions()
            if ref_mod_box:
                r, w = r % box, want % box
            else:
                w = want
            assert np.array_equal(r, w), f"reference: {int((r != w).any(axis=1).sum())} monomers differ"
    assert np.array_equal(pb.r250_get_state(), st_o)
    if ref is not None:
        assert np.array_equal(st_r, st_o)
    assert u.getAge() == o.age() == age + sum(calls)
    att, cand, acc = u.getCounters()
    assert (att, cand, acc) == o.stats() and acc > 0
    return u


def test_c2_full_melt_with_resort_inside():
    s = _melted(systems.ordered_melt(256), 500, seed=31)
    assert s.n == 4096 * 256
    # ages 4880 .. 5120: the re-sort at age 5000 falls in the second call
    three_way(s, [40, 200], age=4880, sort_every=5000, ctype=1, ref_mod_box=True)


def test_c2_full_melt_from_age_zero():
    s = _melted(systems.ordered_melt(256), 300, seed=32)
    three_way(s, [120, 80], age=0, sort_every=5000, ctype=1)


def test_c1_dilute_chains_1000_mcs():
    s = systems.saw_chains(128, 64, box=(128, 128, 128), seed=12345)
    three_way(s, [1, 499, 500], age=0, sort_every=5000, ctype=0)


@pytest.mark.parametrize("shape", [9, 10])
def test_c1_on_one_cluster(shape):
    """C1 on the windowed kernel confined to one cluster of 8 or 16 CTAs
    (cluster barriers instead of grid barriers)"""
    s = systems.saw_chains(128, 64, box=(128, 128, 128), seed=12345)
    pb.r250_seed(4242)
    st = pb.r250_get_state()
    u = pb.UpdaterGPUScBFM_AB_Type().setup(s, rng=pb.Rng.Saru)
    u.setSweepShape(shape)
    assert u.getLaunchInfo()["mode"] == shape and u.getLaunchInfo()["ctas"] == (8 if shape == 9 else 16)
    o = oracle.Sweep(s, rng=2, threads=THREADS)
    for nmcs in (1, 299):
        u.runSimulationOnGPU(nmcs)
        o.run(nmcs, st)
        assert np.array_equal(u.getAllMonomerPositions(), o.positions())
        assert np.array_equal(u.getLattice(), oracle.lattice_words(o.positions(), s.box))


@pytest.mark.parametrize("L,n,phi,star,seed", [(32, 100, 0.35, False, 1), (64, 301, 0.45, True, 2),
                                               (128, 512, 0.2, False, 3), (128, 97, 0.5, True, 4)])
def test_ensemble_systems_solo(L, n, phi, star, seed):
    """systems of the batched-ensemble generator, each run alone"""
    s = systems.ensemble_system(L, n, phi, star, seed=seed)
    three_way(s, [50, 150], age=0, sort_every=120, ctype=1, r250_seed=100 + seed)


def test_c3_star_comb_melt_scaled_to_128():
    s = systems.star_comb_melt(128)
    assert s.n == 210 * 577 and int(s.deg.max()) == 3
    s = _melted(s, 100, seed=33)
    u = three_way(s, [60, 140], age=0, sort_every=100, ctype=1)
    assert u.getNSpecies() == 2      # a forest: the reference's walk gives two colours
