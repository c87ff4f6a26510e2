"""Philox4x32-10: the product's device generator and the oracle's
restatement against curand's own outputs (the reference's Philox option is
curand_init(seed, subsequence = monomer, offset = age) then curand(),
rngs/lemonade_philox.h:48-56), and the whole sweep with Philox against the
oracle and the reference's own build."""
import ctypes

import numpy as np
import pytest

import pscbfm_b200 as pb
from oracle import oracle
from pscbfm_b200 import _native, systems

CASES = [(0, 0, 0), (1234, 5, 0), (0xFFFFFFFF, 7, 3), (42, 524287, 123457), (2 ** 32 - 1, 2 ** 20, 2 ** 33 + 5),
         (987654321, 0, 2 ** 40 + 2)]


def test_oracle_philox_is_deterministic_and_word_ordered():
    o = oracle.orc()
    # consecutive offsets inside one 4-word block share the counter
    blk = [o.orc_philox(7, 3, 8 + k) for k in range(4)]
    assert len(set(blk)) == 4
    assert o.orc_philox(7, 3, 9) == blk[1]


@pytest.mark.gpu
@pytest.mark.parametrize("seed,subseq,offset", CASES)
def test_device_philox_matches_curand_and_oracle(seed, subseq, offset):
    n = 64
    out = np.zeros(2 * n, np.uint32)
    assert _native.lib().bfm_debug_philox_vs_curand(0, seed, subseq, offset, n, out.ctypes.data) == 0
    mine, cur = out[0::2], out[1::2]
    assert np.array_equal(mine, cur)
    o = oracle.orc()
    assert np.array_equal(mine, np.array([o.orc_philox(seed, subseq, offset + k) for k in range(n)], np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["chains", "crosslinked"])
def test_philox_sweep_matches_oracle_and_reference(name):
    s = {"chains": lambda: systems.saw_chains(40, 20, box=(32, 32, 32), seed=61),
         "crosslinked": lambda: systems.add_crosslinks(systems.saw_chains(40, 20, box=(32, 32, 32), seed=62), 40)}[name]()
    pb.r250_seed(808)
    st = pb.r250_get_state()
    st_ref = st.copy()
    u = pb.UpdaterGPUScBFM_AB_Type().setup(s, rng=pb.Rng.Philox, age=4990, steps_between_sortings=17)
    o = oracle.Sweep(s, rng=3, age=4990, sort_every=17, threads=4)
    for nmcs in (6, 25):
        u.runSimulationOnGPU(nmcs)
        o.run(nmcs, st)
        assert np.array_equal(u.getAllMonomerPositions(), o.positions())
    if oracle.ref_gpu() is None:
        pytest.skip("reference build not present")
    ref = oracle.RefUpdater(s, rng=3, age=4990, sort_every=17, ctype=0)
    for nmcs in (6, 25):
        ref.run(nmcs, st_ref)
    assert np.array_equal(ref.positions(), o.positions())
