"""CPU tests of the oracle (test infrastructure) against golden vectors made
by the reference's own code, and its self-consistency."""
import os

import numpy as np
import pytest

from oracle import oracle
from pscbfm_b200 import systems

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def host_gold():
    return np.load(os.path.join(GOLD, "host_vectors.npz"))


def test_saru_matches_reference_vectors(host_gold):
    g = host_gold
    o = oracle.orc()
    got = np.array([o.orc_saru(int(s), int(i) & 0xFFFFFFFF, int(j))
                    for s, i, j in zip(g["saru_seed"], g["saru_iter"], g["saru_sub"])], np.uint32)
    assert np.array_equal(got, g["saru_out"])


def test_hash_matches_reference_vectors(host_gold):
    g = host_gold
    o = oracle.orc()
    got = np.array([o.orc_hash_rng(int(s), int(j)) for s, j in zip(g["saru_seed"], g["saru_sub"])], np.uint32)
    assert np.array_equal(got, g["hash_out"])


def test_coloring_matches_reference_vectors(host_gold):
    g = host_gold
    for idx in range(int(g["ngraphs"][0])):
        deg, nbr = g[f"g{idx}_deg"], g[f"g{idx}_nbr"]
        for uni in (0, 1):
            k, col = oracle.graph_coloring(deg, nbr, uniform=bool(uni))
            assert k == int(g[f"g{idx}_u{uni}_k"][0])
            assert np.array_equal(col, g[f"g{idx}_u{uni}_colors"]), (idx, uni)


def test_coloring_is_proper(host_gold):
    g = host_gold
    for idx in range(int(g["ngraphs"][0])):
        deg, nbr = g[f"g{idx}_deg"], g[f"g{idx}_nbr"]
        _, col = oracle.graph_coloring(deg, nbr, uniform=True)
        for i in range(deg.size):
            for j in nbr[i, : deg[i]]:
                assert col[i] != col[j]


def test_r250_recurrence():
    s = oracle.r250_state(99)
    x = oracle.r250_draw(s, 2000).astype(np.uint64)
    n = np.arange(250, 2000)
    # Maier's index scheme (partner 103 slots ahead in the 250-word ring) gives
    # x[n] = x[n-250] ^ x[n-147], the reciprocal of the trinomial x^250+x^103+1
    assert np.array_equal(x[n], x[n - 250] ^ x[n - 147])


def _check_valid(sysm, pos):
    box = np.array(sysm.box)
    w = pos.astype(np.int64) % box
    cells = set()
    for p in w:
        for dz in (0, 1):
            for dy in (0, 1):
                for dx in (0, 1):
                    c = ((p[0] + dx) % box[0], (p[1] + dy) % box[1], (p[2] + dz) % box[2])
                    assert c not in cells, "excluded volume violated"
                    cells.add(c)
    for i in range(sysm.n):
        for j in sysm.nbr[i, : sysm.deg[i]]:
            d = pos[j].astype(np.int64) - pos[i]
            assert np.all(np.abs(d) <= 3)
            assert sysm.allowed[(d[0] & 7) | ((d[1] & 7) << 3) | ((d[2] & 7) << 6)]


@pytest.mark.parametrize("rng", [1, 2])
def test_oracle_sweep_keeps_model_invariants(rng):
    s = systems.saw_chains(20, 16, box=(32, 32, 32), seed=3)
    sw = oracle.Sweep(s, rng=rng, age=0, sort_every=11, threads=4)
    st = oracle.r250_state(5)
    sw.run(60, st)
    pos = sw.positions()
    assert (pos != s.pos).any()
    _check_valid(s, pos)
    att, cand, acc = sw.stats()
    assert att == 60 * s.n
    assert 0 < acc <= cand <= att


def test_oracle_sweep_thread_count_independent():
    s = systems.add_crosslinks(systems.saw_chains(16, 20, box=(32, 32, 32), seed=8), 20)
    outs = []
    for th in (1, 3, 8):
        sw = oracle.Sweep(s, rng=2, age=123, sort_every=9, threads=th)
        st = oracle.r250_state(77)
        sw.run(40, st)
        outs.append(sw.positions())
    assert np.array_equal(outs[0], outs[1]) and np.array_equal(outs[0], outs[2])


def test_oracle_split_runs_follow_reference_age_rule():
    """currentAge = age + iStep*nSpecies + iSubStep restarts iStep at every
    runSimulationOnGPU call (UpdaterGPUScBFM_AB_Type.cu:3049), so 2 x 10 MCS
    differs from 1 x 20 MCS for Saru (iteration-dependent), not for IntHash."""
    s = systems.saw_chains(12, 16, box=(32, 32, 32), seed=4)
    res = {}
    for rng in (1, 2):
        for split in (False, True):
            sw = oracle.Sweep(s, rng=rng, sort_every=5000, threads=2)
            st = oracle.r250_state(1)
            if split:
                sw.run(10, st)
                sw.run(10, st)
            else:
                sw.run(20, st)
            res[(rng, split)] = sw.positions()
    assert np.array_equal(res[(1, False)], res[(1, True)])
    assert not np.array_equal(res[(2, False)], res[(2, True)])


def test_serial_bfm_keeps_invariants():
    s = systems.saw_chains(10, 16, box=(32, 32, 32), seed=2)
    pos = s.pos.copy()
    acc = oracle.serial_run(s, pos, 50, seed=3)
    assert acc > 0
    _check_valid(s, pos)


def test_oracle_matches_reference_gpu_golden_sweeps():
    """tests/golden/sweep_vectors.npz holds the reference's own updater
    (UpdaterGPUScBFM_AB_Type.cu built for sm_100a) run on a B200 by
    tests/golden/make_golden_sweep.py: chains, star-combs, cross-linked
    (3-colour) systems and a small melt, Saru and IntHash, ages 0 / 17 / 4998,
    several calls.  The CPU oracle must reproduce every call bit for bit.

    One reference defect is allowed for: with 8/16-bit device coordinates and
    a non-zero start age, initialize() runs doSpatialSorting, whose
    kernelTreatOverflows (.cu:1285-1334) compares against
    mPolymerSystemSortedOld before it was ever written (it is only zeroed in
    debug builds, .cu:2073-2077), so some unfolded positions come back shifted
    by whole box lengths.  The trajectory itself is unaffected; for those
    cases positions are compared modulo the box."""
    g = np.load(os.path.join(GOLD, "sweep_vectors.npz"))
    for idx in range(int(g["ncases"][0])):
        rng, age, sort_every, ctype = (int(v) for v in g[f"c{idx}_params"])
        box = tuple(int(v) for v in g[f"c{idx}_box"])
        s = systems.System(box, g[f"c{idx}_pos"], g[f"c{idx}_deg"], g[f"c{idx}_nbr"], g[f"c{idx}_allowed"])
        st = g[f"c{idx}_r250"].copy()
        sw = oracle.Sweep(s, rng=rng, age=age, sort_every=sort_every, threads=4)
        defect = ctype in (1, 2) and age != 0
        for k, nmcs in enumerate(g[f"c{idx}_calls"]):
            sw.run(int(nmcs), st)
            got, want = sw.positions(), g[f"c{idx}_out{k}"]
            name = (str(g[f"c{idx}_name"]), k)
            if defect:
                assert np.array_equal(got % np.array(box), want % np.array(box)), name
                assert np.all((got - want) % np.array(box) == 0), name
            else:
                assert np.array_equal(got, want), name
        assert np.array_equal(st, g[f"c{idx}_r250_end"])
