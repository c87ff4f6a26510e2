"""Batched ensembles (bfm_batch_*): many independent systems advanced by one
persistent kernel, one CTA per system at a time.

Every system must follow exactly the trajectory of a single updater with
the same set-up and R250 state: CPU tests cover the ensemble generator, the
oracle on boxes whose edges are multiples of 8 but not powers of two, and
the argument checks; GPU tests compare each system of mixed batches (RNGs,
ages, sorting intervals, shared-memory and global-memory lattices, 2 and 3
colours, per-system budgets) with the oracle and with single-system runs of
this library, bit for bit on positions, lattice, age, R250 state and
counters."""
import numpy as np
import pytest

import pscbfm_b200 as pb
from oracle import oracle
from pscbfm_b200 import systems


def _valid(s, pos):
    """excluded volume (no two 2x2x2 cubes share a site) and the bond set"""
    pos = np.asarray(pos, np.int64)
    L = np.array(s.box)
    cells = []
    for c in range(8):
        q = (pos + [(c & 1), (c >> 1) & 1, (c >> 2) & 1]) % L
        cells.append((q[:, 0] * L[1] + q[:, 1]) * L[2] + q[:, 2])
    cells = np.concatenate(cells)
    if np.unique(cells).size != cells.size:
        return False
    ids = np.arange(s.n)
    for j in range(int(s.deg.max(initial=0))):
        has = s.deg > j
        d = pos[s.nbr[has, j]] - pos[ids[has]]
        if (np.abs(d) > 3).any() or not s.allowed[(d[:, 0] & 7) | ((d[:, 1] & 7) << 3) | ((d[:, 2] & 7) << 6)].all():
            return False
    return True


@pytest.mark.parametrize("L,n,phi,star,side", [(32, 16, 0.5, False, 0), (48, 100, 0.3, True, 0), (64, 512, 0.1, False, 0),
                                               (40, 40, 0.45, True, 0), (96, 24, 0.2, False, 0), (32, 25, 0.4, False, 8),
                                               (48, 40, 0.3, True, 4)])
def test_ensemble_systems_are_valid(L, n, phi, star, side):
    s = systems.ensemble_system(L, n, phi, star, seed=5, side_every=side, side_len=3 if side else 0)
    assert _valid(s, s.pos)
    assert s.deg.max() == (3 if star or side else 2)
    assert abs(s.n * 8 / L ** 3 - phi) < 0.05 or s.n <= (1 + 3 * ((n - 1) // 3) if star else n)


def test_ensemble_draws_the_configured_ranges():
    sys_, params = systems.ensemble(12, seed=9, boxes=(32, 48, 64))
    assert len(sys_) == 12
    for s, p in zip(sys_, params):
        assert s.box == (p["L"],) * 3 and p["L"] in (32, 48, 64)
        assert 16 <= p["n"] <= 512 and 0.1 <= p["phi"] <= 0.5


@pytest.mark.parametrize("box", [(48, 48, 48), (24, 40, 32)])
def test_oracle_on_boxes_that_are_not_powers_of_two(box):
    s = systems.saw_chains(20, 12, box=box, seed=41)
    o = oracle.Sweep(s, rng=2, sort_every=9, threads=4)
    o.run(150, oracle.r250_state(4))
    p = o.positions()
    assert _valid(s, p)
    assert (p != s.pos).any(axis=1).sum() > s.n // 2
    assert (np.abs(p) >= np.array(box)).any()          # monomers crossed the periodic edges


def test_batch_argument_checks_without_a_gpu():
    b = pb.Batch()
    s = systems.saw_chains(4, 4, box=(32, 32, 32), seed=1)
    with pytest.raises(ValueError):
        b.add(systems.System((20, 32, 32), s.pos, s.deg, s.nbr), rng=pb.Rng.Saru)   # not a multiple of 8
    with pytest.raises(ValueError):
        b.add(s, rng=pb.Rng.Pcg)
    bad = systems.System(s.box, s.pos, s.deg.copy(), s.nbr, s.allowed)
    bad.deg[0] = 9
    with pytest.raises(ValueError, match="8 bonds"):
        b.add(bad)
    with pytest.raises(ValueError):
        b.add(s, r250_state=np.zeros(10, np.uint32))
    assert b.add(s) == 0 and b.add(s, rng=pb.Rng.IntHash) == 1
    assert b.info()["systems"] == 2
    with pytest.raises(ValueError):
        b.set_clusters(3)
    assert b.set_clusters(8).clusters()["size"] == 8


CASES = [
    # system, rng, age, sort_every
    (lambda: systems.saw_chains(20, 16, box=(32, 32, 32), seed=31), pb.Rng.Saru, 0, 5000),
    (lambda: systems.ordered_melt(32), pb.Rng.IntHash, 0, 7),
    (lambda: systems.star_comb(3, arm_len=10, side_every=4, side_len=3, box=(32, 32, 32), seed=32), pb.Rng.Philox, 4999, 5000),
    (lambda: systems.add_crosslinks(systems.saw_chains(24, 16, box=(32, 32, 32), seed=33), 40, seed=1), pb.Rng.Saru, 12345, 13),
    (lambda: systems.ensemble_system(64, 64, 0.4, False, seed=2), pb.Rng.Saru, 3, 3),
    (lambda: systems.ensemble_system(128, 100, 0.2, True, seed=3), pb.Rng.IntHash, 0, 50),
    (lambda: systems.saw_chains(30, 20, box=(16, 64, 32), seed=34), pb.Rng.Philox, 0, 11),
]


def _run_oracle(s, rng, age, sort_every, st, calls):
    o = oracle.Sweep(s, rng=int(rng), age=age, sort_every=sort_every, threads=4)
    for m in calls:
        o.run(int(m), st)
    return o


@pytest.mark.gpu
@pytest.mark.parametrize("clusters", [4, 0, 2, 8, "auto"])
def test_batch_matches_oracle_and_single_runs(clusters):
    """the 128^3 system shared by a cluster of 4, 2 or 8 CTAs, run by one CTA,
    or by the size the autotuner picks after timing all four on the first
    launches of the run: the trajectories are the same"""
    made = [(make(), rng, age, se) for make, rng, age, se in CASES]
    b = pb.Batch()
    if clusters == "auto":
        b.set_autotune(True)
    else:
        b.set_clusters(clusters)
    states = [oracle.r250_state(100 + i) for i in range(len(made))]
    for (s, rng, age, se), st in zip(made, states):
        b.add(s, rng=rng, age=age, sort_every=se, r250_state=st)
    b.initialize()
    budgets = [np.array([5, 17, 0, 9, 30, 3, 21], np.uint32), np.full(len(made), 12, np.uint32)]
    for m in budgets:
        b.run(m)
    for i, ((s, rng, age, se), st0) in enumerate(zip(made, states)):
        st = st0.copy()
        o = _run_oracle(s, rng, age, se, st, [budgets[0][i], budgets[1][i]])
        got = b.positions(i)
        assert np.array_equal(got, o.positions()), f"system {i}"
        a, r250, cnt = b.state(i)
        assert a == o.age() and np.array_equal(r250, st) and cnt == o.stats(), f"system {i}"
        assert np.array_equal(b.lattice(i), oracle.lattice_words(got, s.box)), f"system {i}"
    # one system against a single-system handle of this library
    for i in (1, 3, 5):
        s, rng, age, se = made[i]
        pb.r250_set_state(states[i])
        u = pb.UpdaterGPUScBFM_AB_Type().setup(s, rng=rng, age=age, steps_between_sortings=se)
        for m in budgets:
            if m[i]:
                u.runSimulationOnGPU(int(m[i]))
        assert np.array_equal(u.getAllMonomerPositions(), b.positions(i)), f"system {i}"
    info = b.clusters()
    if clusters == "auto":
        assert info["size"] in (0, 2, 4, 8)
        assert all(v > 0 for v in info["trial_ns_per_move"].values())
        t = b.tuning()
        assert t["tuned"] and t["in_flight"] in (1, 2, 4) and t["cluster_above_words"] in (1024, 8192)
        # every stage ran: the 64^3 system makes the threshold trial count too
        assert all(v > 0 for v in t["trial_ns_per_move"].values())
    else:
        assert info["size"] == clusters


@pytest.mark.gpu
@pytest.mark.parametrize("in_flight,from48", [(1, False), (4, False), (2, True), (4, True)])
def test_batch_tile_shapes_match_oracle(in_flight, from48):
    """every tile shape the autotuner may choose -- 1, 2 or 4 monomers in
    flight per thread; systems of 48^3..64^3 sites on the cluster kernel
    with a global-memory lattice instead of one CTA's shared memory -- gives
    the oracle's trajectories"""
    made = [(make(), rng, age, se) for make, rng, age, se in CASES]
    b = pb.Batch()
    b.set_shape(in_flight, from48)
    states = [oracle.r250_state(300 + i) for i in range(len(made))]
    for (s, rng, age, se), st in zip(made, states):
        b.add(s, rng=rng, age=age, sort_every=se, r250_state=st)
    b.initialize()
    budgets = [np.array([7, 0, 11, 5, 23, 9, 14], np.uint32), np.full(len(made), 10, np.uint32)]
    for m in budgets:
        b.run(m)
    for i, ((s, rng, age, se), st0) in enumerate(zip(made, states)):
        o = _run_oracle(s, rng, age, se, st0.copy(), [budgets[0][i], budgets[1][i]])
        assert np.array_equal(b.positions(i), o.positions()), f"system {i}"
    t = b.tuning()
    assert t["in_flight"] == in_flight and t["cluster_above_words"] == (1024 if from48 else 8192)


@pytest.mark.gpu
@pytest.mark.parametrize("make", [
    lambda: systems.ensemble_system(48, 32, 0.4, False, seed=6),
    lambda: systems.ensemble_system(40, 16, 0.3, True, seed=7),
    lambda: systems.ensemble_system(96, 50, 0.3, False, seed=8),
    lambda: systems.saw_chains(20, 12, box=(24, 40, 32), seed=41),
    lambda: systems.ensemble_system(48, 30, 0.35, True, seed=9, side_every=4, side_len=3),
])
def test_batch_on_boxes_that_are_not_powers_of_two(make):
    s = make()
    st = oracle.r250_state(77)
    b = pb.Batch()
    b.add(s, rng=pb.Rng.Saru, sort_every=19, r250_state=st)
    b.initialize()
    b.run(60)
    o = _run_oracle(s, pb.Rng.Saru, 0, 19, st.copy(), [60])
    assert np.array_equal(b.positions(0), o.positions())
    assert np.array_equal(b.lattice(0), oracle.lattice_words(o.positions(), s.box))
    assert _valid(s, b.positions(0))


@pytest.mark.gpu
def test_batch_ensemble_of_64_systems():
    sys_, params = systems.ensemble(64, seed=21, boxes=(32, 48, 64, 96, 128), n_range=(16, 256))
    b = pb.Batch()
    states = [oracle.r250_state(500 + i) for i in range(len(sys_))]
    for s, st in zip(sys_, states):
        b.add(s, rng=pb.Rng.Saru, r250_state=st)
    b.initialize()
    b.run(20)
    info = b.info()
    assert info["last_attempts"] == 20 * sum(s.n for s in sys_)
    for i, s in enumerate(sys_):
        p = b.positions(i)
        assert _valid(s, p), f"system {i}"
        assert np.array_equal(b.lattice(i), oracle.lattice_words(p, s.box))
    for i in (0, 17, 40, 63):
        o = _run_oracle(sys_[i], pb.Rng.Saru, 0, 5000, states[i].copy(), [20])
        assert np.array_equal(b.positions(i), o.positions()), f"system {i}"


@pytest.mark.gpu
def test_batch_gather_selected_monomers():
    """bfm_batch_gather_positions returns, in the order asked, the same
    unfolded positions as the whole-system read-back, also after a run
    whose re-sorts moved monomers between slots"""
    sys_, _ = systems.ensemble(12, seed=33, boxes=(32, 48, 64, 128), n_range=(16, 128))
    b = pb.Batch()
    for i, s in enumerate(sys_):
        b.add(s, rng=pb.Rng.Saru, sort_every=7, r250_seed=900 + i)
    b.initialize()
    rng = np.random.default_rng(5)
    for mcs in (0, 23, 40):
        if mcs:
            b.run(mcs)
        sel_s = rng.integers(0, len(sys_), 400)
        sel_i = np.array([rng.integers(0, sys_[k].n) for k in sel_s])
        got = b.gather(sel_s, sel_i)
        want = np.stack([b.positions(int(k))[int(i)] for k, i in zip(sel_s, sel_i)])
        assert np.array_equal(got, want)
    with pytest.raises(Exception):
        b.gather([0], [sys_[0].n])
