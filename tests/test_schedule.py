"""The learned run schedule (pscbfm_b200/schedule.py).

CPU: the label extraction on synthetic series with known answers
(exponential approach to a plateau, end vectors of an AR(1) process), the
molecule bookkeeping of the ensemble generator, and the schedule
comparison: with exact predictions of spread equilibration times the
learned budgets cost less than the smallest fixed budget of equal R_e^2
error, and a too-small prediction is extended by the measured drift check.
GPU: the whole pipeline on a 1024-system ensemble (record with the batched
simulator, train the network with the library's kernels, compare), and
that the network predicts the end-to-end autocorrelation time, which the
budgets scale with, better than a constant does (the pipeline is
deterministic: bit-exact simulation, fixed-order sums in training)."""
import math

import numpy as np
import pytest

from pscbfm_b200 import schedule as sch
from pscbfm_b200 import systems


def _series(tau, plateau=100.0, n=500, T=20000.0, every=100.0, seed=0):
    rng = np.random.default_rng(seed)
    t = np.arange(0, T + every, every)
    re2 = plateau * (1 - 0.8 * np.exp(-t / tau)) * (1 + 0.003 * rng.normal(size=t.size))
    return {"t": t, "re2": re2, "rg2": re2 / 6, "ends": np.zeros((t.size, 4, 3), np.float32), "n": n}


def test_equilibration_time_of_an_exponential_approach():
    s = _series(1000.0)
    teq, plat = sch.equilibration_time(s["t"], s["re2"])
    # 0.8 exp(-t/tau) <= 0.1 at t = tau ln 8
    assert abs(teq - 1000.0 * math.log(8)) < 400 and abs(plat - 100.0) < 1.0


def test_relaxation_time_of_ar1_end_vectors():
    rng = np.random.default_rng(2)
    tau, dt = 500.0, 50.0
    a = math.exp(-dt / tau)
    e = np.zeros((600, 400, 3))
    e[0] = rng.normal(size=(400, 3))
    for k in range(1, 600):
        e[k] = a * e[k - 1] + math.sqrt(1 - a * a) * rng.normal(size=(400, 3))
    t = np.arange(600) * dt
    assert abs(sch.relaxation_time(t, e, 0) - tau) < 0.15 * tau


@pytest.mark.parametrize("star,side", [(False, 0), (True, 0), (False, 4), (True, 8)])
def test_molecule_bookkeeping_matches_the_generator(star, side):
    s = systems.ensemble_system(32, 25, 0.3, star, seed=4, side_every=side, side_len=3 if side else 0)
    m = sch.molecules(s, 25, star)
    assert m["count"] * m["size"] == int((s.attributes == 1).sum())
    if side:
        assert (s.attributes == 2).sum() > 0
    re2, rg2, ends = sch.observables(s.pos, m)
    assert re2 > 0 and rg2 > 0 and len(ends) == m["count"] * (3 if star else 1)
    if not star and not side:
        a, b = m["ends"]
        assert (s.deg[a] == 1).all() and (s.deg[b] == 1).all()
    elif star:
        core, tips = m["ends"]
        assert (s.deg[core] == 3).all() and (s.deg[tips] <= 2).all()


def test_learned_budgets_beat_a_fixed_budget_with_exact_predictions():
    taus = np.exp(np.random.default_rng(5).uniform(np.log(100), np.log(5000), 60))
    ser = [_series(tau, seed=i) for i, tau in enumerate(taus)]
    pred = np.log10(taus * math.log(8))
    b = sch.learned_budgets(pred, ser)
    rep = sch.compare(ser, b)
    assert rep["systems_per_hour_ratio"] > 1.5
    assert abs(rep["plain"]["bias_re2"]) <= max(abs(rep["learned"]["bias_re2"]), 0.005) + 1e-12


def test_drift_check_extends_an_underbudgeted_run():
    s = _series(3000.0)
    b = sch.learned_budgets(np.array([np.log10(50.0)]), [s], factor=1.0)
    assert b[0] > 3000.0


@pytest.mark.gpu
def test_pipeline_and_what_the_network_adds():
    rep = sch.run(n_systems=1024, mcs=20000, every=250, epochs=200, seed=3)
    assert rep["systems"] == 1024 and rep["batch_rate_moves_per_s"] > 1e8
    assert rep["train_loss_first_last"][1] < rep["train_loss_first_last"][0]
    assert rep["schedule"]["learned"]["cost_moves"] > 0 and rep["schedule"]["plain"]["cost_moves"] > 0
    assert all(np.isfinite(v) for v in rep["test_rmse"].values())
    # what the network adds: its prediction of the end-to-end autocorrelation
    # time (the quantity the budgets scale with) beats the constant predictor
    key = "log10 end-to-end autocorrelation MCS"
    assert rep["test_rmse"][key] < rep["test_rmse_constant_predictor"][key]


@pytest.mark.gpu
def test_live_schedule_on_the_gpu():
    """The live learned schedule on a small ensemble (384 systems of edges
    32..64, molecules of 16..96 monomers, 40,000 MCS recorded): the live
    runs reproduce the recorded trajectories exactly (bit-exact batched
    simulation from the same seeds), the drift judge ran, and the learned
    schedule's ensemble R_e^2/N stays within 2% of the full-length runs.
    The measured systems-per-hour ratio is reported by bench.py --schedule
    on the full ensemble; here it only has to be positive."""
    rep = sch.live_compare(n_systems=384, mcs=40000, every=500, epochs=200, seed=4, boxes=(32, 48, 64), n_range=(16, 96))
    assert rep["live_runs_reproduce_the_record"]
    assert rep["test_systems_assessed"] >= 20
    assert abs(rep["learned"]["ensemble_re2_per_n_vs_full"]) <= 0.02
    assert rep["learned"]["wall_s"] > 0 and rep["plain"]["wall_s"] > 0 and rep["ratio_learned_vs_plain"] > 0
    assert rep["learned"]["mean_mcs"] <= 40000


def test_driver_logic_with_a_synthetic_record(monkeypatch):
    """schedule.run end to end on the CPU: the batched recorder is replaced by
    synthetic series whose relaxation grows with N, the network by a
    least-squares stand-in; checks the report's structure and that budgets,
    calibration and comparison run."""
    def fake_record(params, total_mcs, every, seed=0, gpu=0, max_vectors=32):
        rng = np.random.default_rng(seed)
        t = np.arange(total_mcs // every + 1) * float(every)
        out = []
        for p in params:
            tau = 20.0 * p["n"] ** 1.5
            re2 = p["n"] * 3.0 * (1 + 0.5 * np.exp(-t / tau)) * (1 + 0.01 * rng.normal(size=t.size))
            a = math.exp(-every / tau)
            e = np.zeros((t.size, 8, 3), np.float32)
            e[0] = rng.normal(size=(8, 3))
            for k in range(1, t.size):
                e[k] = a * e[k - 1] + math.sqrt(1 - a * a) * rng.normal(size=(8, 3))
            out.append({"t": t, "re2": re2, "rg2": re2 / 6, "ends": e, "n": 500, "mol": {"count": 20, "size": p["n"]}})
        return out, None, 1e10

    class Stand:
        def __init__(self, *a, **k):
            pass

        def fit(self, x, y, epochs=1, **k):
            X = np.c_[x, np.ones(len(x))]
            self.w, *_ = np.linalg.lstsq(X, y, rcond=None)
            return [1.0, 0.5]

        def predict(self, x):
            return np.c_[x, np.ones(len(x))] @ self.w

    monkeypatch.setattr(sch, "record", fake_record)
    monkeypatch.setattr(sch, "Surrogate", Stand)
    rep = sch.run(n_systems=96, mcs=20000, every=200, epochs=1, seed=2)
    assert rep["systems"] == 96 and rep["test_systems"] == 24 and rep["test_systems_assessed"] >= 1
    assert rep["schedule"]["learned"]["cost_moves"] > 0 and rep["schedule"]["plain"]["cost_moves"] > 0
    assert rep["budget_factor"] in (2.0, 3.0, 4.0, 6.0, 8.0, 12.0, 16.0)
    assert set(rep["test_rmse"]) == set(sch.TARGETS)


class _FakeBatch:
    """Stand-in for pscbfm_b200.batch.Batch on the CPU: system i's chain
    ends separate linearly in time at rate rates[i] (drift) up to a plateau
    at cap[i] MCS, so the drift check's verdicts are known."""

    rates, caps = None, None

    def __init__(self, gpu=0):
        self.sys, self.t = [], []

    def add(self, system, rng=None, r250_seed=0):
        self.sys.append(system)
        self.t.append(0)
        return len(self.sys) - 1

    def initialize(self):
        pass

    def run(self, mcs):
        m = np.asarray(mcs)
        for j in range(len(self.sys)):
            self.t[j] += int(m[j])
        self._last = int(np.sum(m * np.array([s.n for s in self.sys])))

    def info(self):
        return {"last_attempts": self._last, "last_ms": 1.0}

    def gather(self, sel_s, sel_i):
        out = np.zeros((len(sel_s), 3), np.int32)
        for k, (j, i) in enumerate(zip(sel_s, sel_i)):
            s = self.sys[int(j)]
            key = s.name
            t = min(self.t[int(j)], _FakeBatch.caps[key])
            out[k] = s.pos[int(i)]
            out[k, 0] += int(i) * int(round(_FakeBatch.rates[key] * t))   # ends drift apart along x
        return out

    def close(self):
        pass


def test_live_run_extends_only_drifting_systems(monkeypatch):
    import pscbfm_b200.batch as batch_mod
    a = systems.ensemble_system(32, 16, 0.2, False, seed=1)
    b = systems.ensemble_system(32, 16, 0.2, False, seed=2)
    a.name, b.name = "drifts_long", "settles_early"
    _FakeBatch.rates = {"drifts_long": 0.002, "settles_early": 0.002}
    _FakeBatch.caps = {"drifts_long": 40000, "settles_early": 1000}
    monkeypatch.setattr(batch_mod, "Batch", _FakeBatch)
    mols = [sch.molecules(s, 16, False) for s in (a, b)]
    rec = sch.EndRecorder(mols)
    wall, ran, series, moves, dev = sch.live_run([a, b], [1, 2], [4000, 4000], 200, rec, max_mcs=20000, order=[1, 0])
    assert ran[1] == 4000                  # flat second half: no extension
    assert ran[0] > 4000                   # still relaxing at its budget: extended
    assert ran[0] <= 20000
    assert len(series[0]["t"]) == ran[0] // 200 + 1 and series[0]["t"][-1] == ran[0]


def test_end_recorder_matches_observables():
    sys_ = [systems.ensemble_system(32, 24, 0.3, False, seed=3), systems.ensemble_system(32, 31, 0.3, True, seed=4)]
    mols = [sch.molecules(sys_[0], 24, False), sch.molecules(sys_[1], 31, True)]
    rec = sch.EndRecorder(mols, max_vectors=5)

    class G:
        def gather(self, sel_s, sel_i):
            return np.stack([sys_[int(j)].pos[int(i)] for j, i in zip(sel_s, sel_i)]).astype(np.int32)

    re2, ends = rec.snapshot(G())
    for k, (s, m) in enumerate(zip(sys_, mols)):
        want, _, e = sch.observables(s.pos, m)
        assert abs(re2[k] - want) < 1e-9 * max(1.0, want)
        assert np.allclose(ends[k], e[:5])


class _DetBatch:
    """Deterministic stand-in for Batch: the chain ends of system j drift
    apart as 1 - exp(-t / tau), tau growing with its size, plus a small
    fluctuation fixed by (seed, t) -- so a live run from the same seed
    reproduces the recorded run, as the real bit-exact batch does."""

    def __init__(self, gpu=0):
        self.sys, self.seed, self.t = [], [], []

    def add(self, system, rng=None, r250_seed=0):
        self.sys.append(system)
        self.seed.append(int(r250_seed))
        self.t.append(0)
        return len(self.sys) - 1

    def initialize(self):
        pass

    def run(self, mcs):
        m = np.broadcast_to(np.asarray(mcs), (len(self.sys),))
        for j in range(len(self.sys)):
            self.t[j] += int(m[j])
        self._last = int(np.sum(m * np.array([s.n for s in self.sys])))

    def info(self):
        return {"last_attempts": self._last, "last_ms": 1e-3 * self._last / 1e7}

    def _pos(self, j):
        s = self.sys[j]
        tau = 2.0 * s.n ** 1.2
        t = self.t[j]
        f = 1.0 - math.exp(-t / tau) + 0.01 * np.random.default_rng(self.seed[j] * 1000003 + t).normal()
        p = s.pos.astype(np.int64).copy()
        p[:, 0] += (np.arange(s.n) * 3.0 * f).astype(np.int64)
        return p.astype(np.int32)

    def gather(self, sel_s, sel_i):
        cache = {}
        out = np.zeros((len(sel_s), 3), np.int32)
        for k, (j, i) in enumerate(zip(sel_s, sel_i)):
            j = int(j)
            if j not in cache:
                cache[j] = self._pos(j)
            out[k] = cache[j][int(i)]
        return out

    def all_positions(self):
        return [self._pos(j) for j in range(len(self.sys))]

    def close(self):
        pass


def test_live_compare_plumbing_on_the_cpu(monkeypatch):
    """live_compare end to end with the batch, the network and the solo
    timing replaced by CPU stand-ins: the report's structure and that the
    learned and plain live runs, calibration and ratios come out."""
    import pscbfm_b200.batch as batch_mod

    class Stand:
        def __init__(self, *a, **k):
            pass

        def fit(self, x, y, epochs=1, **k):
            X = np.c_[x, np.ones(len(x))]
            self.w, *_ = np.linalg.lstsq(X, y, rcond=None)
            return [1.0, 0.5]

        def predict(self, x):
            return np.c_[x, np.ones(len(x))] @ self.w

    monkeypatch.setattr(batch_mod, "Batch", _DetBatch)
    monkeypatch.setattr(sch, "Surrogate", Stand)
    monkeypatch.setattr(sch, "solo_rate", lambda *a, **k: 1e9)
    rep = sch.live_compare(n_systems=40, mcs=6000, every=200, epochs=1, seed=5, boxes=(16, 24, 32), n_range=(8, 32),
                           solo_tail=0)
    assert rep["test_systems"] == 10 and rep["test_systems_assessed"] >= 1
    assert rep["learned"]["wall_s"] > 0 and rep["plain"]["wall_s"] > 0
    assert rep["plain"]["budget_mcs"] > 0 and rep["ratio_learned_vs_plain"] > 0
    assert rep["budget_factor"] in (2.0, 3.0, 4.0, 6.0, 8.0, 12.0, 16.0)
    assert rep["systems_per_hour"]["learned"] > 0


def test_live_run_moves_the_tail_to_the_single_system_updater(monkeypatch):
    """with few systems left in the batch, the power-of-two ones continue on
    the single-system updater from the batch's positions, age and R250
    state at a sorting point; stand-ins with a trajectory fixed by (seed,
    MCS) show that every series and budget is the same as without the move,
    and that R_e^2 from whole positions equals the batch's gathered value"""
    import pscbfm_b200.batch as batch_mod
    import pscbfm_b200.updater as upd

    class Batch(_DetBatch):
        def add(self, system, rng=None, r250_seed=0):
            glob["orig"][int(r250_seed)] = system      # the stand-in's trajectory is relative to the start
            return super().add(system, rng=rng, r250_seed=r250_seed)

        current = {}

        def positions(self, j):
            p = self._pos(j)
            Batch.current[self.seed[j]] = p
            return p

        def state(self, j):
            st = np.zeros(251, np.uint32)
            st[0] = self.seed[j]
            return self.t[j], st, (0, 0, 0)

    glob = {"st": np.zeros(251, np.uint32), "orig": {}}
    created = []

    class Updater:
        def setup(self, system, gpu=0, rng=None, age=0, steps_between_sortings=5000):
            self.b = _DetBatch()
            seed = int(glob["st"][0])
            assert np.array_equal(system.pos, Batch.current[seed])   # handed the batch's positions
            self.b.add(glob["orig"][seed], r250_seed=seed)
            self.b.t[0] = int(age)
            created.append(self)
            return self

        def runSimulationOnGPU(self, m):
            self.b.run(m)

        def getLastRunMs(self):
            return 0.1

        def getAllMonomerPositions(self):
            return self.b._pos(0)

        def cleanup(self):
            pass

    monkeypatch.setattr(batch_mod, "Batch", Batch)
    monkeypatch.setattr(upd, "UpdaterGPUScBFM_AB_Type", Updater)
    monkeypatch.setattr(upd, "r250_set_state", lambda st: glob.__setitem__("st", np.array(st, np.uint32)))
    monkeypatch.setattr(upd, "r250_get_state", lambda: glob["st"].copy())
    sys_ = [systems.ensemble_system(L, n, 0.3, False, seed=10 + k) for k, (L, n) in enumerate([(16, 12), (24, 16), (16, 20), (32, 16)])]
    mols = [sch.molecules(s, n, False) for s, n in zip(sys_, (12, 16, 20, 16))]
    budgets = [1000, 3000, 6000, 6000]
    runs = []
    for tail in (0, 2):
        rec = sch.EndRecorder(mols)
        rep = {}
        runs.append(sch.live_run(sys_, [1, 2, 3, 4], budgets, 200, rec, max_mcs=20000, solo_tail=tail, sort_every=1000,
                                 report=rep, solo_min_monomers=0) + (rep,))
    (w0, ran0, ser0, mv0, _, _), (w1, ran1, ser1, mv1, _, rep1) = runs
    assert rep1["moved_to_single_system"] >= 1 and len(created) == rep1["moved_to_single_system"]
    assert np.array_equal(ran0, ran1) and mv0 == mv1
    for a, b in zip(ser0, ser1):
        assert np.array_equal(a["t"], b["t"]) and np.array_equal(a["re2"], b["re2"])
    # only power-of-two boxes move (the 24^3 system stays in the batch)
    assert all(all((v & (v - 1)) == 0 for v in u.b.sys[0].box) for u in created)
