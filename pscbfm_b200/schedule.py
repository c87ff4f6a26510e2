"""Learned run schedule for batched ensembles.

A small network (pscbfm_b200.mlp.MLP, trained on the GPU by the library's
own tensor-core kernels) maps a system's architecture -- monomers per
molecule N, molecule count, volume fraction, arms, box edge, side-chain
spacing -- to the relaxation time of R_e^2, equilibrium R_e^2 and R_g^2
(per monomer) and the end-to-end autocorrelation time.  The schedule gives
each system an MCS budget of a calibrated multiple of its predicted
end-to-end autocorrelation time and admits the longest first; a measured
check on every system's own R_e^2 series (a straight-line fit over the
second half of the run: a significant change of more than 2% means drift)
extends any run the prediction under-budgeted.  The plain schedule, and
the fallback, is one fixed budget for every system.

The MC arithmetic is never touched: budgets only decide how long each
system runs.  Training data come from the batched simulator itself.
"""
from __future__ import annotations

import math

import numpy as np

FEATURES = ("log N", "log molecules", "volume fraction", "arms / 3", "box / 64", "side-chain spacing / 8")
TARGETS = ("log10 R_e^2 relaxation MCS", "R_e^2 / N", "R_g^2 / N", "log10 end-to-end autocorrelation MCS")


# ----------------------------------------------------------- molecules
def molecules(system, n_per_molecule: int, star: bool):
    """index arrays of the ensemble generator's molecules (contiguous ids):
    linear: (first, last, members); star: (core, tips, members).  Side
    chains (attribute 2, ids after every backbone) are not part of them."""
    n = system.n if system.attributes is None else int(np.count_nonzero(np.asarray(system.attributes) == 1))
    if not star:
        size = n_per_molecule
        m = n // size
        first = np.arange(m) * size
        return {"star": False, "ends": (first, first + size - 1), "size": size, "count": m}
    arm = max(1, (n_per_molecule - 1) // 3)
    size = 1 + 3 * arm
    m = n // size
    core = np.arange(m) * size
    tips = np.stack([core + arm, core + 2 * arm, core + 3 * arm], 1)
    return {"star": True, "ends": (core, tips), "size": size, "count": m}


def observables(pos, mol):
    """(R_e^2, R_g^2, end vectors): mean over molecules; for stars R_e^2 is the
    mean squared core-to-tip distance of the arms"""
    p = np.asarray(pos, np.float64)
    size, m = mol["size"], mol["count"]
    q = p[: size * m].reshape(m, size, 3)
    com = q.mean(1)
    rg2 = float(((q - com[:, None, :]) ** 2).sum(2).mean())
    if mol["star"]:
        core, tips = mol["ends"]
        v = p[tips] - p[core][:, None, :]
        re2 = float((v ** 2).sum(2).mean())
        ends = v.reshape(-1, 3)
    else:
        a, b = mol["ends"]
        v = p[b] - p[a]
        re2 = float((v ** 2).sum(1).mean())
        ends = v
    return re2, rg2, ends


# ------------------------------------------------------------ labels
def equilibration_time(t, re2, tol: float = 0.1):
    """first time after which a running mean of R_e^2 stays within tol of the
    plateau (mean of the last third); censored at the last time"""
    t = np.asarray(t, np.float64)
    re2 = np.asarray(re2, np.float64)
    k = max(1, len(re2) // 3)
    plateau = re2[-k:].mean()
    w = max(1, len(re2) // 20)
    run = np.convolve(re2, np.ones(w), mode="same") / np.convolve(np.ones_like(re2), np.ones(w), mode="same")
    ok = np.abs(run - plateau) <= tol * plateau
    bad = np.flatnonzero(~ok[:-1]) if len(ok) > 1 else np.array([], int)
    i = 0 if bad.size == 0 else int(bad[-1]) + 1
    return float(max(t[min(i, len(t) - 1)], t[1] - t[0] if len(t) > 1 else 1.0)), float(plateau)


def relaxation_fit(t, re2, taus=None):
    """least-squares fit R_e^2(t) = A + B exp(-t / tau) over a log grid of
    tau (A, B linear for each tau); returns (tau, A).  Uses the whole
    series, so single-system fluctuations do not decide it."""
    t = np.asarray(t, np.float64)
    y = np.asarray(re2, np.float64)
    if taus is None:
        taus = np.exp(np.linspace(np.log(max(t[1] - t[0], 1.0) / 4), np.log(10.0 * t[-1]), 120))
    best = (np.inf, float(taus[-1]), float(y.mean()))
    for tau in taus:
        e = np.exp(-t / tau)
        A = np.stack([np.ones_like(t), e], 1)
        coef, *_ = np.linalg.lstsq(A, y, rcond=None)
        r = A @ coef - y
        sse = float(r @ r)
        if sse < best[0]:
            best = (sse, float(tau), float(coef[0]))
    return best[1], best[2]


def relaxation_time(t, ends, start: int):
    """end-to-end vector autocorrelation over the snapshots from index start:
    first lag where C drops below 1/e (linear interpolation), censored at
    the window length"""
    t = np.asarray(t, np.float64)
    e = np.asarray(ends[start:], np.float64)      # (snapshots, vectors, 3)
    if len(e) < 3:
        return float(t[-1] - t[start] if len(t) > start else 1.0)
    norm = (e * e).sum(2).mean()
    dt = t[1] - t[0]
    prev = 1.0
    for lag in range(1, len(e)):
        c = float((e[lag:] * e[:-lag]).sum(2).mean() / norm)
        if c < 1.0 / math.e:
            frac = (prev - 1.0 / math.e) / max(prev - c, 1e-12)
            return float(dt * (lag - 1 + frac))
        prev = c
    return float(dt * (len(e) - 1))


def features(p, n_sites_molecules: int):
    """the six inputs of one system's parameters"""
    return np.array([math.log(p["n"]), math.log(max(1, n_sites_molecules)), p["phi"], (3 if p["star"] else 1) / 3.0,
                     p["L"] / 64.0, p.get("side_every", 0) / 8.0], np.float32)


def labels(t, re2, rg2, ends, n_per_molecule):
    """the four targets of one system's recorded series: the equilibration
    time is the fitted relaxation time of R_e^2 (relaxation_fit)"""
    teq, _ = relaxation_fit(t, re2)
    k = max(1, len(re2) // 3)
    re2_eq = float(np.mean(re2[-k:]))
    rg2_eq = float(np.mean(rg2[-k:]))
    start = min(len(t) - 3, int(np.searchsorted(t, teq)))
    tr = relaxation_time(t, ends, max(0, start))
    return np.array([math.log10(teq), re2_eq / n_per_molecule, rg2_eq / n_per_molecule, math.log10(max(tr, 1.0))],
                    np.float32)


# ------------------------------------------------------------ data
def ensemble_params(n_systems: int, seed: int, boxes=(16, 24, 32), n_range=(8, 48), phi_range=(0.1, 0.5)):
    """architectures of a training/test ensemble (small enough to equilibrate)"""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_systems):
        L = int(rng.choice(boxes))
        n = int(round(math.exp(rng.uniform(math.log(n_range[0]), math.log(n_range[1])))))
        star = bool(rng.random() < 0.5)
        if star:
            n = 1 + 3 * max(1, (n - 1) // 3)
        side_every = int(rng.choice((0, 0, 4, 8)))
        side_len = int(rng.integers(2, 5)) if side_every else 0
        out.append({"L": L, "n": n, "phi": float(rng.uniform(*phi_range)), "star": star, "side_every": side_every,
                    "side_len": side_len})
    return out


def record(params, total_mcs: int, every: int, seed: int = 0, gpu: int = 0, max_vectors: int = 32):
    """run every system of the ensemble in one batch for total_mcs MCS,
    recording R_e^2, R_g^2 and (up to max_vectors) end vectors every `every`
    MCS; returns (series, systems, rate in attempted moves/s)"""
    from . import systems as gen
    from .batch import Batch
    from .updater import Rng
    sys_ = [gen.ensemble_system(p["L"], p["n"], p["phi"], p["star"], seed=seed + i, side_every=p.get("side_every", 0),
                                side_len=p.get("side_len", 0)) for i, p in enumerate(params)]
    mols = [molecules(s, p["n"], p["star"]) for s, p in zip(sys_, params)]
    b = Batch(gpu)
    for i, s in enumerate(sys_):
        b.add(s, rng=Rng.Saru, r250_seed=seed + 7919 * i)
    b.initialize()
    nsnap = total_mcs // every + 1
    re2 = np.zeros((len(sys_), nsnap))
    rg2 = np.zeros((len(sys_), nsnap))
    ends = [np.zeros((nsnap, min(max_vectors, m["count"] * (3 if m["star"] else 1)), 3), np.float32) for m in mols]

    def take(k):
        for i, p in enumerate(b.all_positions()):
            a, g, e = observables(p, mols[i])
            re2[i, k], rg2[i, k] = a, g
            ends[i][k] = e[: ends[i].shape[1]]

    take(0)
    moves, ms = 0, 0.0
    for k in range(1, nsnap):
        b.run(every)
        info = b.info()
        moves += info["last_attempts"]
        ms += info["last_ms"]
        take(k)
    t = np.arange(nsnap) * float(every)
    series = [{"t": t, "re2": re2[i], "rg2": rg2[i], "ends": ends[i], "n": sys_[i].n, "mol": mols[i]} for i in range(len(sys_))]
    return series, sys_, moves / (ms / 1e3)


def dataset(params, series):
    x = np.stack([features(p, s["mol"]["count"]) for p, s in zip(params, series)])
    y = np.stack([labels(s["t"], s["re2"], s["rg2"], s["ends"], p["n"]) for p, s in zip(params, series)])
    return x, y


# ------------------------------------------------------------ model
class Surrogate:
    """MLP on standardised inputs and targets"""

    def __init__(self, hidden: int = 128, seed: int = 0, gpu: int = 0):
        from .mlp import MLP
        self.net = MLP(len(FEATURES), hidden, len(TARGETS), seed=seed, gpu=gpu)

    def fit(self, x, y, epochs: int = 300, batch: int = 256, lr: float = 2e-3):
        self.xm, self.xs = x.mean(0), x.std(0) + 1e-6
        self.ym, self.ys = y.mean(0), y.std(0) + 1e-6
        return self.net.fit((x - self.xm) / self.xs, (y - self.ym) / self.ys, epochs=epochs, batch=batch, lr=lr)

    def predict(self, x):
        return self.net.forward((np.asarray(x, np.float32) - self.xm) / self.xs) * self.ys + self.ym


# ---------------------------------------------------------- schedules
def window_estimate(s, budget):
    """R_e^2 a run of `budget` MCS reports: the mean over its second half"""
    t, re2 = s["t"], s["re2"]
    hi = int(np.searchsorted(t, budget, side="right"))
    lo = int(np.searchsorted(t, budget / 2.0, side="left"))
    lo = min(lo, hi - 1)
    return float(re2[lo:hi].mean())


def drifting(s, budget, tol: float = 0.02, z: float = 3.0):
    """the measured check on the second half of the run: a straight-line fit
    of R_e^2 against time; drift when the fitted change across that half is
    more than tol of its mean and the slope is more than z standard errors
    from zero"""
    t, re2 = s["t"], s["re2"]
    hi = int(np.searchsorted(t, budget, side="right"))
    lo = hi // 2
    if hi - lo < 4:
        return True
    x, y = t[lo:hi], re2[lo:hi]
    xc = x - x.mean()
    sxx = float((xc * xc).sum())
    slope = float((xc * (y - y.mean())).sum() / sxx)
    resid = y - y.mean() - slope * xc
    se = math.sqrt(float((resid * resid).sum()) / (len(y) - 2) / sxx)
    change = abs(slope) * float(x[-1] - x[0])
    return change > tol * float(y.mean()) and abs(slope) > z * se


def learned_budgets(pred_log_teq, series, factor: float = 3.0, grow: float = 1.5, floor: float = 200.0):
    """factor x predicted equilibration time, extended by `grow` while the
    measured check sees drift (never past the recorded length)"""
    out = []
    for p, s in zip(pred_log_teq, series):
        tmax = float(s["t"][-1])
        b = min(tmax, max(floor, factor * 10.0 ** float(p)))
        while b < tmax and drifting(s, b):
            b = min(tmax, b * grow)
        out.append(b)
    return np.array(out)


def _errors(series, budgets, truth):
    est = np.array([window_estimate(s, b) for s, b in zip(series, np.broadcast_to(budgets, (len(series),)))])
    rel = (est - truth) / truth
    return est, rel


def compare(series, budgets, plain_grid=None, bias_floor: float = 0.005):
    """Cost (monomers x MCS) and R_e^2 accuracy of the learned budgets
    against fixed budgets.  Accuracy: the per-system relative error of the
    R_e^2 a run reports against its series' plateau, and the ensemble bias
    (mean signed relative error, where single-system noise averages out and
    under-equilibration shows).  Plain: the smallest fixed budget whose bias
    is no larger (at least bias_floor), and the full recorded window."""
    truth = np.array([s["re2"][-max(1, len(s["re2"]) // 3):].mean() for s in series])
    n = np.array([s["n"] for s in series], np.float64)
    _, rel_l = _errors(series, budgets, truth)
    cost_l = float(np.sum(n * budgets))
    tmax = float(series[0]["t"][-1])
    grid = plain_grid if plain_grid is not None else np.unique(np.concatenate([series[0]["t"][1:], [tmax]]))
    target = max(abs(float(rel_l.mean())), bias_floor)
    chosen = tmax
    for b in grid:
        _, rel_p = _errors(series, float(b), truth)
        if abs(rel_p.mean()) <= target:
            chosen = float(b)
            break
    _, rel_p = _errors(series, chosen, truth)
    _, rel_f = _errors(series, tmax, truth)
    est_l = np.array([window_estimate(s, b) for s, b in zip(series, budgets)])
    est_f = np.array([window_estimate(s, tmax) for s in series])
    # ensemble R_e^2 / N over molecules: every molecule counts once, N its length
    cnt = np.array([s.get("mol", {}).get("count", 1) for s in series], np.float64)
    size = np.array([s.get("mol", {}).get("size", s["n"]) for s in series], np.float64)
    wts = cnt / size

    def ens(e, k=slice(None)):
        return float(np.sum(wts[k] * e[k]) / np.sum(cnt[k]))

    dev = ens(est_l) / ens(est_f) - 1.0
    rng = np.random.default_rng(0)
    boot = []
    for _ in range(200):
        k = rng.integers(0, len(series), len(series))
        boot.append(ens(est_l, k) / ens(est_f, k) - 1.0)
    out = {"learned": {"cost_moves": cost_l, "mean_rel_err_re2": float(np.abs(rel_l).mean()), "bias_re2": float(rel_l.mean()),
                       "within_2pct": float(np.mean(np.abs(rel_l) <= 0.02)), "mean_budget_mcs": float(budgets.mean())},
           "plain": {"cost_moves": float(np.sum(n * chosen)), "mean_rel_err_re2": float(np.abs(rel_p).mean()),
                     "bias_re2": float(rel_p.mean()), "within_2pct": float(np.mean(np.abs(rel_p) <= 0.02)), "budget_mcs": chosen},
           "plain_full_window": {"cost_moves": float(np.sum(n * tmax)), "bias_re2": float(rel_f.mean()), "budget_mcs": tmax},
           "ensemble_re2_per_n_learned_vs_full_window": dev,
           "ensemble_re2_per_n_learned_vs_full_window_bootstrap_sd": float(np.std(boot))}
    out["systems_per_hour_ratio"] = out["plain"]["cost_moves"] / cost_l
    out["systems_per_hour_ratio_vs_full_window"] = out["plain_full_window"]["cost_moves"] / cost_l
    return out


def admission_order(pred_log_teq, sizes):
    """longest predicted work first"""
    return np.argsort(-(10.0 ** np.asarray(pred_log_teq, np.float64)) * np.asarray(sizes, np.float64), kind="stable")


# ------------------------------------------------------------ live runs
class EndRecorder:
    """R_e^2 and end vectors of every system of a batch from the positions
    of the molecule ends alone (chain ends; star cores and arm tips), read
    on the device with Batch.gather -- a few percent of the monomers, so a
    snapshot of a whole ensemble costs milliseconds.  For stars R_e^2 is the
    mean squared core-to-tip distance, as in `observables`."""

    def __init__(self, mols, max_vectors: int = 32):
        sel_s, sel_i, a_idx, b_idx, vsys = [], [], [], [], []
        off = 0
        self.keep = []
        for si, m in enumerate(mols):
            if m["star"]:
                core, tips = m["ends"]
                ids = np.concatenate([core, tips.reshape(-1)])
                c = len(core)
                a = np.repeat(np.arange(c), 3)                  # the core of each arm
                b = c + np.arange(3 * c)                        # its tip
            else:
                first, last = m["ends"]
                ids = np.concatenate([first, last])
                c = len(first)
                a, b = np.arange(c), c + np.arange(c)
            sel_s.append(np.full(len(ids), si, np.int64))
            sel_i.append(ids.astype(np.int64))
            nv0 = sum(len(x) for x in a_idx)
            a_idx.append(off + a)
            b_idx.append(off + b)
            vsys.append(np.full(len(a), si, np.int64))
            self.keep.append(np.arange(nv0, nv0 + min(max_vectors, len(a))))
            off += len(ids)
        self.sel_s = np.concatenate(sel_s)
        self.sel_i = np.concatenate(sel_i)
        self.a = np.concatenate(a_idx)
        self.b = np.concatenate(b_idx)
        self.vsys = np.concatenate(vsys)
        self.nsys = len(mols)
        self.count = np.bincount(self.vsys, minlength=self.nsys).astype(np.float64)

    def re2_of(self, i, pos):
        """R_e^2 of system i from its whole position array (original ids)"""
        sel = np.flatnonzero(self.sel_s == i)
        p = np.asarray(pos, np.float64)[self.sel_i[sel]]
        vm = self.vsys == i
        a, b = self.a[vm] - sel[0], self.b[vm] - sel[0]
        v = p[b] - p[a]
        # summed in the same order as `snapshot`, so the values are identical
        w = np.bincount(np.zeros(len(v), np.int64), weights=(v * v).sum(1), minlength=1)[0]
        return float(w / max(self.count[i], 1))

    def snapshot(self, batch, batch_index=None):
        """(R_e^2 per system, end vectors of the first max_vectors molecules
        of each system); batch_index[i]: the batch's index of system i when
        the batch holds them in another order"""
        sel = self.sel_s if batch_index is None else np.asarray(batch_index)[self.sel_s]
        p = batch.gather(sel, self.sel_i).astype(np.float64)
        v = p[self.b] - p[self.a]
        re2 = np.bincount(self.vsys, weights=(v * v).sum(1), minlength=self.nsys) / np.maximum(self.count, 1)
        return re2, [v[k].astype(np.float32) for k in self.keep]


def round_up(x, every):
    return int(every * math.ceil(float(x) / every))


def live_run(systems_, r250_seeds, budgets, every: int, recorder, max_mcs: int | None = None, grow: float = 1.5,
             judge: bool = True, order=None, gpu: int = 0, solo_tail: int = 0, sort_every: int = 5000, report=None,
             solo_min_monomers: int = 16384, clusters: int = 4):
    """Run an ensemble live on the GPU under per-system budgets: system i
    advances `every` MCS per batched launch until its budget is spent; its
    R_e^2 is recorded after every launch; when the budget is spent and the
    drift check (`drifting`, on the second half of its own series) sees the
    run still relaxing, the budget grows by `grow` (up to max_mcs) and the
    system goes on.  Systems are added to the batch in `order` (admission:
    longest predicted work first).

    Tail: once at most `solo_tail` systems are left in the batch, the ones
    of at least `solo_min_monomers` monomers (where one system on the whole
    GPU runs many times faster than on its share of the batch; smaller ones
    run as fast in parallel in the batch) whose box edges are powers of two
    leave it at their next sorting point
    (age a multiple of `sort_every`, where the batch and the single-system
    updater both re-sort by the same keys) and go on, one after another, on
    the single-system updater -- the whole GPU per system -- from the
    batch's positions, age and R250 state, on the same trajectory.  Returns
    (wall seconds, per-system MCS run, per-system series {t, re2},
    attempted moves, device ms); `report` (a dict) receives the systems
    moved to the single-system updater."""
    import time

    from . import updater as upd
    from .batch import Batch
    from .systems import System
    from .updater import Rng
    nsys = len(systems_)
    order = np.arange(nsys) if order is None else np.asarray(order)
    pos_in_batch = np.empty(nsys, np.int64)
    pos_in_batch[order] = np.arange(nsys)
    b = Batch(gpu)
    for i in order:
        b.add(systems_[i], rng=Rng.Saru, r250_seed=int(r250_seeds[i]))
    b.initialize()
    if clusters != 4:
        b.set_clusters(clusters)
    rec = recorder
    remaining = np.array([round_up(x, every) for x in budgets], np.int64)
    ran = np.zeros(nsys, np.int64)
    cap = np.full(nsys, np.iinfo(np.int64).max if max_mcs is None else int(max_mcs), np.int64)
    remaining = np.minimum(remaining, cap)
    series = [{"t": [0.0], "re2": []} for _ in range(nsys)]
    re2, _ = rec.snapshot(b, pos_in_batch)
    for i in range(nsys):
        series[i]["re2"].append(float(re2[i]))
    moves, dev_ms = 0, 0.0
    solo = {}  # system -> [single-system updater, its R250 state]
    launches = []  # (systems in the launch, device ms) per batched launch
    pow2 = np.array([all(v > 0 and (v & (v - 1)) == 0 for v in s.box) and s.n >= solo_min_monomers for s in systems_])
    t0 = time.perf_counter()

    def judged(i):
        if remaining[i] == 0 and judge and ran[i] < cap[i]:
            s_ = {"t": np.asarray(series[i]["t"]), "re2": np.asarray(series[i]["re2"])}
            if drifting(s_, float(ran[i])):
                remaining[i] = min(round_up(ran[i] * grow, every), cap[i]) - ran[i]

    while (remaining > 0).any():
        in_batch = (remaining > 0) & np.array([i not in solo for i in range(nsys)])
        if solo_tail and 0 < in_batch.sum() <= solo_tail:
            for i in np.flatnonzero(in_batch & pow2):
                if ran[i] % sort_every:
                    continue
                j = int(pos_in_batch[i])
                pos = b.positions(j)
                age, st, _ = b.state(j)
                s0 = systems_[i]
                si = System(s0.box, np.ascontiguousarray(pos, dtype=np.int32), s0.deg, s0.nbr, s0.allowed, s0.chains,
                            s0.attributes, s0.name)
                upd.r250_set_state(st)
                u = upd.UpdaterGPUScBFM_AB_Type().setup(si, gpu=gpu, rng=Rng.Saru, age=int(age),
                                                       steps_between_sortings=sort_every)
                solo[i] = [u, upd.r250_get_state()]
                in_batch[i] = False
        step = np.where(in_batch, every, 0).astype(np.uint32)
        if step.any():
            b.run(step[order])
            info = b.info()
            moves += info["last_attempts"]
            dev_ms += info["last_ms"]
            launches.append((int(in_batch.sum()), float(info["last_ms"])))
            ran += step
            remaining -= step
            re2, _ = rec.snapshot(b, pos_in_batch)
            for i in np.flatnonzero(step):
                series[i]["t"].append(float(ran[i]))
                series[i]["re2"].append(float(re2[i]))
                judged(i)
        for i, (u, st) in solo.items():
            if remaining[i] <= 0:
                continue
            upd.r250_set_state(st)
            u.runSimulationOnGPU(every)
            solo[i][1] = upd.r250_get_state()
            moves += systems_[i].n * every
            dev_ms += u.getLastRunMs()
            ran[i] += every
            remaining[i] -= every
            series[i]["t"].append(float(ran[i]))
            series[i]["re2"].append(rec.re2_of(i, u.getAllMonomerPositions()))
            judged(i)
    wall = time.perf_counter() - t0
    for u, _ in solo.values():
        u.cleanup()
    if report is not None:
        report["moved_to_single_system"] = len(solo)
        act = np.array([a for a, _ in launches], np.int64)
        ms = np.array([m for _, m in launches], np.float64)
        report["batched_launches"] = len(launches)
        report["device_ms_by_systems_in_launch"] = {f"<={k}": float(ms[act <= k].sum()) for k in (8, 16, 32, 64, 128)}
        report["device_ms_by_systems_in_launch"]["all"] = float(ms.sum())
    b.close()
    for s in series:
        s["t"] = np.asarray(s["t"])
        s["re2"] = np.asarray(s["re2"])
    return wall, ran, series, moves, dev_ms


def record_live(params, total_mcs: int, every: int, seed: int = 0, gpu: int = 0, max_vectors: int = 32, rg2_snapshots: int = 8):
    """Record an ensemble for total_mcs MCS with the batched simulator:
    R_e^2 and end vectors of every system after every `every` MCS (from the
    gathered molecule ends), R_g^2 from whole-system read-backs at
    rg2_snapshots points of the last third.  Returns (series, systems,
    rate in attempted moves/s, cumulative device seconds at each snapshot)."""
    from . import systems as gen
    from .batch import Batch
    from .updater import Rng
    sys_ = [gen.ensemble_system(p["L"], p["n"], p["phi"], p["star"], seed=seed + i, side_every=p.get("side_every", 0),
                                side_len=p.get("side_len", 0)) for i, p in enumerate(params)]
    mols = [molecules(s, p["n"], p["star"]) for s, p in zip(sys_, params)]
    rec = EndRecorder(mols, max_vectors)
    b = Batch(gpu)
    for i, s in enumerate(sys_):
        b.add(s, rng=Rng.Saru, r250_seed=seed + 7919 * i)
    b.initialize()
    nsnap = total_mcs // every + 1
    re2 = np.zeros((len(sys_), nsnap))
    rg2 = np.full((len(sys_), nsnap), np.nan)
    ends = [np.zeros((nsnap, len(k), 3), np.float32) for k in rec.keep]
    late = set(np.linspace(nsnap - nsnap // 3, nsnap - 1, rg2_snapshots).astype(int).tolist())

    def take(k):
        r, e = rec.snapshot(b)
        re2[:, k] = r
        for i in range(len(sys_)):
            ends[i][k] = e[i]
        if k in late:
            for i, p in enumerate(b.all_positions()):
                rg2[i, k] = observables(p, mols[i])[1]

    take(0)
    moves, ms = 0, 0.0
    cum = np.zeros(nsnap)
    for k in range(1, nsnap):
        b.run(every)
        info = b.info()
        moves += info["last_attempts"]
        ms += info["last_ms"]
        cum[k] = ms / 1e3
        take(k)
    b.close()
    t = np.arange(nsnap) * float(every)
    series = []
    for i in range(len(sys_)):
        rg = rg2[i].copy()
        fill = np.nanmean(rg) if np.isfinite(rg).any() else 0.0
        rg[~np.isfinite(rg)] = fill
        series.append({"t": t, "re2": re2[i], "rg2": rg, "ends": ends[i], "n": sys_[i].n, "mol": mols[i]})
    return series, sys_, moves / (ms / 1e3), cum


def live_compare(n_systems: int = 2048, mcs: int = 200000, every: int = 1000, test_fraction: float = 0.25, epochs: int = 300,
                 seed: int = 3, gpu: int = 0, boxes=(32, 48, 64, 96, 128), n_range=(16, 512), phi_range=(0.1, 0.5),
                 solo_tail: int = 0, solo_tail_alternatives=(), clusters: int = 4):
    """The learned schedule run live against plain fixed budgets.

    An ensemble of the batched configuration's ranges is recorded for `mcs`
    MCS (the full-length runs, whose last third gives each system's plateau
    R_e^2); the network is trained on the training part; on the held-out
    test systems three schedules then run live on the GPU, each from the
    systems' initial states with their own R250 seeds (so every run is a
    prefix of the recorded trajectory):
      learned  budgets = factor x predicted end-to-end autocorrelation time,
               admission longest predicted work first, the drift check
               extending under-budgeted systems by further batched launches;
      plain    the cheapest fixed budget whose ensemble bias of R_e^2 is no
               larger than the learned schedule's, for every system;
      solo     that fixed budget through the single-system updater, one
               system after another (timed on a sample, scaled).
    Systems per hour come from the wall clock of each live run."""
    import time
    params = ensemble_params(n_systems, seed, boxes=boxes, n_range=n_range, phi_range=phi_range)
    t0 = time.perf_counter()
    series, sys_, rate, cum = record_live(params, mcs, every, seed=seed, gpu=gpu)
    t_rec = time.perf_counter() - t0
    x, y = dataset(params, series)
    rng = np.random.default_rng(seed)
    idx = rng.permutation(n_systems)
    n_te = max(1, int(n_systems * test_fraction))
    te, tr = idx[:n_te], idx[n_te:]
    n_cal = max(1, len(tr) // 5)
    cal, fit = tr[:n_cal], tr[n_cal:]
    # labels are trusted where the record saw the system relax: fitted
    # relaxation within a twelfth of the window
    assess = y[:, 0] <= math.log10(mcs / 12.0)
    te_a, cal_a = te[assess[te]], cal[assess[cal]]
    if len(te_a) == 0 or len(cal_a) == 0:
        te_a, cal_a = te, cal
    # the network learns from the training systems whose labels are trusted
    fit_a = fit[assess[fit]]
    if len(fit_a) < 64:
        fit_a = fit
    model = Surrogate(seed=seed, gpu=gpu)
    hist = model.fit(x[fit_a], y[fit_a], epochs=epochs)
    pred_te = model.predict(x[te_a])
    rmse = np.sqrt(((pred_te - y[te_a]) ** 2).mean(0))
    rmse_const = np.sqrt(((y[fit_a].mean(0) - y[te_a]) ** 2).mean(0))
    # budget factor calibrated on held-out training systems (replayed on their records)
    cal_series = [series[i] for i in cal_a]
    pred_cal = model.predict(x[cal_a])
    factor, calib = 8.0, {}
    for f in (2.0, 3.0, 4.0, 6.0, 8.0, 12.0, 16.0):
        c = compare(cal_series, learned_budgets(pred_cal[:, 3], cal_series, factor=f))
        calib[f] = {"ratio": c["systems_per_hour_ratio"], "ensemble_re2_vs_full": c["ensemble_re2_per_n_learned_vs_full_window"]}
    ok = [f for f in calib if abs(calib[f]["ensemble_re2_vs_full"]) <= 0.01]
    if ok:
        factor = max(ok, key=lambda f: calib[f]["ratio"])
    # live runs on the assessable test systems
    test_sys = [sys_[i] for i in te_a]
    seeds = [seed + 7919 * int(i) for i in te_a]
    mols = [series[i]["mol"] for i in te_a]
    truth = np.array([series[i]["re2"][-max(1, len(series[i]["re2"]) // 3):].mean() for i in te_a])
    pred = model.predict(x[te_a])
    budgets = np.maximum(200.0, factor * 10.0 ** pred[:, 3])
    order = admission_order(pred[:, 3], [s.n for s in test_sys])
    rec = EndRecorder(mols)
    rep_l, rep_p = {}, {}
    wall_l, ran_l, ser_l, moves_l, dev_l = live_run(test_sys, seeds, budgets, every, rec, max_mcs=mcs, order=order, gpu=gpu,
                                                    solo_tail=solo_tail, report=rep_l, clusters=clusters)
    est_l = np.array([window_estimate(s, float(r)) for s, r in zip(ser_l, ran_l)])
    # the same learned schedule with other tail thresholds (same trajectories, other executors)
    alternatives = {}
    for k in solo_tail_alternatives:
        rep_k = {}
        w_k, ran_k, _, mv_k, dev_k = live_run(test_sys, seeds, budgets, every, rec, max_mcs=mcs, order=order, gpu=gpu,
                                              solo_tail=int(k), report=rep_k, clusters=clusters)
        alternatives[str(int(k))] = {"wall_s": w_k, "device_s": dev_k / 1e3, "moves": int(mv_k),
                                     "same_mcs": bool(np.array_equal(ran_k, ran_l)), **rep_k}
    rel_l = (est_l - truth) / truth
    # the live runs start from the recorded systems' initial states with the
    # same seeds, so (bit-exact simulation) their R_e^2 series are prefixes of
    # the recorded ones
    prefix = all(np.array_equal(sl["re2"], series[i]["re2"][:len(sl["re2"])]) for sl, i in zip(ser_l, te_a))
    # the plain fixed budget of equal bias, from the recorded trajectories (a
    # plain run of B MCS is their prefix), then run live
    target = max(abs(float(rel_l.mean())), 0.005)
    rec_series = [series[i] for i in te_a]
    B = float(mcs)
    for b_ in series[0]["t"][1:]:
        rel = np.array([(window_estimate(s, float(b_)) - tv) / tv for s, tv in zip(rec_series, truth)])
        if abs(rel.mean()) <= target:
            B = float(b_)
            break
    wall_p, ran_p, ser_p, moves_p, dev_p = live_run(test_sys, seeds, np.full(len(te_a), B), every, rec, judge=False, gpu=gpu,
                                                    solo_tail=solo_tail, report=rep_p, clusters=clusters)
    est_p = np.array([window_estimate(s, float(r)) for s, r in zip(ser_p, ran_p)])
    rel_p = (est_p - truth) / truth
    # ensemble R_e^2 / N over molecules against the full-length runs
    cnt = np.array([m["count"] for m in mols], np.float64)
    size = np.array([m["size"] for m in mols], np.float64)
    ens = lambda e: float(np.sum(cnt / size * e) / np.sum(cnt))
    est_full = np.array([window_estimate(s, float(mcs)) for s in rec_series])
    solo = solo_rate([sys_[i] for i in te_a], seeds, gpu=gpu)
    solo_wall = float(np.sum([s.n for s in test_sys])) * B / solo if solo else None
    return {
        "systems": n_systems, "test_systems": int(n_te), "test_systems_assessed": int(len(te_a)), "recorded_mcs": mcs,
        "snapshot_every": every,
        "ensemble": f"box edges {list(boxes)}, linear chains or 3-arm stars of {n_range[0]}..{n_range[1]} monomers, "
                    f"half of them combs (side chains of 2..4 on every 4th or 8th backbone monomer), volume fraction "
                    f"{phi_range[0]}..{phi_range[1]}, Saru",
        "record_s": t_rec, "batch_rate_moves_per_s": rate, "train_loss_first_last": [hist[0], hist[-1]],
        "training_systems": int(len(fit_a)), "rmse_on": "assessable test systems",
        "test_rmse": dict(zip(TARGETS, map(float, rmse))),
        "test_rmse_constant_predictor": dict(zip(TARGETS, map(float, rmse_const))),
        "budget_factor": factor, "calibration": {str(k): v for k, v in calib.items()},
        "learned": {"wall_s": wall_l, "device_s": dev_l / 1e3, "moves": int(moves_l), "mean_mcs": float(ran_l.mean()),
                    "extended": int(np.sum(ran_l > np.array([round_up(v, every) for v in np.minimum(budgets, mcs)]))),
                    "bias_re2": float(rel_l.mean()), "mean_abs_rel_err_re2": float(np.abs(rel_l).mean()),
                    "ensemble_re2_per_n_vs_full": ens(est_l) / ens(est_full) - 1.0,
                    "moved_to_single_system": rep_l.get("moved_to_single_system", 0),
                    "batched_launches": rep_l.get("batched_launches"),
                    "device_ms_by_systems_in_launch": rep_l.get("device_ms_by_systems_in_launch")},
        "plain": {"budget_mcs": B, "wall_s": wall_p, "device_s": dev_p / 1e3, "moves": int(moves_p),
                  "bias_re2": float(rel_p.mean()), "mean_abs_rel_err_re2": float(np.abs(rel_p).mean()),
                  "ensemble_re2_per_n_vs_full": ens(est_p) / ens(est_full) - 1.0,
                  "moved_to_single_system": rep_p.get("moved_to_single_system", 0),
                  "batched_launches": rep_p.get("batched_launches"),
                  "device_ms_by_systems_in_launch": rep_p.get("device_ms_by_systems_in_launch")},
        "solo": {"moves_per_s": solo, "wall_s_estimate": solo_wall},
        "systems_per_hour": {"learned": len(te_a) / wall_l * 3600.0, "plain": len(te_a) / wall_p * 3600.0,
                             "solo": (len(te_a) / solo_wall * 3600.0) if solo_wall else None},
        "live_runs_reproduce_the_record": bool(prefix),
        "learned_with_other_tail_thresholds": alternatives,
        "clusters": clusters,
        "ratio_learned_vs_plain": wall_p / wall_l,
        "ratio_learned_vs_solo": (solo_wall / wall_l) if solo_wall else None,
    }


def solo_rate(systems_, seeds, gpu: int = 0, sample: int = 24, mcs: int = 2000):
    """attempted moves/s of systems run one after another through the
    single-system updater (power-of-two boxes; a sample, timed on the host
    clock around each runSimulationOnGPU)"""
    import time

    from .updater import Rng, UpdaterGPUScBFM_AB_Type, r250_seed
    rng = np.random.default_rng(11)
    pick = [i for i in rng.permutation(len(systems_)) if not any(v & (v - 1) for v in systems_[i].box)][:sample]
    moves, wall = 0, 0.0
    for i in pick:
        r250_seed(int(seeds[i]))
        u = UpdaterGPUScBFM_AB_Type().setup(systems_[i], gpu=gpu, rng=Rng.Saru)
        u.runSimulationOnGPU(1)
        t0 = time.perf_counter()
        u.runSimulationOnGPU(mcs)
        wall += time.perf_counter() - t0
        moves += systems_[i].n * mcs
        u.cleanup()
    return moves / wall if wall else None


# ------------------------------------------------------------- driver
def run(n_systems: int = 4096, mcs: int = 20000, every: int = 200, test_fraction: float = 0.25, epochs: int = 300,
        seed: int = 1, gpu: int = 0, save: str | None = None):
    """record an ensemble with the batched simulator, train the network on
    part of it, and compare the learned schedule with the plain fixed budget
    on the rest, at equal mean R_e^2 error; returns a report dict"""
    import time
    params = ensemble_params(n_systems, seed)
    t0 = time.perf_counter()
    series, sys_, rate = record(params, mcs, every, seed=seed, gpu=gpu)
    t_rec = time.perf_counter() - t0
    x, y = dataset(params, series)
    if save:
        np.savez_compressed(save, x=x, y=y, t=series[0]["t"], re2=np.stack([s["re2"] for s in series]),
                            rg2=np.stack([s["rg2"] for s in series]), n=np.array([s["n"] for s in series]),
                            rate=np.array([rate]))
    rng = np.random.default_rng(seed)
    idx = rng.permutation(n_systems)
    n_te = max(1, int(n_systems * test_fraction))
    te, tr = idx[:n_te], idx[n_te:]
    # a fifth of the training systems is held out to calibrate the budget
    # factor on predictions the network did not fit
    n_cal = max(1, len(tr) // 5)
    cal, fit = tr[:n_cal], tr[n_cal:]
    model = Surrogate(seed=seed, gpu=gpu)
    t0 = time.perf_counter()
    hist = model.fit(x[fit], y[fit], epochs=epochs)
    t_fit = time.perf_counter() - t0
    pred = model.predict(x[te])
    rmse = np.sqrt(((pred - y[te]) ** 2).mean(0))
    rmse_const = np.sqrt(((y[fit].mean(0) - y[te]) ** 2).mean(0))
    # systems whose fitted relaxation time exceeds a twelfth of the recorded
    # window cannot be assessed by it (neither schedule equilibrates them in
    # the record); they are left out of the schedule comparison
    assessable = y[:, 0] <= math.log10(mcs / 12.0)
    if assessable[te].any() and assessable[cal].any():
        te, cal_j = te[assessable[te]], cal[assessable[cal]]
    else:
        cal_j = cal
    pred = model.predict(x[te])
    test_series = [series[i] for i in te]
    # the budget factor is calibrated on the held-out training systems: of the
    # factors whose ensemble R_e^2 / N stays within 1% of the value of
    # full-length runs, the one with the largest gain over the cheapest fixed
    # budget of equal bias
    train_series = [series[i] for i in cal_j]
    pred_tr = model.predict(x[cal_j])
    # budgets scale with the predicted end-to-end autocorrelation time, the
    # target the network predicts best
    factor, calib = 8.0, {}
    for f in (2.0, 3.0, 4.0, 6.0, 8.0, 12.0, 16.0):
        c = compare(train_series, learned_budgets(pred_tr[:, 3], train_series, factor=f))
        calib[f] = {"bias": c["learned"]["bias_re2"], "ratio": c["systems_per_hour_ratio"],
                    "ensemble_re2_vs_full": c["ensemble_re2_per_n_learned_vs_full_window"],
                    "ratio_vs_full": c["systems_per_hour_ratio_vs_full_window"]}
    ok = [f for f in calib if abs(calib[f]["ensemble_re2_vs_full"]) <= 0.01]
    if ok:
        factor = max(ok, key=lambda f: calib[f]["ratio"])
    budgets = learned_budgets(pred[:, 3], test_series, factor=factor)
    cmp = compare(test_series, budgets)
    # the same schedule fed the constant (training-mean) prediction: what the network adds
    const_budgets = learned_budgets(np.full(len(te), y[fit, 3].mean()), test_series, factor=factor)
    cmp_const = compare(test_series, const_budgets)
    per_hour = lambda cost: len(te) / (cost / rate) * 3600.0
    order = admission_order(pred[:, 3], [series[i]["n"] for i in te])
    return {
        "systems": n_systems, "test_systems": int(n_te), "test_systems_assessed": int(len(te)), "recorded_mcs": mcs, "snapshot_every": every,
        "ensemble": "boxes 16/24/32, linear chains or 3-arm stars of 8..48 backbone monomers, half of them combs (a side "
                    "chain of 2..4 on every 4th or 8th backbone monomer), volume fraction 0.1..0.5, Saru",
        "batch_rate_moves_per_s": rate, "record_s": t_rec, "fit_s": t_fit,
        "train_loss_first_last": [hist[0], hist[-1]],
        "test_rmse": dict(zip(TARGETS, map(float, rmse))),
        "test_rmse_constant_predictor": dict(zip(TARGETS, map(float, rmse_const))),
        "schedule": cmp, "budget_factor": factor, "calibration_on_held_out_training_systems": {str(k): v for k, v in calib.items()},
        "systems_per_hour": {"learned": per_hour(cmp["learned"]["cost_moves"]), "plain": per_hour(cmp["plain"]["cost_moves"])},
        "schedule_without_network": {"cost_moves": cmp_const["learned"]["cost_moves"],
                                     "mean_rel_err_re2": cmp_const["learned"]["mean_rel_err_re2"],
                                     "bias_re2": cmp_const["learned"]["bias_re2"],
                                     "ratio_vs_plain": cmp_const["systems_per_hour_ratio"]},
        "admission_order_head": [int(te[i]) for i in order[:8]],
    }


def main(argv=None):
    import argparse
    import json
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--systems", type=int, default=4096)
    ap.add_argument("--mcs", type=int, default=200000)
    ap.add_argument("--every", type=int, default=1000)
    ap.add_argument("--epochs", type=int, default=300)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--out", default=None)
    ap.add_argument("--save", default=None, help="npz with the features, labels and recorded series")
    a = ap.parse_args(argv)
    rep = run(a.systems, a.mcs, a.every, epochs=a.epochs, seed=a.seed, save=a.save)
    s = json.dumps(rep)
    print(s, flush=True)
    if a.out:
        with open(a.out, "w") as fh:
            fh.write(s + "\n")


if __name__ == "__main__":
    main()
