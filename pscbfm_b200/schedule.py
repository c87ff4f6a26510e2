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
