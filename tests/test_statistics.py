"""Statistics: the colored two-phase sweep and a serial random-sequential BFM
sample the same physics.  R_e^2, R_g^2 and the middle-monomer MSD g1 of the
colored algorithm must agree within 2 sigma with the serial updater
(LeMonADE's serial updater is not in the reference tree; the oracle's serial
Metropolis BFM stands in for it).

Sigma is the standard error of the difference of the two means, estimated
from per-chain time averages (chains are independent samples)."""
import numpy as np
import pytest

import pscbfm_b200 as pb
from oracle import oracle
from pscbfm_b200 import analysis, systems


def _collect(step, pos0, chains, n_eq, n_blocks, block):
    """run n_eq, then n_blocks blocks of `block` MCS; per-chain means of
    R_e^2, R_g^2 and g1 over block lags"""
    pos = step(pos0, n_eq)
    re2, rg2, g1 = [], [], []
    c_prev = analysis.centres(pos, chains)
    for _ in range(n_blocks):
        pos = step(pos, block)
        a, b = analysis.re2_rg2_per_chain(pos, chains)
        re2.append(a)
        rg2.append(b)
        c_now = analysis.centres(pos, chains)
        g1.append(analysis.msd(c_prev, c_now, len(chains))["g1"])
        c_prev = c_now
    return np.mean(re2, axis=0), np.mean(rg2, axis=0), np.mean(g1, axis=0)


def _within(a, b, k=2.0):
    n = a.size
    se = np.sqrt(a.var(ddof=1) / n + b.var(ddof=1) / b.size)
    return abs(a.mean() - b.mean()) <= k * se, a.mean(), b.mean(), se


def _serial_stepper(sysm, seed):
    state = {"seed": seed}

    def step(pos, nmcs):
        p = np.ascontiguousarray(pos, dtype=np.int32).copy()
        oracle.serial_run(sysm, p, nmcs, seed=state["seed"])
        state["seed"] += 1
        return p
    return step


@pytest.mark.gpu
def test_cuda_sweep_statistics_match_serial_bfm():
    s = systems.saw_chains(64, 16, box=(64, 64, 64), seed=101)
    pb.r250_seed(55)
    u = pb.UpdaterGPUScBFM_AB_Type().setup(s, rng=pb.Rng.Saru)

    def gpu_step(pos, nmcs):
        u.runSimulationOnGPU(nmcs)
        return u.getAllMonomerPositions()

    col = _collect(gpu_step, s.pos, s.chains, 3000, 40, 400)
    ser = _collect(_serial_stepper(s, 7), s.pos, s.chains, 3000, 40, 400)
    for name, a, b in zip(("R_e^2", "R_g^2", "g1(400 MCS)"), col, ser):
        ok, ma, mb, se = _within(a, b)
        assert ok, f"{name}: colored {ma:.3f} vs serial {mb:.3f}, 2 sigma = {2 * se:.3f}"


@pytest.mark.gpu
def test_c1_statistics_match_serial_bfm():
    """Configuration C1 itself (128 self-avoiding chains x 64 on 128^3):
    after 10,000 MCS of equilibration, 20 blocks of 1000 MCS."""
    s = systems.saw_chains(128, 64, box=(128, 128, 128), seed=12345)
    pb.r250_seed(56)
    u = pb.UpdaterGPUScBFM_AB_Type().setup(s, rng=pb.Rng.Saru)

    def gpu_step(pos, nmcs):
        u.runSimulationOnGPU(nmcs)
        return u.getAllMonomerPositions()

    col = _collect(gpu_step, s.pos, s.chains, 10000, 20, 1000)
    ser = _collect(_serial_stepper(s, 8), s.pos, s.chains, 10000, 20, 1000)
    for name, a, b in zip(("R_e^2", "R_g^2", "g1(1000 MCS)"), col, ser):
        ok, ma, mb, se = _within(a, b)
        assert ok, f"{name}: colored {ma:.3f} vs serial {mb:.3f}, 2 sigma = {2 * se:.3f}"


def test_oracle_colored_statistics_match_serial_bfm():
    """The same check for the CPU restatement of the colored algorithm, on
    a smaller system (runs without a GPU)."""
    s = systems.saw_chains(48, 12, box=(64, 64, 64), seed=202)
    sw = oracle.Sweep(s, rng=2, sort_every=5000, threads=4)
    st = oracle.r250_state(9)

    def col_step(pos, nmcs):
        sw.run(nmcs, st)
        return sw.positions()

    col = _collect(col_step, s.pos, s.chains, 1500, 30, 300)
    ser = _collect(_serial_stepper(s, 11), s.pos, s.chains, 1500, 30, 300)
    for name, a, b in zip(("R_e^2", "R_g^2", "g1(300 MCS)"), col, ser):
        ok, ma, mb, se = _within(a, b)
        assert ok, f"{name}: colored {ma:.3f} vs serial {mb:.3f}, 2 sigma = {2 * se:.3f}"
