#!/usr/bin/env python
"""Throughput of the colored BFM sweep: attempted moves per second on one B200.

Workloads (--config):
  c2 (default)  dense linear melt, 4096 chains x N=256 (1,048,576 monomers) on
                a 256^3 periodic lattice, volume fraction 0.5, two colours,
                Saru RNG; the start is a serpentine crystal melted by the sweep
                itself before warm-up.  A step is 1000 MCS.
  c1            dilute linear chains, 128 self-avoiding walks x N=64 (8,192
                monomers) on a 128^3 periodic lattice, Saru RNG.  A step is
                1000 MCS (10 steps = the 10,000 MCS run).
  c3            dense melt of 3-arm star-combs (arm 64, a 16-monomer side
                chain on every 8th backbone monomer), 115,600 stars x 577 =
                66,701,200 monomers on a 1024^3 periodic lattice, volume
                fraction 0.497, Saru RNG.  A step is 100 MCS.

  value  attempted moves/s from CUDA events around each step's kernels on the
         library stream, state resident in HBM (L2 flushed before each step)
  e2e    the same through the public C ABI with host buffers: each step is
         runSimulationOnGPU (host-drawn colour/seed schedule copied H2D from
         pinned memory) plus the read-back of all positions (D2H)

Multi-GPU (torchrun): independent replicas, one system per rank, no
collective on the data path ("weak" scaling); times are the max over ranks.

--impl reference runs the reference's own UpdaterGPUScBFM_AB_Type (built for
sm_100a from its sources into oracle/_ref/) on the same workload, from the
same R250 state, through its own API: value from CUDA events around its
runSimulationOnGPU, e2e on the host clock including its position getters.
Without that library it times the CPU oracle port on all host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import numpy as np  # noqa: E402

WORKLOAD = ("dense linear melt: 4096 chains x N=256 (1,048,576 monomers), 256^3 periodic lattice, "
            "volume fraction 0.5, 108-vector bond set, 2 colours, Saru RNG")
METRIC = "attempted moves/s on 1 B200; batched+surrogate vs plain at equal R_e² error"
UNIT = "attempted moves/s"

# per workload: generator, MCS per step, untimed melt, the reference
# instantiation (coordinate type) and where the state lives
CONFIGS = {
    "c1": {"mcs_per_step": 1000, "melt_mcs": 0, "ref_ctype": 0, "ref_type": "int32_t", "resident": "l2",
           "desc": "dilute linear chains: 128 chains x N=64 (8,192 monomers), self-avoiding walks from seed 12345, "
                   "128^3 periodic lattice, volume fraction 0.031, 108-vector bond set, Saru RNG"},
    "c2": {"mcs_per_step": 1000, "melt_mcs": 2000, "ref_ctype": 1, "ref_type": "uint8_t", "resident": "l2",
           "desc": WORKLOAD},
    "c3": {"mcs_per_step": 100, "melt_mcs": 200, "ref_ctype": None, "ref_type": None, "resident": "hbm",
           "desc": "dense star-comb melt: 115,600 3-arm stars (arm 64, side chain of 16 on every 8th backbone "
                   "monomer) x 577 = 66,701,200 monomers, 1024^3 periodic lattice, volume fraction 0.497, "
                   "108-vector bond set, Saru RNG"},
}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--config", default="c2", choices=sorted(CONFIGS),
                   help="c2: the 256^3 linear melt (default); c1: 128 chains x 64 on 128^3; c3: the 1024^3 star-comb melt")
    p.add_argument("--mcs-per-step", type=int, default=None, help="default: 1000 (c1, c2), 100 (c3)")
    p.add_argument("--melt-mcs", type=int, default=None, help="untimed MCS before warm-up (default per config)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--cpu-seconds", type=float, default=12.0)
    p.add_argument("--box", type=int, default=None,
                   help="c2: edge of the cubic linear melt (256: the 4096 x 256 benchmark melt; 512, 1024: the same "
                        "density with chains of L monomers, states beyond L2); c3: edge of the star-comb melt "
                        "(1024: the benchmark; 256, 512: the same construction in a smaller box)")
    p.add_argument("--sweep-shape", type=int, default=-1,
                   help="persistent-kernel shape (-1 automatic; see bfm_set_sweep_shape)")
    p.add_argument("--batch", type=int, default=0,
                   help="time a batched ensemble of this many systems instead (box edges 32..128, chains or "
                        "3-arm stars of 16..512 monomers, volume fraction 0.1..0.5), against the same systems "
                        "run one after another through the single-system updater")
    p.add_argument("--plain-sample", type=int, default=48,
                   help="systems of the ensemble timed one by one for the plain comparison")
    p.add_argument("--schedule", type=int, default=0,
                   help="run the learned schedule live against plain fixed budgets on an ensemble of this many "
                        "systems (batched-ensemble ranges), recorded for --schedule-mcs MCS")
    p.add_argument("--schedule-mcs", type=int, default=100000)
    p.add_argument("--schedule-every", type=int, default=500)
    p.add_argument("--schedule-solo-tail", type=int, default=0,
                   help="systems left in the batch at which power-of-two ones move to the single-system updater")
    p.add_argument("--schedule-clusters", type=int, default=4,
                   help="CTAs per cluster for the large systems in the schedule's batched runs")
    p.add_argument("--schedule-solo-tail-alt", default="",
                   help="comma-separated other thresholds to time the learned schedule with as well")
    a = p.parse_args()
    cfg = CONFIGS[a.config]
    if a.mcs_per_step is None:
        a.mcs_per_step = cfg["mcs_per_step"]
    if a.melt_mcs is None:
        a.melt_mcs = cfg["melt_mcs"]
    if a.box is None:
        a.box = {"c1": 128, "c2": 256, "c3": 1024}[a.config]
    if a.config == "c1" and a.box != 128:
        p.error("c1 is the 128^3 system")
    return a


# ------------------------------------------------------------------ ranks
class Ranks:
    """One process per GPU (torchrun environment); NCCL on GPUs, gloo on CPU.
    Only the timing reductions cross ranks: every replica is independent."""

    def __init__(self, backend: str | None = None):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        self.device = None
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            if backend is None:
                backend = "nccl" if torch.cuda.is_available() else "gloo"
            kw = {}
            if backend == "nccl":
                torch.cuda.set_device(self.local)
                self.device = torch.device("cuda", self.local)
                kw["device_id"] = self.device
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120), **kw)
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, v: float) -> float:
        if not self.pg:
            return v
        import torch
        t = torch.tensor([v], dtype=torch.float64, device=self.device or "cpu")
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


def aggregate(ranks, attempts: int, dev_s: float, e2e_s: float):
    """Whole-job throughput of independent replicas: the attempts of all
    ranks over the slowest rank's time (device-timed and end-to-end)."""
    dev = ranks.max(dev_s)
    e2e = ranks.max(e2e_s)
    total = attempts * ranks.world
    return total / dev, total / e2e, total


# ------------------------------------------------------------------ clocks
class Clocks:
    """nvidia-smi sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        hi = max(sm)
        loaded = [v for v in sm if v >= 0.5 * hi] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def flush_l2(buf):
    """Write a buffer larger than the 126 MB L2 (torch, current stream)."""
    import torch
    buf.zero_()
    torch.cuda.synchronize()


def peaks():
    path = os.path.join(HERE, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# --------------------------------------------------------------- workload
def make_workload(config: str = "c2", box: int = 256):
    from pscbfm_b200 import systems
    if config == "c1":
        return systems.saw_chains(128, 64, box=(128, 128, 128), seed=12345)
    if config == "c3":
        return systems.star_comb_melt(box)
    return systems.ordered_melt(box)


def workload_name(config: str, box: int, system) -> str:
    if config == "c3" and box != 1024:
        stars = system.n // 577
        return (f"dense star-comb melt: {stars:,} 3-arm stars (arm 64, side chain of 16 on every 8th backbone monomer) "
                f"x 577 = {system.n:,} monomers, {box}^3 periodic lattice, volume fraction {8 * system.n / box ** 3:.3f}, "
                f"108-vector bond set, Saru RNG")
    if config != "c2" or box == 256:
        return CONFIGS[config]["desc"]
    chains = len(system.chains)
    return (f"dense linear melt: {chains} chains x N={system.n // chains} ({system.n:,} monomers), {box}^3 periodic "
            f"lattice, volume fraction 0.5, 108-vector bond set, 2 colours, Saru RNG")


def workload_tag(config: str, box: int) -> str:
    """file tag of the committed ncu summaries for this workload"""
    return {"c1": "c1_128", "c3": f"starcomb{box}"}.get(config, f"melt{box}")


def algorithmic_bytes(c: float, a: float, kbar: float, C: int = 4):
    """Bytes per attempted move of the check and perform kernels: own
    coordinate C (4 B up to 256 per axis, 8 B beyond, the reference's
    coordinate record), bond count 1, per bond a 4-byte id and an 8-byte
    coordinate gather, nine 4-byte lattice probes, the target bit for
    candidates (c); perform: nine probes of the target lattice for
    candidates, coordinate write and two lattice bit updates for accepted
    moves (a)."""
    check = C + 1 + 12 * kbar + 36 + 4 * c
    perform = 36 * c + C * a + 8 * a
    return check, perform


def cpu_baseline(system, pos_now, seconds: float, what: str = "256^3 melt"):
    """The oracle (CPU restatement of the colored sweep, OpenMP over the
    monomers of a colour) on a bounded sample: as many MCS of the same melt
    as fit in about `seconds` of host time, on all host cores; plus the
    serial random-sequential BFM on one core."""
    from oracle import oracle
    from pscbfm_b200.systems import System
    s = System(system.box, pos_now.copy(), system.deg, system.nbr, system.allowed, system.chains)
    cores = os.cpu_count() or 1
    sw = oracle.Sweep(s, rng=2, age=0, sort_every=5000, threads=cores)
    st = oracle.r250_state(5)
    t = time.perf_counter()
    sw.run(1, st)
    one = max(time.perf_counter() - t, 1e-3)
    m = max(1, min(200, int(seconds / one)))
    t = time.perf_counter()
    sw.run(m, st)
    dt = time.perf_counter() - t
    colored = s.n * m / dt
    pos = pos_now.copy()
    t = time.perf_counter()
    oracle.serial_run(s, pos, 1, seed=3)
    dts = time.perf_counter() - t
    serial = s.n / dts
    return {"value": colored, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{m} MCS of the same {what} ({s.n * m:.3g} attempted moves), colored two-phase "
                      f"algorithm, OpenMP over the monomers of a colour",
            "serial_1core": {"value": serial, "unit": UNIT, "cores": 1,
                             "sample": f"1 MCS random-sequential Metropolis BFM on the same {what}"}}


# ------------------------------------------------------------------- arms
def run_b200(args, ranks):
    import torch

    import pscbfm_b200 as pb
    gpu = ranks.local
    torch.cuda.set_device(gpu)
    cfg = CONFIGS[args.config]
    system = make_workload(args.config, args.box)
    pb.r250_seed(1000 + ranks.rank)
    u = pb.UpdaterGPUScBFM_AB_Type().setup(system, gpu=gpu, rng=pb.Rng.Saru)
    if args.sweep_shape != -1:
        u.setSweepShape(args.sweep_shape)
    else:
        # the launch-shape autotuner times the candidate shapes on the first
        # chunk of the untimed melt (or warm-up) and keeps the fastest
        u.setSweepAutotune(True)
    S = args.mcs_per_step
    if args.melt_mcs:
        u.runSimulationOnGPU(args.melt_mcs)    # melt the ordered start (untimed)
    flushbuf = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{gpu}")
    # the caller's page-locked position buffer, filled by one device-to-host copy per step
    pinned = torch.empty((system.n, 3), dtype=torch.int32, pin_memory=True)
    hostpos = pinned.numpy()
    for _ in range(args.warmup):
        flush_l2(flushbuf)
        u.runSimulationOnGPU(S)
        u.getAllMonomerPositions(out=hostpos)
    launch_info = u.getLaunchInfo()
    tuning = u.getSweepTuning()

    # live timing of every sweep-kernel launch for the roofline (same path)
    a0, c0, s0 = u.getCounters()
    kmcs = min(S, 2048)
    k_ms, k_launches, k_attempts = u.timeKernels(kmcs)
    a1, c1, s1 = u.getCounters()
    cand = (c1 - c0) / max(a1 - a0, 1)
    acc = (s1 - s0) / max(a1 - a0, 1)

    clocks = Clocks(gpu)
    torch.cuda.synchronize()
    ranks.barrier()
    torch.cuda.synchronize()
    clocks.start()
    t_begin = time.perf_counter()
    dev_ms, e2e_s, launches = 0.0, 0.0, 0
    step_ms = []
    acnt0 = u.getCounters()
    for _ in range(args.steps):
        flush_l2(flushbuf)
        t0 = time.perf_counter()
        u.runSimulationOnGPU(S)
        pos = u.getAllMonomerPositions(out=hostpos)
        e2e_s += time.perf_counter() - t0
        ms = u.getLastRunMs()
        dev_ms += ms
        step_ms.append(ms)
        launches += u.getLastRunLaunches() + 1    # + the read-back unpack kernel
    torch.cuda.synchronize()
    ranks.barrier()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t_begin
    clk = clocks.stop()
    acnt1 = u.getCounters()

    attempts = acnt1[0] - acnt0[0]
    value, e2e, total_attempts = aggregate(ranks, attempts, dev_ms / 1e3, e2e_s)

    kbar = float(system.deg.mean())
    coord_bytes = 4 if max(system.box) <= 256 else 8
    b_check, b_perf = algorithmic_bytes(cand, acc, kbar, coord_bytes)
    nspec = u.getNSpecies()
    hbm, hbm_kind = peaks()
    t_launch = k_ms / max(k_launches, 1) / 1e3
    bytes_launch = (b_check + b_perf) * k_attempts / max(k_launches, 1)
    achieved = bytes_launch / t_launch / 1e9
    traffic = None
    l2 = None
    kname = "k_sweep_w" if launch_info.get("mode", 0) >= 6 else "k_sweep"
    prof = os.path.join(HERE, "profiles", f"{kname}_{workload_tag(args.config, args.box)}_traffic.json")
    if os.path.exists(prof):
        try:
            # DRAM (and L2) bytes per attempted move from one ncu capture of a
            # shorter launch, scaled to this launch's attempted moves
            tr = json.load(open(prof))
            traffic = tr["dram_bytes_per_attempt"] * k_attempts / max(k_launches, 1)
            if "l2_bytes_per_attempt" in tr:
                l2 = {"lts_throughput_pct": tr.get("lts_throughput_pct"),
                      "l2_bytes_per_attempt": tr["l2_bytes_per_attempt"],
                      "algorithmic_bytes_per_attempt": b_check + b_perf,
                      "dram_bytes_per_attempt": tr["dram_bytes_per_attempt"],
                      "source": os.path.relpath(prof, HERE)}
        except Exception:
            traffic = None
    whole_bytes = (b_check + b_perf) * total_attempts / ranks.world
    resident = "l2" if max(system.box) <= 256 else "hbm"
    if resident == "l2":
        bound = "l2/latency"
        bound_note = ("the state is L2-resident: the algorithmic bytes are served by L2/L1, not DRAM; the kernel is "
                      "bound by integer issue, L2 round trips and two grid barriers per colour substep. frac is "
                      "against the measured HBM copy bandwidth, as the scope table's formula defines it")
    else:
        bound = "hbm"
        bound_note = "the state (GB) is beyond L2: monomer streams and lattice words come from DRAM"
    line = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": ranks.world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": dev_ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u32",
        "data": ("synthetic (seeded self-avoiding walks)" if args.config == "c1" else
                 "synthetic (ordered start of the stated shape, melted in place before warm-up)"),
        "config": {"workload": workload_name(args.config, args.box, system), "config": args.config, "mcs_per_step": S,
                   "monomers": system.n, "box": [int(b) for b in system.box],
                   "colours": nspec, "replicas": ranks.world,
                   "l2": ("flushed before every step (256 MiB write); the state is L2-resident within a step"
                          if resident == "l2" else
                          "flushed before every step (256 MiB write); the state is larger than L2"),
                   "launch": "one persistent cooperative kernel per chunk of up to 4096 colour substeps",
                   "kernel_shape": launch_info, "shape_tuning": tuning},
        "e2e": {"value": e2e, "unit": UNIT,
                "h2d_bytes_per_step": S * nspec * 16,
                "d2h_bytes_per_step": system.n * 12,
                "host_buffers": "schedule from the engine's page-locked ring; positions into the caller's "
                                "page-locked (n, 3) int32 array"},
        "gpu_launches": launches,
        "roofline": {"bound": bound, "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": traffic, "kernel": kname, "peak_source": f"{hbm_kind} hbm_gbs",
                     "note": bound_note, "l2": l2, "coord_bytes": coord_bytes,
                     "bytes_per_attempt": {"check": b_check, "perform": b_perf},
                     "attempts_per_launch": k_attempts / max(k_launches, 1),
                     "launch_ms": t_launch * 1e3, "launches_timed": k_launches,
                     "candidate_fraction": cand, "accept_fraction": acc,
                     "whole_step_gbs": whole_bytes / (dev_ms / 1e3) / 1e9},
        "clocks": clk,
        "wall_s": wall,
    }
    if ranks.rank == 0 and ranks.world == 1 and not args.no_cpu_baseline:
        what = {"c1": "128^3 dilute system", "c3": f"{args.box}^3 star-comb melt"}.get(args.config, f"{args.box}^3 melt")
        line["cpu_baseline"] = cpu_baseline(system, pos, args.cpu_seconds, what)
    if ranks.rank == 0:
        print(json.dumps(line), flush=True)


def run_batch(args, ranks):
    """Batched ensemble: every system advances args.mcs_per_step MCS per step
    in one bfm_batch_run (persistent kernel, one CTA per system).  The plain
    comparison runs a random sample of the same systems one after another
    through the single-system updater (its own persistent kernel per
    system), the way a plain ensemble would be run, and reports the
    aggregate rate of that sample."""
    import torch

    import pscbfm_b200 as pb
    from pscbfm_b200 import systems
    gpu = ranks.local
    torch.cuda.set_device(gpu)
    t = time.perf_counter()
    sys_, params = systems.ensemble(args.batch, seed=12345 + 1000 * ranks.rank)
    t_gen = time.perf_counter() - t
    b = pb.Batch(gpu)
    for i, s in enumerate(sys_):
        b.add(s, rng=pb.Rng.Saru, r250_seed=12345 + i)
    t = time.perf_counter()
    b.initialize()
    t_init = time.perf_counter() - t
    S = args.mcs_per_step
    b.set_autotune(True)          # the first warm-up launches time the cluster sizes
    for _ in range(args.warmup):
        b.run(S)
    tuning = b.clusters()
    clocks = Clocks(gpu)
    torch.cuda.synchronize()
    ranks.barrier()
    clocks.start()
    dev_ms, e2e_s, attempts, launches = 0.0, 0.0, 0, 0
    d2h = 0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        b.run(S)
        info = b.info()
        # read back one system per step (the observable a driver would look at)
        b.positions(_ % len(sys_))
        e2e_s += time.perf_counter() - t0
        dev_ms += info["last_ms"]
        attempts += info["last_attempts"]
        launches += info["last_launches"]
        d2h += sys_[_ % len(sys_)].n * 12
    torch.cuda.synchronize()
    ranks.barrier()
    clk = clocks.stop()
    value, e2e, total = aggregate(ranks, attempts, dev_ms / 1e3, e2e_s)

    # plain: a sample of the same systems one by one through the single-system updater
    rng = np.random.default_rng(7)
    pick = rng.choice(len(sys_), size=min(args.plain_sample, len(sys_)), replace=False)
    p_att, p_ms, p_wall, p_n = 0, 0.0, 0.0, 0
    for i in pick:
        s = sys_[i]
        if any(v & (v - 1) for v in s.box):
            continue      # the single-system updater, like the reference, takes powers of two only
        pb.r250_seed(12345 + int(i))
        u = pb.UpdaterGPUScBFM_AB_Type().setup(s, gpu=gpu, rng=pb.Rng.Saru)
        u.runSimulationOnGPU(1)
        t0 = time.perf_counter()
        u.runSimulationOnGPU(S)
        p_wall += time.perf_counter() - t0
        p_ms += u.getLastRunMs()
        p_att += s.n * S
        p_n += 1
        u.cleanup()
    plain = p_att / (p_ms / 1e3) if p_ms else None
    boxes = {}
    for prm in params:
        boxes[prm["L"]] = boxes.get(prm["L"], 0) + 1
    line = {
        "metric": "attempted moves/s, batched ensemble on 1 B200",
        "value": value, "unit": UNIT, "n_gpus": ranks.world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dev_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32", "data": "synthetic (seeded ensemble generator)",
        "config": {"workload": f"batched ensemble: {len(sys_)} systems, {total // max(1, args.steps * S) // ranks.world:,} "
                               f"monomers, box edges {dict(sorted(boxes.items()))}, chains or 3-arm stars of 16..512 "
                               f"monomers, volume fraction 0.1..0.5, Saru, 2 colours per system",
                   "mcs_per_step": S, "systems": len(sys_), "generate_s": t_gen, "initialize_s": t_init,
                   "clusters": tuning,
                   "l2": "ensemble state beyond L2 (lattices and monomer arrays of all systems)"},
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": len(sys_) * 16 + 4 * len(sys_),
                "d2h_bytes_per_step": d2h // max(1, args.steps)},
        "gpu_launches": launches,
        "plain": {"value": plain, "unit": UNIT, "systems_timed": p_n,
                  "wall_rate": p_att / p_wall if p_wall else None,
                  "how": "sampled systems of the same ensemble, each through the single-system updater in turn"},
        "speedup_vs_plain": (value / plain) if plain else None,
        "clocks": clk,
    }
    if ranks.rank == 0:
        print(json.dumps(line), flush=True)


def run_schedule(args, ranks):
    """The learned run schedule, live: systems equilibrated per hour on the
    wall clock, learned budgets (with admission order and the drift judge
    extending runs on the GPU) against the cheapest plain fixed budget of
    equal R_e^2 bias, batched and solo."""
    if ranks.rank != 0:
        return
    import torch

    from pscbfm_b200 import schedule as sch
    torch.cuda.set_device(ranks.local)
    clocks = Clocks(ranks.local)
    clocks.start()
    rep = sch.live_compare(args.schedule, args.schedule_mcs, args.schedule_every, gpu=ranks.local,
                           solo_tail=args.schedule_solo_tail, clusters=args.schedule_clusters,
                           solo_tail_alternatives=[int(v) for v in args.schedule_solo_tail_alt.split(",") if v])
    clk = clocks.stop()
    line = {"metric": "systems equilibrated per hour on 1 B200, learned schedule vs plain fixed budget at equal R_e^2 bias",
            "value": rep["systems_per_hour"]["learned"], "unit": "systems/hour", "n_gpus": 1, "higher_is_better": True,
            "vs_baseline": None, "dtype": "u32 (sweep), bf16/fp32 (network)", "data": "synthetic (seeded ensemble generator)",
            "config": {"workload": "learned schedule on batched ensembles", "systems": args.schedule,
                       "recorded_mcs": args.schedule_mcs, "snapshot_every": args.schedule_every},
            "ratio_learned_vs_plain": rep["ratio_learned_vs_plain"], "ratio_learned_vs_solo": rep["ratio_learned_vs_solo"],
            "report": rep, "clocks": clk}
    print(json.dumps(line), flush=True)


def run_reference(args, ranks):
    """The reference's own updater on the same workload, from the same R250
    state as the B200 arm (seed 1000 for rank 0), through its public API:
    set-up, an untimed melt, warm-up, then timed runSimulationOnGPU calls
    (value: CUDA events on the legacy stream around each call, which waits
    for the updater's own stream; e2e: host clock around the call and the
    read-back through its per-index position getters)."""
    if ranks.rank != 0:
        return
    cfg = CONFIGS[args.config]
    if cfg["ref_ctype"] is None or args.box > 256:
        print(json.dumps({"impl": "reference", "unavailable": "the reference's device coordinates take boxes of at "
                                                               "most 256 per axis (UpdaterGPUScBFM_AB_Type.cu:2468-2478)"}),
              flush=True)
        return
    from oracle import oracle
    system = make_workload(args.config, args.box)
    S = args.mcs_per_step
    config = {"workload": workload_name(args.config, args.box, system), "config": args.config, "mcs_per_step": S,
              "monomers": system.n, "box": [int(b) for b in system.box], "colours": None, "replicas": 1,
              "l2": ("flushed before every step (256 MiB write); the state is L2-resident within a step"
                     if cfg["resident"] == "l2" else "flushed before every step (256 MiB write)"),
              "launch": f"the reference's UpdaterGPUScBFM_AB_Type<{cfg['ref_type']}>: check, perform and clear "
                        f"kernels per colour substep, launched from the host"}
    if oracle.ref_gpu() is not None:
        import torch
        ref = oracle.RefUpdater(system, rng=2, age=0, sort_every=5000, ctype=cfg["ref_ctype"], gpu=ranks.local)
        st = oracle.r250_state(1000)
        if args.melt_mcs:
            ref.run(args.melt_mcs, st)
        flushbuf = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{ranks.local}")
        for _ in range(args.warmup):
            flush_l2(flushbuf)
            ref.run(S, st)
            ref.positions()
        config["colours"] = int(oracle.graph_coloring(system.deg, system.nbr)[0])
        clocks = Clocks(ranks.local)
        torch.cuda.synchronize()
        clocks.start()
        dev_ms, tot = 0.0, 0.0
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        for _ in range(args.steps):
            flush_l2(flushbuf)
            t0 = time.perf_counter()
            e0.record()
            ref.run(S, st)            # synchronous, ends with its own copy-back
            e1.record()
            ref.positions()
            tot += time.perf_counter() - t0
            e1.synchronize()
            dev_ms += e0.elapsed_time(e1)
        clk = clocks.stop()
        value = system.n * S * args.steps / (dev_ms / 1e3)
        e2e = system.n * S * args.steps / tot
        desc = {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                "sample": f"{args.steps} x {S} MCS of the same workload through the reference's "
                          f"UpdaterGPUScBFM_AB_Type<{cfg['ref_type']}> (its own CUDA kernels, built for sm_100a), "
                          f"one host thread driving the B200"}
        d2h = system.n * 16           # doCopyBack: mPolymerSystem->pop(), int4 per monomer (.cu:3468-3471)
        ms_per_step = dev_ms / args.steps
        del ref                       # its destructor logs to stdout: before the JSON line, not after
        import gc
        gc.collect()
    else:
        clk = None
        what = {"c1": "128^3 dilute system"}.get(args.config, "256^3 melt")
        c = cpu_baseline(system, system.pos, args.cpu_seconds, what)
        value = e2e = c["value"]
        desc = {k: c[k] for k in ("value", "unit", "cores", "kind", "sample")}
        d2h = 0
        ms_per_step = None
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": ("synthetic (seeded self-avoiding walks)" if args.config == "c1" else
                     "synthetic (ordered start of the stated shape, melted in place before warm-up)"),
            "config": config, "cpu_baseline": desc,
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": d2h},
            "clocks": clk}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    ranks = Ranks()
    try:
        if args.impl == "reference":
            run_reference(args, ranks)
        elif args.schedule:
            run_schedule(args, ranks)
        elif args.batch:
            run_batch(args, ranks)
        else:
            run_b200(args, ranks)
    finally:
        ranks.close()


if __name__ == "__main__":
    main()
