#!/usr/bin/env python
"""Throughput of the colored BFM sweep: attempted moves per second on one B200.

Workload: dense linear melt, 4096 chains x N=256 (1,048,576 monomers) on a
256^3 periodic lattice, volume fraction 0.5, standard 108-vector bond set,
two colours (bipartite chains), Saru RNG.  The start is a serpentine crystal
melted by the sweep itself before warm-up.  A "step" is --mcs-per-step
Monte-Carlo steps (default 1000; 100 steps = the 100,000 MCS run).

  value  attempted moves/s from CUDA events around each step's kernels on the
         library stream, state resident in HBM (L2 flushed before each step)
  e2e    the same through the public C ABI with host buffers: each step is
         runSimulationOnGPU (host-drawn colour/seed schedule copied H2D from
         pinned memory) plus the read-back of all positions (D2H)

Multi-GPU (torchrun): independent replicas, one system per rank, no
collective on the data path ("weak" scaling); times are the max over ranks.

--impl reference runs the reference's own UpdaterGPUScBFM_AB_Type (built for
sm_100a from its sources into oracle/_ref/) on the same workload through its
own API; without that library it times the CPU oracle port on all host cores.
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


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--mcs-per-step", type=int, default=1000)
    p.add_argument("--melt-mcs", type=int, default=2000)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--cpu-seconds", type=float, default=12.0)
    p.add_argument("--box", type=int, default=256,
                   help="edge of the cubic melt (256: the 4096 x 256 benchmark melt; 512, 1024: the same density "
                        "with chains of L monomers, states beyond L2)")
    p.add_argument("--sweep-shape", type=int, default=-1,
                   help="persistent-kernel shape (-1 automatic; see bfm_set_sweep_shape)")
    p.add_argument("--batch", type=int, default=0,
                   help="time a batched ensemble of this many systems instead (box edges 32..128, chains or "
                        "3-arm stars of 16..512 monomers, volume fraction 0.1..0.5), against the same systems "
                        "run one after another through the single-system updater")
    p.add_argument("--plain-sample", type=int, default=48,
                   help="systems of the ensemble timed one by one for the plain comparison")
    return p.parse_args()


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
def make_workload(box: int = 256):
    from pscbfm_b200 import systems
    return systems.ordered_melt(box)


def workload_name(box: int, system) -> str:
    if box == 256:
        return WORKLOAD
    chains = len(system.chains)
    return (f"dense linear melt: {chains} chains x N={system.n // chains} ({system.n:,} monomers), {box}^3 periodic "
            f"lattice, volume fraction 0.5, 108-vector bond set, 2 colours, Saru RNG")


def algorithmic_bytes(c: float, a: float, kbar: float, C: int = 4):
    """Bytes per attempted move of the check and perform kernels: own
    coordinate C, bond count 1, per bond a 4-byte id and an 8-byte coordinate
    gather, nine 4-byte lattice probes, the target bit for candidates (c);
    perform: nine probes of the target lattice for candidates, coordinate
    write and two lattice bit updates for accepted moves (a)."""
    check = C + 1 + 12 * kbar + 36 + 4 * c
    perform = 36 * c + C * a + 8 * a
    return check, perform


def cpu_baseline(system, pos_now, seconds: float):
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
            "sample": f"{m} MCS of the same 256^3 melt ({s.n * m:.3g} attempted moves), colored two-phase "
                      f"algorithm, OpenMP over the monomers of a colour",
            "serial_1core": {"value": serial, "unit": UNIT, "cores": 1,
                             "sample": "1 MCS random-sequential Metropolis BFM on the same melt"}}


# ------------------------------------------------------------------- arms
def run_b200(args, ranks):
    import torch

    import pscbfm_b200 as pb
    gpu = ranks.local
    torch.cuda.set_device(gpu)
    system = make_workload(args.box)
    pb.r250_seed(1000 + ranks.rank)
    u = pb.UpdaterGPUScBFM_AB_Type().setup(system, gpu=gpu, rng=pb.Rng.Saru)
    if args.sweep_shape != -1:
        u.setSweepShape(args.sweep_shape)
    S = args.mcs_per_step
    u.runSimulationOnGPU(args.melt_mcs)        # melt the serpentine crystal (untimed)
    launch_info = u.getLaunchInfo()
    flushbuf = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{gpu}")
    for _ in range(args.warmup):
        flush_l2(flushbuf)
        u.runSimulationOnGPU(S)
        u.getAllMonomerPositions()

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
        pos = u.getAllMonomerPositions()
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
    b_check, b_perf = algorithmic_bytes(cand, acc, kbar)
    nspec = u.getNSpecies()
    hbm, hbm_kind = peaks()
    t_launch = k_ms / max(k_launches, 1) / 1e3
    bytes_launch = (b_check + b_perf) * k_attempts / max(k_launches, 1)
    achieved = bytes_launch / t_launch / 1e9
    traffic = None
    kname = "k_sweep_w" if launch_info.get("mode", 0) >= 6 else "k_sweep"
    prof = os.path.join(HERE, "profiles", f"{kname}_melt{args.box}_traffic.json")
    if os.path.exists(prof):
        try:
            # DRAM bytes per attempted move from one ncu capture of a shorter
            # launch, scaled to this launch's attempted moves
            traffic = json.load(open(prof))["dram_bytes_per_attempt"] * k_attempts / max(k_launches, 1)
        except Exception:
            traffic = None
    whole_bytes = (b_check + b_perf) * total_attempts / ranks.world
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
        "data": "synthetic (seeded serpentine melt of the stated shape, melted in place before warm-up)",
        "config": {"workload": workload_name(args.box, system), "mcs_per_step": S, "monomers": system.n, "box": list(system.box),
                   "colours": nspec, "replicas": ranks.world,
                   "l2": "flushed before every step (256 MiB write); the 19 MiB state is L2-resident within a step",
                   "launch": "one persistent cooperative kernel per chunk of up to 4096 colour substeps",
                   "kernel_shape": launch_info},
        "e2e": {"value": e2e, "unit": UNIT,
                "h2d_bytes_per_step": S * nspec * 16,
                "d2h_bytes_per_step": system.n * 12},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": traffic, "kernel": kname, "peak_source": f"{hbm_kind} hbm_gbs",
                     "bytes_per_attempt": {"check": b_check, "perform": b_perf},
                     "attempts_per_launch": k_attempts / max(k_launches, 1),
                     "launch_ms": t_launch * 1e3, "launches_timed": k_launches,
                     "candidate_fraction": cand, "accept_fraction": acc,
                     "whole_step_gbs": whole_bytes / (dev_ms / 1e3) / 1e9},
        "clocks": clk,
        "wall_s": wall,
    }
    if ranks.rank == 0 and ranks.world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(system, pos, args.cpu_seconds)
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


def run_reference(args, ranks):
    if ranks.rank != 0:
        return
    if args.box != 256:
        print(json.dumps({"impl": "reference", "unavailable": "the reference's 8-bit device coordinates take boxes of "
                                                               "at most 256 per axis"}), flush=True)
        return
    from oracle import oracle
    system = make_workload()
    S = args.mcs_per_step
    if oracle.ref_gpu() is not None:
        import torch
        ref = oracle.RefUpdater(system, rng=2, age=0, sort_every=5000, ctype=1, gpu=ranks.local)
        st = oracle.r250_state(7)
        ref.run(args.melt_mcs, st)
        flushbuf = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{ranks.local}")
        for _ in range(args.warmup):
            flush_l2(flushbuf)
            ref.run(S, st)
            ref.positions()
        clocks = Clocks(ranks.local)
        torch.cuda.synchronize()
        clocks.start()
        tot = 0.0
        for _ in range(args.steps):
            flush_l2(flushbuf)
            t0 = time.perf_counter()
            ref.run(S, st)            # synchronous, ends with its own copy-back
            ref.positions()
            tot += time.perf_counter() - t0
        clk = clocks.stop()
        value = system.n * S * args.steps / tot
        desc = {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                "sample": f"{args.steps} x {S} MCS of the same melt through the reference's "
                          f"UpdaterGPUScBFM_AB_Type<uint8_t> (its own CUDA kernels, built for sm_100a), "
                          f"one host thread driving the B200"}
    else:
        clk = None
        c = cpu_baseline(system, system.pos, args.cpu_seconds)
        value = c["value"]
        desc = {k: c[k] for k in ("value", "unit", "cores", "kind", "sample")}
        tot = None
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": (tot / args.steps * 1e3) if tot else None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic", "config": {"workload": WORKLOAD, "mcs_per_step": S},
            "cpu_baseline": desc,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "clocks": clk}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    ranks = Ranks()
    try:
        if args.impl == "reference":
            run_reference(args, ranks)
        elif args.batch:
            run_batch(args, ranks)
        else:
            run_b200(args, ranks)
    finally:
        ranks.close()


if __name__ == "__main__":
    main()
