"""ctypes bindings of the oracle libraries (test infrastructure only).

``liboracle.so``           CPU restatement of the reference's colored sweep
``_ref/libref_host.so``    the reference's own Saru/Hash/graph colouring
``_ref/libref_pscbfm.so``  the reference's own GPU updater built for sm_100a
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_HOST_SO = os.path.join(HERE, "_ref", "libref_host.so")
REF_GPU_SO = os.path.join(HERE, "_ref", "libref_pscbfm.so")
# the reference checkout: $PSCBFM_REFERENCE, else a sibling of the repository
REF_ROOT = os.environ.get("PSCBFM_REFERENCE", os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))
REF_SRC = os.path.join(REF_ROOT, "src", "pscbfm")

_c = ctypes
_P = _c.c_void_p


def build(reference: bool | None = None) -> None:
    """Build liboracle.so; also the reference libraries when the reference
    sources are present (this container) and they are missing or stale."""
    subprocess.run(["make", "-s", "liboracle.so"], cwd=HERE, check=True)
    if reference is None:
        reference = os.path.isdir(REF_SRC)
    if reference:
        subprocess.run(["make", "-s", "ref", f"REF_SRC={REF_SRC}"], cwd=HERE, check=True)


_orc = None


def orc() -> ctypes.CDLL:
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_SO):
            build(reference=False)
        L = ctypes.CDLL(ORACLE_SO)
        L.orc_saru.restype = _c.c_uint32
        L.orc_saru.argtypes = [_c.c_uint32] * 3
        L.orc_hash_rng.restype = _c.c_uint32
        L.orc_hash_rng.argtypes = [_c.c_uint32] * 2
        L.orc_philox.restype = _c.c_uint32
        L.orc_philox.argtypes = [_c.c_uint64] * 3
        L.orc_zindex.restype = _c.c_uint32
        L.orc_zindex.argtypes = [_c.c_int64] * 3 + [_c.c_uint32] * 3
        L.orc_r250_seed_u64.argtypes = [_P, _c.c_uint64]
        L.orc_r250_seed_words.argtypes = [_P, _P]
        L.orc_r250_draw.argtypes = [_P, _P, _c.c_size_t]
        L.orc_graph_coloring.restype = _c.c_int
        L.orc_graph_coloring.argtypes = [_c.c_uint32, _P, _P, _c.c_int, _P]
        L.orc_sweep_create.restype = _P
        L.orc_sweep_create.argtypes = [_c.c_uint32] * 4 + [_P, _P, _P, _P, _c.c_int, _c.c_int64, _c.c_int64, _c.c_int]
        L.orc_sweep_destroy.argtypes = [_P]
        L.orc_sweep_set_periodicity.argtypes = [_P, _c.c_int, _c.c_int, _c.c_int]
        L.orc_sweep_run.argtypes = [_P, _c.c_uint32, _P]
        L.orc_sweep_get.argtypes = [_P, _P]
        L.orc_sweep_age.restype = _c.c_int64
        L.orc_sweep_age.argtypes = [_P]
        L.orc_sweep_nspecies.restype = _c.c_uint32
        L.orc_sweep_nspecies.argtypes = [_P]
        L.orc_sweep_colors.argtypes = [_P, _P]
        L.orc_sweep_slab.restype = _c.c_uint32
        L.orc_sweep_slab.argtypes = [_P, _c.c_uint32, _P]
        L.orc_sweep_stats.argtypes = [_P, _P]
        L.orc_sweep_set_filter_stats.argtypes = [_P, _c.c_int]
        L.orc_sweep_filter_stats.argtypes = [_P, _P]
        L.orc_serial_run.restype = _c.c_uint64
        L.orc_serial_run.argtypes = [_c.c_uint32] * 4 + [_P, _P, _P, _P, _c.c_uint64, _c.c_uint64]
        _orc = L
    return _orc


def r250_state(seed: int) -> np.ndarray:
    s = np.zeros(251, np.uint32)
    orc().orc_r250_seed_u64(s.ctypes.data, seed)
    return s


def r250_state_words(words) -> np.ndarray:
    w = np.ascontiguousarray(words, dtype=np.uint32)
    s = np.zeros(251, np.uint32)
    orc().orc_r250_seed_words(s.ctypes.data, w.ctypes.data)
    return s


def r250_draw(state: np.ndarray, n: int) -> np.ndarray:
    out = np.zeros(n, np.uint32)
    orc().orc_r250_draw(state.ctypes.data, out.ctypes.data, n)
    return out


def graph_coloring(deg, nbr8, uniform=True):
    d = np.ascontiguousarray(deg, dtype=np.uint32)
    b = np.ascontiguousarray(nbr8, dtype=np.uint32)
    out = np.zeros(d.size, np.uint32)
    k = orc().orc_graph_coloring(d.size, d.ctypes.data, b.ctypes.data, int(uniform), out.ctypes.data)
    return k, out


class Sweep:
    """Stateful CPU emulation of the reference's colored sweep."""

    def __init__(self, system, rng=2, age=0, sort_every=5000, threads=None, periodic=(True, True, True)):
        L = orc()
        self.n = system.n
        self._pos = np.ascontiguousarray(system.pos, dtype=np.int32)
        self._deg = np.ascontiguousarray(system.deg, dtype=np.uint32)
        self._nbr = np.ascontiguousarray(system.nbr, dtype=np.uint32)
        self._allowed = np.ascontiguousarray(system.allowed, dtype=np.uint8)
        forbidden = (1 - self._allowed).astype(np.uint8)
        threads = threads or os.cpu_count() or 1
        bx, by, bz = system.box
        self._h = L.orc_sweep_create(bx, by, bz, self.n, self._pos.ctypes.data, self._deg.ctypes.data,
                                     self._nbr.ctypes.data, forbidden.ctypes.data, int(rng), int(age),
                                     int(sort_every), int(threads))
        if not self._h:
            raise RuntimeError("oracle sweep set-up failed")
        L.orc_sweep_set_periodicity(self._h, *(int(bool(p)) for p in periodic))

    def run(self, nmcs: int, r250: np.ndarray):
        orc().orc_sweep_run(self._h, int(nmcs), r250.ctypes.data)

    def positions(self) -> np.ndarray:
        out = np.zeros((self.n, 3), np.int32)
        orc().orc_sweep_get(self._h, out.ctypes.data)
        return out

    def age(self) -> int:
        return int(orc().orc_sweep_age(self._h))

    def nspecies(self) -> int:
        return int(orc().orc_sweep_nspecies(self._h))

    def colors(self) -> np.ndarray:
        out = np.zeros(self.n, np.uint32)
        orc().orc_sweep_colors(self._h, out.ctypes.data)
        return out

    def slab(self, sp: int) -> np.ndarray:
        m = orc().orc_sweep_slab(self._h, sp, None)
        out = np.zeros(m, np.uint32)
        orc().orc_sweep_slab(self._h, sp, out.ctypes.data)
        return out

    def stats(self):
        out = np.zeros(3, np.uint64)
        orc().orc_sweep_stats(self._h, out.ctypes.data)
        return tuple(int(v) for v in out)

    def set_filter_stats(self, mode: int):
        """0 off; 1 counted as the reference's count kernels do; 2 the moves made"""
        orc().orc_sweep_set_filter_stats(self._h, int(mode))

    def filter_stats(self) -> np.ndarray:
        """(species, 5 filters, [min, mean, stddev, max, substeps]) of the latest run"""
        out = np.zeros((self.nspecies(), 5, 5), np.float64)
        orc().orc_sweep_filter_stats(self._h, out.ctypes.data)
        return out

    def __del__(self):
        if getattr(self, "_h", None):
            orc().orc_sweep_destroy(self._h)
            self._h = None


def serial_run(system, pos: np.ndarray, nmcs: int, seed: int) -> int:
    """Random-sequential serial BFM, in place on pos; returns accepted moves."""
    d = np.ascontiguousarray(system.deg, dtype=np.uint32)
    b = np.ascontiguousarray(system.nbr, dtype=np.uint32)
    f = (1 - np.ascontiguousarray(system.allowed, dtype=np.uint8)).astype(np.uint8)
    bx, by, bz = system.box
    return int(orc().orc_serial_run(bx, by, bz, system.n, pos.ctypes.data, d.ctypes.data, b.ctypes.data,
                                    f.ctypes.data, int(nmcs), int(seed)))


def lattice_words(pos: np.ndarray, box) -> np.ndarray:
    """Occupation bit lattice (Z-order, 32-bit words) of corner positions;
    edges that are not powers of two are padded to the next one."""
    from pscbfm_b200.systems import System  # noqa: F401  (keeps import graph explicit)
    Lm = 1
    while Lm < max(box):
        Lm *= 2
    words = np.zeros(Lm ** 3 // 32, np.uint32)
    p = np.asarray(pos, dtype=np.int64) % np.array(box)
    code = _zcode(p[:, 0]) | (_zcode(p[:, 1]) << 1) | (_zcode(p[:, 2]) << 2)
    np.bitwise_or.at(words, code >> 5, (np.uint32(1) << (code & 31).astype(np.uint32)).astype(np.uint32))
    return words


def _zcode(v):
    x = np.asarray(v, dtype=np.uint64) & np.uint64(0x3FF)
    x = (x | (x << np.uint64(16))) & np.uint64(0x030000FF)
    x = (x | (x << np.uint64(8))) & np.uint64(0x0300F00F)
    x = (x | (x << np.uint64(4))) & np.uint64(0x030C30C3)
    x = (x | (x << np.uint64(2))) & np.uint64(0x09249249)
    return x.astype(np.int64)


# ---------------------------------------------------------- reference libs
_ref_host = None
_ref_gpu = None


def ref_host():
    global _ref_host
    if _ref_host is None:
        if not os.path.exists(REF_HOST_SO):
            return None
        L = ctypes.CDLL(REF_HOST_SO)
        L.ref_saru.restype = _c.c_uint32
        L.ref_saru.argtypes = [_c.c_uint32, _c.c_uint64, _c.c_uint32]
        L.ref_hash.restype = _c.c_uint32
        L.ref_hash.argtypes = [_c.c_uint32, _c.c_uint32]
        L.ref_graph_coloring.restype = _c.c_int
        L.ref_graph_coloring.argtypes = [_c.c_uint32, _P, _P, _c.c_int, _P]
        _ref_host = L
    return _ref_host


def ref_gpu():
    global _ref_gpu
    if _ref_gpu is None:
        if not os.path.exists(REF_GPU_SO):
            return None
        L = ctypes.CDLL(REF_GPU_SO)
        L.ref_last_error.restype = _c.c_char_p
        L.ref_create.restype = _P
        L.ref_create.argtypes = [_c.c_int, _c.c_int] + [_c.c_uint32] * 4 + [_P, _P, _P, _P, _c.c_int, _c.c_int64, _c.c_int64]
        L.ref_set_periodicity.argtypes = [_c.c_int]
        L.ref_run.restype = _c.c_int
        L.ref_run.argtypes = [_P, _c.c_uint32]
        L.ref_get.argtypes = [_P, _P, _c.c_uint32]
        L.ref_run_stats.restype = _c.c_long
        L.ref_run_stats.argtypes = [_P, _c.c_uint32, _P, _c.c_size_t]
        L.ref_age.restype = _c.c_int64
        L.ref_age.argtypes = [_P]
        L.ref_destroy.argtypes = [_P]
        L.ref_r250_set.argtypes = [_P]
        L.ref_r250_get.argtypes = [_P]
        _ref_gpu = L
    return _ref_gpu


class RefUpdater:
    """The reference's own UpdaterGPUScBFM_AB_Type<T> on the GPU (oracle/_ref)."""

    def __init__(self, system, rng=2, age=0, sort_every=5000, ctype=0, gpu=0, periodic=(True, True, True)):
        L = ref_gpu()
        if L is None:
            raise RuntimeError("oracle/_ref/libref_pscbfm.so is not built")
        L.ref_set_periodicity(sum(1 << a for a in range(3) if periodic[a]))
        self.n = system.n
        self._pos = np.ascontiguousarray(system.pos, dtype=np.int32)
        self._deg = np.ascontiguousarray(system.deg, dtype=np.uint32)
        self._nbr = np.ascontiguousarray(system.nbr, dtype=np.uint32)
        self._allowed = np.ascontiguousarray(system.allowed, dtype=np.uint8)
        bx, by, bz = system.box
        self._h = L.ref_create(gpu, ctype, bx, by, bz, self.n, self._pos.ctypes.data, self._deg.ctypes.data,
                               self._nbr.ctypes.data, self._allowed.ctypes.data, int(rng), int(age), int(sort_every))
        if not self._h:
            raise RuntimeError("reference set-up failed: " + (L.ref_last_error() or b"").decode())

    def run(self, nmcs: int, r250: np.ndarray):
        L = ref_gpu()
        L.ref_r250_set(r250.ctypes.data)
        if L.ref_run(self._h, int(nmcs)) != 0:
            raise RuntimeError("reference run failed: " + (L.ref_last_error() or b"").decode())
        L.ref_r250_get(r250.ctypes.data)

    def positions(self) -> np.ndarray:
        out = np.zeros((self.n, 3), np.int32)
        ref_gpu().ref_get(self._h, out.ctypes.data, self.n)
        return out

    def run_stats(self, nmcs: int, r250: np.ndarray) -> str:
        """run with the reference's "Stats" log active; returns what it printed"""
        L = ref_gpu()
        L.ref_r250_set(r250.ctypes.data)
        buf = ctypes.create_string_buffer(1 << 16)
        if L.ref_run_stats(self._h, int(nmcs), buf, len(buf)) < 0:
            raise RuntimeError("reference run failed: " + (L.ref_last_error() or b"").decode())
        L.ref_r250_get(r250.ctypes.data)
        return buf.value.decode()

    def __del__(self):
        if getattr(self, "_h", None):
            ref_gpu().ref_destroy(self._h)
            self._h = None


def parse_filter_analysis(text: str):
    """The reference's printed filter analysis (.cu:3351-3374, one block
    "=== Group X (n) ===" per species, then per filter
    "name: min(p%) | mean(p%) +- stddev | max(p%)") as
    (group sizes, array (groups, 5, 4) of min, mean, stddev, max)."""
    sizes, rows = [], []
    for line in text.splitlines():
        if line.startswith("=== Group "):
            sizes.append(int(line.split("(")[1].split(")")[0]))
            rows.append([])
        elif rows and len(rows[-1]) < 5 and ": " in line and " | " in line and " +- " in line:
            vals = line.split(": ", 1)[1]
            lo, mid, hi = vals.split(" | ")
            mean, std = mid.split(" +- ")
            num = lambda t: float(t.split("(")[0])
            rows[-1].append([num(lo), num(mean), float(std), num(hi)])
    return sizes, np.array(rows, dtype=np.float64).reshape(len(rows), 5, 4)


# ---------------------------------------------------------------- chain analysis
def linear_chains(deg, nbr):
    """Restatement of AnalyzerMsd::getLinearPolymerSystemInfo
    (src/AnalyzerMsd.tpp:193-280) for test use: chains in order of their
    lowest id, walked with a stack; end monomers in the order met; the middle
    monomer floor(n/2) bonds from the first end.  Returns (first, middle,
    last, members) with members a list of id arrays."""
    n = len(deg)
    visited = np.zeros(n, dtype=bool)
    first, middle, last, members = [], [], [], []
    for i0 in range(n):
        if visited[i0]:
            continue
        ends, todo, mem = [], [i0], [i0]
        visited[i0] = True
        while todo:
            m = todo.pop()
            nn = int(deg[m])
            if nn > 2:
                raise ValueError("not linear chains")
            if nn <= 1:
                ends.append(m)
            for b in range(nn):
                q = int(nbr[m][b])
                if not visited[q]:
                    visited[q] = True
                    todo.append(q)
                    mem.append(q)
        if len(mem) == 1 and len(ends) == 1:
            ends.append(ends[0])
        if len(ends) != 2:
            raise ValueError("not exactly two chain ends")
        mid = prev = ends[0]
        for _ in range(len(mem) // 2):
            nxt = int(nbr[mid][0]) if int(nbr[mid][0]) != prev else int(nbr[mid][1])
            prev, mid = mid, nxt
        first.append(ends[0]); middle.append(mid); last.append(ends[1]); members.append(np.array(mem))
    return np.array(first), np.array(middle), np.array(last), members


def chain_observables(pos, first, middle, last, members, origin=None):
    """<R_e^2>, <R_g^2>, per-chain centres and g1..g5 against `origin` (the
    dict this function returns for the origin state), as AnalyzerMsd
    computes them (src/AnalyzerMsd.tpp:304-421), in float64."""
    p = np.asarray(pos, dtype=np.float64)
    com = np.stack([p[m].mean(axis=0) for m in members])
    re2 = ((p[last] - p[first]) ** 2).sum(axis=1)
    rg2 = np.array([((p[m] - p[m].mean(axis=0)) ** 2).sum(axis=1).mean() for m in members])
    box = com.mean(axis=0)
    vals = [p[first], p[middle], p[last], com, p[middle] - com]
    g = [0.0] * 5
    ac = 0.0
    if origin is not None:
        r0 = origin["vals"][2] - origin["vals"][0]
        den = float((r0 * r0).sum())
        ac = float(((p[last] - p[first]) * r0).sum() / den) if den > 0 else 0.0
        drift = box - origin["box"] if len(members) > 1 else np.zeros(3)
        for k in range(5):
            d = vals[k] - origin["vals"][k] - (drift if k < 4 else 0.0)
            g[k] = float((d * d).sum(axis=1).mean())
    return {"re2": float(re2.mean()), "rg2": float(rg2.mean()), "re2_chain": re2, "rg2_chain": rg2,
            "com": com, "box": box, "vals": vals, "g": g, "end_autocorr": ac}
