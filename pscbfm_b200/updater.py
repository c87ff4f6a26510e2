"""Host-side mirror of the reference's ``UpdaterGPUScBFM_AB_Type<T>``.

Same method names, argument meaning, dependency order and exception types as
src/pscbfm/UpdaterGPUScBFM_AB_Type.h:453-514 of lgh0504/pscbfm, forwarding
to the C ABI of ``libpscbfm_b200.so`` (include/pscbfm_b200.h).  The
reference's ``std::invalid_argument`` becomes ``ValueError`` and its
``std::runtime_error`` becomes ``RuntimeError``; CUDA failures, which the
reference answers with ``exit()`` (cudacommon.hpp:36-51), raise
:class:`CudaError`.

The template parameter of the reference (the device coordinate type) has no
counterpart: positions are always kept as 32-bit Z-order codes plus image
counters on the device.
"""
from __future__ import annotations

import ctypes
import enum

import numpy as np

from . import _native


class CudaError(RuntimeError):
    """A CUDA runtime call failed inside the library."""


class DeviceTimeout(TimeoutError):
    """A bounded device-side wait gave up."""


class Rng(enum.IntEnum):
    """``UpdaterGPUScBFM_AB_Type::Rng`` (UpdaterGPUScBFM_AB_Type.h:413-420)."""

    IntHash = 1
    Saru = 2
    Philox = 3
    Pcg = 4
    Xorwow = 5


def _raise(status: int, msg: str):
    if status == _native.BFM_OK:
        return
    if status == _native.BFM_EINVAL:
        raise ValueError(msg)
    if status == _native.BFM_ECUDA:
        raise CudaError(msg)
    if status == _native.BFM_ETIMEOUT:
        raise DeviceTimeout(msg)
    raise RuntimeError(msg)


class UpdaterGPUScBFM_AB_Type:
    """One simulated BFM system on one GPU (see module docstring)."""

    Rng = Rng

    def __init__(self):
        self._lib = _native.lib()
        h = ctypes.c_void_p()
        _raise(self._lib.bfm_create(ctypes.byref(h)), "bfm_create failed")
        self._h = h
        self._n = 0
        self._nchains = 0
        self._steps_between_sortings = 5000

    # ------------------------------------------------------------ plumbing
    def _check(self, status: int):
        if status != _native.BFM_OK:
            msg = self._lib.bfm_last_error(self._h)
            _raise(status, msg.decode() if msg else f"status {status}")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.bfm_destroy(h)
            self._h = None

    def destruct(self):
        """Free every resource (``destruct``, UpdaterGPUScBFM_AB_Type.h:455)."""
        self._check(self._lib.bfm_cleanup(self._h))

    # ------------------------------------------------------------ setters
    def setGpu(self, iGpuToUse: int):
        self._check(self._lib.bfm_set_gpu(self._h, int(iGpuToUse)))

    def copyBondSet(self, dx: int, dy: int, dz: int, bondForbidden: bool):
        self._check(self._lib.bfm_copy_bond_set(self._h, int(dx), int(dy), int(dz), 1 if bondForbidden else 0))

    def setNrOfAllMonomers(self, nAllMonomers: int):
        self._check(self._lib.bfm_set_nr_of_all_monomers(self._h, int(nAllMonomers)))
        self._n = int(nAllMonomers)

    def setAttribute(self, i: int, attribute: int):
        self._check(self._lib.bfm_set_attribute(self._h, int(i), int(attribute)))

    def setMonomerCoordinates(self, i: int, x: int, y: int, z: int):
        self._check(self._lib.bfm_set_monomer_coordinates(self._h, int(i), int(x), int(y), int(z)))

    def setConnectivity(self, monoidx1: int, monoidx2: int):
        self._check(self._lib.bfm_set_connectivity(self._h, int(monoidx1), int(monoidx2)))

    def setLatticeSize(self, boxX: int, boxY: int, boxZ: int):
        self._check(self._lib.bfm_set_lattice_size(self._h, int(boxX), int(boxY), int(boxZ)))

    def setPeriodicity(self, isPeriodicX: bool, isPeriodicY: bool, isPeriodicZ: bool):
        self._check(self._lib.bfm_set_periodicity(self._h, int(bool(isPeriodicX)), int(bool(isPeriodicY)), int(bool(isPeriodicZ))))

    def setAge(self, rAge: int):
        self._check(self._lib.bfm_set_age(self._h, int(rAge)))

    def getAge(self) -> int:
        v = ctypes.c_int64()
        self._check(self._lib.bfm_get_age(self._h, ctypes.byref(v)))
        return v.value

    def setRng(self, x):
        self._check(self._lib.bfm_set_rng(self._h, int(x)))

    def getRng(self) -> Rng:
        v = ctypes.c_int()
        self._check(self._lib.bfm_get_rng(self._h, ctypes.byref(v)))
        return Rng(v.value)

    def setStepsBetweenSortings(self, rnStepsBetweenSortings: int):
        self._check(self._lib.bfm_set_steps_between_sortings(self._h, int(rnStepsBetweenSortings)))
        self._steps_between_sortings = int(rnStepsBetweenSortings)

    def getStepsBetweenSortings(self) -> int:
        return self._steps_between_sortings

    # ------------------------------------------------------------ life cycle
    def initialize(self):
        self._check(self._lib.bfm_initialize(self._h))

    def execute(self) -> bool:
        return True

    def runSimulationOnGPU(self, nrMCS_per_Call: int):
        self._check(self._lib.bfm_run(self._h, int(nrMCS_per_Call)))

    def cleanup(self):
        self._check(self._lib.bfm_cleanup(self._h))
        self._n = 0

    # ------------------------------------------------------------ getters
    def _pos(self, i: int):
        x, y, z = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        self._check(self._lib.bfm_get_monomer_position(self._h, int(i), ctypes.byref(x), ctypes.byref(y), ctypes.byref(z)))
        return x.value, y.value, z.value

    def getMonomerPositionInX(self, i: int) -> int:
        return self._pos(i)[0]

    def getMonomerPositionInY(self, i: int) -> int:
        return self._pos(i)[1]

    def getMonomerPositionInZ(self, i: int) -> int:
        return self._pos(i)[2]

    # ------------------------------------------------------------ bulk API
    def setAllMonomerCoordinates(self, xyz):
        a = np.ascontiguousarray(xyz, dtype=np.int32).reshape(-1, 3)
        self._check(self._lib.bfm_set_all_coordinates(self._h, a.ctypes.data, a.shape[0]))

    def setAllConnectivity(self, deg, nbr8):
        d = np.ascontiguousarray(deg, dtype=np.uint8)
        b = np.ascontiguousarray(nbr8, dtype=np.uint32).reshape(-1, 8)
        self._check(self._lib.bfm_set_all_connectivity(self._h, d.ctypes.data, b.ctypes.data, d.shape[0]))

    def setBondSet(self, allowed512):
        """allowed512[(dx&7)|(dy&7)<<3|(dz&7)<<6] for dx,dy,dz in [-4,3], the
        loop of the LeMonADE adapter (GPUScBFM_AB_Type.h:168-175)."""
        allowed = np.asarray(allowed512, dtype=bool)
        for dx in range(-4, 4):
            for dy in range(-4, 4):
                for dz in range(-4, 4):
                    self.copyBondSet(dx, dy, dz, not allowed[(dx & 7) | ((dy & 7) << 3) | ((dz & 7) << 6)])

    def getAllMonomerPositions(self, out: np.ndarray = None) -> np.ndarray:
        """unfolded positions, (n, 3) int32; `out` (optional) is filled and
        returned -- page-locked memory there takes one device-to-host copy"""
        if out is None:
            out = np.empty((self._n, 3), dtype=np.int32)
        elif out.shape != (self._n, 3) or out.dtype != np.int32 or not out.flags.c_contiguous:
            raise ValueError(f"out must be a C-contiguous ({self._n}, 3) int32 array")
        self._check(self._lib.bfm_get_positions(self._h, out.ctypes.data, self._n))
        return out

    def setColoring(self, mode: int):
        """colouring at initialize: 0 host walk (default), 1 device for forests"""
        self._check(self._lib.bfm_set_coloring(self._h, int(mode)))

    def getColoring(self):
        """(mode, whether the last initialize coloured on the device)"""
        m, d = ctypes.c_int(), ctypes.c_int()
        self._check(self._lib.bfm_get_coloring(self._h, ctypes.byref(m), ctypes.byref(d)))
        return m.value, bool(d.value)

    # ---- the reference's "Stats" filter analysis
    FILTERS = ("Box Boundaries", "Invalid Bonds", "Volume Exclusion", "! Invalid Bonds && Volume Exclusion",
               "! Invalid Bonds && ! Volume Exclusion && Parallel Volume Exclusion")

    def setFilterStats(self, mode: int = 1):
        """count, in the following runs, the moves each filter refuses per
        colour substep (the per-substep kernels run while this is on).
        mode 1: the reference's printed numbers (IntHash directions for
        filters 0-3; filter 4 after the move, read through the reference's
        byte fetch of its bit-packed target lattice); 2: the moves this RNG
        made, filter 4 = candidates refused; 0: off."""
        self._check(self._lib.bfm_set_filter_stats(self._h, int(mode)))
        return self

    def getFilterStats(self) -> np.ndarray:
        """(species, 5 filters, [min, mean, stddev, max, substeps]) over the
        colour substeps of the last run; filter names in FILTERS"""
        out = np.zeros((self.getNSpecies(), 5, 5), dtype=np.float64)
        self._check(self._lib.bfm_get_filter_stats(self._h, out.ctypes.data, out.size))
        return out

    # ---- chain analysis on the device (the reference's AnalyzerMsd)
    def analyzerInit(self) -> int:
        """Find the linear chains (first end, middle, last end) by the
        reference analyzer's rule; ValueError if the system is not made of
        linear chains.  Returns the number of chains."""
        nc = ctypes.c_uint32()
        self._check(self._lib.bfm_analyzer_init(self._h, ctypes.byref(nc)))
        self._nchains = nc.value
        return nc.value

    def analyze(self, set_origin: bool = False) -> dict:
        """Chain observables of the current state, computed on the GPU:
        <R_e^2>, <R_g^2>, g1..g5 against the time origin (zero before one is
        set), the box centre of mass and the end-to-end vector
        autocorrelation against the origin.  set_origin makes the current
        state the origin of later calls."""
        out = np.zeros(12, dtype=np.float64)
        self._check(self._lib.bfm_analyze(self._h, int(bool(set_origin)), out.ctypes.data, out.size))
        return {"chains": int(out[0]), "re2": float(out[1]), "rg2": float(out[2]),
                "g": [float(v) for v in out[3:8]], "box_com": out[8:11].copy(), "end_autocorr": float(out[11])}

    def analyzerChainIds(self):
        nc = self._nchains
        f, m, l = (np.empty(nc, dtype=np.uint32) for _ in range(3))
        self._check(self._lib.bfm_analyzer_chain_ids(self._h, f.ctypes.data, m.ctypes.data, l.ctypes.data, nc))
        return f, m, l

    def analyzePerChain(self):
        """per-chain R_e^2, R_g^2 and centre of mass of the last analyze()"""
        nc = self._nchains
        re2, rg2 = np.empty(nc), np.empty(nc)
        com = np.empty((nc, 3))
        self._check(self._lib.bfm_analyze_per_chain(self._h, re2.ctypes.data, rg2.ctypes.data, com.ctypes.data, nc))
        return re2, rg2, com

    def getLattice(self) -> np.ndarray:
        nw = ctypes.c_size_t()
        self._check(self._lib.bfm_get_lattice_words(self._h, ctypes.byref(nw)))
        out = np.empty(nw.value, dtype=np.uint32)
        self._check(self._lib.bfm_get_lattice(self._h, out.ctypes.data, nw.value))
        return out

    def getNSpecies(self) -> int:
        v = ctypes.c_uint32()
        self._check(self._lib.bfm_get_nspecies(self._h, ctypes.byref(v)))
        return v.value

    def getColors(self) -> np.ndarray:
        out = np.empty(self._n, dtype=np.uint32)
        self._check(self._lib.bfm_get_colors(self._h, out.ctypes.data, self._n))
        return out

    def getSpeciesOrder(self, sp: int) -> np.ndarray:
        cnt = ctypes.c_size_t()
        self._check(self._lib.bfm_get_species_order(self._h, int(sp), None, 0, ctypes.byref(cnt)))
        out = np.empty(cnt.value, dtype=np.uint32)
        self._check(self._lib.bfm_get_species_order(self._h, int(sp), out.ctypes.data, cnt.value, ctypes.byref(cnt)))
        return out

    def getCounters(self):
        """(attempted moves, candidates after the check phase, accepted moves)."""
        out = np.zeros(3, dtype=np.uint64)
        self._check(self._lib.bfm_get_counters(self._h, out.ctypes.data))
        return int(out[0]), int(out[1]), int(out[2])

    def getLastRunMs(self) -> float:
        v = ctypes.c_double()
        self._check(self._lib.bfm_get_last_run_ms(self._h, ctypes.byref(v)))
        return v.value

    def getLastRunLaunches(self) -> int:
        v = ctypes.c_uint64()
        self._check(self._lib.bfm_get_last_run_launches(self._h, ctypes.byref(v)))
        return v.value

    def timeKernels(self, nmcs: int):
        """Run nmcs MCS with CUDA events around every sweep-kernel launch;
        returns (device ms, launches, attempted moves) summed over the run."""
        ms, n, a = ctypes.c_double(), ctypes.c_uint64(), ctypes.c_uint64()
        self._check(self._lib.bfm_time_kernels(self._h, int(nmcs), ctypes.byref(ms), ctypes.byref(n), ctypes.byref(a)))
        return ms.value, n.value, a.value

    def getLaunchInfo(self) -> dict:
        """Shape of the persistent kernel: bond mode (0 gather, 1 stored, 2 staged),
        CTAs, threads per CTA, dynamic shared memory per CTA."""
        m, g, t, b = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_size_t()
        self._check(self._lib.bfm_get_launch_info(self._h, ctypes.byref(m), ctypes.byref(g), ctypes.byref(t), ctypes.byref(b)))
        return {"mode": m.value, "ctas": g.value, "threads": t.value, "smem_bytes": b.value}

    def setSweepShape(self, shape: int):
        """-1 automatic; 0 gather, 1 stored bond codes (bonds tested first), 2 staged; +3 global
        candidate lists; 6..8 windowed with 1, 2, 4 items per thread in flight (8: bonds tested
        first, the leading face only of the items that pass); 9, 10 windowed on one cluster."""
        self._check(self._lib.bfm_set_sweep_shape(self._h, int(shape)))

    def setSweepAutotune(self, on: bool = True):
        """time the persistent-kernel shapes on the first chunk of the next run, keep the fastest"""
        self._check(self._lib.bfm_set_sweep_autotune(self._h, int(bool(on))))

    def getSweepTuning(self) -> dict:
        tuned = ctypes.c_int()
        n = ctypes.c_uint32()
        cap = 16
        sh, ex, th = (ctypes.c_int * cap)(), (ctypes.c_int * cap)(), (ctypes.c_int * cap)()
        ns = (ctypes.c_double * cap)()
        self._check(self._lib.bfm_get_sweep_tuning(self._h, ctypes.byref(tuned), ctypes.byref(n), sh, ex, th, ns, cap))
        k = min(n.value, cap)
        return {"tuned": bool(tuned.value),
                "trials": [{"shape": sh[i], "extra_rounds": ex[i], "threads": th[i], "ns_per_move": ns[i]} for i in range(k)]}

    def setBarrierTimeoutMs(self, ms: int):
        self._check(self._lib.bfm_set_barrier_timeout_ms(self._h, int(ms)))

    def setLaunchMode(self, mode: int):
        self._check(self._lib.bfm_set_launch_mode(self._h, int(mode)))

    # ------------------------------------------------------------ convenience
    def setup(self, system, *, gpu: int = 0, rng=Rng.Saru, age: int = 0, steps_between_sortings: int = 5000):
        """All setters of the LeMonADE adapter (GPUScBFM_AB_Type.h:121-184) for
        a :class:`pscbfm_b200.systems.System`, then ``initialize``."""
        self.setGpu(gpu)
        self.setRng(rng)
        self.setAge(age)
        self.setStepsBetweenSortings(steps_between_sortings)
        self.setPeriodicity(*getattr(system, "periodic", (True, True, True)))
        self.setLatticeSize(*system.box)
        self.setNrOfAllMonomers(system.n)
        self.setAllMonomerCoordinates(system.pos)
        self.setAllConnectivity(system.deg, system.nbr)
        self.setBondSet(system.allowed)
        self.initialize()
        return self


def color_graph(deg, nbr, uniform: bool = True, device: bool = False, gpu: int = 0):
    """The species colouring initialize() uses (the reference's
    graphColoring with uniform rebalancing).  device=True computes the same
    colours with the tree components on the GPU (see bfm_color_graph_device).
    Returns (colours, number of colours, how: 0 host, 1 device, 2 the tree
    components on the device and the cyclic ones on the host)."""
    d = np.ascontiguousarray(deg, dtype=np.uint8)
    b = np.ascontiguousarray(nbr, dtype=np.uint32)
    n = d.size
    col = np.zeros(n, dtype=np.uint32)
    nc = ctypes.c_uint32()
    lib = _native.lib()
    if device:
        dev = ctypes.c_int()
        st = lib.bfm_color_graph_device(int(gpu), n, d.ctypes.data, b.ctypes.data, int(uniform), col.ctypes.data,
                                        ctypes.byref(nc), ctypes.byref(dev))
        on_dev = int(dev.value)
    else:
        st = lib.bfm_color_graph(n, d.ctypes.data, b.ctypes.data, int(uniform), col.ctypes.data, ctypes.byref(nc))
        on_dev = 0
    if st != _native.BFM_OK:
        _raise(st, f"colouring failed (status {st})")
    return col, nc.value, on_dev


# process-global R250 colour/seed generator (LeMonADE's RandomNumberGenerators)
def r250_seed(seed: int):
    _native.lib().bfm_r250_seed(int(seed))


def r250_seed_words(words):
    w = np.ascontiguousarray(words, dtype=np.uint32)
    if w.size < 250:
        raise ValueError("R250 needs at least 250 seed words")
    _native.lib().bfm_r250_seed_words(w.ctypes.data, w.size)


def r250_get_state() -> np.ndarray:
    out = np.zeros(251, dtype=np.uint32)
    _native.lib().bfm_r250_get_state(out.ctypes.data)
    return out


def r250_set_state(state):
    s = np.ascontiguousarray(state, dtype=np.uint32)
    if s.size != 251 or s[250] >= 250:
        raise ValueError("R250 state must be 250 words + an index below 250")
    _native.lib().bfm_r250_set_state(s.ctypes.data)


def r250_rand32() -> int:
    return int(_native.lib().bfm_r250_rand32())
