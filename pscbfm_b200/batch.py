"""Batched ensembles: many independent BFM systems advanced by one
persistent kernel (``bfm_batch_*`` in include/pscbfm_b200.h).

Each system follows exactly the trajectory of a single
:class:`UpdaterGPUScBFM_AB_Type` with the same set-up and R250 state; its
colour and seed draws come from its own R250 stream.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native
from .updater import Rng


class BatchError(RuntimeError):
    pass


class Batch:
    """Set up with :meth:`add` per system and :meth:`initialize`, then
    :meth:`run` with one MCS count per system (or one for all)."""

    def __init__(self, gpu: int = 0):
        self._lib = _native.lib()
        h = ctypes.c_void_p()
        self._check(self._lib.bfm_batch_create(int(gpu), ctypes.byref(h)), None)
        self._h = h
        self._sizes = []
        self._keep = []

    def _check(self, status, h=-1):
        if status == _native.BFM_OK:
            return
        msg = ""
        hh = self._h if h == -1 else h
        if hh is not None:
            msg = (self._lib.bfm_batch_last_error(hh) or b"").decode()
        if status == _native.BFM_EINVAL:
            raise ValueError(msg)
        raise BatchError(f"status {status}: {msg}")

    def add(self, system, rng=Rng.Saru, age: int = 0, sort_every: int = 5000, r250_state=None, r250_seed: int = 0) -> int:
        """Add a system (a pscbfm_b200.systems.System); returns its index."""
        pos = np.ascontiguousarray(system.pos, dtype=np.int32)
        deg = np.ascontiguousarray(system.deg, dtype=np.uint8)
        nbr = np.ascontiguousarray(system.nbr, dtype=np.uint32)
        allowed = np.ascontiguousarray(system.allowed, dtype=np.uint8)
        st = None if r250_state is None else np.ascontiguousarray(r250_state, dtype=np.uint32)
        if st is not None and st.size != 251:
            raise ValueError("an R250 state has 251 words")
        sid = ctypes.c_uint32()
        bx, by, bz = (int(v) for v in system.box)
        self._check(self._lib.bfm_batch_add_system(self._h, bx, by, bz, int(system.n), pos.ctypes.data, deg.ctypes.data,
                                                   nbr.ctypes.data, allowed.ctypes.data, int(rng), int(age),
                                                   int(sort_every), None if st is None else st.ctypes.data,
                                                   int(r250_seed), ctypes.byref(sid)))
        self._sizes.append(int(system.n))
        return sid.value

    def set_clusters(self, size):
        """CTAs sharing a system whose lattice is in global memory: 2, 4
        (default; True selects it), 8, or 0 / False for one CTA each"""
        size = 4 if size is True else (0 if size is False else int(size))
        self._check(self._lib.bfm_batch_set_clusters(self._h, size))
        return self

    def set_autotune(self, on: bool = True):
        """time cluster sizes 4, 2, 8 and off on the next run's first launches, keep the fastest"""
        self._check(self._lib.bfm_batch_set_autotune(self._h, int(bool(on))))
        return self

    def clusters(self) -> dict:
        size, tuned = ctypes.c_int(), ctypes.c_int()
        ns = np.zeros(4, np.float64)
        self._check(self._lib.bfm_batch_get_clusters(self._h, ctypes.byref(size), ctypes.byref(tuned), ns.ctypes.data))
        return {"size": size.value, "tuned": bool(tuned.value), "trial_ns_per_move": dict(zip((4, 2, 8, 0), ns.tolist()))}

    def set_shape(self, in_flight: int = 2, clusters_from_48: bool = False):
        """monomers per thread in flight (1, 2, 4); systems of 48^3..64^3 on clusters too"""
        self._check(self._lib.bfm_batch_set_shape(self._h, int(in_flight), int(bool(clusters_from_48))))

    def tuning(self) -> dict:
        cs, f, tuned = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        above = ctypes.c_uint32()
        ns = (ctypes.c_double * 7)()
        self._check(self._lib.bfm_batch_get_tuning(self._h, ctypes.byref(cs), ctypes.byref(f), ctypes.byref(above),
                                                   ctypes.byref(tuned), ns))
        names = ("clusters 4", "clusters 2", "clusters 8", "clusters off", "1 in flight", "4 in flight",
                 "clusters from 48^3")
        return {"cluster_size": cs.value, "in_flight": f.value, "cluster_above_words": above.value,
                "tuned": bool(tuned.value), "trial_ns_per_move": dict(zip(names, list(ns)))}

    def initialize(self):
        self._check(self._lib.bfm_batch_initialize(self._h))
        return self

    def __len__(self):
        return len(self._sizes)

    def run(self, mcs):
        """Advance system s by mcs[s] MCS (an int advances every system alike)."""
        m = np.full(len(self), int(mcs), np.uint32) if np.isscalar(mcs) else np.ascontiguousarray(mcs, dtype=np.uint32)
        self._check(self._lib.bfm_batch_run(self._h, m.ctypes.data, m.size))

    def positions(self, sys: int) -> np.ndarray:
        out = np.empty((self._sizes[sys], 3), np.int32)
        self._check(self._lib.bfm_batch_get_positions(self._h, int(sys), out.ctypes.data, self._sizes[sys]))
        return out

    def all_positions(self) -> list:
        """positions of every system (one bulk read-back), as a list of (n, 3) arrays"""
        total = sum(self._sizes)
        out = np.empty((total, 3), np.int32)
        self._check(self._lib.bfm_batch_get_all_positions(self._h, out.ctypes.data, total))
        cuts = np.cumsum([0] + self._sizes)
        return [out[cuts[i]:cuts[i + 1]] for i in range(len(self._sizes))]

    def gather(self, systems, ids) -> np.ndarray:
        """unfolded positions (m, 3) of the monomers ids[k] of systems[k]
        (original monomer ids), read on the device"""
        sy = np.asarray(systems, np.uint64).reshape(-1)
        ii = np.asarray(ids, np.uint64).reshape(-1)
        if sy.size != ii.size:
            raise ValueError("one system index per monomer id")
        g = np.ascontiguousarray((sy << np.uint64(32)) | ii, dtype=np.uint64)
        out = np.empty((g.size, 3), np.int32)
        if g.size:
            self._check(self._lib.bfm_batch_gather_positions(self._h, g.ctypes.data, g.size, out.ctypes.data))
        return out

    def state(self, sys: int):
        """(age, R250 state of 251 words, (attempts, candidates, accepts))"""
        age = ctypes.c_int64()
        st = np.zeros(251, np.uint32)
        cnt = np.zeros(3, np.uint64)
        self._check(self._lib.bfm_batch_get_state(self._h, int(sys), ctypes.byref(age), st.ctypes.data, cnt.ctypes.data))
        return age.value, st, tuple(int(v) for v in cnt)

    def lattice(self, sys: int) -> np.ndarray:
        need = ctypes.c_size_t()
        self._check(self._lib.bfm_batch_get_lattice(self._h, int(sys), None, 0, ctypes.byref(need)))
        out = np.zeros(need.value, np.uint32)
        self._check(self._lib.bfm_batch_get_lattice(self._h, int(sys), out.ctypes.data, out.size, None))
        return out

    def info(self) -> dict:
        ns, k = ctypes.c_uint32(), ctypes.c_uint32()
        mono, launches, att = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        ms = ctypes.c_double()
        self._check(self._lib.bfm_batch_info(self._h, ctypes.byref(ns), ctypes.byref(mono), ctypes.byref(k),
                                             ctypes.byref(ms), ctypes.byref(launches), ctypes.byref(att)))
        return {"systems": ns.value, "monomers": mono.value, "species_max": k.value, "last_ms": ms.value,
                "last_launches": launches.value, "last_attempts": att.value}

    def close(self):
        if getattr(self, "_h", None):
            self._lib.bfm_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()
