"""The no-allocation entry point bfm_substep_noalloc against bfm_run.

bfm_substep_noalloc exists for callers that cannot call cudaMalloc while they
step a system -- a host simulation that gives the library slices of a device
pool it manages itself, or one running under a fixed device-memory budget
where allocation (which may also synchronize the device) is not allowed.
Here the caller's arrays come from torch (the test plays that caller); the
entry point itself must allocate nothing and must reproduce, substep by
substep, exactly what the handle-based bfm_run computes.
"""
import ctypes

import numpy as np
import pytest

import pscbfm_b200 as pb
from pscbfm_b200 import _native, systems

pytestmark = pytest.mark.gpu


def _dilate(v):
    x = np.asarray(v, dtype=np.uint64) & np.uint64(0x3FF)
    for sh, m in ((16, 0x030000FF), (8, 0x0300F00F), (4, 0x030C30C3), (2, 0x09249249)):
        x = (x | (x << np.uint64(sh))) & np.uint64(m)
    return x


def _undilate(v):
    x = np.asarray(v, dtype=np.uint64) & np.uint64(0x09249249)
    for sh, m in ((2, 0x030C30C3), (4, 0x0300F00F), (8, 0x030000FF), (16, 0x3FF)):
        x = (x | (x >> np.uint64(sh))) & np.uint64(m)
    return x.astype(np.int64)


class _CallerArrays:
    """The caller's own layout of a system that a handle also runs: compact
    colour slabs in the library's slot order, positions as Z-order codes of
    the wrapped coordinates, arrays in device memory the caller allocated
    (torch plays that caller)."""

    def __init__(self, s, u, with_img):
        import torch

        box = np.array(s.box)
        self.box = box
        self.nspec = u.getNSpecies()
        orders = [u.getSpeciesOrder(sp) for sp in range(self.nspec)]
        self.counts = [len(o) for o in orders]
        self.offs = np.concatenate([[0], np.cumsum(self.counts)[:-1]]).astype(np.int64)
        self.npad = int(sum(self.counts))
        slot_of = np.empty(s.n, np.int64)
        for sp, o in enumerate(orders):
            slot_of[o] = self.offs[sp] + np.arange(len(o))
        self.slot_of = slot_of
        pos0 = s.pos.astype(np.int64)
        wrapped = pos0 % box
        img0 = (pos0 - wrapped) // box
        codes = np.zeros(self.npad, np.uint32)
        codes[slot_of] = (_dilate(wrapped[:, 0]) | (_dilate(wrapped[:, 1]) << np.uint64(1))
                          | (_dilate(wrapped[:, 2]) << np.uint64(2))).astype(np.uint32)
        img = np.zeros((3, self.npad), np.int32)
        img[:, slot_of] = img0.T
        deg = np.zeros(self.npad, np.uint8)
        deg[slot_of] = s.deg
        rows = max(int(s.deg.max()), 1)
        nbr = np.zeros((rows, self.npad), np.uint32)
        for j in range(rows):
            has = s.deg > j
            nbr[j, slot_of[has]] = slot_of[s.nbr[has, j]]
        lm = int(box.max())
        lat = np.zeros(lm ** 3 // 32, np.uint32)
        np.bitwise_or.at(lat, codes >> 5, (np.uint32(1) << (codes & 31)).astype(np.uint32))
        dev = torch.device("cuda", 0)
        self.d_pos = torch.from_numpy(codes.view(np.int32)).to(dev)
        self.d_img = torch.from_numpy(img).to(dev) if with_img else None
        self.d_nbr = torch.from_numpy(nbr.view(np.int32)).to(dev)
        self.d_deg = torch.from_numpy(deg).to(dev)
        self.d_lat = torch.from_numpy(lat.view(np.int32)).to(dev)
        self.allowed = np.ascontiguousarray(s.allowed, dtype=np.uint8)
        self.stream = torch.cuda.current_stream(dev)

    def substep(self, lib, sp, seed, iteration, rng):
        return lib.bfm_substep_noalloc(self.d_pos.data_ptr(), self.d_img.data_ptr() if self.d_img is not None else None,
                                       self.d_nbr.data_ptr(), self.d_deg.data_ptr(), self.npad, self.d_lat.data_ptr(),
                                       int(self.box[0]), int(self.box[1]), int(self.box[2]), self.allowed.ctypes.data,
                                       int(self.offs[sp]), self.counts[sp], seed, iteration & 0xFFFFFFFF, int(rng),
                                       ctypes.c_void_p(self.stream.cuda_stream))

    def positions(self):
        """unfolded positions (with image counters) or wrapped ones (without)"""
        c = self.d_pos.cpu().numpy().view(np.uint32)[self.slot_of].astype(np.uint64)
        w = np.stack([_undilate(c), _undilate(c >> np.uint64(1)), _undilate(c >> np.uint64(2))], axis=1)
        if self.d_img is None:
            return w
        return w + self.d_img.cpu().numpy()[:, self.slot_of].T.astype(np.int64) * self.box


CASES = [
    ("saru_cubic_img", pb.Rng.Saru, (32, 32, 32), True),
    ("inthash_cubic_img", pb.Rng.IntHash, (32, 32, 32), True),
    ("saru_noncubic_noimg", pb.Rng.Saru, (32, 16, 64), False),
    ("inthash_noncubic_noimg", pb.Rng.IntHash, (32, 16, 64), False),
]


@pytest.mark.parametrize("name,rng,box,with_img", CASES, ids=[c[0] for c in CASES])
def test_noalloc_substeps_match_run_two_calls(name, rng, box, with_img):
    """Two MCS in a row: after each, the caller's arrays stepped by
    bfm_substep_noalloc equal the handle's positions and lattice, bit for
    bit (with image counters: unfolded positions; without: wrapped ones)."""
    lib = _native.lib()
    s = systems.saw_chains(30, 20, box=box, seed=41)
    pb.r250_seed(17)
    u = pb.UpdaterGPUScBFM_AB_Type().setup(s, rng=rng, age=0)
    ca = _CallerArrays(s, u, with_img)
    for call in range(2):
        st = pb.r250_get_state()
        age = u.getAge()
        u.runSimulationOnGPU(1)
        want = u.getAllMonomerPositions().astype(np.int64)
        st_after = pb.r250_get_state()
        pb.r250_set_state(st)                 # replay the draws of that MCS
        for sub in range(ca.nspec):
            sp = pb.r250_rand32() % ca.nspec
            seed = pb.r250_rand32()
            assert ca.substep(lib, sp, seed, age + sub, rng) == 0
        ca.stream.synchronize()
        assert np.array_equal(pb.r250_get_state(), st_after)
        got = ca.positions()
        if not with_img:
            want = want % ca.box
        assert np.array_equal(got, want), f"call {call}: {int((got != want).any(axis=1).sum())} monomers differ"
        assert np.array_equal(ca.d_lat.cpu().numpy().view(np.uint32), u.getLattice())
        assert (got != (s.pos if with_img else s.pos % ca.box)).any()


def test_noalloc_allocates_nothing_across_many_calls():
    """After the first call on the device (address look-up and kernel
    loading), further calls with either generator leave the device's free
    memory unchanged."""
    import torch

    lib = _native.lib()
    s = systems.saw_chains(30, 20, box=(32, 32, 32), seed=43)
    pb.r250_seed(5)
    u = pb.UpdaterGPUScBFM_AB_Type().setup(s, rng=pb.Rng.Saru, age=0)
    ca = _CallerArrays(s, u, True)
    assert ca.substep(lib, 0, 1, 0, pb.Rng.Saru) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    for k in range(200):
        rng = pb.Rng.Saru if k % 2 else pb.Rng.IntHash
        assert ca.substep(lib, k % ca.nspec, 1000 + k, k, rng) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0


def test_noalloc_rejects_sizes_beyond_its_maximum():
    import torch

    lib = _native.lib()
    allowed = np.ascontiguousarray(systems.ALLOWED_108, dtype=np.uint8)
    buf = torch.zeros(1 << 20, dtype=torch.int32, device="cuda:0")
    p = buf.data_ptr()
    rc = lib.bfm_substep_noalloc(p, None, p, p, 1 << 20, p, 256, 256, 256, allowed.ctypes.data,
                                 0, 1000, 1, 0, int(pb.Rng.Saru), None)
    assert rc == _native.BFM_ETOOLARGE
    rc = lib.bfm_substep_noalloc(p, None, p, p, 1 << 20, p, 64, 64, 64, allowed.ctypes.data,
                                 0, (1 << 18) + 1, 1, 0, int(pb.Rng.Saru), None)
    assert rc == _native.BFM_ETOOLARGE
    torch.cuda.synchronize()
    # a bond table that does not allow exactly 108 vectors is a bad argument
    bad = allowed.copy()
    bad[np.flatnonzero(bad)[0]] = 0
    rc = lib.bfm_substep_noalloc(p, None, p, p, 1 << 20, p, 32, 32, 32, bad.ctypes.data,
                                 0, 1000, 1, 0, int(pb.Rng.Saru), None)
    assert rc == _native.BFM_EINVAL
    # Philox is not taken by this entry point
    rc = lib.bfm_substep_noalloc(p, None, p, p, 1 << 20, p, 32, 32, 32, allowed.ctypes.data,
                                 0, 1000, 1, 0, int(pb.Rng.Philox), None)
    assert rc == _native.BFM_EINVAL
    torch.cuda.synchronize()
