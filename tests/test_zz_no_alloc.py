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


def test_noalloc_substeps_match_run_two_calls():
    import torch

    lib = _native.lib()
    s = systems.saw_chains(30, 20, box=(32, 32, 32), seed=41)
    box = np.array(s.box)
    pb.r250_seed(17)
    u = pb.UpdaterGPUScBFM_AB_Type().setup(s, rng=pb.Rng.Saru, age=0)
    nspec = u.getNSpecies()
    orders = [u.getSpeciesOrder(sp) for sp in range(nspec)]

    # the caller's own layout: compact colour slabs in the library's slot order
    counts = [len(o) for o in orders]
    offs = np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.int64)
    npad = int(sum(counts))
    slot_of = np.empty(s.n, np.int64)
    for sp, o in enumerate(orders):
        slot_of[o] = offs[sp] + np.arange(len(o))
    pos0 = s.pos.astype(np.int64)
    wrapped = pos0 % box
    img0 = (pos0 - wrapped) // box
    codes = np.zeros(npad, np.uint32)
    codes[slot_of] = (_dilate(wrapped[:, 0]) | (_dilate(wrapped[:, 1]) << np.uint64(1))
                      | (_dilate(wrapped[:, 2]) << np.uint64(2))).astype(np.uint32)
    img = np.zeros((3, npad), np.int32)
    img[:, slot_of] = img0.T
    deg = np.zeros(npad, np.uint8)
    deg[slot_of] = s.deg
    rows = max(int(s.deg.max()), 1)
    nbr = np.zeros((rows, npad), np.uint32)
    for j in range(rows):
        has = s.deg > j
        nbr[j, slot_of[has]] = slot_of[s.nbr[has, j]]
    lat = np.zeros(32 ** 3 // 32, np.uint32)
    np.bitwise_or.at(lat, codes >> 5, (np.uint32(1) << (codes & 31)).astype(np.uint32))

    dev = torch.device("cuda", 0)
    d_pos = torch.from_numpy(codes.view(np.int32)).to(dev)
    d_img = torch.from_numpy(img).to(dev)
    d_nbr = torch.from_numpy(nbr.view(np.int32)).to(dev)
    d_deg = torch.from_numpy(deg).to(dev)
    d_lat = torch.from_numpy(lat.view(np.int32)).to(dev)
    allowed = np.ascontiguousarray(s.allowed, dtype=np.uint8)
    stream = torch.cuda.current_stream(dev)

    for call in range(2):
        st = pb.r250_get_state()
        age = u.getAge()
        u.runSimulationOnGPU(1)
        want = u.getAllMonomerPositions()
        st_after = pb.r250_get_state()
        pb.r250_set_state(st)                 # replay the draws of that MCS
        for sub in range(nspec):
            sp = pb.r250_rand32() % nspec
            seed = pb.r250_rand32()
            rc = lib.bfm_substep_noalloc(d_pos.data_ptr(), d_img.data_ptr(), d_nbr.data_ptr(), d_deg.data_ptr(), npad,
                                         d_lat.data_ptr(), 32, 32, 32, allowed.ctypes.data, int(offs[sp]),
                                         counts[sp], seed, (age + sub) & 0xFFFFFFFF, int(pb.Rng.Saru),
                                         ctypes.c_void_p(stream.cuda_stream))
            assert rc == 0
        stream.synchronize()
        assert np.array_equal(pb.r250_get_state(), st_after)
        c = d_pos.cpu().numpy().view(np.uint32)[slot_of].astype(np.uint64)
        im = d_img.cpu().numpy()[:, slot_of].T.astype(np.int64)
        got = np.stack([_undilate(c), _undilate(c >> np.uint64(1)), _undilate(c >> np.uint64(2))], axis=1) + im * box
        assert np.array_equal(got, want), f"call {call}: {int((got != want).any(axis=1).sum())} monomers differ"
        assert np.array_equal(d_lat.cpu().numpy().view(np.uint32), u.getLattice())
        assert (got != s.pos).any()


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
