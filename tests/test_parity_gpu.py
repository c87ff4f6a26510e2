"""GPU parity: the CUDA sweep (through the C ABI) against the CPU oracle and
against the reference's own updater built for sm_100a, bit for bit on final
positions and on the occupation lattice."""
import numpy as np
import pytest

import pscbfm_b200 as pb
from oracle import oracle
from pscbfm_b200 import systems

pytestmark = pytest.mark.gpu


def _directed(base):
    """Drop the back-pointer of a few bonds: the reference's setConnectivity
    is directed (UpdaterGPUScBFM_AB_Type.cu:2616-2634), so a bond may be
    listed on one side only; it then constrains only that side."""
    s = systems.System(base.box, base.pos.copy(), base.deg.copy(), base.nbr.copy(), base.allowed.copy())
    for i in (5, 40, 77):
        j = int(s.nbr[i, s.deg[i] - 1])
        s.deg[i] -= 1
        s.nbr[i, s.deg[i]] = 0
        assert j != i
    return s


def _systems():
    return {
        "dilute_chains": systems.saw_chains(40, 24, box=(64, 64, 64), seed=21),
        "dense_chains": systems.saw_chains(60, 32, box=(32, 32, 32), seed=22),
        "star_comb": systems.star_comb(6, arm_len=20, side_every=5, side_len=4, box=(32, 32, 32), seed=23),
        "crosslinked": systems.add_crosslinks(systems.saw_chains(40, 20, box=(32, 32, 32), seed=24), 60, seed=2),
        "melt_L32": systems.ordered_melt(32),
        "lone_monomers": systems.saw_chains(50, 1, box=(16, 16, 16), seed=25),
        "directed_bonds": _directed(systems.saw_chains(60, 32, box=(32, 32, 32), seed=26)),
    }


SYSTEMS = _systems()


def run_pair(s, rng, age, sort_every, calls, r250_seed=1234, mode=0):
    pb.r250_seed(r250_seed)
    st = pb.r250_get_state()
    u = pb.UpdaterGPUScBFM_AB_Type()
    u.setLaunchMode(mode)
    u.setup(s, gpu=0, rng=rng, age=age, steps_between_sortings=sort_every)
    o = oracle.Sweep(s, rng=int(rng), age=age, sort_every=sort_every, threads=4)
    for nmcs in calls:
        u.runSimulationOnGPU(nmcs)
        o.run(nmcs, st)
        got, want = u.getAllMonomerPositions(), o.positions()
        assert np.array_equal(got, want), f"{int((got != want).any(axis=1).sum())} monomers differ after {nmcs} MCS"
        assert np.array_equal(u.getLattice(), oracle.lattice_words(got, s.box))
    assert np.array_equal(pb.r250_get_state(), st)
    assert u.getAge() == o.age()
    return u, o


@pytest.mark.parametrize("name", list(SYSTEMS))
@pytest.mark.parametrize("rng", [pb.Rng.Saru, pb.Rng.IntHash])
def test_sweep_matches_oracle(name, rng):
    s = SYSTEMS[name]
    u, o = run_pair(s, rng, age=0, sort_every=13, calls=[1, 30, 17])
    assert np.array_equal(u.getColors(), o.colors())
    for sp in range(u.getNSpecies()):
        assert np.array_equal(u.getSpeciesOrder(sp), o.slab(sp))
    att, cand, acc = u.getCounters()
    oatt, ocand, oacc = o.stats()
    assert (att, cand, acc) == (oatt, ocand, oacc)


@pytest.mark.parametrize("age,sort_every", [(4999, 5000), (12345, 7), (3, 1), (0, 5000)])
def test_age_and_sorting_cadence(age, sort_every):
    run_pair(SYSTEMS["dense_chains"], pb.Rng.Saru, age=age, sort_every=sort_every, calls=[9, 1, 25])


@pytest.mark.parametrize("mode", [1, 2])
@pytest.mark.parametrize("name", ["crosslinked", "melt_L32", "dilute_chains"])
def test_split_kernel_paths_match_oracle(name, mode):
    """The per-substep kernels (CUDA graphs, direct launches) give the same
    trajectory as the persistent kernel and the oracle."""
    run_pair(SYSTEMS[name], pb.Rng.Saru, 0, 50, [70, 130], mode=mode)


@pytest.mark.parametrize("shape", [0, 1, 2, 3, 4, 6, 7, 8, 9, 10])
@pytest.mark.parametrize("name", ["dense_chains", "crosslinked", "star_comb", "melt_L32"])
def test_every_persistent_kernel_shape_matches_oracle(name, shape):
    """gather / stored / staged / windowed bond handling, candidate lists in
    shared or global memory, grid or cluster barriers: all bit-exact
    against the oracle."""
    s = SYSTEMS[name]
    pb.r250_seed(4321)
    st = pb.r250_get_state()
    u = pb.UpdaterGPUScBFM_AB_Type().setup(s, rng=pb.Rng.Saru, steps_between_sortings=29)
    u.setSweepShape(shape)
    assert u.getLaunchInfo()["mode"] == (shape if shape >= 6 else shape % 3)
    o = oracle.Sweep(s, rng=2, sort_every=29, threads=4)
    for nmcs in (17, 40):
        u.runSimulationOnGPU(nmcs)
        o.run(nmcs, st)
        assert np.array_equal(u.getAllMonomerPositions(), o.positions())
        assert np.array_equal(u.getLattice(), oracle.lattice_words(o.positions(), s.box))


def test_large_box_global_list_path():
    """The 512^3 melt (8.4 M monomers): too large to stage in shared memory,
    so the automatic shape uses stored codes with global candidate lists;
    size-independent properties after a short run."""
    s = systems.ordered_melt(512)
    pb.r250_seed(12)
    u = pb.UpdaterGPUScBFM_AB_Type().setup(s, rng=pb.Rng.Saru)
    info = u.getLaunchInfo()
    # the face-mask table and the bonds-first chunk (4 items x 1024 threads, 8 B each)
    assert info["mode"] == 1 and info["smem_bytes"] == 4 * 192 * 8 * 8 + 4 * 1024 * 8
    u.runSimulationOnGPU(20)
    pos = u.getAllMonomerPositions().astype(np.int64)
    assert np.array_equal(u.getLattice(), oracle.lattice_words(pos, s.box))
    att, cand, acc = u.getCounters()
    assert att == 20 * s.n and acc > 0
    w = pos % 512
    assert np.unique((w[:, 0] << 18) | (w[:, 1] << 9) | w[:, 2]).size == s.n
    for j in range(2):
        has = s.deg > j
        d = pos[s.nbr[has, j]] - pos[np.arange(s.n)[has]]
        assert s.allowed[(d[:, 0] & 7) | ((d[:, 1] & 7) << 3) | ((d[:, 2] & 7) << 6)].all()


def test_large_box_bonds_first_chunks_bit_exact():
    """The 512^3 melt on the stored-code kernel: 28,000 items per CTA and
    colour, so its bonds-first check runs seven chunks per substep with the
    two alternating counters; bit-exact against the oracle."""
    s = systems.ordered_melt(512)
    pb.r250_seed(77)
    st = pb.r250_get_state()
    u = pb.UpdaterGPUScBFM_AB_Type().setup(s, rng=pb.Rng.Saru)
    assert u.getLaunchInfo()["mode"] == 1
    o = oracle.Sweep(s, rng=2, threads=8)
    for nmcs in (2, 1):
        u.runSimulationOnGPU(nmcs)
        o.run(nmcs, st)
        got = u.getAllMonomerPositions()
        assert np.array_equal(got, o.positions())
        assert np.array_equal(u.getLattice(), oracle.lattice_words(got, s.box))


def test_windowed_bonds_first_several_blocks_per_warp():
    """Shape 8 on 30,000 lone monomers (no bonds: every item passes the bond
    test): about 200 list entries per CTA of 64 threads, so each warp takes
    several blocks of 64 in the face pass; bit-exact against the oracle."""
    s = systems.saw_chains(30000, 1, box=(128, 128, 128), seed=31)
    pb.r250_seed(78)
    st = pb.r250_get_state()
    u = pb.UpdaterGPUScBFM_AB_Type().setup(s, rng=pb.Rng.Saru, steps_between_sortings=11)
    u.setSweepShape(8)
    info = u.getLaunchInfo()
    assert info["mode"] == 8 and info["threads"] == 64
    o = oracle.Sweep(s, rng=2, sort_every=11, threads=4)
    for nmcs in (7, 20):
        u.runSimulationOnGPU(nmcs)
        o.run(nmcs, st)
        got = u.getAllMonomerPositions()
        assert np.array_equal(got, o.positions())
        assert np.array_equal(u.getLattice(), oracle.lattice_words(got, s.box))


def test_launch_paths_agree_and_can_be_switched():
    s = SYSTEMS["crosslinked"]
    out = []
    for mode in (0, 1, 2):
        a, _ = run_pair(s, pb.Rng.Saru, 0, 50, [200], mode=mode)
        out.append(a.getAllMonomerPositions())
    assert np.array_equal(out[0], out[1]) and np.array_equal(out[0], out[2])
    # switching paths between calls on one handle keeps the trajectory
    pb.r250_seed(1234)
    st = pb.r250_get_state()
    u = pb.UpdaterGPUScBFM_AB_Type().setup(s, rng=pb.Rng.Saru, steps_between_sortings=50)
    o = oracle.Sweep(s, rng=2, sort_every=50, threads=4)
    for mode, nmcs in ((0, 30), (2, 20), (1, 70), (0, 45)):
        u.setLaunchMode(mode)
        u.runSimulationOnGPU(nmcs)
        o.run(nmcs, st)
        assert np.array_equal(u.getAllMonomerPositions(), o.positions())


def test_timed_run_keeps_trajectory():
    """bfm_time_kernels advances the system exactly like bfm_run."""
    s = SYSTEMS["dense_chains"]
    pb.r250_seed(3)
    st = pb.r250_get_state()
    u = pb.UpdaterGPUScBFM_AB_Type().setup(s, rng=pb.Rng.Saru)
    o = oracle.Sweep(s, rng=2, threads=4)
    ms, launches, attempts = u.timeKernels(40)
    o.run(40, st)
    assert np.array_equal(u.getAllMonomerPositions(), o.positions())
    assert ms > 0 and launches >= 1 and attempts == 40 * s.n


def test_barrier_wait_is_bounded_and_reported():
    """Failure detection without a GPU fault: a grid barrier that expects one
    CTA more than exists can never complete; every wait must give up after
    its bound, the call must report BFM_ETIMEOUT, and the context must stay
    usable (a normal sweep afterwards is still bit-exact)."""
    import ctypes
    from pscbfm_b200 import _native
    lib = _native.lib()
    ms = ctypes.c_double()
    assert lib.bfm_barrier_selftest(0, 200, 0, 64, ctypes.byref(ms)) == _native.BFM_OK
    assert lib.bfm_barrier_selftest(0, 100, 1, 4, ctypes.byref(ms)) == _native.BFM_ETIMEOUT
    assert 50.0 < ms.value < 5000.0
    run_pair(SYSTEMS["dense_chains"], pb.Rng.Saru, 0, 13, [10])


def test_three_colours_present():
    u, _ = run_pair(SYSTEMS["crosslinked"], pb.Rng.Saru, 0, 5000, [3])
    assert u.getNSpecies() >= 3


def test_wrapping_and_image_counters():
    """Long dilute run: monomers cross the periodic box many times; the
    unfolded positions still match the oracle."""
    s = systems.saw_chains(8, 4, box=(8, 8, 8), seed=5)
    u, o = run_pair(s, pb.Rng.Saru, 0, 100, [500, 500])
    pos = u.getAllMonomerPositions()
    assert (np.abs(pos) >= 8).any()


REF_CASES = [
    ("dilute_chains", 0), ("dense_chains", 0), ("crosslinked", 0), ("melt_L32", 0), ("star_comb", 1),
    ("dense_chains", 1),
]


@pytest.mark.parametrize("name,ctype", REF_CASES)
@pytest.mark.parametrize("rng", [pb.Rng.Saru, pb.Rng.IntHash])
def test_sweep_matches_reference_build(name, ctype, rng):
    """The reference's own UpdaterGPUScBFM_AB_Type<T> (oracle/_ref), driven
    with the same R250 stream: positions after each call must be identical
    to the product's and to the oracle's."""
    if oracle.ref_gpu() is None:
        pytest.skip("oracle/_ref/libref_pscbfm.so not built")
    s = SYSTEMS[name]
    pb.r250_seed(77)
    st_ref = pb.r250_get_state()
    u, o = run_pair(s, rng, age=0, sort_every=11, calls=[5, 20], r250_seed=77)
    ref = oracle.RefUpdater(s, rng=int(rng), age=0, sort_every=11, ctype=ctype)
    ref.run(5, st_ref)
    ref.run(20, st_ref)
    assert np.array_equal(ref.positions(), o.positions())
    assert np.array_equal(ref.positions(), u.getAllMonomerPositions())


def test_full_size_melt_properties():
    """The 256^3 melt (1,048,576 monomers): size-independent properties after
    a short run -- lattice equals the positions' lattice, bonds stay in the
    set, no two corners coincide, a second identical run is identical."""
    s = systems.ordered_melt(256)
    outs = []
    for _ in range(2):
        pb.r250_seed(9)
        u = pb.UpdaterGPUScBFM_AB_Type().setup(s, rng=pb.Rng.Saru)
        u.runSimulationOnGPU(200)
        pos = u.getAllMonomerPositions()
        outs.append(pos)
        assert np.array_equal(u.getLattice(), oracle.lattice_words(pos, s.box))
        att, cand, acc = u.getCounters()
        assert att == 200 * s.n and acc > 0
    assert np.array_equal(outs[0], outs[1])
    pos = outs[0].astype(np.int64)
    ids = np.arange(s.n)
    for j in range(2):
        has = s.deg > j
        d = pos[s.nbr[has, j]] - pos[ids[has]]
        assert np.all(np.abs(d) <= 3)
        assert s.allowed[(d[:, 0] & 7) | ((d[:, 1] & 7) << 3) | ((d[:, 2] & 7) << 6)].all()
    w = pos % 256
    codes = w[:, 0] * 65536 + w[:, 1] * 256 + w[:, 2]
    assert np.unique(codes).size == s.n


@pytest.mark.parametrize("name", ["melt_L32", "dense_chains", "star_comb"])
def test_shape_autotuner_keeps_the_trajectory(name):
    """the autotuner's trial launches (every shape that fits, each on a share
    of the first chunk) are part of the run: positions stay bit-exact
    against the oracle, and the tuner reports its trials and a choice"""
    s = SYSTEMS[name]
    pb.r250_seed(99)
    st = pb.r250_get_state()
    u = pb.UpdaterGPUScBFM_AB_Type().setup(s, rng=pb.Rng.Saru, steps_between_sortings=40)
    u.setSweepAutotune(True)
    o = oracle.Sweep(s, rng=2, sort_every=40, threads=4)
    for nmcs in (60, 25):
        u.runSimulationOnGPU(nmcs)
        o.run(nmcs, st)
        assert np.array_equal(u.getAllMonomerPositions(), o.positions())
        assert np.array_equal(u.getLattice(), oracle.lattice_words(o.positions(), s.box))
    info = u.getSweepTuning()
    assert info["tuned"] and len(info["trials"]) >= 3
    assert all(t["ns_per_move"] > 0 for t in info["trials"])
    assert u.getLaunchInfo()["mode"] in {t["shape"] for t in info["trials"]}


def test_positions_into_page_locked_buffer():
    """a page-locked output buffer is filled by one device-to-host copy;
    the positions equal those of the staging path and of the per-index
    getters, before and after further runs"""
    import torch
    s = SYSTEMS["dense_chains"]
    pb.r250_seed(77)
    u = pb.UpdaterGPUScBFM_AB_Type().setup(s, rng=pb.Rng.Saru)
    pinned_t = torch.empty((s.n, 3), dtype=torch.int32, pin_memory=True)
    pinned = pinned_t.numpy()
    for nmcs in (10, 25):
        u.runSimulationOnGPU(nmcs)
        pinned[:] = -1
        got = u.getAllMonomerPositions(out=pinned)
        assert got is pinned
        want = u.getAllMonomerPositions()
        assert np.array_equal(pinned, want)
        assert [u.getMonomerPositionInX(7), u.getMonomerPositionInY(7), u.getMonomerPositionInZ(7)] == list(want[7])
    with pytest.raises(ValueError):
        u.getAllMonomerPositions(out=np.empty((s.n, 2), np.int32))
