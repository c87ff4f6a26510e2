"""The reference's "Stats" filter analysis (UpdaterGPUScBFM_AB_Type.cu:
kernelCountFilteredCheck :1033-1097, kernelCountFilteredPerform :1192-1216,
accumulation :2917-2936 and :3316-3330, report :3348-3387).

Per colour substep the sweep counts the moves refused by [0] the box walls,
[1] an invalid bond, [2] an occupied leading face, [3] an occupied face with
valid bonds, [4] a parallel candidate's target; per species the run reports
min, mean, standard deviation and max over its substeps.  Mode 1 counts as
the reference does: IntHash directions for filters 0-3, and filter 4 after
the move with checkFront's byte fetch on the reference's bit-packed target
lattice; mode 2 counts the moves actually made.

CPU: the oracle's mode 1 against the reference's own printed analysis
(tests/golden/filter_stats_reference.npz); its mode-2 counts add up to its
candidate and accept counters; counting changes no trajectory.  GPU: the
CUDA path against the oracle bit for bit in both modes, for every RNG and
with walls; the oracle's mode 1 against the reference build live."""
import os

import numpy as np
import pytest

import pscbfm_b200 as pb
from oracle import oracle
from pscbfm_b200 import systems

MIN, MEAN, STD, MAX, CNT = range(5)


def _sizes(o):
    return np.array([len(o.slab(sp)) for sp in range(o.nspecies())], dtype=np.float64)


def _oracle(s, rng, mode, periodic=(True, True, True), sort_every=23):
    o = oracle.Sweep(s, rng=rng, sort_every=sort_every, periodic=periodic, threads=4)
    o.set_filter_stats(mode)
    return o


def _check_totals(fs, sizes, d_att, d_cand, d_acc):
    """mode-2 counts against the counters: every attempt of a substep is
    refused by the walls, a bond, the face, or becomes a candidate; every
    candidate is accepted or refused by filter 4."""
    cnt = fs[:, 0, CNT]
    assert np.all(fs[:, :, CNT] == cnt[:, None])
    tot = lambda f: int(round(float(np.sum(fs[:, f, MEAN] * cnt))))
    assert int(round(float(np.sum(sizes * cnt)))) == d_att
    assert d_att - tot(0) - tot(1) - tot(3) == d_cand
    assert d_cand - tot(4) == d_acc
    assert np.all(fs[:, :, MIN] <= fs[:, :, MEAN] + 1e-9) and np.all(fs[:, :, MEAN] <= fs[:, :, MAX] + 1e-9)
    assert np.all(fs[:, 2, MEAN] >= fs[:, 3, MEAN])


@pytest.mark.parametrize("rng", [1, 2, 3])
@pytest.mark.parametrize("walls", [False, True])
def test_oracle_counts_add_up_to_the_counters(rng, walls):
    if walls:
        periodic = (False, True, False)
        s = systems.open_box_chains(20, 12, box=(32, 32, 32), seed=91, periodic=periodic)
    else:
        periodic = (True, True, True)
        s = systems.add_crosslinks(systems.saw_chains(30, 16, box=(32, 32, 32), seed=92), 30, seed=3)
    o = _oracle(s, rng, 2, periodic)
    st = oracle.r250_state(8)
    for nmcs in (7, 40):
        before = o.stats()
        o.run(nmcs, st)
        after = o.stats()
        fs = o.filter_stats()
        assert fs[:, 0, CNT].sum() == nmcs * o.nspecies()
        _check_totals(fs, _sizes(o), *(a - b for a, b in zip(after, before)))
        assert (fs[:, 0, MAX].max() > 0) == walls


def test_oracle_modes_agree_for_inthash_and_counting_keeps_the_trajectory():
    s = systems.saw_chains(40, 20, box=(32, 32, 32), seed=93)
    runs = {}
    for mode in (0, 1, 2):
        o = _oracle(s, 1, mode)
        o.run(30, oracle.r250_state(5))
        runs[mode] = (o.positions(), o.filter_stats() if mode else None)
    assert np.array_equal(runs[0][0], runs[1][0]) and np.array_equal(runs[0][0], runs[2][0])
    m1, m2 = runs[1][1], runs[2][1]
    assert np.array_equal(m1[:, :4], m2[:, :4])             # same directions for IntHash
    assert not np.array_equal(m1[:, 4], m2[:, 4])           # the reference's filter 4 is another count


GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "filter_stats_reference.npz")


def test_oracle_mode1_matches_the_reference_printout_fixture():
    """The reference's own printed analysis (make_golden_filter_stats.py,
    run on a B200) for IntHash, Saru and Philox systems of 2 and 3 species:
    the oracle's mode 1 reproduces every printed min, mean, stddev and max
    to the printout's six significant digits, and the same positions."""
    g = np.load(GOLD)
    for c in range(int(g["ncases"][0])):
        k = lambda key: g[f"c{c}_{key}"]
        s = systems.System(tuple(int(v) for v in k("box")), k("pos"), k("deg"), k("nbr"), k("allowed"))
        rng, sort_every = (int(v) for v in k("params"))
        st = k("r250").copy()
        o = _oracle(s, rng, 1, sort_every=sort_every)
        for j, nmcs in enumerate(k("calls")):
            o.run(int(nmcs), st)
            sizes, printed = oracle.parse_filter_analysis(str(k(f"text{j}")))
            assert sizes == [int(v) for v in _sizes(o)], str(k("name"))
            np.testing.assert_allclose(printed, o.filter_stats()[..., :4], rtol=2e-5, atol=1e-4, equal_nan=True,
                                       err_msg=f"{k('name')} call {j}")
        assert np.array_equal(o.positions(), k("out"))


GPU_CASES = {
    "crosslinked": (lambda: systems.add_crosslinks(systems.saw_chains(40, 20, box=(32, 32, 32), seed=24), 60, seed=2),
                    (True, True, True)),
    "melt_L32": (lambda: systems.ordered_melt(32), (True, True, True)),
    "walls": (lambda: systems.open_box_chains(24, 12, box=(32, 32, 32), seed=82, periodic=(False, True, False)),
              (False, True, False)),
}


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [1, 2])
@pytest.mark.parametrize("rng", [pb.Rng.IntHash, pb.Rng.Saru, pb.Rng.Philox])
@pytest.mark.parametrize("case", list(GPU_CASES))
def test_filter_stats_match_oracle(case, rng, mode):
    make, periodic = GPU_CASES[case]
    s = make()
    pb.r250_seed(31)
    st = pb.r250_get_state()
    u = pb.UpdaterGPUScBFM_AB_Type().setup(s, rng=rng, steps_between_sortings=23)
    u.setFilterStats(mode)
    o = _oracle(s, int(rng), mode, periodic)
    for nmcs in (3, 41):
        u.runSimulationOnGPU(nmcs)
        o.run(nmcs, st)
        assert np.array_equal(u.getAllMonomerPositions(), o.positions())
        got, want = u.getFilterStats(), o.filter_stats()
        np.testing.assert_array_equal(got[..., [MIN, MAX, CNT]], want[..., [MIN, MAX, CNT]])
        np.testing.assert_allclose(got[..., MEAN], want[..., MEAN], rtol=1e-12, atol=0)
        np.testing.assert_allclose(got[..., STD], want[..., STD], rtol=1e-9, atol=1e-9, equal_nan=True)
        assert got[:, 0, CNT].sum() == nmcs * u.getNSpecies()


@pytest.mark.gpu
def test_filter_stats_counts_add_up_on_the_gpu_and_the_fast_path_resumes():
    """mode 2 against the device's own counters; switching counting off
    returns to the persistent kernel on the same trajectory."""
    s = systems.add_crosslinks(systems.saw_chains(40, 20, box=(32, 32, 32), seed=24), 60, seed=2)
    pb.r250_seed(44)
    st = pb.r250_get_state()
    u = pb.UpdaterGPUScBFM_AB_Type().setup(s, rng=pb.Rng.Saru, steps_between_sortings=50)
    o = oracle.Sweep(s, rng=2, sort_every=50, threads=4)
    sizes = np.array([len(u.getSpeciesOrder(sp)) for sp in range(u.getNSpecies())], dtype=np.float64)
    for mode, nmcs in ((0, 20), (2, 60), (0, 30), (2, 5)):
        u.setFilterStats(mode)
        before = u.getCounters()
        u.runSimulationOnGPU(nmcs)
        o.run(nmcs, st)
        after = u.getCounters()
        assert np.array_equal(u.getAllMonomerPositions(), o.positions())
        if mode:
            fs = u.getFilterStats()
            assert fs[:, 0, CNT].sum() == nmcs * u.getNSpecies()   # fresh per run
            _check_totals(fs, sizes, *(a - b for a, b in zip(after, before)))


@pytest.mark.gpu
@pytest.mark.parametrize("rng", [pb.Rng.IntHash, pb.Rng.Saru])
@pytest.mark.parametrize("name", ["dense_chains", "crosslinked"])
def test_oracle_mode1_matches_the_reference_printout(name, rng):
    """The reference's own build (oracle/_ref) with its "Stats" log active
    prints the analysis; the oracle's mode-1 statistics (and so the CUDA
    path's) equal the printed values to its six significant digits."""
    if oracle.ref_gpu() is None:
        pytest.skip("oracle/_ref/libref_pscbfm.so not built")
    s = {"dense_chains": lambda: systems.saw_chains(60, 32, box=(32, 32, 32), seed=22),
         "crosslinked": GPU_CASES["crosslinked"][0]}[name]()
    pb.r250_seed(61)
    st_ref = pb.r250_get_state()
    st = st_ref.copy()
    ref = oracle.RefUpdater(s, rng=int(rng), sort_every=17)
    o = _oracle(s, int(rng), 1, sort_every=17)
    u = pb.UpdaterGPUScBFM_AB_Type().setup(s, rng=rng, steps_between_sortings=17)
    u.setFilterStats(1)
    for nmcs in (12, 30):
        text = ref.run_stats(nmcs, st_ref)
        o.run(nmcs, st)
        u.runSimulationOnGPU(nmcs)
        sizes, printed = oracle.parse_filter_analysis(text)
        want = o.filter_stats()
        assert sizes == [int(v) for v in _sizes(o)]
        np.testing.assert_allclose(printed, want[..., :4], rtol=2e-5, atol=1e-4, equal_nan=True)
        np.testing.assert_array_equal(u.getFilterStats()[..., [MIN, MAX, CNT]], want[..., [MIN, MAX, CNT]])
        assert np.array_equal(ref.positions(), o.positions())


CPP_DRIVER = r'''
#include "UpdaterGPUScBFM_AB_Type.h"
#include <cstdio>
#include <vector>
/* reads box, n, positions, bond counts, partners and the 512 allowed-bond
 * flags; sets up the drop-in like the LeMonADE adapter; runs with "Stats" */
int main(int argc, char **argv)
{
    FILE *f = std::fopen(argv[1], "rb");
    uint32_t hdr[4];
    if (std::fread(hdr, 4, 4, f) != 4) return 2;
    const uint32_t n = hdr[3];
    std::vector<int32_t> pos(3 * (size_t)n);
    std::vector<uint32_t> deg(n), nbr(8 * (size_t)n);
    std::vector<uint8_t> allowed(512);
    if (std::fread(pos.data(), 4, pos.size(), f) != pos.size() || std::fread(deg.data(), 4, n, f) != n ||
        std::fread(nbr.data(), 4, nbr.size(), f) != nbr.size() || std::fread(allowed.data(), 1, 512, f) != 512)
        return 2;
    std::fclose(f);
    bfm_r250_seed(77);
    UpdaterGPUScBFM_AB_Type<int32_t> u;
    u.setGpu(0);
    u.setRng(UpdaterGPUScBFM_AB_Type<int32_t>::Rng::Saru);
    u.setStepsBetweenSortings(17);
    u.setLatticeSize(hdr[0], hdr[1], hdr[2]);
    u.setNrOfAllMonomers(n);
    for (uint32_t i = 0; i < n; ++i) u.setMonomerCoordinates(i, pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
    for (uint32_t i = 0; i < n; ++i) u.setAttribute(i, 1);
    for (uint32_t i = 0; i < n; ++i)
        for (uint32_t j = 0; j < deg[i]; ++j) u.setConnectivity(i, nbr[8 * (size_t)i + j]);
    for (int dx = -4; dx < 4; ++dx)
        for (int dy = -4; dy < 4; ++dy)
            for (int dz = -4; dz < 4; ++dz)
                u.copyBondSet(dx, dy, dz, !allowed[(dx & 7) | ((dy & 7) << 3) | ((dz & 7) << 6)]);
    u.initialize();
    u.mLog.activate("Stats");
    u.runSimulationOnGPU(12);
    u.runSimulationOnGPU(30);
    return 0;
}
'''


@pytest.mark.gpu
def test_cpp_dropin_prints_the_reference_analysis(tmp_path):
    """A C++ program on the drop-in header with the "Stats" level active
    prints, after every run, the analysis in the reference's format; its
    numbers are the oracle's mode-1 statistics."""
    import os
    import subprocess
    from pscbfm_b200 import _native
    s = systems.saw_chains(60, 32, box=(32, 32, 32), seed=22)
    inp = tmp_path / "system.bin"
    with open(inp, "wb") as fh:
        fh.write(np.array(list(s.box) + [s.n], np.uint32).tobytes())
        fh.write(np.ascontiguousarray(s.pos, np.int32).tobytes())
        fh.write(np.ascontiguousarray(s.deg, np.uint32).tobytes())
        fh.write(np.ascontiguousarray(s.nbr, np.uint32).tobytes())
        fh.write(np.ascontiguousarray(s.allowed, np.uint8).tobytes())
    src, exe = tmp_path / "drive.cpp", tmp_path / "drive"
    src.write_text(CPP_DRIVER)
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    libdir = os.path.dirname(_native.LIBPATH)
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(root, "include"), str(src), "-o", str(exe),
                    "-L", libdir, "-lpscbfm_b200", "-Wl,-rpath," + libdir], check=True)
    run = subprocess.run([str(exe), str(inp)], capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stderr[-2000:]
    blocks = run.stderr.split("Filter analysis. Format:")[1:]
    assert len(blocks) == 2
    pb.r250_seed(77)
    st = pb.r250_get_state()
    o = _oracle(s, 2, 1, sort_every=17)
    for block, nmcs in zip(blocks, (12, 30)):
        o.run(nmcs, st)
        sizes, printed = oracle.parse_filter_analysis(block)
        assert sizes == [int(v) for v in _sizes(o)]
        np.testing.assert_allclose(printed, o.filter_stats()[..., :4], rtol=2e-5, atol=1e-4, equal_nan=True)
