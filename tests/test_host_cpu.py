"""CPU tests of the product's host side and C ABI (no GPU compute)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import pscbfm_b200 as pb
from pscbfm_b200 import _native, systems
from oracle import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")


def header_functions():
    names = []
    for h in ("pscbfm_b200.h",):
        txt = open(os.path.join(ROOT, "include", h)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names += re.findall(r"\b(bfm_\w+)\s*\(", txt)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    L = _native.lib()
    declared = header_functions()
    assert declared, "no declarations parsed"
    for name in declared:
        assert hasattr(L, name), name
    assert sorted(_native.exported_symbols()) == declared


def test_product_coloring_matches_reference_vectors():
    g = np.load(os.path.join(GOLD, "host_vectors.npz"))
    L = _native.lib()
    for idx in range(int(g["ngraphs"][0])):
        deg = g[f"g{idx}_deg"].astype(np.uint8)
        nbr = np.ascontiguousarray(g[f"g{idx}_nbr"], dtype=np.uint32)
        for uni in (0, 1):
            out = np.zeros(deg.size, np.uint32)
            k = ctypes.c_uint32()
            assert L.bfm_color_graph(deg.size, deg.ctypes.data, nbr.ctypes.data, uni, out.ctypes.data, ctypes.byref(k)) == 0
            assert k.value == int(g[f"g{idx}_u{uni}_k"][0])
            assert np.array_equal(out, g[f"g{idx}_u{uni}_colors"]), (idx, uni)


def test_product_r250_matches_oracle():
    for seed in (0, 1, 2 ** 40 + 5):
        pb.r250_seed(seed)
        st = oracle.r250_state(seed)
        assert np.array_equal(pb.r250_get_state(), st)
        want = oracle.r250_draw(st, 1000)
        got = np.array([pb.r250_rand32() for _ in range(1000)], np.uint32)
        assert np.array_equal(got, want)
    words = np.arange(1, 301, dtype=np.uint32) * 2654435761
    pb.r250_seed_words(words)
    st = oracle.r250_state_words(words[:250])
    assert np.array_equal(pb.r250_get_state(), st)
    pb.r250_set_state(st)
    assert np.array_equal(pb.r250_get_state(), st)
    with pytest.raises(ValueError):
        pb.r250_set_state(np.zeros(250, np.uint32))


def _fresh(n=4, box=(32, 32, 32)):
    u = pb.UpdaterGPUScBFM_AB_Type()
    u.setLatticeSize(*box)
    u.setNrOfAllMonomers(n)
    return u


def test_setter_errors_follow_reference_exceptions():
    u = _fresh()
    with pytest.raises(RuntimeError):          # setNrOfAllMonomers twice (.cu:2550-2556)
        u.setNrOfAllMonomers(4)
    for k in range(8):
        u.setConnectivity(0, 1)
    with pytest.raises(ValueError):            # > MAX_CONNECTIVITY (.cu:2626-2633)
        u.setConnectivity(0, 1)
    with pytest.raises(ValueError):
        u.setMonomerCoordinates(4, 0, 0, 0)
    with pytest.raises(RuntimeError):          # not a power of two (.cu:2673-2683)
        u.setLatticeSize(48, 32, 32)
    with pytest.raises(RuntimeError):
        u.setLatticeSize(2048, 32, 32)
    with pytest.raises(ValueError):
        u.setRng(9)
    with pytest.raises(RuntimeError):          # run before initialize
        u.runSimulationOnGPU(1)


def test_initialize_rejects_wrong_bond_set():
    s = systems.saw_chains(2, 4, box=(16, 16, 16), seed=1)
    u = pb.UpdaterGPUScBFM_AB_Type()
    u.setLatticeSize(*s.box)
    u.setNrOfAllMonomers(s.n)
    u.setAllMonomerCoordinates(s.pos)
    u.setAllConnectivity(s.deg, s.nbr)
    allowed = s.allowed.copy()
    allowed[np.flatnonzero(allowed)[0]] = False   # 107 allowed (.cu:1524-1533)
    u.setBondSet(allowed)
    with pytest.raises(RuntimeError, match="108"):
        u.initialize()


def test_initialize_rejects_overlap_and_bad_bonds():
    s = systems.saw_chains(2, 4, box=(16, 16, 16), seed=1)
    bad = s.pos.copy()
    bad[1] = bad[0] + np.array([1, 0, 0])       # overlapping cubes
    u = pb.UpdaterGPUScBFM_AB_Type()
    u.setLatticeSize(*s.box)
    u.setNrOfAllMonomers(s.n)
    u.setAllMonomerCoordinates(bad)
    u.setAllConnectivity(np.zeros(s.n, np.uint8), np.zeros((s.n, 8), np.uint32))
    u.setBondSet(s.allowed)
    with pytest.raises(ValueError, match="excluded volume|share"):
        u.initialize()
    far = s.pos.copy()
    far[1] = far[0] + np.array([4, 4, 4])       # bond (4,4,4) not in the set
    u2 = pb.UpdaterGPUScBFM_AB_Type()
    u2.setLatticeSize(*s.box)
    u2.setNrOfAllMonomers(s.n)
    u2.setAllMonomerCoordinates(far)
    u2.setAllConnectivity(s.deg, s.nbr)
    u2.setBondSet(s.allowed)
    with pytest.raises(ValueError, match="bond"):
        u2.initialize()


def test_cpp_dropin_header_compiles(tmp_path):
    src = tmp_path / "use.cpp"
    src.write_text(r'''
#include "UpdaterGPUScBFM_AB_Type.h"
#include <cstdio>
int main() {
    UpdaterGPUScBFM_AB_Type<uint8_t> u;
    u.setLatticeSize(32, 32, 32);
    u.setNrOfAllMonomers(2);
    try { u.setNrOfAllMonomers(2); } catch (std::runtime_error const &) { std::puts("ok"); }
    u.mLog.activate("Stats");
    u.setFilterStats(2);
    try { u.printFilterAnalysis(std::cerr); } catch (std::runtime_error const &) { std::puts("stats before init"); }
    return u.mLog.isActive("Stats") ? 0 : 1;
}
''')
    exe = tmp_path / "use"
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    "-L", os.path.dirname(_native.LIBPATH), "-lpscbfm_b200",
                    "-Wl,-rpath," + os.path.dirname(_native.LIBPATH)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    assert "ok" in out and "stats before init" in out
