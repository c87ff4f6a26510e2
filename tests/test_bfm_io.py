"""The .bfm / .seeds formats: Python writer -> C++ reader and writer of the
pscbfm CLI (--dry-run, no GPU) -> Python reader, and the CLI's simulation
against the Python API on the GPU."""
import os
import subprocess

import numpy as np
import pytest

import pscbfm_b200 as pb
from pscbfm_b200 import _native, bfm_io, systems


def _same(a, b):
    assert a.box == b.box
    assert np.array_equal(a.pos, b.pos)
    for i in range(a.n):
        assert sorted(a.nbr[i, : a.deg[i]].tolist()) == sorted(b.nbr[i, : b.deg[i]].tolist())
    assert np.array_equal(a.attributes, b.attributes)


def _cli():
    _native.build()
    return _native.CLI


@pytest.mark.parametrize("kind", ["chains", "stars", "crosslinked"])
def test_bfm_round_trip_through_cpp_cli(tmp_path, kind):
    s = {"chains": lambda: systems.saw_chains(12, 20, box=(32, 32, 32), seed=1),
         "stars": lambda: systems.star_comb(3, arm_len=10, side_every=3, side_len=2, box=(32, 32, 32), seed=2),
         "crosslinked": lambda: systems.add_crosslinks(systems.saw_chains(10, 12, box=(32, 32, 32), seed=3), 15)}[kind]()
    if s.attributes is None:
        s.attributes = np.ones(s.n, np.int32)
    src = tmp_path / "in.bfm"
    moved = s.pos + np.array([3, -40, 7], dtype=np.int32)   # unfolded positions outside the box
    bfm_io.write_bfm(str(src), s, [(0, s.pos), (1234, moved)])
    back, age = bfm_io.read_bfm(str(src))
    assert age == 1234
    s2 = systems.System(s.box, moved, s.deg, s.nbr, s.allowed, attributes=s.attributes)
    _same(back, s2)
    out = tmp_path / "out.bfm"
    subprocess.run([_cli(), "--dry-run", "-i", str(src), "-o", str(out)], check=True)
    back2, age2 = bfm_io.read_bfm(str(out))
    assert age2 == 1234
    _same(back2, s2)
    assert np.array_equal(back2.allowed, s.allowed)


def test_cli_rejects_missing_conformation(tmp_path):
    p = tmp_path / "bad.bfm"
    p.write_text("!number_of_monomers=2\n!box_x=32\n!box_y=32\n!box_z=32\n")
    r = subprocess.run([_cli(), "--dry-run", "-i", str(p), "-o", str(tmp_path / "o.bfm")], capture_output=True, text=True)
    assert r.returncode != 0 and "No conformation" in r.stderr


def test_seeds_round_trip(tmp_path):
    w = (np.arange(300, dtype=np.uint64) * 2654435761).astype(np.uint32)
    p = tmp_path / "x.seeds"
    bfm_io.write_seeds(str(p), w)
    assert np.array_equal(bfm_io.read_seeds(str(p)), w)


@pytest.mark.gpu
def test_cli_simulation_matches_python_api(tmp_path):
    """pscbfm -i in.bfm -e x.seeds -m 300 -s 100 -r 2 appends frames at ages
    100/200/300 (+ the start); each equals the Python API run with the same
    seeds, including the two draws the reference's main discards."""
    s = systems.saw_chains(40, 16, box=(32, 32, 32), seed=9)
    s.attributes = np.ones(s.n, np.int32)
    src, out, seeds = tmp_path / "in.bfm", tmp_path / "out.bfm", tmp_path / "x.seeds"
    bfm_io.write_bfm(str(src), s, [(0, s.pos)])
    words = (np.arange(258, dtype=np.uint64) * 40503 + 7).astype(np.uint32)
    bfm_io.write_seeds(str(seeds), words)
    subprocess.run([_cli(), "-i", str(src), "-e", str(seeds), "-o", str(out), "-m", "300", "-s", "100", "-r", "2"],
                   check=True)
    got, age = bfm_io.read_bfm(str(out))
    assert age == 300
    pb.r250_seed_words(words)
    pb.r250_rand32()
    pb.r250_rand32()
    u = pb.UpdaterGPUScBFM_AB_Type().setup(s, rng=pb.Rng.Saru)
    for _ in range(3):
        u.runSimulationOnGPU(100)
    assert np.array_equal(got.pos, u.getAllMonomerPositions())
