"""The workload generators of the benchmark configurations, checked on the
host: every bond in the 108 set, no two 2x2x2 cubes overlapping, the
topology and the sizes the configurations name."""
import numpy as np
import pytest

from pscbfm_b200 import systems


def _check_valid(s):
    L = np.array(s.box)
    pos = s.pos.astype(np.int64)
    cells = np.zeros(tuple(s.box), np.uint8)
    for c in systems._CUBE:
        q = (pos + c) % L
        np.add.at(cells, (q[:, 0], q[:, 1], q[:, 2]), 1)
    assert cells.max() == 1, "excluded volume violated"
    ids = np.repeat(np.arange(s.n), 8).reshape(s.n, 8)
    has = np.arange(8)[None, :] < s.deg[:, None]
    a, b = ids[has], s.nbr[has].astype(np.int64)
    d = pos[b] - pos[a]
    assert (np.abs(d) <= 3).all()
    assert s.allowed[(d[:, 0] & 7) | ((d[:, 1] & 7) << 3) | ((d[:, 2] & 7) << 6)].all()
    # every bond listed from both ends
    fwd = set(zip(a.tolist(), b.tolist()))
    assert all((y, x) in fwd for x, y in fwd)


@pytest.mark.parametrize("L,stars", [(128, 210), (256, 1764)])
def test_star_comb_melt_is_valid(L, stars):
    s = systems.star_comb_melt(L)
    assert s.n == stars * 577
    _check_valid(s)
    assert int(s.deg.max()) == 3
    # per star: 1 core of degree 3, 24 anchors of degree 3 (the last backbone
    # monomer of each arm carries a side chain: degree 2), 24 side-chain tips
    deg = s.deg.reshape(stars, 577)
    assert (deg[:, 0] == 3).all()
    assert ((deg == 3).sum(axis=1) == 1 + 3 * 7).all()
    assert ((deg == 1).sum(axis=1) == 3 * 8).all()
    # attributes: backbone and core A (1), side chains B (2)
    attr = s.attributes.reshape(stars, 577)
    assert ((attr == 1).sum(axis=1) == 1 + 3 * 64).all()
    assert 0.46 < 8 * s.n / L ** 3 < 0.5


def test_star_comb_melt_1024_counts():
    """the C3 sizes without building the 6.7e7-monomer arrays: the same
    formula the generator uses"""
    L, A = 1024, 64
    G = L // 2
    stars = (G // 6) * (G // A) * ((2 * (L // 4)) // 3)
    assert stars == 115600 and stars * 577 == 66701200
    assert abs(8 * stars * 577 / L ** 3 - 0.497) < 1e-3


def test_star_comb_melt_is_a_forest():
    s = systems.star_comb_melt(128)
    bonds = int(s.deg.sum()) // 2
    assert bonds == s.n - 210          # one tree per star


def test_c1_chains_are_valid():
    s = systems.saw_chains(128, 64, box=(128, 128, 128), seed=12345)
    assert s.n == 8192
    _check_valid(s)
