"""Species colouring on the device (bfm_color_graph_device) against the
host walk that restates the reference's graphColoring: the same colours,
node for node, on linear chains, shuffled ids, branched trees (stars,
combs), isolated monomers, and crosslinked graphs whose cyclic components
go to the host walk.  A sweep set up with device colouring is bit-exact against the oracle
(which colours on the host)."""
import numpy as np
import pytest

import pscbfm_b200 as pb
from oracle import oracle
from pscbfm_b200 import systems

pytestmark = pytest.mark.gpu


def with_isolated(s, k, seed):
    """k extra unbonded monomers at free sites, at random ids"""
    rng = np.random.default_rng(seed)
    occ = set()
    for p in s.pos % np.array(s.box):
        for d in np.array(np.meshgrid([0, 1], [0, 1], [0, 1])).T.reshape(-1, 3):
            occ.add(tuple((p + d) % np.array(s.box)))
    extra = []
    while len(extra) < k:
        q = rng.integers(0, s.box, size=3)
        cells = [tuple((q + d) % np.array(s.box)) for d in np.array(np.meshgrid([0, 1], [0, 1], [0, 1])).T.reshape(-1, 3)]
        if any(c in occ for c in cells):
            continue
        occ.update(cells)
        extra.append(q)
    n0, n = s.n, s.n + k
    order = rng.permutation(n)           # new id of old monomer i (old ids n0.. are the isolated ones)
    inv = np.argsort(order)
    pos = np.concatenate([s.pos, np.array(extra, dtype=np.int32)])[inv]
    deg0 = np.concatenate([s.deg, np.zeros(k, np.uint8)])
    nbr0 = np.concatenate([s.nbr, np.zeros((k, 8), np.uint32)])
    deg = deg0[inv]
    nbr = np.zeros_like(nbr0)
    for new in range(n):
        old = inv[new]
        for j in range(int(deg0[old])):
            nbr[new, j] = order[nbr0[old, j]]
    return systems.System(s.box, pos.astype(np.int32), deg, nbr, s.allowed, [])


CASES = {
    "chains": lambda: systems.saw_chains(60, 33, box=(64, 64, 64), seed=91),
    "melt": lambda: systems.ordered_melt(64),
    "stars": lambda: systems.star_comb(6, arm_len=20, side_every=4, side_len=5, box=(64, 64, 64), seed=92),
    "isolated": lambda: with_isolated(systems.saw_chains(30, 17, box=(32, 32, 32), seed=93), 25, 94),
}


@pytest.mark.parametrize("name", list(CASES))
def test_device_colouring_equals_host_walk(name):
    s = CASES[name]()
    host, kh, _ = pb.color_graph(s.deg, s.nbr)
    dev, kd, on_dev = pb.color_graph(s.deg, s.nbr, device=True)
    assert on_dev == 1
    assert kd == kh and np.array_equal(dev, host)
    assert np.array_equal(oracle.graph_coloring(s.deg, s.nbr)[1], host)


@pytest.mark.parametrize("links", [3, 30, 400])
def test_graph_with_cycles_keeps_the_host_colours(links):
    """crosslinks close cycles in a few components (3 links: 3 of 40), in
    many (30: 14 of 34) or join everything into cyclic networks (400: 5 of
    5): tree components are coloured on the device, cyclic ones by the host
    walk, and the result equals the walk over the whole graph"""
    s = systems.add_crosslinks(systems.saw_chains(40, 20, box=(32, 32, 32), seed=95), links)
    host, kh, _ = pb.color_graph(s.deg, s.nbr)
    dev, kd, on_dev = pb.color_graph(s.deg, s.nbr, device=True)
    assert on_dev == 2 and kd == kh and np.array_equal(dev, host)
    assert np.array_equal(oracle.graph_coloring(s.deg, s.nbr)[1], host)


def test_sweep_with_device_colouring_matches_oracle():
    s = systems.star_comb(4, arm_len=24, side_every=6, side_len=6, box=(64, 64, 64), seed=96)
    pb.r250_seed(77)
    st = pb.r250_get_state()
    u = pb.UpdaterGPUScBFM_AB_Type()
    u.setColoring(1)
    u.setup(s, rng=pb.Rng.Saru)
    assert u.getColoring() == (1, True)
    o = oracle.Sweep(s, rng=2, threads=4)
    assert np.array_equal(u.getColors(), o.colors())
    for nmcs in (20, 90):
        u.runSimulationOnGPU(nmcs)
        o.run(nmcs, st)
        assert np.array_equal(u.getAllMonomerPositions(), o.positions())
