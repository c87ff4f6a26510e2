"""Chain analysis on the device against the oracle's restatement of the
reference's AnalyzerMsd (src/AnalyzerMsd.tpp): chain discovery (ends in the
order met, middle floor(n/2) bonds from the first end), per-chain R_e^2
(exact integers), R_g^2 and centre of mass, and g1..g5 against a time origin
with the box centre-of-mass drift removed for more than one chain.

Tolerances: per-chain R_e^2 bit-exact (integer); R_g^2 and the centres of
mass to 1e-12 relative (the device divides exact 64-bit integer sums once,
numpy sums floats); the chain means and g1..g5 to 1e-9 relative (float64
sums in a different order)."""
import numpy as np
import pytest

import pscbfm_b200 as pb
from oracle import oracle
from pscbfm_b200 import systems

pytestmark = pytest.mark.gpu


def permuted(s, seed):
    """the same system with monomer ids shuffled (chain discovery then
    starts walks in the middle of chains)"""
    rng = np.random.default_rng(seed)
    perm = rng.permutation(s.n)            # new id of old monomer i
    inv = np.argsort(perm)
    pos = s.pos[inv]
    deg = s.deg[inv]
    nbr = np.zeros_like(s.nbr)
    for new in range(s.n):
        old = inv[new]
        for j in range(int(s.deg[old])):
            nbr[new, j] = perm[s.nbr[old, j]]
    return systems.System(s.box, pos, deg, nbr, s.allowed, [])


CASES = {
    "chains": lambda: systems.saw_chains(48, 24, box=(32, 32, 32), seed=71),
    "shuffled": lambda: permuted(systems.saw_chains(40, 17, box=(32, 32, 32), seed=72), 5),
    "one_chain": lambda: systems.saw_chains(1, 64, box=(64, 64, 64), seed=73),
    "short_chains": lambda: systems.saw_chains(200, 3, box=(32, 32, 32), seed=74),
}


def _check(obs, ref, u, rel_means=1e-9):
    assert obs["chains"] == len(ref["re2_chain"])
    re2, rg2, com = u.analyzePerChain()
    assert np.array_equal(re2, ref["re2_chain"])
    np.testing.assert_allclose(rg2, ref["rg2_chain"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(com, ref["com"], rtol=1e-12, atol=1e-9)
    assert obs["re2"] == pytest.approx(ref["re2"], rel=rel_means)
    assert obs["rg2"] == pytest.approx(ref["rg2"], rel=rel_means)
    np.testing.assert_allclose(obs["box_com"], ref["box"], rtol=1e-12, atol=1e-9)
    for a, b in zip(obs["g"], ref["g"]):
        assert a == pytest.approx(b, rel=rel_means, abs=1e-9)
    assert obs["end_autocorr"] == pytest.approx(ref["end_autocorr"], rel=1e-9, abs=1e-12)


@pytest.mark.parametrize("name", list(CASES))
def test_analyzer_matches_reference_rule(name):
    s = CASES[name]()
    pb.r250_seed(31)
    u = pb.UpdaterGPUScBFM_AB_Type().setup(s, rng=pb.Rng.Saru)
    nc = u.analyzerInit()
    first, middle, last, members = oracle.linear_chains(s.deg, s.nbr)
    assert nc == len(first)
    f, m, l = u.analyzerChainIds()
    assert np.array_equal(f, first) and np.array_equal(m, middle) and np.array_equal(l, last)

    u.runSimulationOnGPU(50)
    obs = u.analyze(set_origin=True)
    ref0 = oracle.chain_observables(u.getAllMonomerPositions(), first, middle, last, members)
    _check(obs, ref0, u)
    assert obs["g"] == [0.0] * 5
    for nmcs in (30, 200):
        u.runSimulationOnGPU(nmcs)
        obs = u.analyze()
        ref = oracle.chain_observables(u.getAllMonomerPositions(), first, middle, last, members, origin=ref0)
        _check(obs, ref, u)
        assert all(g > 0 for g in obs["g"])


def test_analyzer_rejects_branched_systems():
    s = systems.add_crosslinks(systems.saw_chains(40, 20, box=(32, 32, 32), seed=75), 10)
    u = pb.UpdaterGPUScBFM_AB_Type().setup(s, rng=pb.Rng.Saru)
    with pytest.raises(ValueError):
        u.analyzerInit()


def test_analyzer_on_the_full_melt():
    """the 256^3 melt (4096 chains x 256): device results against numpy"""
    s = systems.ordered_melt(256)
    pb.r250_seed(32)
    u = pb.UpdaterGPUScBFM_AB_Type().setup(s, rng=pb.Rng.Saru)
    assert u.analyzerInit() == 4096
    u.runSimulationOnGPU(20)
    obs0 = u.analyze(set_origin=True)
    u.runSimulationOnGPU(100)
    obs = u.analyze()
    pos = u.getAllMonomerPositions().astype(np.float64)
    c = pos.reshape(4096, 256, 3)
    re2 = ((c[:, -1] - c[:, 0]) ** 2).sum(axis=1)
    rg2 = ((c - c.mean(axis=1, keepdims=True)) ** 2).sum(axis=2).mean(axis=1)
    assert obs["re2"] == pytest.approx(re2.mean(), rel=1e-9)
    assert obs["rg2"] == pytest.approx(rg2.mean(), rel=1e-9)
    assert obs0["chains"] == 4096 and obs["g"][1] > 0
