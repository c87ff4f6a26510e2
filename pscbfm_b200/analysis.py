"""Polymer observables of unfolded BFM positions.

Chain-level observables as the reference's analyzer defines them
(src/AnalyzerMsd.tpp:304-421): for linear chains given as (first id, length)
the end-to-end vector, the radius of gyration, and the mean-square
displacements g1 (middle monomer), g3 (chain centre of mass) and the
first / last monomers, with the drift of the whole box's centre of mass
subtracted when there is more than one chain (AnalyzerMsd.tpp:386-390).
"""
from __future__ import annotations

import numpy as np


def chain_arrays(chains):
    first = np.array([c[0] for c in chains], dtype=np.int64)
    length = np.array([c[1] for c in chains], dtype=np.int64)
    return first, length


def re2_rg2_per_chain(pos, chains):
    """(R_e^2, R_g^2) of every chain, as float64 arrays."""
    p = np.asarray(pos, dtype=np.float64)
    first, length = chain_arrays(chains)
    if np.all(length == length[0]):
        L = int(length[0])
        idx = first[:, None] + np.arange(L)[None, :]
        c = p[idx]                                    # chains x L x 3
        re2 = ((c[:, -1] - c[:, 0]) ** 2).sum(axis=1)
        rg2 = ((c - c.mean(axis=1, keepdims=True)) ** 2).sum(axis=2).mean(axis=1)
        return re2, rg2
    re2, rg2 = [], []
    for f, L in zip(first, length):
        c = p[f:f + L]
        re2.append(((c[-1] - c[0]) ** 2).sum())
        rg2.append(((c - c.mean(axis=0)) ** 2).sum(axis=1).mean())
    return np.array(re2), np.array(rg2)


def centres(pos, chains):
    """Middle monomer, first, last monomer and centre of mass of every chain."""
    p = np.asarray(pos, dtype=np.float64)
    first, length = chain_arrays(chains)
    mid = p[first + length // 2]
    com = np.stack([p[f:f + L].mean(axis=0) for f, L in zip(first, length)])
    return {"middle": mid, "first": p[first], "last": p[first + length - 1], "com": com}


def msd(c0, c1, chains_count):
    """g1 (middle), g3 (centre of mass) between two snapshots of `centres`,
    box centre-of-mass drift removed for more than one chain."""
    drift = c1["com"].mean(axis=0) - c0["com"].mean(axis=0) if chains_count > 1 else 0.0
    out = {}
    for key, name in (("middle", "g1"), ("com", "g3"), ("first", "g_first"), ("last", "g_last")):
        d = c1[key] - c0[key] - drift
        out[name] = (d * d).sum(axis=1)
    return out
