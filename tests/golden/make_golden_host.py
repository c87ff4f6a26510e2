"""Generate tests/golden/host_vectors.npz from the reference's own code.

Runs the reference's rngs/Saru.h, rngs/Hash.h and graphColoring.tpp, compiled
from the reference sources into oracle/_ref/libref_host.so (oracle/Makefile,
target `ref`), on seeded inputs and stores inputs and outputs.  Needs the
reference tree; run from the repository root:

    make -C oracle ref && python tests/golden/make_golden_host.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle  # noqa: E402
from pscbfm_b200 import systems  # noqa: E402


def random_graph(rng, n, m):
    deg = np.zeros(n, np.uint32)
    nbr = np.zeros((n, 8), np.uint32)
    for _ in range(m):
        a, b = (int(v) for v in rng.integers(0, n, 2))
        if a == b or deg[a] >= 8 or deg[b] >= 8:
            continue
        nbr[a, deg[a]] = b
        deg[a] += 1
        nbr[b, deg[b]] = a
        deg[b] += 1
    return deg, nbr


def main():
    ref = oracle.ref_host()
    if ref is None:
        raise SystemExit("oracle/_ref/libref_host.so missing: run `make -C oracle ref` first")
    rng = np.random.default_rng(20240611)
    k = 4096
    seeds = rng.integers(0, 2 ** 32, k, dtype=np.uint64)
    iters = rng.integers(0, 2 ** 40, k, dtype=np.uint64)
    subs = rng.integers(0, 2 ** 32, k, dtype=np.uint64)
    # also the small structured corner: iteration/subsequence 0..63
    seeds[:64] = 0
    iters[:64] = np.arange(64)
    subs[:64] = np.arange(64)
    saru = np.array([ref.ref_saru(int(s), int(i), int(j)) for s, i, j in zip(seeds, iters, subs)], np.uint32)
    hsh = np.array([ref.ref_hash(int(s) & 0xFFFFFFFF, int(j)) for s, j in zip(seeds, subs)], np.uint32)

    graphs = {}
    cases = []
    for t in range(40):
        n = int(rng.integers(1, 300))
        m = int(rng.integers(0, 3 * n))
        cases.append(random_graph(rng, n, m))
    # polymer topologies: linear chains, star-combs, cross-linked chains
    s1 = systems.saw_chains(6, 20, box=(32, 32, 32), seed=5)
    s2 = systems.star_comb(3, arm_len=12, side_every=4, side_len=3, box=(32, 32, 32), seed=6)
    s3 = systems.add_crosslinks(systems.saw_chains(8, 24, box=(32, 32, 32), seed=9), 30, seed=4)
    for s in (s1, s2, s3):
        cases.append((s.deg.astype(np.uint32), s.nbr.astype(np.uint32)))
    for idx, (deg, nbr) in enumerate(cases):
        for uni in (0, 1):
            out = np.zeros(deg.size, np.uint32)
            kcol = ref.ref_graph_coloring(deg.size, deg.ctypes.data, nbr.ctypes.data, uni, out.ctypes.data)
            graphs[f"g{idx}_deg"] = deg
            graphs[f"g{idx}_nbr"] = nbr
            graphs[f"g{idx}_u{uni}_colors"] = out
            graphs[f"g{idx}_u{uni}_k"] = np.array([kcol], np.int32)
    np.savez_compressed(os.path.join(ROOT, "tests", "golden", "host_vectors.npz"),
                        saru_seed=seeds.astype(np.uint32), saru_iter=iters, saru_sub=subs.astype(np.uint32),
                        saru_out=saru, hash_out=hsh, ngraphs=np.array([len(cases)]), **graphs)
    print("wrote host_vectors.npz with", k, "RNG vectors and", len(cases), "graphs")


if __name__ == "__main__":
    main()
