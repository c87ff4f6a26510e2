"""Generate tests/golden/sweep_vectors.npz by running the reference's own GPU
updater (src/pscbfm/UpdaterGPUScBFM_AB_Type.cu, built for sm_100a into
oracle/_ref/libref_pscbfm.so by `make -C oracle ref`) on small seeded systems.

Needs a B200.  Usage (repository root):
    python tests/golden/make_golden_sweep.py [output.npz]
The stored inputs (positions, bonds, R250 seed, RNG, age, sort cadence, MCS
per call) and the reference's unfolded positions after every call let the CPU
tests pin the oracle to the reference's kernels without a GPU.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle  # noqa: E402
from pscbfm_b200 import systems  # noqa: E402

CASES = [
    # name, system factory, rng, age, sort_every, calls, ctype
    ("chains_saru", lambda: systems.saw_chains(20, 16, box=(32, 32, 32), seed=31), 2, 0, 5000, (3, 10), 0),
    ("chains_hash", lambda: systems.saw_chains(20, 16, box=(32, 32, 32), seed=31), 1, 0, 7, (3, 10), 0),
    ("stars_saru_age", lambda: systems.star_comb(4, arm_len=12, side_every=4, side_len=3, box=(32, 32, 32), seed=32),
     2, 4998, 5000, (4, 6), 1),
    ("xlinked_saru", lambda: systems.add_crosslinks(systems.saw_chains(24, 16, box=(32, 32, 32), seed=33), 40, seed=1),
     2, 17, 5, (5, 5, 5), 0),
    ("melt32_saru", lambda: systems.ordered_melt(32), 2, 0, 5000, (20,), 2),
]


def main(out_path):
    data = {}
    for idx, (name, make, rng, age, sort_every, calls, ctype) in enumerate(CASES):
        s = make()
        st = oracle.r250_state(1000 + idx)
        data[f"c{idx}_name"] = np.array(name)
        data[f"c{idx}_box"] = np.array(s.box, np.int32)
        data[f"c{idx}_pos"] = s.pos
        data[f"c{idx}_deg"] = s.deg
        data[f"c{idx}_nbr"] = s.nbr
        data[f"c{idx}_allowed"] = s.allowed
        data[f"c{idx}_r250"] = st.copy()
        data[f"c{idx}_params"] = np.array([rng, age, sort_every, ctype], np.int64)
        data[f"c{idx}_calls"] = np.array(calls, np.int64)
        ref = oracle.RefUpdater(s, rng=rng, age=age, sort_every=sort_every, ctype=ctype)
        for k, nmcs in enumerate(calls):
            ref.run(nmcs, st)
            data[f"c{idx}_out{k}"] = ref.positions()
        data[f"c{idx}_r250_end"] = st.copy()
        print(name, "n =", s.n, "moved:", int((data[f"c{idx}_out{len(calls) - 1}"] != s.pos).any(axis=1).sum()))
    data["ncases"] = np.array([len(CASES)])
    np.savez_compressed(out_path, **data)
    print("wrote", out_path)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden", "sweep_vectors.npz"))
