"""Generate tests/golden/filter_stats_reference.npz: the filter analysis that
the reference's own GPU updater prints with its "Stats" log level active
(src/pscbfm/UpdaterGPUScBFM_AB_Type.cu:3348-3387), for small seeded systems.

The updater is built from the reference sources for sm_100a into
oracle/_ref/libref_pscbfm.so (`make -C oracle ref`); oracle/ref_gpu.cu
switches the log level on around one runSimulationOnGPU call and returns what
it printed.  Needs a B200.  Usage (repository root):
    python tests/golden/make_golden_filter_stats.py [output.npz]
Stored per case: the system, R250 state, RNG, sort cadence, MCS per call, and
the printed text of every call, so that CPU tests can pin the oracle's
statistics to the reference's output without a GPU.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle  # noqa: E402
from pscbfm_b200 import systems  # noqa: E402

CASES = [
    # name, system factory, rng, sort_every, calls
    ("chains_hash", lambda: systems.saw_chains(60, 32, box=(32, 32, 32), seed=22), 1, 17, (12, 30)),
    ("chains_saru", lambda: systems.saw_chains(60, 32, box=(32, 32, 32), seed=22), 2, 17, (12, 30)),
    ("xlinked_hash", lambda: systems.add_crosslinks(systems.saw_chains(40, 20, box=(32, 32, 32), seed=24), 60, seed=2),
     1, 9, (7, 25)),
    ("melt32_philox", lambda: systems.ordered_melt(32), 3, 5000, (10,)),
]


def main(out_path):
    data = {}
    for idx, (name, make, rng, sort_every, calls) in enumerate(CASES):
        s = make()
        st = oracle.r250_state(2000 + idx)
        data[f"c{idx}_name"] = np.array(name)
        data[f"c{idx}_box"] = np.array(s.box, np.int32)
        data[f"c{idx}_pos"] = s.pos
        data[f"c{idx}_deg"] = s.deg
        data[f"c{idx}_nbr"] = s.nbr
        data[f"c{idx}_allowed"] = s.allowed
        data[f"c{idx}_r250"] = st.copy()
        data[f"c{idx}_params"] = np.array([rng, sort_every], np.int64)
        data[f"c{idx}_calls"] = np.array(calls, np.int64)
        ref = oracle.RefUpdater(s, rng=rng, sort_every=sort_every)
        for k, nmcs in enumerate(calls):
            text = ref.run_stats(nmcs, st)
            data[f"c{idx}_text{k}"] = np.array(text)
            sizes, printed = oracle.parse_filter_analysis(text)
            print(name, nmcs, "MCS, groups", sizes, "filter 4 means", printed[:, 4, 1])
        data[f"c{idx}_out"] = ref.positions()
    data["ncases"] = np.array([len(CASES)])
    np.savez_compressed(out_path, **data)
    print("wrote", out_path)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden", "filter_stats_reference.npz"))
