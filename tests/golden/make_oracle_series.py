"""Generates tests/golden/oracle_<workload>_<steps>.npz: the FP64 oracle's
probe series for a full-size benchmark workload (nlos_lbm/workloads.py), so
that the GPU tests can hold the FP32 and FP16 paths to it at full size and
full length without running the oracle (which takes minutes on the host).

    python tests/golden/make_oracle_series.py scatter 2000

The oracle is pinned to the unmodified reference by tests/test_oracle_pinning.py;
these series are its output, not the reference's.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [REPO, os.path.join(REPO, "city-scale-nlos-acoustic-engine-code_b200")]

from nlos_lbm import workloads  # noqa: E402
from oracle import OracleSolver  # noqa: E402


def main(name, steps):
    w = workloads.build(name)
    o = OracleSolver(w["cfg"], w["sources"], w["probes"], triangles=w["triangles"])
    t0 = time.time()
    o.step(steps)
    path = os.path.join(HERE, f"oracle_{name}_{steps}.npz")
    np.savez_compressed(path, probes=o.get_probes(), steps=np.array(steps), dims_halo=np.array(o.dims_halo))
    print(path, f"{time.time() - t0:.0f} s")


if __name__ == "__main__":
    main(sys.argv[1], int(sys.argv[2]))
