#!/usr/bin/env python3
"""Golden result of the CPU oracle on the full-size workload.

The 20,000-sphere globule (seed 1002, lmax 10, 590 points, eta 0.1,
eps 78.3553, iconv 10) takes minutes on a CPU, too long for the test suite, so
the oracle's energy, iteration counts, cavity size and forces are stored here
once.  Run from the repository root:  python tests/golden/make_config2.py
"""
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from ddpcm_b200 import molecules as M  # noqa: E402
from oracle import oracle as O  # noqa: E402


def main():
    c = M.CONFIGS[2]
    m = M.to_bohr(M.config_molecule(2))
    t = time.time()
    r = O.energy_forces(m, c["lmax"], c["ngrid"], c["iconv"], c["eps"], c["eta"])
    out = os.path.join(ROOT, "tests", "golden", "config2_oracle.npz")
    np.savez_compressed(out, esolv=r["esolv"], iters=np.array(r["iters"]), ncav=r["ncav"],
                        fx=r["fx"], seconds=time.time() - t, threads=O.num_threads())
    print(out, r["esolv"], r["iters"], r["ncav"])


if __name__ == "__main__":
    main()
