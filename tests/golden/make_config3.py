#!/usr/bin/env python3
"""Golden results of the CPU oracle for the batched workload.

The batch is 256 globules with sphere counts log-uniform in [20, 2000]
(ddpcm_b200.molecules.batch_molecules with BATCH_CONFIG: lmax 6, 302 points,
eta 0.1, eps 78.3553, iconv 10).  Solving all of them on a CPU takes many
minutes, so the oracle's energy, iteration counts and forces are stored for
a sample of 16 molecules: the six largest (1,700-1,952 spheres) and ten
spread evenly over the size order.  Run from the repository root:
    python tests/golden/make_config3.py
"""
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from ddpcm_b200 import molecules as M  # noqa: E402
from oracle import oracle as O  # noqa: E402


def sample_indices(sizes):
    order = np.argsort(sizes, kind="stable")
    pick = list(order[-6:]) + list(order[np.linspace(0, len(order) - 7, 10).astype(int)])
    return sorted(set(int(k) for k in pick))


def main():
    c = M.BATCH_CONFIG
    mols = M.batch_molecules(count=c["count"], lo=c["lo"], hi=c["hi"], seed=c["seed"])
    sizes = np.array([m["n"] for m in mols])
    idx = sample_indices(sizes)
    t = time.time()
    esolv, iters, fx, off = [], [], [], [0]
    for k in idx:
        r = O.energy_forces(M.to_bohr(mols[k]), c["lmax"], c["ngrid"], c["iconv"], c["eps"],
                            c["eta"])
        esolv.append(r["esolv"])
        iters.append(r["iters"])
        fx.append(np.asarray(r["fx"]).reshape(-1, 3))
        off.append(off[-1] + len(fx[-1]))
        print(k, sizes[k], r["esolv"], r["iters"], flush=True)
    out = os.path.join(ROOT, "tests", "golden", "config3_oracle.npz")
    np.savez_compressed(out, index=np.array(idx), nsph=sizes[idx], esolv=np.array(esolv),
                        iters=np.array(iters), fx=np.concatenate(fx), off=np.array(off),
                        seconds=time.time() - t, threads=O.num_threads())
    print(out, len(idx), "molecules", time.time() - t, "s")


if __name__ == "__main__":
    main()
