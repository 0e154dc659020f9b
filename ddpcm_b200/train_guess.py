#!/usr/bin/env python3
"""Train the learned initial guess on solutions that the solver generates.

Data: synthetic globules (the benchmark's generator, ddpcm_b200.molecules)
with sphere counts log-uniform in [50, 1500], plus MD-like trajectories
(every frame moves each centre by a Gaussian of 0.05 angstrom per
coordinate).  Each batch of molecules is solved by the plain FP64 method
(reference guess, tol 10^-iconv) in one ddc_batch_energy_forces call; the
library then writes one training row per sphere to device memory
(ddc_guess_features / ddc_guess_targets): the sphere's right-hand side,
adjoint right-hand side, radius and 16-bin neighbour-distance histogram, and
the corrections X - facl g and S - facl psi that the network learns.

Training runs in the library (ddc_guess_train_epoch: BF16 weights, FP32
accumulation, Adam) on one GPU; torch is used only to hold the device arrays
and draw the shuffling permutation.  The trained parameters are written to an
.npz that GuessModel.load reads.

    python -m ddpcm_b200.train_guess --out ddpcm_b200/guess_lmax6_g302.npz
"""
import argparse
import json
import math
import os
import sys
import time

import numpy as np

if __package__ in (None, ""):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

from ddpcm_b200 import molecules as M  # noqa: E402
from ddpcm_b200.ddcosmo import DDCosmo, GuessModel  # noqa: E402

# seeds: training molecules and trajectories live in their own seed ranges,
# away from the benchmark's (1000-1009, 3000-3256) and the held-out
# evaluation globules (EVAL_SEEDS)
TRAIN_SEED0 = 500000
TRAJ_SEED0 = 700000
EVAL_SEEDS = (900001, 900002, 900003, 900004)


def _make(args):
    return M.make_molecule(*args)


def training_molecules(count, lo, hi, seed, procs=None):
    """`count` globules of log-uniform size in [lo, hi], generated on all host
    cores (a spawned pool, started before any GPU work)."""
    import multiprocessing as mp
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(math.log(lo), math.log(hi), size=count)).astype(int)
    jobs = [(int(n), seed + 1 + k) for k, n in enumerate(sizes)]
    with mp.get_context("spawn").Pool(procs or os.cpu_count()) as pool:
        return pool.map(_make, jobs, chunksize=8)


def collect(dd, model, mols, feats, tgts, dev):
    """Solve `mols` in one batched call and append their training rows."""
    import torch
    out = dd.batch_energy_forces([M.to_bohr(m) for m in mols])
    n = int(out["off"][-1])
    f = torch.empty((n, model.nfeat), dtype=torch.float32, device=dev)
    t = torch.empty((n, model.nout), dtype=torch.float32, device=dev)
    dd.guess_rows(f.data_ptr(), t.data_ptr())
    feats.append(f)
    tgts.append(t)
    return out["iters"]


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--lmax", type=int, default=6)
    ap.add_argument("--ngrid", type=int, default=302)
    ap.add_argument("--iconv", type=int, default=10)
    ap.add_argument("--eta", type=float, default=0.1)
    ap.add_argument("--eps", type=float, default=78.3553)
    ap.add_argument("--molecules", type=int, default=5000)
    ap.add_argument("--lo", type=int, default=50)
    ap.add_argument("--hi", type=int, default=1500)
    ap.add_argument("--trajectories", type=int, default=10)
    ap.add_argument("--frames", type=int, default=200)
    ap.add_argument("--hidden", type=int, default=256)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--per-call", type=int, default=256, help="molecules per batched solve")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--out", required=True)
    a = ap.parse_args(argv)

    t0 = time.time()
    mols = training_molecules(a.molecules, a.lo, a.hi, TRAIN_SEED0)
    import torch
    dev = torch.device("cuda", a.device)
    torch.cuda.set_device(dev)
    model = GuessModel(a.lmax, a.hidden, a.device)
    feats, tgts = [], []
    with DDCosmo(lmax=a.lmax, ngrid=a.ngrid, iconv=a.iconv, eps=a.eps, eta=a.eta,
                 device=a.device) as dd:
        dd.set_guess_model(model)  # row widths of the training data
        for k in range(0, len(mols), a.per_call):
            collect(dd, model, mols[k:k + a.per_call], feats, tgts, dev)
        rng = np.random.default_rng(TRAJ_SEED0)
        sizes = np.exp(rng.uniform(math.log(a.lo), math.log(a.hi), size=a.trajectories))
        for j, n in enumerate(sizes.astype(int)):
            frames = M.trajectory(M.make_molecule(int(n), TRAJ_SEED0 + 1 + j), a.frames,
                                  sigma=0.05, seed=TRAJ_SEED0 + 1000 + j)
            per = max(1, min(a.frames, 200000 // max(int(n), 1)))
            for k in range(0, len(frames), per):
                collect(dd, model, frames[k:k + per], feats, tgts, dev)
        dd.set_guess_model(None)
    feat = torch.cat(feats)
    tgt = torch.cat(tgts)
    del feats, tgts
    t_data = time.time() - t0
    n = feat.shape[0]
    # 5% of the rows held out for the validation loss
    perm = torch.randperm(n, device=dev, generator=torch.Generator(device=dev).manual_seed(1))
    nval = max(1, n // 20)
    val_idx, tr_idx = perm[:nval], perm[nval:]
    ftr, ttr = feat[tr_idx].contiguous(), tgt[tr_idx].contiguous()
    fva, tva = feat[val_idx].contiguous(), tgt[val_idx].contiguous()
    del feat, tgt
    ntr = ftr.shape[0]
    model.fit_scaling(ftr.data_ptr(), ttr.data_ptr(), ntr)
    model.init_random(seed=7)
    scale = torch.tensor(model.get_params()[-model.nout:], device=dev)
    gen = torch.Generator(device=dev).manual_seed(11)
    hist = []
    pred = torch.empty_like(tva)

    def val_loss():
        model.predict(fva.data_ptr(), pred.data_ptr(), fva.shape[0])
        return float(((pred - tva / scale) ** 2).mean())

    base = float(((tva / scale) ** 2).mean())  # loss of the reference guess (zero correction)
    t1 = time.time()
    for ep in range(a.epochs):
        lr = a.lr * (0.02 + 0.98 * 0.5 * (1.0 + math.cos(math.pi * ep / max(a.epochs - 1, 1))))
        order = torch.randperm(ntr, device=dev, generator=gen).to(torch.int32)
        tl = model.train_epoch(ftr.data_ptr(), ttr.data_ptr(), order.data_ptr(), ntr, a.batch, lr)
        vl = val_loss()
        hist.append((ep, lr, tl, vl))
        print(f"epoch {ep:3d} lr {lr:.2e} train {tl:.5f} val {vl:.5f} (reference guess {base:.5f})",
              flush=True)
    t_train = time.time() - t1
    meta = dict(rows=n, train_rows=ntr, val_rows=nval, epochs=a.epochs, batch=a.batch,
                lr=a.lr, molecules=a.molecules, lo=a.lo, hi=a.hi, trajectories=a.trajectories,
                frames=a.frames, ngrid=a.ngrid, iconv=a.iconv, eta=a.eta, eps=a.eps,
                data_seconds=t_data, train_seconds=t_train, val_loss=hist[-1][3],
                val_loss_reference_guess=base)
    model.save(a.out, history=np.array(hist), meta=json.dumps(meta))
    print(json.dumps(meta), flush=True)
    return meta


if __name__ == "__main__":
    main()
