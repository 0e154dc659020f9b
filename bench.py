#!/usr/bin/env python3
"""Benchmark of the ddCOSMO energy+force path on B200.

Workload (one "step"): the reference's main.f90 flow -- ddinit, mkrhs, direct
solve, energy, adjoint solve, forces_dd, ddmkzeta and the two efld
contractions -- on the 20,000-sphere globule (lmax 10, 590 Lebedev points,
eta 0.1, eps 78.3553, tol 1e-10), synthetic seeded input.  Metric: energy+force
solves per second.

* ``value``: whole-job solves/s with the inputs (charges, centres, radii)
  already resident in HBM (C ABI in device-pointer mode), timed with CUDA
  events on the library's stream, max over ranks.
* ``e2e``: the same through the C ABI with host arrays: the host->device copy
  of the inputs and the device->host copy of Esolv and the forces are inside
  the timed region.
* ``roofline``: the dominant kernel of the step, timed live inside the timed
  region with the library's CUDA-event stage timers (only that stage is
  timed there; ``stage_ms_per_step`` comes from one untimed step after the
  warm-up with every stage timed).
* ``cpu_baseline``: the CPU oracle (restatement of the reference, OpenMP over
  all host cores) on a bounded sample of the same workload, scaled to one
  solve.

Multi-GPU: the path does not shard (one molecule per GPU); ``--gpus N`` runs N
independent replicas, one per rank, and reports the aggregate ("weak").

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

WORKLOAD = 2  # 20,000 spheres, lmax 10, ngrid 590 (override: --workload)
METRIC = "energy+force solves/s"
UNIT = "solves/s"


def _workload_config():
    from ddpcm_b200 import molecules as M
    c = dict(M.CONFIGS[WORKLOAD])
    mol = M.to_bohr(M.config_molecule(WORKLOAD))
    return c, mol


def _config_json(c, nranks, extra=None):
    d = {"workload": f"globule N={c['n']} lmax={c['lmax']} ngrid={c['ngrid']} eta={c['eta']} "
                     f"tol=1e-{c['iconv']} energy+forces",
         "nsph": c["n"], "lmax": c["lmax"], "ngrid": c["ngrid"], "eta": c["eta"],
         "eps": c["eps"], "iconv": c["iconv"], "seed": c["seed"],
         "parallelism": f"replicas x{nranks}" if nranks > 1 else "single GPU",
         "l2": "working set > L2 (DIIS history ~1 GB, grid fields ~0.5 GB); no flush needed",
         "guess": "reference (facl*rhs)", "precision": "fp64"}
    if extra:
        d.update(extra)
    return d


# ---------------------------------------------------------------------------
# distributed plumbing (one process per GPU; replicas, no data collective)
# ---------------------------------------------------------------------------
def _dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        backend = os.environ.get("DDC_BENCH_BACKEND", "nccl")
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def _max_over_ranks(value, pg, device=None):
    if pg is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def _barrier(pg, device=None):
    if pg is None:
        return
    import torch
    t = torch.zeros(1, device=device)
    pg.all_reduce(t)


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# roofline bookkeeping
# ---------------------------------------------------------------------------
def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p.get("hbm_gbs", 6650.0), "measured"
    except OSError:
        return 6650.0, "fallback"


def _stage_work(stage, info, c):
    """Algorithmic FLOPs of one launch of a stage (FP64 pipe)."""
    N, NC, NY, G, T = info["nsph"], info["ncav"], info["nylm"], info["ngrid"], info["ntriples"]
    if stage == "coulomb_pot":
        return 10.0 * N * NC                    # mkrhs: 10 flops per pair
    if stage == "efield":
        return 20.0 * N * NC                    # efld: 20 flops per pair (per launch)
    if stage in ("lx_pot", "uchi_pot", "lstarx"):
        return 6.0 * NY * T                     # 4*nylm (Y t^l) + 2*nylm (contraction)
    if stage == "lx_lstarx":
        return 12.0 * NY * T                    # L and L* applications, 6*nylm each
    if stage in ("proj_gemm", "xi_gemm"):
        return 2.0 * NY * G * N
    return None


def _traffic_from_profiles(kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, if any
    (the figures there are for the 20,000-sphere workload)."""
    if WORKLOAD != 2:
        return None
    path = os.path.join(ROOT, "profiles", "dram_traffic.txt")
    try:
        for ln in open(path):
            f = ln.split()
            if len(f) >= 2 and f[0] == kernel:
                return float(f[1])
    except OSError:
        pass
    return None


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def dd_stages(stages):
    return {k: v for k, v in stages.items() if v[1] > 0}


VARIANTS = {
    # name: (precision, guess, paired direct/adjoint solves); the first is the headline
    "mixed_ref_guess": (1, 0, 1),
    "fp64_ref_guess": (0, 0, 1),
    "fp64_zero_guess": (0, 1, 1),
    "mixed_zero_guess": (1, 1, 1),
    "fp64_ref_guess_unpaired": (0, 0, 0),
    "mixed_ref_guess_unpaired": (1, 0, 0),
}


def _oracle_fixture():
    """FP64 oracle result of the benchmark workload (tests/golden/make_config2.py)."""
    if WORKLOAD != 2:
        return None
    path = os.path.join(ROOT, "tests", "golden", "config2_oracle.npz")
    try:
        return np.load(path)
    except OSError:
        return None


def measure_batch(dev, stream, precision=None):
    """The batched workload: 256 uneven globules solved in one library call
    (per-molecule Jacobi/DIIS; FP64, or the mixed refinement per molecule).
    One warm-up call, one timed call."""
    import torch
    from ddpcm_b200 import molecules as M
    from ddpcm_b200.ddcosmo import DDCosmo, PREC_FP64, PREC_MIXED
    prec = PREC_FP64 if precision is None else precision
    bc = M.BATCH_CONFIG
    mols = [M.to_bohr(m) for m in M.batch_molecules(bc["count"], bc["lo"], bc["hi"], bc["seed"])]
    with DDCosmo(lmax=bc["lmax"], ngrid=bc["ngrid"], iconv=bc["iconv"], eps=bc["eps"],
                 eta=bc["eta"], stream=stream.cuda_stream, precision=prec) as db:
        db.batch_energy_forces(mols)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = db.batch_energy_forces(mols)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1)
    it = out["iters"]
    sizes = [len(m["q"]) for m in mols]
    err = None
    try:
        gold = np.load(os.path.join(ROOT, "tests", "golden", "config3_oracle.npz"))
        e_rel, f_abs, e_big = [], [], []
        for j, k in enumerate(gold["index"]):
            k = int(k)
            ref_e = float(gold["esolv"][j])
            ref_f = gold["fx"][gold["off"][j]:gold["off"][j + 1]]
            e_rel.append(abs(out["esolv"][k] - ref_e) / abs(ref_e))
            f_abs.append(float(np.abs(out["fx"][k] - ref_f).max()))
            if gold["nsph"][j] > 60:
                e_big.append(e_rel[-1])
        err = {"esolv_rel_max": max(e_rel), "esolv_rel_max_above_60_spheres": max(e_big),
               "forces_max_abs": max(f_abs),
               "molecules_checked": len(e_rel),
               "largest_checked": int(gold["nsph"].max()),
               "against": "FP64 CPU oracle, 16 of the 256 molecules incl. the six largest "
                          "(tests/golden/config3_oracle.npz)"}
    except OSError:
        pass
    return {"workload": f"{bc['count']} globules, N log-uniform [{bc['lo']}, {bc['hi']}] "
                        f"(total {sum(sizes)} spheres), lmax={bc['lmax']} ngrid={bc['ngrid']} "
                        f"eta={bc['eta']} tol=1e-{bc['iconv']}, energy+forces, "
                        f"{'mixed' if prec == PREC_MIXED else 'FP64'}",
            "solves_per_s": bc["count"] / (ms * 1e-3), "ms_per_batch": ms,
            "iterations_direct": {"min": int(it[:, 0].min()), "median": float(np.median(it[:, 0])),
                                  "max": int(it[:, 0].max())},
            "iterations_adjoint": {"min": int(it[:, 1].min()),
                                   "median": float(np.median(it[:, 1])),
                                   "max": int(it[:, 1].max())},
            "error": err, "host_arrays": True}


def measure_learned(dev, stream, weights=None, nmol=4, n=2000):
    """Learned initial guess on held-out globules (the learned-guess
    configuration): `nmol` globules of `n` spheres at lmax 6 / 302 points,
    tol 1e-10, seeds outside the training set.  Each is solved by energy +
    forces from the FP64 zero guess (the plain method, also the accuracy
    reference), the reference guess, the learned guess (FP64 and mixed) and,
    for frame 1 of a 0.05 angstrom trajectory from the molecule, frame 0's
    solutions.  One warm-up and one timed call each, device arrays, CUDA
    events on the library's stream."""
    import torch
    from ddpcm_b200 import molecules as M
    from ddpcm_b200.ddcosmo import (GUESS_LEARNED, GUESS_REFERENCE, GUESS_USER, GUESS_ZERO,
                                    DDCosmo, GuessModel)
    from ddpcm_b200.train_guess import EVAL_SEEDS
    weights = weights or os.path.join(ROOT, "ddpcm_b200", "guess_lmax6_g302.npz")
    if not os.path.exists(weights):
        return {"unavailable": f"no trained model at {os.path.relpath(weights, ROOT)}"}
    model = GuessModel.load(weights, device=dev.index or 0)
    p = dict(lmax=6, ngrid=302, iconv=10, eps=78.3553, eta=0.1, device=dev.index or 0)
    keys = "qxyzr"
    runs = {}
    names = ("fp64_zero_guess", "fp64_ref_guess", "fp64_learned_guess", "mixed_learned_guess",
             "mixed_ref_guess", "fp64_prev_frame_guess", "mixed_prev_frame_guess")
    for k in range(nmol):
        m0, m1 = (M.to_bohr(f) for f in M.trajectory(M.make_molecule(n, EVAL_SEEDS[k]), 2,
                                                      sigma=0.05, seed=EVAL_SEEDS[k] + 77))
        nylm = 49
        d_in = {kk: torch.tensor(m1[kk], dtype=torch.float64, device=dev) for kk in keys}
        d0 = {kk: torch.tensor(m0[kk], dtype=torch.float64, device=dev) for kk in keys}
        sig = torch.zeros((n, nylm), dtype=torch.float64, device=dev)
        ss = torch.zeros_like(sig)
        fx = torch.zeros((n, 3), dtype=torch.float64, device=dev)
        prev = {}
        for prec in (0, 1):  # frame 0's solutions, the trajectory guess
            with DDCosmo(precision=prec, guess=GUESS_REFERENCE, device_pointers=1,
                         stream=stream.cuda_stream, **p) as dd:
                dd.energy_forces_ptr(*(d0[kk].data_ptr() for kk in keys), n, sig.data_ptr(),
                                     ss.data_ptr(), fx.data_ptr())
                prev[prec] = (sig.clone(), ss.clone())
        ref = None
        for name in names:
            prec = 1 if name.startswith("mixed") else 0
            guess = (GUESS_ZERO if "zero" in name else GUESS_REFERENCE if "ref_" in name else
                     GUESS_LEARNED if "learned" in name else GUESS_USER)
            with DDCosmo(precision=prec, guess=guess, device_pointers=1,
                         stream=stream.cuda_stream, **p) as dd:
                if guess == GUESS_LEARNED:
                    dd.set_guess_model(model)

                def step():
                    if guess == GUESS_USER:
                        sig.copy_(prev[prec][0])
                        ss.copy_(prev[prec][1])
                    return dd.energy_forces_ptr(*(d_in[kk].data_ptr() for kk in keys), n,
                                                sig.data_ptr(), ss.data_ptr(), fx.data_ptr())
                step()
                torch.cuda.synchronize(dev)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                info = step()
                e1.record(stream)
                torch.cuda.synchronize(dev)
                ms = e0.elapsed_time(e1)
            r = {"ms": ms, "iterations": [info["direct"]["iterations"],
                                          info["adjoint"]["iterations"]],
                 "esolv": info["esolv"], "fx": fx.cpu().numpy().copy()}
            if ref is None:
                ref = r
            r["esolv_rel_err"] = abs(r["esolv"] - ref["esolv"]) / abs(ref["esolv"])
            r["forces_max_abs_err"] = float(np.abs(r["fx"] - ref["fx"]).max())
            runs.setdefault(name, []).append(r)
    out = {"workload": f"{nmol} held-out globules of {n} spheres (seeds {EVAL_SEEDS[:nmol]}), "
                       "lmax=6 ngrid=302 eta=0.1 tol=1e-10, energy+forces, frame 1 of a "
                       "0.05 angstrom trajectory from each",
           "model": os.path.relpath(weights, ROOT), "variants": {}}
    base = sum(r["ms"] for r in runs["fp64_zero_guess"])
    for name, rs in runs.items():
        ms = sum(r["ms"] for r in rs)
        out["variants"][name] = {
            "ms_per_solve": ms / len(rs),
            "iterations_direct": [r["iterations"][0] for r in rs],
            "iterations_adjoint": [r["iterations"][1] for r in rs],
            "speedup_vs_fp64_zero_guess": base / ms,
            "esolv_rel_err_max": max(r["esolv_rel_err"] for r in rs),
            "forces_max_abs_err": max(r["forces_max_abs_err"] for r in rs),
            "against": "FP64 zero-guess GPU solve of the same frame"}
    return out


def measure_previous_frame(make, timed, d_in, keys, c, dev):
    """Trajectory guess: frame 1 of a trajectory (every centre of the workload
    moved by a Gaussian 0.05 angstrom per coordinate) solved with frame 0's
    X and S as the initial guesses (ddc_energy_forces with DDC_GUESS_USER).
    Compared with the FP64 zero-guess solve of the same frame 1, which is also
    the accuracy reference.  One warm-up and one timed step each; every step
    restores the guesses first (two device copies, inside the timed region)."""
    import torch
    from ddpcm_b200 import molecules as M
    from ddpcm_b200.ddcosmo import GUESS_USER, GUESS_ZERO
    f0, f1 = (M.to_bohr(f) for f in M.trajectory(M.config_molecule(WORKLOAD), 2, sigma=0.05,
                                                  seed=77))
    d1 = {k: torch.tensor(f1[k], dtype=torch.float64, device=dev) for k in keys}
    N = len(f1["q"])
    nylm = (c["lmax"] + 1) ** 2
    w_sig = torch.zeros((N, nylm), dtype=torch.float64, device=dev)
    w_s = torch.zeros_like(w_sig)
    fx = torch.zeros((N, 3), dtype=torch.float64, device=dev)

    def step(dd, inputs, sig0=None, s0=None):
        def run():
            if sig0 is not None:
                w_sig.copy_(sig0)
                w_s.copy_(s0)
            return dd.energy_forces_ptr(*(inputs[k].data_ptr() for k in keys), N,
                                        w_sig.data_ptr(), w_s.data_ptr(), fx.data_ptr())
        return run

    out = {}
    d0 = make(0, GUESS_ZERO, device_pointers=1)
    ms_cold, info_cold, _, _ = timed(d0, step(d0, d1), 1, 1)
    fx_ref = fx.clone()
    es_ref = info_cold["esolv"]
    out["fp64_zero_guess_frame1"] = {
        "ms_per_solve": ms_cold,
        "iterations": [info_cold["direct"]["iterations"], info_cold["adjoint"]["iterations"]]}
    d0.close()
    for name, prec in (("mixed_prev_frame_guess", 1), ("fp64_prev_frame_guess", 0)):
        dv = make(prec, GUESS_USER, device_pointers=1)
        w_sig.zero_()
        w_s.zero_()
        dv.energy_forces_ptr(*(d_in[k].data_ptr() for k in keys), N, w_sig.data_ptr(),
                             w_s.data_ptr(), fx.data_ptr())
        g_sig, g_s = w_sig.clone(), w_s.clone()
        msv, infov, _, _ = timed(dv, step(dv, d1, g_sig, g_s), 1, 1)
        out[name] = {"ms_per_solve": msv,
                     "iterations": [infov["direct"]["iterations"],
                                    infov["adjoint"]["iterations"]],
                     "refinements": [infov["direct"]["refinements"],
                                     infov["adjoint"]["refinements"]],
                     "error": {"esolv_rel": abs(infov["esolv"] - es_ref) / abs(es_ref),
                               "forces_max_abs": float((fx - fx_ref).abs().max()),
                               "against": "FP64 zero-guess GPU solve of the same frame"},
                     "speedup_vs_fp64_zero_guess": ms_cold / msv,
                     "workload": "frame 1 of a 0.05 angstrom Gaussian-step trajectory of the "
                                 "benchmark globule, frame 0's X and S as guesses"}
        dv.close()
    return out


def run_ours(args):
    import torch

    world, rank, local, pg = _dist_setup()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    from ddpcm_b200.ddcosmo import DDCosmo, fp32_peak_gflops, fp64_peak_gflops

    c, mol = _workload_config()
    stream = torch.cuda.current_stream(dev)
    keys = "qxyzr"
    d_in = {k: torch.tensor(mol[k], dtype=torch.float64, device=dev) for k in keys}
    N = len(mol["q"])
    nylm = (c["lmax"] + 1) ** 2
    d_sig = torch.zeros((N, nylm), dtype=torch.float64, device=dev)
    d_s = torch.zeros_like(d_sig)
    d_fx = torch.zeros((N, 3), dtype=torch.float64, device=dev)
    common = dict(lmax=c["lmax"], ngrid=c["ngrid"], iconv=c["iconv"], eps=c["eps"], eta=c["eta"],
                  device=local)
    ref = _oracle_fixture()

    def make(prec, guess, **kw):
        return DDCosmo(precision=prec, guess=guess, stream=stream.cuda_stream, **common, **kw)

    def timed(dd, step, warmup, steps, clocks=False):
        for _ in range(warmup):
            info = step()
        torch.cuda.synchronize(dev)
        dd.reset_stage_times()
        l0 = dd.launches
        _barrier(pg, dev)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        clk = ClockSampler(local) if clocks else None
        if clk:
            clk.__enter__()
        e0.record(stream)
        for _ in range(steps):
            info = step()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        if clk:
            clk.__exit__(None, None, None)
        _barrier(pg, dev)
        ms = _max_over_ranks(e0.elapsed_time(e1), pg, dev)
        return ms, info, (dd.launches - l0) // max(steps, 1), clk

    def accuracy(info):
        if ref is None:
            return None
        fx = d_fx.cpu().numpy()
        return {"esolv_rel": abs(info["esolv"] - float(ref["esolv"])) / abs(float(ref["esolv"])),
                "forces_max_abs": float(np.abs(fx - ref["fx"]).max()),
                "against": "FP64 CPU oracle (tests/golden/config2_oracle.npz)"}

    def dev_step(dd):
        return lambda: dd.energy_forces_ptr(*(d_in[k].data_ptr() for k in keys), N,
                                            d_sig.data_ptr(), d_s.data_ptr(), d_fx.data_ptr())

    # headline: mixed precision (FP32 operator in FP64 refinement), reference guess
    names = list(VARIANTS)
    prec, guess, paired = VARIANTS[names[0]]
    # After the warm-up, one untimed step with every stage timed gives the
    # stage breakdown and the dominant stage; the timed region then records
    # events around the dominant stage only (its live launch times feed the
    # roofline), which keeps the other stages' event records off the host
    # path between a solver step's reductions and its next launches.
    dd = make(prec, guess, device_pointers=1, timing=1, pair_solves=paired)
    step = dev_step(dd)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    dd.reset_stage_times()
    step()
    profile_stages = dd.stage_times()
    per = {k: v for k, v in profile_stages.items() if v[1] > 0 and k != "init"}
    dom = max(per, key=lambda k: per[k][0])
    dd.set_timed_stages([dom])
    ms, info, launches, clk = timed(dd, step, 0, args.steps, clocks=True)
    stages = dd.stage_times()
    acc_head = accuracy(info)
    ms_step = ms / args.steps
    value = world * args.steps / (ms * 1e-3)

    # comparison variants: one warm-up, one timed step each
    variants = {names[0]: {"ms_per_solve": ms_step,
                           "iterations": [info["direct"]["iterations"],
                                          info["adjoint"]["iterations"]],
                           "refinements": [info["direct"]["refinements"],
                                           info["adjoint"]["refinements"]],
                           "error": acc_head}}
    if not args.no_variants:
        for name in names[1:]:
            pv, gv, pp = VARIANTS[name]
            dv = make(pv, gv, device_pointers=1, pair_solves=pp)
            msv, infov, _, _ = timed(dv, dev_step(dv), 1, 1)
            variants[name] = {"ms_per_solve": msv,
                              "iterations": [infov["direct"]["iterations"],
                                             infov["adjoint"]["iterations"]],
                              "refinements": [infov["direct"]["refinements"],
                                              infov["adjoint"]["refinements"]],
                              "error": accuracy(infov)}
            dv.close()
        base = variants["fp64_zero_guess"]["ms_per_solve"]
        for v in variants.values():
            v["speedup_vs_fp64_zero_guess"] = base / v["ms_per_solve"]
        variants.update(measure_previous_frame(make, timed, d_in, keys, c, dev))

    batch = None
    if not args.no_batch and world == 1:
        from ddpcm_b200.ddcosmo import PREC_MIXED
        batch = measure_batch(dev, stream)
        batch["mixed"] = measure_batch(dev, stream, PREC_MIXED)
    learned = None
    if not args.no_variants and world == 1:
        learned = measure_learned(dev, stream)

    if args.no_e2e:
        dd.close()
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                              "ms_per_step": ms_step, "profile_run": True,
                              "stage_ms_per_step": {k: round(v[0], 3) for k, v in
                                                    dd_stages(profile_stages).items()},
                              "variants": variants,
                              "info": {k: info[k] for k in ("nsph", "ncav", "ntriples",
                                                            "npairs")}}), flush=True)
        if pg is not None:
            pg.destroy_process_group()
        return

    # end to end: host arrays in pinned memory, copies inside the timed region
    de = make(prec, guess, pair_solves=paired)
    h_in = {k: torch.tensor(mol[k], dtype=torch.float64).pin_memory() for k in keys}
    h_fx = torch.zeros((N, 3), dtype=torch.float64).pin_memory()

    def step_host():
        return de.energy_forces_ptr(*(h_in[k].data_ptr() for k in keys), N, 0, 0,
                                    h_fx.data_ptr())

    for _ in range(max(1, args.warmup // 2)):
        step_host()
    torch.cuda.synchronize(dev)
    _barrier(pg, dev)
    t0 = time.perf_counter()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(args.steps):
        step_host()
    e3.record(stream)
    torch.cuda.synchronize(dev)
    wall = time.perf_counter() - t0
    ms_e2e = max(e2.elapsed_time(e3), wall * 1e3)
    ms_e2e = _max_over_ranks(ms_e2e, pg, dev)
    e2e_value = world * args.steps / (ms_e2e * 1e-3)
    h2d = 5 * N * 8
    d2h = 3 * N * 8 + 8

    # dominant kernel and its roofline (its events in the timed region)
    dom_ms, dom_calls = stages[dom]
    work = _stage_work(dom, info, c)
    fp64 = fp64_peak_gflops(local) if rank == 0 else None
    fp32 = fp32_peak_gflops(local) if rank == 0 else None
    hbm, hbm_src = _peaks()
    avg_ms = dom_ms / dom_calls
    f32_kernel = prec == 1 and dom in ("lx_pot", "lstarx", "lx_lstarx", "lx_gather",
                                       "proj_gemm", "xi_gemm")
    peak = fp32 if f32_kernel else fp64
    roof = {"kernel": dom, "bound": "fp32" if f32_kernel else "fp64", "unit": "TFLOP/s",
            "achieved": (work / (avg_ms * 1e-3) / 1e12) if work else None,
            "peak": peak / 1e3 if peak else None,
            "peak_source": ("measured FP32 FMA probe (ddc_fp32_peak), this run" if f32_kernel
                            else "measured FP64 FMA probe (ddc_fp64_peak), this run"),
            "launch_ms": avg_ms, "launches_per_step": dom_calls / args.steps,
            "traffic": _traffic_from_profiles(dom)}
    if dom == "lx_lstarx":
        roof["note"] = ("fused L / L* pass: algorithmic flops count both operator "
                        "applications (6*nylm per triple each); the stage also holds the few "
                        "FP64 launches of the refinement steps" if prec == 1 else
                        "fused L / L* pass: algorithmic flops count both operator "
                        "applications (6*nylm per triple each)")
    if roof["achieved"] and roof["peak"]:
        roof["frac"] = roof["achieved"] / roof["peak"]
    stage_ms = {k: round(v[0], 3) for k, v in profile_stages.items() if v[1] > 0}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64 (FP32 operator inside FP64 refinement)",
            "data": "synthetic (seeded globule, PCG64)",
            "config": _config_json(c, world, {"precision": "mixed (FP32 operator, FP64 "
                                                            "refinement/DIIS/energy/forces)"}),
            "iterations": {"direct": info["direct"]["iterations"],
                           "adjoint": info["adjoint"]["iterations"]},
            "sizes": {k: info[k] for k in ("nsph", "ncav", "nylm", "ngrid", "ntriples",
                                           "npairs")},
            "esolv_hartree": info["esolv"], "error_vs_fp64_oracle": acc_head,
            "variants": variants, "batch": batch, "learned_guess": learned,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": ms_e2e / args.steps},
            "gpu_launches": launches, "stage_ms_per_step": stage_ms,
            "stage_ms_note": "one untimed step after the warm-up with every stage timed",
            "roofline": roof, "clocks": clk.summary(),
            "peaks": {"fp64_gflops_measured": fp64, "fp32_gflops_measured": fp32,
                      "hbm_gbs": hbm, "hbm_source": hbm_src}}
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(variants.get("fp64_ref_guess", variants[names[0]]),
                                            budget_s=args.cpu_budget)
    dd.close()
    de.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()


# ---------------------------------------------------------------------------
# CPU baseline: the oracle on a bounded sample of the workload
# ---------------------------------------------------------------------------
ORACLE_ITERS = None  # filled from a measured run when available


def cpu_sample(c, mol, iters, frac=64, diis_iters=32):
    """Time the oracle (OpenMP, all host threads) on a bounded sample of one
    energy+force solve and scale it to one solve.  Sample: the full ddinit;
    one lx and one lstarx application and `diis_iters` iterations of the
    reference's serial Jacobi/DIIS vector work (history copies, Gram row,
    Gauss-Jordan, extrapolation, H-norm), each scaled by the solve's iteration
    counts; mkrhs on every frac-th cavity point; forces_dd on 1/frac of the
    spheres in eight ranges spread over the molecule; both efld calls on
    1/frac of their targets."""
    from oracle import oracle as O
    t = {}
    nthreads = O.num_threads()
    d = O.RefDD(c["lmax"], c["ngrid"], c["iconv"], 1, c["eps"], c["eta"])
    t0 = time.perf_counter()
    d.init(mol["x"], mol["y"], mol["z"], mol["r"])
    t["init"] = time.perf_counter() - t0
    ccav = d.get("ccav")
    NC, N, NY = d.ncav, d.nsph, d.nylm
    sub = ccav[::frac]
    t0 = time.perf_counter()
    phi_s, psi = O.mkrhs(mol["q"], mol["x"], mol["y"], mol["z"], sub, NY)
    t["mkrhs"] = (time.perf_counter() - t0) * NC / max(len(sub), 1)
    rng = np.random.default_rng(0)
    x = rng.standard_normal((N, NY)) * 1e-3
    t0 = time.perf_counter()
    d.lx(x)
    t["lx"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    d.lstarx(x)
    t["lstarx"] = time.perf_counter() - t0
    t["diis_per_iter"] = d.diis_sample(diis_iters) / diis_iters
    phi = rng.standard_normal(NC) * 1e-2
    # the per-call set-up (xi and the expanded phi over the whole molecule)
    # is timed alone and counted once; the per-sphere work is scaled
    nr = 8 if N >= 8 * frac else 1
    width = max(1, N // (frac * nr))
    ranges = [((k * N) // nr, min(N, (k * N) // nr + width)) for k in range(nr)]
    done = sum(b - a for a, b in ranges)
    t0 = time.perf_counter()
    d.forces_dd_ranges(phi, x, x, [(0, 0)])
    t_setup = time.perf_counter() - t0
    t0 = time.perf_counter()
    d.forces_dd_ranges(phi, x, x, ranges)
    t_rg = time.perf_counter() - t0
    t["forces"] = t_setup + max(t_rg - t_setup, 0.0) * N / done
    csph = d.get("csph")
    t0 = time.perf_counter()
    O.efld(mol["q"], csph, sub)
    t["efld1"] = (time.perf_counter() - t0) * NC / max(len(sub), 1)
    zeta = rng.standard_normal(NC) * 1e-4
    n1 = max(1, N // frac)
    t0 = time.perf_counter()
    O.efld(zeta, ccav, csph[:n1])
    t["efld2"] = (time.perf_counter() - t0) * N / n1
    total = (t["init"] + t["mkrhs"] + iters[0] * t["lx"] + iters[1] * t["lstarx"]
             + (iters[0] + iters[1]) * t["diis_per_iter"] + t["forces"] + t["efld1"]
             + t["efld2"])
    return total, t, nthreads


def cpu_model_check():
    """The sampling model against a full oracle run on the same host: the
    600-sphere globule (lmax 8, 302 points) solved in full (energy, adjoint,
    forces), and the model's estimate from a sample of it."""
    from ddpcm_b200 import molecules as M
    from oracle import oracle as O
    c = M.CONFIGS[1]
    mol = M.to_bohr(M.config_molecule(1))
    t0 = time.perf_counter()
    r = O.energy_forces(mol, c["lmax"], c["ngrid"], c["iconv"], c["eps"], c["eta"])
    full = time.perf_counter() - t0
    model, _, _ = cpu_sample(c, mol, r["iters"], frac=8, diis_iters=16)
    return {"workload": "globule N=600 lmax=8 ngrid=302 (full oracle energy+forces)",
            "full_s": full, "model_s": model, "model_error": model / full - 1.0}


def cpu_baseline(variant, budget_s=None):
    c, mol = _workload_config()
    iters = _reference_iters() if WORKLOAD == 2 else tuple(variant["iterations"])
    t0 = time.perf_counter()
    total, parts, nth = cpu_sample(c, mol, iters)
    check = cpu_model_check()
    spent = time.perf_counter() - t0
    return {"value": 1.0 / total, "unit": UNIT, "cores": nth, "kind": "port",
            "sample": (f"oracle (C restatement of the reference, OpenMP {nth} threads): full "
                       f"ddinit + one lx + one lstarx + 32 iterations of the serial Jacobi/DIIS "
                       f"vector work, scaled by the reference's {iters[0]}/{iters[1]} "
                       f"iterations, + 1/64 of mkrhs, forces_dd (8 spread ranges) and both "
                       f"efld, scaled to one solve; {spent:.1f} s of CPU wall time"),
            "seconds_per_solve": total, "parts_s": {k: round(v, 4) for k, v in parts.items()},
            "model_check": check, "model_error": check["model_error"]}


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    c, mol = _workload_config()
    iters = _reference_iters()
    vals = []
    spent = []
    for k in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        total, parts, nth = cpu_sample(c, mol, iters)
        if k >= args.warmup:
            vals.append(total)
            spent.append(time.perf_counter() - t0)
    sec = statistics.mean(vals)
    value = 1.0 / sec
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded globule, PCG64)", "impl": "reference",
            "config": _config_json(c, 1),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nth, "kind": "port",
                             "sample": (f"per step: full ddinit + one lx + one lstarx + 32 "
                                        f"iterations of the serial Jacobi/DIIS vector work, "
                                        f"scaled by {iters[0]}/{iters[1]} iterations, + 1/64 of "
                                        f"mkrhs, forces_dd (8 spread ranges) and both efld, "
                                        f"scaled to one solve; {statistics.mean(spent):.1f} s "
                                        f"CPU wall per step")},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _reference_iters():
    """Jacobi/DIIS iteration counts of the reference algorithm on this workload
    (direct, adjoint): those of the stored full-size oracle run
    (tests/golden/config2_oracle.npz, the reference's algorithm in FP64 from
    the reference guess); for other workloads a typical count."""
    ref = _oracle_fixture()
    if ref is not None:
        it = ref["iters"]
        return int(it[0]), int(it[1])
    return 45, 45


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline sample")
    ap.add_argument("--cpu-budget", type=float, default=None)
    ap.add_argument("--workload", type=int, default=WORKLOAD, choices=[0, 1, 2, 9],
                    help="molecule configuration (2: the benchmark workload)")
    ap.add_argument("--no-variants", action="store_true",
                    help="skip the comparison variants (plain FP64, zero guess)")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the batched-molecules measurement")
    ap.add_argument("--no-e2e", action="store_true",
                    help="time only the device-resident step (profiling runs)")
    args = ap.parse_args()
    globals()["WORKLOAD"] = args.workload
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
