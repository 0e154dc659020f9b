#!/usr/bin/env python3
"""Build the golden fixtures in this folder from the reference's regression data.

The reference ships six input decks (tests/<mol>.txt, Input.txt format read by
main.f90:129-148) and the output logs of its own driver on them
(tests/<mol>.log).  This script reads both, as text, and writes one JSON file
per molecule with:

* ``params``: iprint, nproc, lmax, ngrid, iconv, igrad, eps, eta;
* ``atoms``: rows of ``q x y z r`` in angstrom, exactly as in the deck;
* ``energy_kcal``: the printed solvation energy (main.f90:190);
* ``norms_direct`` / ``norms_adjoint``: the per-iteration increment norms
  printed by jacobi_diis (jacobi_diis.f90:143-150);
* ``forces``: the final ddCOSMO forces (main.f90:270-277), when printed;
* for the iprint >= 3/4 decks, every dumped intermediate (facs, facl, basis,
  grid, weights, inl/nl, fi, ui, ccav, rhs, X, adjoint rhs, S, xi, the
  ddCOSMO-only forces and zeta), as printed by prtsph/ptcart
  (ddcosmo.f90:667-780).

Printed numbers carry 8 decimals (f14.8 / f16.8), energies 6 (f14.6) and
norms 4 significant digits, which bounds the tolerance of every check.

Run in a container that has the reference checked out:
    python tests/golden/make_golden.py /path/to/reference/tests
"""
import json
import os
import re
import sys

MOLS = ["formaldehyde", "benzene", "caffeine", "taxol", "ala25", "crambin"]
FNUM = r"[-+]?\d*\.\d+(?:[DdEe][-+]?\d+)?"


def fnum(s):
    return float(s.replace("D", "E").replace("d", "e"))


def read_deck(path):
    lines = open(path).read().splitlines()
    vals = [ln.split()[0] for ln in lines[:9]]
    params = dict(iprint=int(vals[0]), nproc=int(vals[1]), lmax=int(vals[2]), ngrid=int(vals[3]),
                  iconv=int(vals[4]), igrad=int(vals[5]), eps=float(vals[6]), eta=float(vals[7]))
    n = int(vals[8])
    atoms = [[fnum(t) for t in ln.split()[:5]] for ln in lines[9:9 + n]]
    return params, atoms


def find(lines, pat, start=0):
    for i in range(start, len(lines)):
        if pat in lines[i]:
            return i
    return -1


def parse_block_matrix(lines, start, nrow, ncol, sph):
    """Parse a prtsph (sph=True, rows 'l m v...') or ptcart (rows 'i v...')
    dump with ncol > 1 starting after the label line ``start``.  Returns
    column-major values as a list of columns, and the index after the block."""
    cols = []
    i = start + 1
    nfull = ncol - ncol % 5
    blocks = list(range(0, nfull, 5)) + [nfull]
    for b0 in blocks:
        width = 5 if b0 < nfull else ncol % 5
        i += 1  # header line with column numbers
        block = [[] for _ in range(width)]
        for _ in range(nrow):
            toks = lines[i].split()
            vals = toks[2:] if sph else toks[1:]
            assert len(vals) == width, (lines[i], width)
            for k in range(width):
                block[k].append(float(vals[k]))
            i += 1
        cols.extend(block)
    return cols, i


def parse_single(lines, start, nrow):
    vals = []
    for k in range(nrow):
        vals.append(float(lines[start + 1 + k].split()[-1]))
    return vals


def parse_forces(lines, start, n):
    return [[float(t) for t in lines[start + 2 + k].split()[1:4]] for k in range(n)]


def parse_log(path, params, n):
    lines = open(path).read().splitlines()
    out = {}
    e = find(lines, "solvation energy (kcal/mol)")
    out["energy_kcal"] = float(lines[e].split()[-1])
    norms = [(i, fnum(ln.split()[-1])) for i, ln in enumerate(lines) if "iter=" in ln]
    # direct block precedes the energy line, adjoint block follows it
    out["norms_direct"] = [v for i, v in norms if i < e]
    out["norms_adjoint"] = [v for i, v in norms if i > e]
    f = find(lines, "ddCOSMO forces (atomic units)")
    if f >= 0:
        out["forces"] = parse_forces(lines, f, n)
    iprint = params["iprint"]
    lmax = params["lmax"]
    nylm = (lmax + 1) ** 2
    ngrid = int(re.search(r"number of grid points:\s+(\d+)", "\n".join(lines)).group(1))
    out["ngrid_snapped"] = ngrid
    if iprint >= 3:
        k = find(lines, "solution to the ddCOSMO equation")
        out["X"], _ = parse_block_matrix(lines, k, nylm, n, True)
        k = find(lines, "solution to the ddCOSMO adjoint equation")
        out["S"], _ = parse_block_matrix(lines, k, nylm, n, True)
    if iprint >= 4:
        k = find(lines, "facs (column")
        out["facs"] = parse_single(lines, k, nylm)
        k = find(lines, "facl (column")
        out["facl_as_printed"] = parse_single(lines, k, nylm)  # prints facs (ddcosmo.f90:276)
        k = find(lines, "   basis")
        out["basis"], _ = parse_block_matrix(lines, k, nylm, ngrid, True)
        k = find(lines, "   grid")
        out["grid_as_printed"], _ = parse_block_matrix(lines, k, ngrid, 3, False)
        k = find(lines, "weights (column")
        out["weights"] = parse_single(lines, k, ngrid)
        k = find(lines, "inl:")
        inl = []
        j = k + 1
        while lines[j].strip():
            inl.extend(int(t) for t in lines[j].split())
            j += 1
        out["inl"] = inl
        nl = []
        for s in range(n):
            j = find(lines, "neighbours of sphere", j)
            j += 1
            while j < len(lines) and lines[j].strip() and "neighbours" not in lines[j]:
                nl.extend(int(t) for t in lines[j].split())
                j += 1
        out["nl"] = nl
        k = find(lines, "   fi")
        out["fi"], _ = parse_block_matrix(lines, k, ngrid, n, False)
        k = find(lines, "   ui")
        out["ui"], _ = parse_block_matrix(lines, k, ngrid, n, False)
        k = find(lines, "external cavity points:")
        ccav = []
        j = k + 1
        while lines[j].strip():
            ccav.append([float(t) for t in lines[j].split()[1:4]])
            j += 1
        out["ccav"] = ccav
        k = find(lines, "rhs of the ddCOSMO equation")
        out["rhs"], _ = parse_block_matrix(lines, k, nylm, n, True)
        k = find(lines, "rhs of the ddCOSMO adjoint equation")
        out["psi"], _ = parse_block_matrix(lines, k, nylm, n, True)
        k = find(lines, "   xi")
        out["xi"], _ = parse_block_matrix(lines, k, ngrid, n, False)
        k = find(lines, "ddCOSMO-only contributions to the forces")
        out["forces_dd"] = parse_forces(lines, k, n)
        k = find(lines, "   zeta")
        zcols, _ = parse_block_matrix(lines, k, ngrid, n, False)
        flat = [v for col in zcols for v in col]
        out["zeta"] = flat[: len(ccav)]  # beyond ncav the dump reads past the array
    return out


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: python make_golden.py <reference tests/ directory>")
    src = sys.argv[1]
    here = os.path.dirname(os.path.abspath(__file__))
    for mol in MOLS:
        params, atoms = read_deck(os.path.join(src, mol + ".txt"))
        res = parse_log(os.path.join(src, mol + ".log"), params, len(atoms))
        res.update(dict(name=mol, params=params, atoms=atoms,
                        source=f"tests/{mol}.txt, tests/{mol}.log"))
        with open(os.path.join(here, mol + ".json"), "w") as fh:
            json.dump(res, fh, separators=(",", ":"))
        print(mol, len(atoms), "atoms", res["energy_kcal"], "kcal/mol",
              len(res["norms_direct"]), len(res["norms_adjoint"]), "iters")


if __name__ == "__main__":
    main()
