#!/usr/bin/env python3
"""Generate ``lebedev_orbits.inc``: the Lebedev-Laikov quadrature parameters.

The reference loads its angular grids through ``llgrid`` (llgnew.f:5-91), which
calls one ``LDnnnn`` routine per grid size (llgnew.f:682 onwards).  Each of those
routines is a flat list of symmetry orbits: it sets the orbit parameters
``A``, ``B`` (for orbit codes 4/5/6) and the weight ``V`` and then expands the
orbit with ``GEN_OH(code, ...)`` (llgnew.f:93-681).  The numbers themselves are
the published Lebedev-Laikov constants (Lebedev & Laikov, Doklady Math. 59,
1999, 477-481), so this script only *reads* them: it parses every
``Call GEN_OH`` line together with the current ``A``/``B``/``V`` values and
writes them as a C table of ``{code, a, b, v}`` records, one block per grid
size.  The orbit expansion itself (the point order inside an orbit) is
``expand_orbit`` in ``ddc_api.cu``.

The decimal literals are copied digit-for-digit (``D`` exponent replaced by
``e``), so that ``strtod`` rounds them to exactly the same doubles as the
Fortran compiler does.

Usage: python gen_lebedev_table.py <path/to/llgnew.f> <out.inc>
"""
import re
import sys

SIZES = [6, 14, 26, 38, 50, 74, 86, 110, 146, 170, 194, 230, 266, 302, 350,
         434, 590, 770, 974, 1202, 1454, 1730, 2030, 2354, 2702, 3074, 3470,
         3890, 4334, 4802, 5294, 5810]
NPTS = {1: 6, 2: 12, 3: 8, 4: 24, 5: 24, 6: 48}


def parse(path):
    text = open(path).read().splitlines()
    grids = {}
    cur = None
    state = {"A": "0.0", "B": "0.0", "V": "0.0"}
    sub_re = re.compile(r"^\s+SUBROUTINE\s+LD(\d{4})\(", re.I)
    asg_re = re.compile(r"^\s+([ABV])=([-+0-9.Dd]+)\s*$")
    call_re = re.compile(r"^\s+Call\s+GEN_OH\(\s*(\d)\s*,", re.I)
    for line in text:
        m = sub_re.match(line)
        if m:
            cur = int(m.group(1))
            grids[cur] = []
            state = {"A": "0.0", "B": "0.0", "V": "0.0"}
            continue
        if cur is None:
            continue
        m = asg_re.match(line)
        if m:
            state[m.group(1).upper()] = m.group(2).replace("D", "e").replace("d", "e")
            continue
        m = call_re.match(line)
        if m:
            grids[cur].append((int(m.group(1)), state["A"], state["B"], state["V"]))
    return grids


def main():
    src, out = sys.argv[1], sys.argv[2]
    grids = parse(src)
    lines = ["/* Generated by gen_lebedev_table.py from the Lebedev-Laikov orbit",
             " * parameters (published constants; llgnew.f LDnnnn routines).",
             " * One record per symmetry orbit: {code, a, b, v}. Do not edit. */",
             ""]
    offs, counts = [], []
    recs = []
    for n in SIZES:
        orb = grids[n]
        npts = sum(NPTS[c] for c, _, _, _ in orb)
        if npts != n:
            raise SystemExit(f"grid {n}: orbits expand to {npts} points")
        offs.append(len(recs))
        counts.append(len(orb))
        recs.extend(orb)
    lines.append(f"#define LEB_NSIZES {len(SIZES)}")
    lines.append(f"#define LEB_NORBITS {len(recs)}")
    lines.append("static const int leb_sizes[LEB_NSIZES] = {" + ", ".join(map(str, SIZES)) + "};")
    lines.append("static const int leb_orbit_off[LEB_NSIZES] = {" + ", ".join(map(str, offs)) + "};")
    lines.append("static const int leb_orbit_cnt[LEB_NSIZES] = {" + ", ".join(map(str, counts)) + "};")
    lines.append("static const struct leb_orbit_rec { int code; double a, b, v; } leb_orbits[LEB_NORBITS] = {")
    for c, a, b, v in recs:
        lines.append(f"  {{{c}, {a}, {b}, {v}}},")
    lines.append("};")
    open(out, "w").write("\n".join(lines) + "\n")


if __name__ == "__main__":
    main()
