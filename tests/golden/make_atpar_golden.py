"""Generate tests/golden/mgo_atpar.json: the inputs and printed results of
lapw1's radial set-up (ATPAR) and eigenvalues from the reference's shipped
MgO runs.

The WIEN2k tree ships complete MgO SCF runs under
SRC_elast/example-MgO/elast/{eos,rhomb,tetra} whose last cycle wrote the spherical
(case.vsp) and non-spherical (case.vns) potentials that its lapw1 read, and
whose lapw1 printed (case.output1_*).  The input files are kept as text
(the case-file readers of hack_wein2k_b200.case_files parse them in the
tests); of the output the script keeps the numbers lapw1 printed:

  * the searched energy parameters (E(BOTTOM), E(TOP)) and the POTENTIAL
    PARAMETERS table U(R), U'(R), DU/DE, DU'/DE, NORM-U' per l and atom
    (atpar.f:150-300), the LO coefficients A, B, C (abc.f), the Gaunt
    factors and radial integrals U V U, UE V UE, U V UE of the
    non-spherical potential (atpar.f:330-480);
  * the eigenvalues of every k-point (to 1e-7 Ry).

This script reads those text files (in the build container, where the
reference tree is mounted) and writes the extracted numbers; the tests use
only the committed JSON.  Usage:

    python tests/golden/make_atpar_golden.py /path/to/reference
"""
from __future__ import annotations

import glob
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from make_golden import parse_struct  # noqa: E402


def parse_output1_atpar(path, nat):
    """Per atom: searched energies, the POTENTIAL PARAMETERS rows (l < ltop,
    then the LO rows), LO coefficients and the non-spherical integral lines."""
    txt = open(path).read().split("\n")
    atoms = []
    j = 0
    for a in range(nat):
        while "ATOMIC SPHERE DEPENDENT PARAMETERS" not in txt[j]:
            j += 1
        j += 2
        es = []
        while "POTENTIAL PARAMETERS" not in txt[j]:
            m = re.search(r"E\(\s*(\d+)\)=\s*([-\d.]+)(?:\s+E\(BOTTOM\)=\s*([-\d.]+)\s+E\(TOP\)=\s*([-\d.]+))?",
                          txt[j])
            if m:
                es.append(dict(l=int(m.group(1)), e=float(m.group(2)),
                               bottom=float(m.group(3)) if m.group(3) else None,
                               top=float(m.group(4)) if m.group(4) else None))
            j += 1
        j += 2
        rows, locoef, ns = [], [], []
        while j < len(txt) and "NUMBER OF RADIAL INTEGRALS" not in txt[j]:
            x = txt[j]
            m = re.match(r"\s+(\d+)\s+(-?\d\.\d+E[+-]\d+)\s+(-?\d\.\d+E[+-]\d+)\s+(-?\d\.\d+E[+-]\d+)\s+"
                         r"(-?\d\.\d+E[+-]\d+)\s+(-?\d\.\d+E[+-]\d+)\s+(\d)\s+(\d)\s+(\d)", x)
            if m:
                rows.append([int(m.group(1))] + [float(m.group(q)) for q in range(2, 7)] +
                            [int(m.group(q)) for q in range(7, 10)])
            m = re.match(r"LO COEFFICIENT: l,A,B,C\s+(\d+)\s+([-\d.]+)\s+([-\d.]+)\s+([-\d.]+)", x)
            if m:
                locoef.append([int(m.group(1))] + [float(m.group(q)) for q in (2, 3, 4)])
            m = re.match(r"(lo)?\s+(-?\d+)\s+(-?\d+)\s+(-?\d+)\s+(-?\d+)\s+(-?\d+)\s+(-?\d+)\s+([-\d.]+)\s+([-\d.]+)"
                         r"(?:\s+([-\d.]+)\s+([-\d.]+)\s+([-\d.]+)\s+(\d+))?\s*$", x)
            if m and "E" not in x:
                ent = dict(lo=bool(m.group(1)), idx=[int(m.group(q)) for q in range(2, 8)],
                           gnt=[float(m.group(8)), float(m.group(9))])
                if m.group(10):
                    ent["v"] = [float(m.group(q)) for q in (10, 11, 12)]
                    ent["lm1"] = int(m.group(13))
                ns.append(ent)
            if a + 1 < nat and "ATOMIC SPHERE DEPENDENT PARAMETERS" in x:
                break
            j += 1
        atoms.append(dict(energies=es, params=rows, lo_coef=locoef, nonspherical=ns))
    return atoms


def parse_eigenvalues(paths):
    """Per k-block: the k vector as printed, 'MATRIX SIZE' and the
    eigenvalues below 'EIGENVALUES ARE:'."""
    res = []
    for p in paths:
        txt = open(p).read().split("\n")
        j = 0
        while j < len(txt):
            m = re.match(r"\s+K=\s+([-\d.]+)\s+([-\d.]+)\s+([-\d.]+)\s+\d+\s*$", txt[j])
            if m and j + 2 < len(txt) and "MATRIX SIZE" in txt[j + 1] and "EIGENVALUES ARE" in txt[j + 2]:
                size = int(re.search(r"MATRIX SIZE\s+(\d+)", txt[j + 1]).group(1))
                vals = []
                jj = j + 3
                while "EIGENVALUES BELOW" not in txt[jj]:
                    vals.extend(float(v) for v in txt[jj].split())
                    jj += 1
                res.append(dict(kprint=[float(m.group(q)) for q in (1, 2, 3)], size=size, eig=vals))
                j = jj
            j += 1
    return res


def main(ref):
    base = os.path.join(ref, "SRC_elast", "example-MgO", "elast")
    out = {"source": "SRC_elast/example-MgO/elast/{eos,rhomb,tetra} of the reference tree: the input files case.struct, "
                     "case.in1, case.klist, case.vsp, case.vns as text, and numbers printed by its lapw1 in "
                     "case.output1_*", "cases": {}}
    for case in ("eos", "rhomb", "tetra"):
        d = os.path.join(base, case)
        files = {ext: open(os.path.join(d, case + "." + ext)).read() for ext in ("struct", "in1", "klist", "vsp", "vns")}
        st = parse_struct(os.path.join(d, case + ".struct"))
        nat = len(st["atoms"])
        outs = sorted(glob.glob(os.path.join(d, case + ".output1_*")))
        atp = parse_output1_atpar(outs[0], nat)
        eig = parse_eigenvalues(outs)
        out["cases"][case] = dict(files=files, atpar=atp, eigenvalues=eig)
        print(case, "atoms", nat, "k-blocks with eigenvalues", len(eig))
    with open(os.path.join(HERE, "mgo_atpar.json"), "w") as f:
        json.dump(out, f, separators=(",", ":"))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_atpar_golden.py <reference tree root>")
    main(sys.argv[1])
