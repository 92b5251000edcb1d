"""Generate tests/golden/mgo_golden.json from the reference's shipped MgO runs.

The WIEN2k tree ships three complete MgO SCF runs under
SRC_elast/example-MgO/elast/{tetra,eos,rhomb}.  Their inputs (.struct,
.in1, .klist, .vns) and lapw1 outputs (.output1_*) are the only known
answers the reference holds for this path:

  * MATRIX SIZE per k-point      -> pins COORS + LOPW (basis construction)
  * the printed star expansion   -> pins SETWAR/STERN (WAVE members, TAUP
    of the warped interstitial     phases, WARPING = POTK * conj(TAUP))
    potential (setwar.f:88-115)

This script reads those text files once (in the build container, where the
reference tree is mounted) and writes the extracted numbers; the tests use
only the committed JSON.  Usage:

    python tests/golden/make_golden.py /path/to/reference
"""
from __future__ import annotations

import glob
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def parse_struct(path):
    lines = open(path).read().split("\n")
    lattic = lines[1][0:4].strip()
    nat = int(re.search(r"NONEQUIV\.\s*ATOMS:\s*(\d+)", lines[1]).group(1))
    a, b, c, al, be, ga = (float(lines[3][i * 10:(i + 1) * 10]) for i in range(6))
    atoms = []
    i = 4
    for _ in range(nat):
        pos = []
        x = lines[i]
        pos.append([float(x[12:22]), float(x[25:35]), float(x[38:48])])
        mult = int(lines[i + 1][15:17])
        for m in range(1, mult):
            x = lines[i + 1 + m]
            pos.append([float(x[12:22]), float(x[25:35]), float(x[38:48])])
        rl = lines[i + 1 + mult]
        name = rl[0:10].strip()
        rmt = float(re.search(r"RMT=\s*([\d.]+)", rl).group(1))
        rot = [[float(lines[i + 2 + mult + r][20 + 10 * c2:30 + 10 * c2]) for c2 in range(3)] for r in range(3)]
        atoms.append(dict(name=name, pos=pos, mult=mult, rmt=rmt, rotloc=rot))
        i += 5 + mult
    nsym = int(lines[i][0:4])
    i += 1
    ops = []
    for _ in range(nsym):
        imat, tau = [], []
        for r in range(3):
            x = lines[i + r]
            imat.append([int(x[0:2]), int(x[2:4]), int(x[4:6])])
            tau.append(float(x[6:17]))
        ops.append(dict(imat=imat, tau=tau))
        i += 4
    return dict(lattic=lattic, abc=[a, b, c], angles=[al, be, ga], atoms=atoms, symops=ops)


def parse_in1(path, nat):
    lines = [x for x in open(path).read().split("\n")]
    rkmax = float(lines[1].split()[0])
    lmax = int(lines[1].split()[1])
    lnsmax = int(lines[1].split()[2])
    i = 2
    lo = []
    for _ in range(nat):
        nlr = int(lines[i].split()[1])
        seen, los = set(), []
        for q in range(nlr):
            l = int(lines[i + 1 + q].split()[0])
            if l in seen:
                los.append(l)
            seen.add(l)
        lo.append(los)
        i += 1 + nlr
    return dict(rkmax=rkmax, lmax=lmax, lnsmax=lnsmax, lo_l=lo)


def parse_klist(path):
    out = []
    for line in open(path):
        if line.startswith("END"):
            break
        f = line[10:].split()
        out.append([int(f[0]), int(f[1]), int(f[2]), int(f[3])])
    return out


def parse_sizes(paths):
    """Per k-block of the output: the k vector, 'MATRIX SIZE' (the 2001
    build's PRTKPT printed NV there) and the solver's preceding
    'matrix size' line (NV+NLO)."""
    res = []
    for p in paths:
        txt = open(p).read().split("\n")
        last_full = None
        for j, line in enumerate(txt):
            mf = re.match(r"\s*matrix size\s+(\d+)", line)
            if mf:
                last_full = int(mf.group(1))
            m = re.match(r"\s+K=\s+([-\d.]+)\s+([-\d.]+)\s+([-\d.]+)\s+\d+\s*$", line)
            if m and j + 1 < len(txt) and "MATRIX SIZE" in txt[j + 1]:
                size = int(re.search(r"MATRIX SIZE\s+(\d+)", txt[j + 1]).group(1))
                res.append(([float(m.group(k)) for k in (1, 2, 3)], size, last_full))
                last_full = None
    return res


def parse_stars(path):
    """The star blocks SETWAR prints (setwar.f:88,113): K, IND, members."""
    txt = open(path).read().split("\n")
    stars = []
    j = 0
    while j < len(txt):
        m = re.match(r"\s+K=\s+(-?\d+)\s+(-?\d+)\s+(-?\d+)\s+IND=\s*(\d+)", txt[j])
        if m:
            k = [int(m.group(q)) for q in (1, 2, 3)]
            ind = int(m.group(4))
            mem = []
            jj = j + 1
            while jj + 1 < len(txt):
                w = re.match(r"\s+(\d+)\. WAVE=\s*(-?\d+)\s+(-?\d+)\s+(-?\d+)\s+TAUP=\s*([-\d.]+)\s+([-\d.]+)", txt[jj])
                if not w:
                    break
                wp = re.search(r"WARPING=\s*([-\d.]+)\s+([-\d.]+)", txt[jj + 1])
                mem.append(dict(wave=[int(w.group(q)) for q in (2, 3, 4)],
                                taup=[float(w.group(5)), float(w.group(6))],
                                warping=[float(wp.group(1)), float(wp.group(2))]))
                jj += 2
            stars.append(dict(k=k, ind=ind, members=mem))
            j = jj
            if len(stars) >= 9:
                break
        else:
            j += 1
    return stars


def parse_vns_interstitial(path, nmax=None):
    txt = open(path).read().split("\n")
    j = [i for i, x in enumerate(txt) if "TOTAL POTENTIAL IN INTERSTITIAL" in x][0]
    npw = int(re.search(r"NUMBER OF PW\s+(\d+)", txt[j + 2]).group(1))
    pw = []
    for x in txt[j + 3:j + 3 + npw]:
        ja, jb, jc = int(x[3:8]), int(x[8:13]), int(x[13:18])
        re_, im_ = float(x[18:37]), float(x[37:56])
        pw.append([ja, jb, jc, re_, im_])
    return pw[:nmax] if nmax else pw


def main(ref):
    base = os.path.join(ref, "SRC_elast", "example-MgO", "elast")
    out = {"source": "SRC_elast/example-MgO/elast/{tetra,eos,rhomb} of the reference tree", "cases": {}}
    for case in ("tetra", "eos", "rhomb"):
        d = os.path.join(base, case)
        st = parse_struct(os.path.join(d, case + ".struct"))
        in1 = parse_in1(os.path.join(d, case + ".in1"), len(st["atoms"]))
        kl = parse_klist(os.path.join(d, case + ".klist"))
        # the k-parallel chunk files belong to the final .struct; a stray
        # case.output1 (eos) was written at another volume
        outs = sorted(glob.glob(os.path.join(d, case + ".output1_*")))
        sizes = parse_sizes(outs)
        kmap = {}
        for (ix, iy, iz, idv) in kl:
            kmap.setdefault(tuple(round(v / idv, 5) for v in (ix, iy, iz)), (ix, iy, iz, idv))
        ks = []
        for kv, size, full in sizes:
            key = tuple(round(v, 5) for v in kv)
            hit = kmap.get(key)
            if hit is None:  # printed rounding: search the nearest
                best = min(kmap, key=lambda q: sum(abs(a - b) for a, b in zip(q, kv)))
                if sum(abs(a - b) for a, b in zip(best, kv)) < 2e-5:
                    hit = kmap[best]
            if hit is not None:
                ks.append(dict(k=list(hit), nv=size, hsrows=full))
        # unique k entries (a k-point may appear in several output files)
        seen, uniq = set(), []
        for e in ks:
            t = tuple(e["k"])
            if t not in seen:
                seen.add(t)
                uniq.append(e)
        stars = parse_stars(outs[0])
        pw = parse_vns_interstitial(os.path.join(d, case + ".vns"), nmax=len(stars) + 2)
        out["cases"][case] = dict(struct=st, in1=in1, kpoints=uniq, stars=stars, potk=pw,
                                  n_klist=len(kl))
        print(case, "k-points with sizes:", len(uniq), "of", len(kl), "stars:", len(stars))
    with open(os.path.join(HERE, "mgo_golden.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <reference tree root>")
    main(sys.argv[1])
