"""Readers of the WIEN2k case files that lapw1 reads before the matrix setup.

The drop-in takes the radial parameters, potentials and basis as plain
arrays (include/lapw1gpu.h); a host that is not lapw1 itself builds them
from the same files lapw1 reads.  These readers follow the reference's
fixed formats:

  read_struct  case.struct   inilpw.f:230-300 (formats 5000-5060),
                              latgen.f:311-315 (symmetry operations)
  read_in1     case.in1      inilpw.f:302-332, atpar.f:130-208
                              (format 5000 of atpar.f)
  read_vsp     case.vsp      atpar.f:86-99: r V_00(r) per atom, Rydberg
  read_vns     case.vns      atpar.f:345-372 (MT parts, format 5040),
                              rdswar.f:19-30 (interstitial plane waves)
  read_klist   case.klist    inilpw.f:409-420 (format 5100)

Every reader takes the file's text (so that callers and tests need not
touch the file system) and returns plain Python / numpy values.
"""
from __future__ import annotations

import re
from dataclasses import dataclass, field
from typing import List

import numpy as np


def _f(s: str) -> float:
    """A Fortran F/E field: blanks around the number, D exponents allowed."""
    s = s.strip().replace("D", "E").replace("d", "e")
    return float(s) if s else 0.0


def _i(s: str) -> int:
    s = s.strip()
    return int(s) if s else 0


@dataclass
class StructAtom:
    name: str
    iatnr: int                 # > 0: cubic site (cubic harmonics, CBCOMB)
    pos: np.ndarray            # [mult, 3] fractional
    jrj: int                   # radial mesh points (NPT)
    r0: float
    rmt: float                 # as recomputed from the mesh (inilpw.f:290)
    dx: float                  # logarithmic step DH
    z: float
    rotloc: np.ndarray         # C view [col][row] of ROTLOC(3,3)

    @property
    def mult(self) -> int:
        return int(self.pos.shape[0])


@dataclass
class Struct:
    title: str
    lattic: str
    rel: bool
    abc: tuple
    angles: tuple              # degrees
    atoms: List[StructAtom]
    imat: np.ndarray           # [nsym][line r][col c] as written: IMAT(c+1, r+1)
    tau: np.ndarray            # [nsym][3]


_FNUM = r"(-?\d*\.?\d+(?:[EeDd][+-]?\d+)?)"


def read_struct(text: str) -> Struct:
    """The fields of inilpw.f's formats 5010-5060, read by label rather
    than by column: the files of older WIEN2k versions (the reference's
    shipped MgO runs write 'ATOM=  1: X=...' and 'ATOMS: 2') shift the
    columns those formats name."""
    L = text.split("\n")
    title = L[0].rstrip()
    lattic = L[1][0:4].strip()
    nat = int(re.search(r"ATOMS\s*:?\s*(\d+)", L[1]).group(1))
    m = re.search(r"MODE OF CALC\s*=\s*(\w+)", L[2])
    irel = m.group(1) if m else "RELA"
    vals = [_f(L[3][10 * q:10 * (q + 1)]) for q in range(6)]
    abc = tuple(vals[:3])
    angles = tuple(v if v != 0.0 else 90.0 for v in vals[3:])

    def atom_line(x):
        iat = int(re.search(r"ATOM\s*=?\s*(-?\d+)", x).group(1))
        xyz = [_f(re.search(c + r"\s*=\s*" + _FNUM, x).group(1)) for c in ("X", "Y", "Z")]
        return iat, xyz

    atoms = []
    i = 4
    for _ in range(nat):
        iatnr, p0 = atom_line(L[i])
        pos = [p0]
        mult = int(re.search(r"MULT\s*=\s*(\d+)", L[i + 1]).group(1))
        i += 2
        for _m in range(mult - 1):
            pos.append(atom_line(L[i])[1])
            i += 1
        x = L[i]
        name = x[0:10].strip()
        jrj = int(re.search(r"NPT\s*=\s*(\d+)", x).group(1))
        r0 = _f(re.search(r"R0\s*=\s*" + _FNUM, x).group(1))
        rmt = _f(re.search(r"RMT\s*=\s*" + _FNUM, x).group(1))
        z = _f(re.search(r"Z\s*:\s*" + _FNUM, x).group(1))
        dx = np.log(rmt / r0) / (jrj - 1)
        rmt = r0 * np.exp(dx * (jrj - 1))  # inilpw.f:289-290
        rot = []
        for r in range(3):
            y = L[i + 1 + r]
            y = y.split(":", 1)[1] if ":" in y else y[20:]
            rot.append([_f(v) for v in re.findall(_FNUM, y)[:3]])
        atoms.append(StructAtom(name=name, iatnr=iatnr, pos=np.array(pos, dtype=np.float64), jrj=jrj, r0=r0,
                                rmt=float(rmt), dx=float(dx), z=z, rotloc=np.array(rot, dtype=np.float64)))
        i += 4
    nsym = _i(L[i][0:4])
    i += 1
    imat = np.zeros((nsym, 3, 3), dtype=np.int64)
    tau = np.zeros((nsym, 3))
    for s in range(nsym):
        for r in range(3):
            x = L[i + r]
            imat[s, r] = [_i(x[0:2]), _i(x[2:4]), _i(x[4:6])]
            tau[s, r] = _f(x[6:17])
        i += 4
    return Struct(title=title, lattic=lattic, rel=(irel != "NREL"), abc=abc, angles=angles, atoms=atoms,
                  imat=imat, tau=tau)


@dataclass
class In1Line:
    l: int
    e: float
    de: float
    switch: str
    napw: int


@dataclass
class In1Atom:
    e: float
    napw: int
    lines: List[In1Line]


@dataclass
class In1:
    mode: str
    rkmax: float
    lmax: int
    lnsmax: int
    atoms: List[In1Atom] = field(default_factory=list)
    emin: float = -1.0e70
    emax: float = 1.0e70


def read_in1(text: str, nat: int) -> In1:
    L = text.split("\n")
    mode = L[0][0:5]
    f = L[1].split()
    res = In1(mode=mode, rkmax=_f(f[0]), lmax=_i(f[1]), lnsmax=_i(f[2]))
    i = 2
    for _ in range(nat):
        g = L[i].split()
        ei, nlr = _f(g[0]), _i(g[1])
        napw = _i(g[2]) if len(g) > 2 and re.fullmatch(r"-?\d+", g[2]) else 0
        lines = []
        for q in range(nlr):
            x = L[i + 1 + q].ljust(28)
            lines.append(In1Line(l=_i(x[1:2]), e=_f(x[2:12]), de=_f(x[12:22]), switch=x[22:26].strip(),
                                 napw=_i(x[26:28])))
        res.atoms.append(In1Atom(e=ei, napw=napw, lines=lines))
        i += 1 + nlr
    # K-VECTORS line (format 20X,I1,2F10.1): the energy window
    x = L[i] if i < len(L) else ""
    if x.strip():
        res.emin, res.emax = _f(x[21:31]), _f(x[31:41])
    return res


_NUM = re.compile(r"-?\d*\.\d+[EeDd][+-]\d+")


def _radial_blocks(text: str, npts: List[int]):
    """Per atom, the (L, M, values) blocks of a VLM file and the line where
    the atom section ends."""
    T = text.split("\n")
    out = []
    j = 0
    for a in range(len(npts)):
        while "ATOMNUMBER" not in T[j]:
            j += 1
        nlm = _i(re.search(r"NUMBER OF LM=\s*(\d+)", T[j + 1]).group(1))
        j += 2
        blocks = []
        for _ in range(nlm):
            while "VLM(R) FOR L=" not in T[j]:
                j += 1
            m = re.search(r"L=\s*(-?\d+)\s+M=\s*(-?\d+)", T[j])
            vals = []
            j += 1
            while len(vals) < npts[a]:
                vals.extend(float(v.replace("D", "E")) for v in _NUM.findall(T[j]))
                j += 1
            blocks.append((int(m.group(1)), int(m.group(2)), np.array(vals[: npts[a]], dtype=np.float64)))
        out.append(blocks)
    return out, j


def read_vsp(text: str, npts: List[int]) -> List[np.ndarray]:
    """r V_00(r) of each atom (Rydberg), the array ATPAR halves into Hartree."""
    blocks, _ = _radial_blocks(text, npts)
    return [b[0][2] for b in blocks]


@dataclass
class Vns:
    lm: List[List[tuple]]      # per atom [(L, M), ...] as written (L < 0: sine-like)
    vlm: List[List[np.ndarray]]
    potk: list                 # [(JA, JB, JC, complex)] interstitial plane waves


def read_vns(text: str, npts: List[int]) -> Vns:
    blocks, j = _radial_blocks(text, npts)
    T = text.split("\n")
    potk = []
    k = next((q for q in range(j, len(T)) if "TOTAL POTENTIAL IN INTERSTITIAL" in T[q]), None)
    if k is not None:
        npw = _i(re.search(r"NUMBER OF PW\s+(\d+)", T[k + 2]).group(1))
        for x in T[k + 3:k + 3 + npw]:
            potk.append((_i(x[3:8]), _i(x[8:13]), _i(x[13:18]), complex(_f(x[18:37]), _f(x[37:56]))))
    return Vns(lm=[[(b[0], b[1]) for b in bl] for bl in blocks], vlm=[[b[2] for b in bl] for bl in blocks],
               potk=potk)


def read_klist(text: str):
    """[(name, (ISX, ISY, ISZ), IDV, weight)] up to the END line (format 5100)."""
    out = []
    for x in text.split("\n"):
        if x.startswith("END") or not x.strip():
            break
        x = x.ljust(50)
        out.append((x[0:10].strip(), (_i(x[10:15]), _i(x[15:20]), _i(x[20:25])), _i(x[25:30]), _f(x[30:35])))
    return out
