"""Writers (and a reader) of lapw1's output files case.vector and case.energy.

lapw2 reads lapw1's eigenvalues and eigenvectors from these two files; a
host that sets up and solves k-points with this library writes them the way
lapw1 does, so that the rest of a WIEN2k run takes them unchanged:

  write_header   inilpw.f:440-445  per atom: E_l (l = 0..LMAX-1) and the
                                   LO energies ELO(0:LOMAX, 1:NLOAT)
  write_kpoint   tapewf.F:44-59    per k-point: SX, SY, SZ, KNAME, NV, NE,
                                   WEIGHT, IPGR; the KZZ of the NV(+NLO)
                                   rows; per state I, E(I) and the
                                   conjugated eigenvector (complex build)
  energy_lines   tapewf.F:46,50    the formatted twin (case.energy)
  write_nsh      atpar.f:112-115,345,563-570, forfhs.f:26-69
                                   case.nsh (unit 71, read by lapw2's
                                   force terms): per atom the Gaunt
                                   factor x non-spherical radial integral
                                   of every LQNS entry

case.vector is a Fortran sequential unformatted file: every record is
framed by its byte length as a 4-byte integer before and after (the
default of gfortran and ifort).  Integers are 4-byte, reals 8-byte,
COMPLEX*16 two 8-byte reals.
"""
from __future__ import annotations

import struct
from typing import BinaryIO, List, Sequence

import numpy as np


def _record(f: BinaryIO, payload: bytes) -> None:
    n = struct.pack("<i", len(payload))
    f.write(n)
    f.write(payload)
    f.write(n)


def write_header(f: BinaryIO, e: np.ndarray, elo: np.ndarray) -> None:
    """e: [nat, LMAX] E_l (Ry); elo: [nat, NLOAT, LOMAX+1] LO energies
    (the Problem's layout).  Two records per atom (inilpw.f:442-443)."""
    e = np.asarray(e, dtype="<f8")
    elo = np.asarray(elo, dtype="<f8")
    for a in range(e.shape[0]):
        _record(f, e[a].tobytes())
        _record(f, elo[a].reshape(-1).tobytes())   # ELO(J, k) with J fastest = [k][J]


def _kpoint_sx(k, lattic: str, ortho: bool):
    sx, sy, sz = (float(v) for v in k)
    if not ortho and lattic.strip().upper().startswith("CXZ"):
        sx, sz = sx + sz, -sx + sz
    return sx, sy, sz


def write_kpoint(f: BinaryIO, k: Sequence[float], kname: str, kzz: np.ndarray, eig: np.ndarray, z: np.ndarray,
                 weight: float, ipgr: str = "", lattic: str = "P", ortho: bool = True) -> None:
    """One k-point (tapewf.F:44-59).  kzz: [n, 3] rows of the basis (plane
    waves then LOs); eig: [ne]; z: [n, ne] complex eigenvectors as the
    eigen-solve returns them (the file holds their conjugates)."""
    sx, sy, sz = _kpoint_sx(k, lattic, ortho)
    n = int(kzz.shape[0])
    ne = int(len(eig))
    name = kname.encode()[:10].ljust(10)
    pg = ipgr.encode()[:3].ljust(3)
    _record(f, struct.pack("<3d", sx, sy, sz) + name + struct.pack("<2id", n, ne, float(weight)) + pg)
    _record(f, np.ascontiguousarray(kzz, dtype="<i4").tobytes())
    zc = np.conj(np.asarray(z, dtype=np.complex128))
    for i in range(ne):
        _record(f, struct.pack("<id", i + 1, float(eig[i])))
        _record(f, np.ascontiguousarray(zc[:n, i]).astype("<c16").tobytes())


def energy_lines(k, kname: str, n: int, eig, weight: float, ipgr: str = "", lattic: str = "P",
                 ortho: bool = True) -> List[str]:
    """The lines of case.energy for one k-point: '(3e19.12,a10,2i6,f5.1,a3)'
    then one 'I E(I)' line per state."""
    sx, sy, sz = _kpoint_sx(k, lattic, ortho)
    head = "".join(_e19(v) for v in (sx, sy, sz)) + kname[:10].ljust(10) + f"{n:6d}{len(eig):6d}" + \
        f"{weight:5.1f}" + ipgr[:3].ljust(3)
    return [head] + [f"{i + 1:12d}{float(e):25.15E}" for i, e in enumerate(eig)]


def _e19(v: float) -> str:
    """Fortran E19.12: 0.dddddddddddd E+xx (mantissa in [0.1, 1))."""
    if v == 0.0:
        return "0.000000000000E+00".rjust(19)
    m, e = f"{abs(v):.11E}".split("E")
    mant = m.replace(".", "")
    exp = int(e) + 1
    s = ("-" if v < 0 else "") + "0." + mant + ("E+" if exp >= 0 else "E-") + f"{abs(exp):02d}"
    return s.rjust(19)


def read_vector(f: BinaryIO, nat: int):
    """Parse a case.vector written by write_header / write_kpoint: returns
    (header [(E, ELO)] per atom, [k-point dicts])."""
    def rec():
        h = f.read(4)
        if not h:
            return None
        (n,) = struct.unpack("<i", h)
        b = f.read(n)
        (m,) = struct.unpack("<i", f.read(4))
        if m != n:
            raise ValueError("broken record frame")
        return b
    head = []
    for _ in range(nat):
        e = np.frombuffer(rec(), dtype="<f8").copy()
        elo = np.frombuffer(rec(), dtype="<f8").copy()
        head.append((e, elo))
    kps = []
    while True:
        b = rec()
        if b is None:
            break
        sx, sy, sz = struct.unpack("<3d", b[:24])
        kname = b[24:34].decode().strip()
        n, ne, w = struct.unpack("<2id", b[34:50])
        ipgr = b[50:53].decode().strip()
        kzz = np.frombuffer(rec(), dtype="<i4").reshape(n, 3).copy()
        eig = np.zeros(ne)
        z = np.zeros((n, ne), dtype=np.complex128)
        for i in range(ne):
            idx, ei = struct.unpack("<id", rec())
            assert idx == i + 1
            eig[i] = ei
            z[:, i] = np.conj(np.frombuffer(rec(), dtype="<c16"))
        kps.append(dict(k=(sx, sy, sz), kname=kname, weight=w, ipgr=ipgr, kzz=kzz, eig=eig, z=z))
    return head, kps


def _nsh_pair(v) -> str:
    return _e19(v.real) + _e19(v.imag)


def write_nsh(f, rads, lomax: int = 3) -> None:
    """case.nsh from the host ATPAR's per-atom Gaunt lists and radial
    integrals (hack_wein2k_b200.atpar.AtomRadial): the header, then per
    atom its ' .Atom' line, for every LQNS entry (l0, ll, lp, m, mm, mp)
    the products GFAC x (uVu, dVd, uVd, dVu) and, when l0 or lp carries a
    local orbital, GFAC x (loVu 21, loVu 12, loVlo 22, loVd 21, loVd 12),
    and a closing line of zeros.  f: a text stream."""
    f.write(" non-spherical Matrixelements x Gaunt-Coefficient (d=du/dE):\n"
            " l0 ll lp m0 mm mp     uVu dVd\n"
            "                       uVd dVu\n")
    pad = " " * 18
    zero = 0j
    for ja, rad in enumerate(rads):
        f.write(f"{ja + 1:3d} .Atom \n")
        for (l0, ll, lp, lm1, m, mp, g) in rad.gaunts:
            uvu, dvd, uvd = rad.vns[(l0, lm1, lp)]
            dvu = rad.vns[(lp, lm1, l0)][2]
            mm = rad.lm[lm1 - 1][1]
            f.write(f"{l0:3d}{ll:3d}{lp:3d}{m:3d}{mm:3d}{mp:3d}" + _nsh_pair(g * uvu) + _nsh_pair(g * dvd) + "\n")
            f.write(pad + _nsh_pair(g * uvd) + _nsh_pair(g * dvu) + "\n")
            if l0 <= lomax or lp <= lomax:
                t21 = t12 = t22 = d21 = d12 = zero
                lo0 = l0 <= lomax and bool(rad.loor[l0])
                if lo0:
                    lv = rad.vnslo[(l0, lm1, lp)]
                    t21, d21 = g * lv[0], g * lv[1]
                if lp <= lomax and bool(rad.loor[lp]):
                    lv = rad.vnslo[(lp, lm1, l0)]
                    if lo0:
                        t22 = g * rad.vnslo[(l0, lm1, lp)][2]
                    t12, d12 = g * lv[0], g * lv[1]
                f.write(pad + _nsh_pair(t21) + _nsh_pair(t12) + _nsh_pair(t22) + "\n")
                f.write(pad + _nsh_pair(d21) + _nsh_pair(d12) + "\n")
        f.write("".join(f"{0:3d}" for _ in range(6)) + _e19(0.0) * 4 + "\n" + pad + _e19(0.0) * 4 + "\n")


def read_nsh(f):
    """Parse a case.nsh written by write_nsh (or lapw1): {atom: [entry]},
    entry = dict(idx=(l0, ll, lp, m, mm, mp), t=[tuu, tdd, tud, tdu],
    lo=[tuu21, tuu12, tuu22, tud21, tdu12] or None).  lo lines follow an
    entry exactly when l0 or lp is at most lomax (3)."""
    lines = f.read().splitlines()[3:]
    out, atom, i = {}, None, 0

    def cvals(s, n):
        return [complex(float(s[19 * (2 * k):19 * (2 * k + 1)]), float(s[19 * (2 * k + 1):19 * (2 * k + 2)]))
                for k in range(n)]
    while i < len(lines):
        ln = lines[i]
        if ln.strip().endswith(".Atom"):
            atom = int(ln.split()[0])
            out[atom] = []
            i += 1
            continue
        idx = tuple(int(ln[3 * k:3 * k + 3]) for k in range(6))
        t = cvals(ln[18:], 2) + cvals(lines[i + 1][18:], 2)
        i += 2
        if idx == (0,) * 6 and all(v == 0 for v in t):
            continue
        lo = None
        if idx[0] <= 3 or idx[2] <= 3:
            lo = cvals(lines[i][18:], 3) + cvals(lines[i + 1][18:], 2)
            i += 2
        out[atom].append(dict(idx=idx, t=t, lo=lo))
    return out
