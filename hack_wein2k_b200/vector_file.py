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
