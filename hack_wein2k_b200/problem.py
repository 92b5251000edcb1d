"""Host-side description of one k-point's H/S setup problem.

`Problem` carries exactly the inputs that WIEN2k lapw1's HAMILT, HNS and
HORB read (SRC_lapw1/hamilt.F:1-2, hns.F:1-3, horb.F:1-2 and the module
state they use: matrices, loabc, lolog, out, struk, rotmat, orb).  It is
marshalled into the `lapw1gpu_problem` C struct of include/lapw1gpu.h, the
same struct the Fortran caller fills through ISO_C_BINDING.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field, fields
from typing import Optional

import numpy as np

LOMAX = 3
NLOAT = 3
NSL2 = 25
NTNS = 9

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class CProblem(C.Structure):
    """ctypes mirror of `lapw1gpu_problem` (include/lapw1gpu.h)."""

    _fields_ = [
        ("n", C.c_int), ("nv", C.c_int), ("nlo", C.c_int), ("nat", C.c_int),
        ("ndf", C.c_int), ("ltop", C.c_int), ("ldl", C.c_int), ("lnsmax", C.c_int),
        ("ins", C.c_int), ("nohns", C.c_int), ("vi", C.c_double), ("bkzz", C.c_double * 9),
        ("mult", _ip), ("rmt", _dp), ("v", _dp), ("pos", _dp), ("rotij", _dp), ("rotloc", _dp),
        ("kzz", _ip), ("xk", _dp), ("yk", _dp), ("zk", _dp), ("rk", _dp),
        ("p", _dp), ("pe", _dp), ("dp", _dp), ("dpe", _dp), ("pei", _dp), ("e", _dp),
        ("lapw", _ip),
        ("ilo", _ip), ("loor", _ip), ("alo", _dp), ("blo", _dp), ("clo", _dp), ("elo", _dp),
        ("pi12lo", _dp), ("pe12lo", _dp), ("dplo", _dp),
        ("warp1", C.c_int), ("warp2", C.c_int), ("warp3", C.c_int), ("warp", _dp),
        ("tns", _dp),
        ("natorb", C.c_int), ("iatom", _ip), ("nlorb", _ip), ("lorb", _ip), ("vorb", _dp),
    ]


class CStats(C.Structure):
    """ctypes mirror of `lapw1gpu_stats`."""

    _fields_ = [(k, C.c_double) for k in (
        "ms_total", "ms_albl", "ms_spherical", "ms_lo", "ms_hns", "ms_horb",
        "ms_h2d", "ms_d2h", "flops_fp64_equiv", "kernel_launches", "ms_sph_main", "ms_hns_main",
        "ms_k_albl", "ms_table", "ms_sph_slice", "ms_host")]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def _c(a, dtype):
    a = np.ascontiguousarray(a, dtype=dtype)
    return a


@dataclass
class Problem:
    """Inputs of one k-point.  Shapes follow include/lapw1gpu.h (C order)."""

    nv: int
    nlo: int
    ltop: int                  # lmax + 1
    lnsmax: int
    vi: float
    mult: np.ndarray           # [nat] int
    rmt: np.ndarray            # [nat]
    v: np.ndarray              # [nat]
    pos: np.ndarray            # [ndf, 3]
    rotij: np.ndarray          # [ndf, 3, 3]  (C view of Fortran ROTIJ(3,3,ndf): [a][col][row])
    rotloc: np.ndarray         # [nat, 3, 3]
    kzz: np.ndarray            # [n, 3] int
    xk: np.ndarray             # [n]
    yk: np.ndarray
    zk: np.ndarray
    rk: np.ndarray
    p: np.ndarray              # [nat, ldl] U(R)
    pe: np.ndarray             # Udot(R)
    dp: np.ndarray             # U'(R)
    dpe: np.ndarray            # Udot'(R)
    pei: np.ndarray            # |Udot|^2
    e: np.ndarray              # E_l
    lapw: np.ndarray           # [nat, ldl] int
    ilo: np.ndarray            # [nat, 4] int
    loor: np.ndarray           # [nat, 4] int
    alo: np.ndarray            # [nat, 3, 4]
    blo: np.ndarray
    clo: np.ndarray
    elo: np.ndarray
    pi12lo: np.ndarray         # [nat, 4]
    pe12lo: np.ndarray
    dplo: np.ndarray
    warp: np.ndarray           # complex [2w3+1, 2w2+1, 2w1+1]
    bkzz: np.ndarray           # [3, 3]: Cartesian k+G = k + bkzz @ KZZ
    tns: np.ndarray            # complex [nat, 9, 25, 25]
    ins: int = 0
    nohns: int = 0
    iatom: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))   # 1-based atom types
    nlorb: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    lorb: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.int32))
    vorb: np.ndarray = field(default_factory=lambda: np.zeros((0, 4, 7, 7), np.complex128))
    name: str = ""
    meta: dict = field(default_factory=dict)

    # ---- derived sizes ----
    @property
    def n(self) -> int:
        return self.nv + self.nlo

    @property
    def nat(self) -> int:
        return int(len(self.mult))

    @property
    def ndf(self) -> int:
        return int(np.sum(self.mult))

    @property
    def ldl(self) -> int:
        return int(self.p.shape[1])

    @property
    def natorb(self) -> int:
        return int(len(self.iatom))

    @property
    def warp_half(self):
        w3, w2, w1 = self.warp.shape
        return (w1 - 1) // 2, (w2 - 1) // 2, (w3 - 1) // 2

    def validate(self) -> None:
        n, nat, ndf = self.n, self.nat, self.ndf
        assert self.kzz.shape == (n, 3)
        for a in (self.xk, self.yk, self.zk, self.rk):
            assert a.shape == (n,)
        assert self.pos.shape == (ndf, 3) and self.rotij.shape == (ndf, 3, 3)
        assert self.rotloc.shape == (nat, 3, 3)
        assert self.p.shape == (nat, self.ldl) and self.ldl >= self.ltop
        assert self.ilo.shape == (nat, LOMAX + 1)
        nlo = int(sum((2 * l + 1) * self.mult[a] * self.ilo[a, l]
                      for a in range(nat) for l in range(LOMAX + 1)))
        assert nlo == self.nlo, (nlo, self.nlo)
        assert self.tns.shape == (nat, NTNS, NSL2, NSL2)
        assert np.asarray(self.bkzz).shape == (3, 3)

    def to_c(self) -> CProblem:
        """Marshal into the C struct.  The returned struct keeps references
        to the contiguous arrays it points into (attribute `_keep`)."""
        self.validate()
        keep = []

        def dptr(a):
            a = np.ascontiguousarray(a, dtype=np.float64)
            keep.append(a)
            return a.ctypes.data_as(_dp)

        def cptr(a):
            a = np.ascontiguousarray(a, dtype=np.complex128)
            keep.append(a)
            return a.ctypes.data_as(_dp)

        def iptr(a):
            a = np.ascontiguousarray(a, dtype=np.int32)
            keep.append(a)
            return a.ctypes.data_as(_ip)

        w1, w2, w3 = self.warp_half
        s = CProblem(
            n=self.n, nv=self.nv, nlo=self.nlo, nat=self.nat, ndf=self.ndf,
            ltop=self.ltop, ldl=self.ldl, lnsmax=self.lnsmax, ins=self.ins,
            nohns=self.nohns, vi=float(self.vi),
            bkzz=(C.c_double * 9)(*np.asarray(self.bkzz, dtype=np.float64).reshape(9)),
            mult=iptr(self.mult), rmt=dptr(self.rmt), v=dptr(self.v), pos=dptr(self.pos),
            rotij=dptr(self.rotij), rotloc=dptr(self.rotloc),
            kzz=iptr(self.kzz), xk=dptr(self.xk), yk=dptr(self.yk), zk=dptr(self.zk),
            rk=dptr(self.rk),
            p=dptr(self.p), pe=dptr(self.pe), dp=dptr(self.dp), dpe=dptr(self.dpe),
            pei=dptr(self.pei), e=dptr(self.e), lapw=iptr(self.lapw),
            ilo=iptr(self.ilo), loor=iptr(self.loor), alo=dptr(self.alo), blo=dptr(self.blo),
            clo=dptr(self.clo), elo=dptr(self.elo), pi12lo=dptr(self.pi12lo),
            pe12lo=dptr(self.pe12lo), dplo=dptr(self.dplo),
            warp1=w1, warp2=w2, warp3=w3, warp=cptr(self.warp),
            tns=cptr(self.tns),
            natorb=self.natorb, iatom=iptr(self.iatom if self.natorb else np.zeros(1)),
            nlorb=iptr(self.nlorb if self.natorb else np.zeros(1)),
            lorb=iptr(self.lorb if self.natorb else np.zeros((1, 3))),
            vorb=cptr(self.vorb if self.natorb else np.zeros((1, 4, 7, 7))),
        )
        s._keep = keep
        return s

    def hs_bytes(self) -> int:
        return self.n * self.n * 16

    def copy(self, **changes) -> "Problem":
        d = {f.name: getattr(self, f.name) for f in fields(self)}
        d.update(changes)
        return Problem(**d)


def hermitian_from_packed(hs: np.ndarray, hsdiag: np.ndarray):
    """Hermitian H and S of the generalized problem H x = e S x that SECLR4
    solves from the packed state (seclr4.F:158-296): it conjugates HS and
    HSDIAG, reduces H from the lower triangle including the diagonal
    (ZHCGST / ZHEEVX2 'L'), and factors the upper triangle with HSDIAG as
    its diagonal (ZPOTRF 'U'), which ZHCGST takes as the Cholesky factor of
    S**T (zhcgst.f:34-42).  So S(i,j) = conj(HS(j,i)) for i > j: S is the
    transpose of the Hermitian matrix the upper triangle stores, and H and S
    carry the same structure-factor phases."""
    hc = np.conj(hs)
    low = np.tril(hc, -1)
    H = low + low.conj().T + np.diag(np.diag(hc).real)
    up = np.triu(hc, 1).T                      # S(i,j) = conj(HS(j,i)), i > j
    S = up + up.conj().T + np.diag(np.conj(hsdiag).real)
    return H, S
