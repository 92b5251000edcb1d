"""lapw1's radial set-up (ATPAR) on the host, and a k-point problem from the case files.

The drop-in boundary takes what ATPAR computes once per run as plain arrays
(include/lapw1gpu.h: U, U', Udot, Udot', |Udot|^2, E_l, the LO
coefficients and the non-spherical T blocks).  This module computes them
from the WIEN2k case files the way lapw1 does, so that a host other than
lapw1 can drive the library, and so that the library's matrices can be
checked end to end against the eigenvalues lapw1 printed for the
reference's shipped runs:

  outwin     SRC_lapw1/outwin.f:1-113  scalar-relativistic outward
                                       integration (Rydberg units inside)
  rint13     SRC_lapw1/rint13.f:1-70   radial integral of large and small
                                       components on the logarithmic mesh
  select     SRC_lapw1/select.f:1-148  energy search between the band
                                       bottom (u' = 0) and top (u = 0)
  atpar      SRC_lapw1/atpar.f:67-565  energy parameters, u, udot, LO
                                       functions, ABC coefficients, Gaunt
                                       list and radial integrals of VLM
  abc        SRC_lapw1/abc.f:35-63
  cbcomb     SRC_lapw1/cbcomb.f:1-114  cubic-harmonic combination of VLM
  gaunt      SRC_lapw1/gaunt1.f, gaunt2.f: the Gaunt integral, here from
             the closed form with Wigner 3j symbols (the reference
             evaluates the same integral by 12-point Gauss quadrature,
             exact for these degrees)
  rotdef     SRC_lapw1/rotdef.f        ROTIJ of each equivalent atom
  locdef     SRC_lapw1/locdef.f        ROTIJ for non-orthogonal lattices

`problem_from_case` assembles a `Problem` for one k-point (COORS/LOPW from
`lattice`, the warped interstitial table from `warp`).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from fractions import Fraction
from functools import lru_cache
from typing import List, Optional

import numpy as np

from . import lattice, warp
from .case_files import In1, Struct, Vns
from .problem import LOMAX, NLOAT, Problem

CLIGHT = 137.0359895
NSLMAX = 5           # param.inc: lmax_ns + 1 upper bound
LDL = 13             # param.inc LMAX: per-l array length
DELE = 2.0e-3        # atpar.f DELE: energy shift of the udot difference (Hartree)
TRAPLEVEL = 1.0e-3   # atpar.f: |U(R)| below this shifts E_l down once by 0.05 Ry


# ----------------------------------------------------------------- radial ODE
def outwin(rel: bool, v: np.ndarray, rnot: float, dh: float, jri: int, eh: float, fl: float, z: float):
    """Scalar-relativistic radial equation integrated outward (outwin.f).
    v: r V(r) in Hartree on the mesh r_i = rnot exp(dh (i-1)); eh in
    Hartree.  Returns (u(R), u'(R), nodes, A, B): large and small
    components (B scaled by c/2 as the reference leaves it)."""
    e = eh * 2.0
    rnet = rnot * np.exp(dh * np.arange(jri, dtype=np.float64))
    nodes = 0
    zz = z + z
    c = 2.0 * CLIGHT if rel else 1.0e10
    fllp1 = fl * (fl + 1.0)
    r83sq = 64.0 / 9.0
    r1 = 1.0 / 9.0
    r2 = -5.0 * r1
    r3 = 19.0 * r1
    h83 = 8.0 / 3.0
    g0 = 1.0
    if z < 0.9:
        s = fl + 1.0
        sf = fl
        f0 = fl / c
    else:
        aa = zz / c
        s = math.sqrt(fllp1 + 1.0 - aa * aa)
        sf = s
        f0 = g0 * (s - 1.0) / aa
    A = np.zeros(jri)
    B = np.zeros(jri)
    d = np.zeros((2, 3))
    for k in range(3):
        r = rnet[k]
        drdi = dh * r
        A[k] = (r ** s) * g0
        B[k] = (r ** sf) * f0
        d[0, k] = drdi * A[k] * s / r
        d[1, k] = drdi * B[k] * sf / r
    dg1, dg2, dg3 = d[0, 0], d[0, 1], d[0, 2]
    df1, df2, df3 = d[1, 0], d[1, 1], d[1, 2]
    vv = [float(x) for x in v[:jri]]
    rr = [float(x) for x in rnet]
    a_prev, b_prev = A[2], B[2]
    Al, Bl = list(A), list(B)
    for k in range(3, jri):
        r = rr[k]
        drdi = dh * r
        phi = (e - 2.0 * vv[k] / r) * drdi / c
        u = drdi * c + phi
        x = -drdi / r
        y = -fllp1 * x * x / u + phi
        det = r83sq - x * x + u * y
        b11 = a_prev * h83 + r1 * dg1 + r2 * dg2 + r3 * dg3
        b22 = b_prev * h83 + r1 * df1 + r2 * df2 + r3 * df3
        ak = (b11 * (h83 - x) + b22 * u) / det
        bk = (b22 * (h83 + x) - b11 * y) / det
        if ak * a_prev < 0.0:
            nodes += 1
        Al[k], Bl[k] = ak, bk
        dg1, dg2, dg3 = dg2, dg3, u * bk - x * ak
        df1, df2, df3 = df2, df3, x * bk - y * ak
        a_prev, b_prev = ak, bk
    A = np.array(Al)
    B = np.array(Bl) * (c / 2.0)
    val = A[jri - 1] / rr[jri - 1]
    slo = dg3 / (dh * rr[jri - 1])
    slo = (slo - val) / rr[jri - 1]
    return val, slo, nodes, A, B


def rint13(c1: float, c2: float, a, b, x, y, rnot: float, dx: float, jri: int) -> float:
    """Radial integral sum_j (c1 a_j x_j + c2 b_j y_j) r_j dx by the
    Simpson rule on the logarithmic mesh (rint13.f)."""
    d = math.exp(dx)
    j = 3 - (jri % 2)          # 1-based index of the first Simpson point
    j1 = j - 1
    r = rnot * d ** (j - 1)
    rr1 = r / d
    z4 = 0.0
    z2 = 0.0
    while True:
        g1 = c1 * a[j - 1] * x[j - 1]
        g2 = c2 * b[j - 1] * y[j - 1]
        z4 = z4 + r * (g1 + g2)
        if z4 == 0.0:
            z4 = 2.0e-55
        r = r * d
        j = j + 1
        if j >= jri:
            break
        z2 = z2 + r * (c1 * a[j - 1] * x[j - 1] + c2 * b[j - 1] * y[j - 1])
        r = r * d
        j = j + 1
    p1 = rnot * (c1 * a[0] * x[0] + c2 * b[0] * y[0])
    p2 = rr1 * (c1 * a[j1 - 1] * x[j1 - 1] + c2 * b[j1 - 1] * y[j1 - 1])
    s = 2 * z2 + 4 * z4 + r * (c1 * a[j - 1] * x[j - 1] + c2 * b[j - 1] * y[j - 1]) + p2
    s = (dx * s + p1) / 3.0
    if j1 > 1:
        s = s + 0.5 * dx * (p1 + p2)
    return s


class EnergySearchError(RuntimeError):
    """SELECT found no energy limits (select.f:141-147: 'STOP - Error')."""


def select(l: int, ei: float, de: float, emain: str, rel: bool, vr, rnot: float, dx: float, jri: int, z: float):
    """Automatic energy search (select.f): from ei (Ry) in steps de (Ry)
    up (and down) until u' (bottom) and u (top) change sign; returns
    (E, E_bottom, E_top) in Ry."""
    fl = float(l)
    ei = ei * 0.5
    de = de * 0.5
    u, du = outwin(rel, vr, rnot, dx, jri, ei, fl, z)[:2]
    eiup = eidn = ei
    e1 = e2 = -100.0
    upold, dupold = u, du
    dnold, ddnold = u, du
    state = 10
    while True:
        if state == 10:
            eiup = eiup + de
            uup, duup = outwin(rel, vr, rnot, dx, jri, eiup, fl, z)[:2]
            utst, dutst = upold * uup, dupold * duup
            upold, dupold = uup, duup
            if utst < 0.0:
                e2 = eiup
                if e1 > -30.0:
                    break
            if dutst < 0.0:
                e1 = eiup
                if e2 > -30.0:
                    break
            if e1 < -30.0 and eiup < 2.5:
                state = 20
            elif eiup < 0.5:
                state = 10
            else:
                break
        else:  # state 20: one step down
            eidn = eidn - de
            udn, dudn = outwin(rel, vr, rnot, dx, jri, eidn, fl, z)[:2]
            utst, dutst = dnold * udn, ddnold * dudn
            dnold, ddnold = udn, dudn
            if utst < 0.0:
                e2 = eidn
                if e1 > -30.0:
                    break
            if dutst < 0.0:
                e1 = eidn
                if e2 > -30.0:
                    break
            if e2 < -30.0:
                state = 10
            elif eidn > ei - 3.0:
                state = 20
            else:
                break
    ei, e1, e2 = ei * 2.0, e1 * 2.0, e2 * 2.0
    if e1 < -60.0 and e2 < -60.0:
        if emain == "STOP":
            raise EnergySearchError(f"no energy limits found for L={l}")
        ei = 2.0
    elif e2 < -60.0:
        if emain == "STOP":
            raise EnergySearchError(f"no energy limits found for L={l}")
        ei = max(e1, ei)
    elif e1 < -60.0:
        raise EnergySearchError(f"no energy limits found for L={l}")
    else:
        ei = (e1 + e2) * 0.5
    return ei, e1, e2


# ----------------------------------------------------------------- Gaunt integral
def _fac(n: int) -> int:
    return math.factorial(n)


@lru_cache(maxsize=None)
def wigner3j(j1: int, j2: int, j3: int, m1: int, m2: int, m3: int) -> float:
    """Wigner 3j symbol by the Racah formula, exact up to the final square root."""
    if m1 + m2 + m3 != 0 or j3 < abs(j1 - j2) or j3 > j1 + j2:
        return 0.0
    if abs(m1) > j1 or abs(m2) > j2 or abs(m3) > j3:
        return 0.0
    tri = Fraction(_fac(j1 + j2 - j3) * _fac(j1 - j2 + j3) * _fac(-j1 + j2 + j3), _fac(j1 + j2 + j3 + 1))
    pre = tri * _fac(j1 + m1) * _fac(j1 - m1) * _fac(j2 + m2) * _fac(j2 - m2) * _fac(j3 + m3) * _fac(j3 - m3)
    s = Fraction(0)
    for k in range(max(0, j2 - j3 - m1, j1 - j3 + m2), min(j1 + j2 - j3, j1 - m1, j2 + m2) + 1):
        s += Fraction((-1) ** k, _fac(k) * _fac(j1 + j2 - j3 - k) * _fac(j1 - m1 - k) * _fac(j2 + m2 - k)
                      * _fac(j3 - j2 + m1 + k) * _fac(j3 - j1 - m2 + k))
    sign = -1 if (j1 - j2 - m3) % 2 else 1
    return sign * float(s) * math.sqrt(float(pre))


@lru_cache(maxsize=None)
def gaunt(lp: int, l: int, ls: int, mp: int, m: int, ms: int) -> float:
    """The integral of conj(Y_lp,mp) Y_l,m Y_ls,ms over the sphere
    (Condon-Shortley Y_lm), the quantity GAUNT1(LP,L,LS,MP,M,MS) returns."""
    if -mp + m + ms != 0:
        return 0.0
    pre = math.sqrt((2 * lp + 1) * (2 * l + 1) * (2 * ls + 1) / (4.0 * math.pi))
    sgn = -1.0 if mp % 2 else 1.0
    return sgn * pre * wigner3j(lp, l, ls, 0, 0, 0) * wigner3j(lp, l, ls, -mp, m, ms)


# ----------------------------------------------------------------- cubic harmonics
def _c_kub():
    c = np.zeros((11, 11))
    c[0, 0] = 1.0
    c[3, 2] = 1.0
    c[4, 0] = 0.5 * math.sqrt(7.0 / 3.0)
    c[4, 4] = 0.5 * math.sqrt(5.0 / 3.0)
    c[6, 0] = 0.5 * math.sqrt(0.5)
    c[6, 2] = 0.25 * math.sqrt(11.0)
    c[6, 4] = -0.5 * math.sqrt(7.0 / 2.0)
    c[6, 6] = -0.25 * math.sqrt(5.0)
    c[7, 2] = 0.5 * math.sqrt(13.0 / 6.0)
    c[7, 6] = 0.5 * math.sqrt(11.0 / 6.0)
    c[8, 0] = 0.125 * math.sqrt(33.0)
    c[8, 4] = 0.25 * math.sqrt(7.0 / 3.0)
    c[8, 8] = 0.125 * math.sqrt(65.0 / 3.0)
    c[9, 2] = 0.25 * math.sqrt(3.0)
    c[9, 4] = 0.5 * math.sqrt(17.0 / 6.0)
    c[9, 6] = -0.25 * math.sqrt(13.0)
    c[9, 8] = -0.5 * math.sqrt(7.0 / 6.0)
    c[10, 0] = 0.125 * math.sqrt(65.0 / 6.0)
    c[10, 2] = 0.125 * math.sqrt(247.0 / 6.0)
    c[10, 4] = -0.25 * math.sqrt(11.0 / 2.0)
    c[10, 6] = 0.0625 * math.sqrt(19.0 / 3.0)
    c[10, 8] = -0.125 * math.sqrt(187.0 / 6.0)
    c[10, 10] = -0.0625 * math.sqrt(85.0)
    return c


def cbcomb(lm: List[tuple], vlm: List[np.ndarray]) -> None:
    """Combine the radial potential coefficients of a cubic site in place
    (cbcomb.f): the groups (4,0)+(4,4), (6,0)+(6,4), ... of the cubic
    harmonics, (-3,2) scaled by -1/sqrt 2."""
    ck = _c_kub()
    sqrt2 = math.sqrt(2.0)
    i = 0
    n = len(lm)
    while i < n:
        L, M = lm[i]
        if L == 0 and M == 0:
            i += 1
        elif L == -3 and M == 2:
            vlm[i] = -vlm[i] / sqrt2
            i += 1
        elif L in (4, 6, -7, -9):
            sq1 = 1.0 if M == 0 else sqrt2
            c1, c2 = ck[abs(L), M], ck[abs(L), M + 4]
            v = vlm[i] * c1 + vlm[i + 1] * c2
            vlm[i + 1] = v * c2 / sqrt2
            vlm[i] = v * c1 / sq1
            i += 2
        elif L in (8, 10):
            sq1 = 1.0 if M == 0 else sqrt2
            c1, c2, c3 = ck[abs(L), M], ck[abs(L), M + 4], ck[abs(L), M + 8]
            v = vlm[i] * c1 + vlm[i + 1] * c2 + vlm[i + 2] * c3
            vlm[i + 1] = v * c2 / sqrt2
            vlm[i + 2] = v * c3 / sqrt2
            vlm[i] = v * c1 / sq1
            i += 3
        else:
            raise ValueError("UNCORRECT LM LIST FOR CUBIC STRUCTURE")


# ----------------------------------------------------------------- ATPAR
@dataclass
class AtomRadial:
    """ATPAR's per-atom results (atspdt, loabc, lolog, loint modules)."""
    e: np.ndarray                 # E_l (Ry), [LDL]
    p: np.ndarray                 # U(R)
    dp: np.ndarray                # U'(R)
    pe: np.ndarray                # Udot(R)
    dpe: np.ndarray               # Udot'(R)
    pei: np.ndarray               # |Udot|^2
    nodes: np.ndarray             # [ltop, 3]: nodes at E-DELE, E, E+DELE
    lapw: np.ndarray              # [LDL] int
    ilo: np.ndarray               # [LOMAX+1] int
    loor: np.ndarray              # [LOMAX+1] int
    elo: np.ndarray               # [NLOAT, LOMAX+1]
    alo: np.ndarray
    blo: np.ndarray
    clo: np.ndarray
    plo: np.ndarray               # [LOMAX+1]
    dplo: np.ndarray
    pi12lo: np.ndarray
    pe12lo: np.ndarray
    searched: list = field(default_factory=list)   # [(l, E, E_bottom, E_top)]
    # non-spherical part (INS = 0)
    lm: list = field(default_factory=list)          # [(L, M)] kept (|L| <= 2 lnsmax)
    gaunts: list = field(default_factory=list)      # LQNS/GFAC entries: (l0, ll, lp, lmx(1-based), m, mp, gfac)
    vns: dict = field(default_factory=dict)         # (l0, lm1, lp) -> (uVu, ueVue, uVue)
    vnslo: dict = field(default_factory=dict)       # (l0, lm1, lp) -> (lo V u, lo V ue, lo V lo)


def atpar(struct: Struct, in1: In1, vsp: List[np.ndarray], vns: Optional[Vns], ltop: int, lnsmax: int):
    """ATPAR for every inequivalent atom (atpar.f:67-565).  ltop = NT =
    lmax + 1.  Returns [AtomRadial]."""
    out = []
    for ja, at in enumerate(struct.atoms):
        rel = struct.rel
        c1f, c2f = (1.0, 1.0 / CLIGHT ** 2) if rel else (1.0, 1.0e-22)
        vr = np.asarray(vsp[ja], dtype=np.float64) / 2.0      # r V in Hartree
        rnot, dx, jri, z = at.r0, at.dx, at.jrj, at.z
        ri = lambda a, b, x, y: rint13(c1f, c2f, a, b, x, y, rnot, dx, jri)  # noqa: E731
        ow = lambda eh, fl: outwin(rel, vr, rnot, dx, jri, eh, fl, z)        # noqa: E731
        a1 = in1.atoms[ja]
        lapw = np.ones(LDL, dtype=np.int32)
        if a1.napw == 1:
            lapw[:] = 0
        ilo = np.zeros(LOMAX + 1, dtype=np.int32)
        loor = np.zeros(LOMAX + 1, dtype=np.int32)
        elo = np.zeros((NLOAT, LOMAX + 1))
        for l in range(LOMAX + 1):
            elo[:, l] = 999.0 if lapw[l] else 997.0
        e = np.full(LDL, a1.e)
        searched = []
        lalt = -1
        for ln in a1.lines:
            l, ei = ln.l, ln.e
            if ln.de > 1.0e-5:
                ei, eb, et = select(l, ei, ln.de, ln.switch, rel, vr, rnot, dx, jri, z)
                searched.append((l, ei, eb, et))
            if l == lalt:
                ilo[l] += 1
                elo[ilo[l] - 1, l] = ei
                loor[l] = 1
            else:
                if ln.napw == 1:
                    lapw[l] = 0
                    ilo[l] = 1
                    elo[0, l] = ei
                    elo[1, l] = 997.0
                e[l] = ei
            lalt = l
        delei = 0.25 / DELE
        p, dp, pe, dpe, pei = (np.zeros(LDL) for _ in range(5))
        nodes = np.zeros((ltop, 3), dtype=np.int32)
        A1, B1, AE1, BE1 = {}, {}, {}, {}
        for j in range(ltop):
            dotrap = True
            while True:
                fl = float(j)
                ei = e[j] / 2.0
                uvb, duvb, nodel, A, B = ow(ei - DELE, fl)
                trx = 1.0 / math.sqrt(ri(A, B, A, B))
                AE, BE = trx * A, trx * B
                uvb, duvb = trx * uvb, trx * duvb
                uve, duve, nodeu, A, B = ow(ei + DELE, fl)
                trx = 1.0 / math.sqrt(ri(A, B, A, B))
                uve = delei * (trx * uve - uvb)
                duve = delei * (trx * duve - duvb)
                AE = delei * (trx * A - AE)
                BE = delei * (trx * B - BE)
                uv, duv, nods, A, B = ow(ei, fl)
                trx = 1.0 / math.sqrt(ri(A, B, A, B))
                p[j], dp[j] = trx * uv, trx * duv
                A, B = trx * A, trx * B
                cross = ri(A, B, AE, BE)
                tr_ = -cross
                AE = AE + tr_ * A
                BE = BE + tr_ * B
                pe[j] = uve + tr_ * p[j]
                dpe[j] = duve + tr_ * dp[j]
                pei[j] = ri(AE, BE, AE, BE)
                if j < NSLMAX:
                    A1[j], B1[j], AE1[j], BE1[j] = A, B, AE, BE
                if abs(p[j]) < TRAPLEVEL and dotrap:
                    dotrap = False
                    e[j] = e[j] - 0.05
                    continue
                nodes[j] = (nodel, nods, nodeu)
                break
        plo, dplo, pi12lo, pe12lo = (np.zeros(LOMAX + 1) for _ in range(4))
        A1LO, B1LO = {}, {}
        for l in range(LOMAX + 1):
            if loor[l]:
                ei = elo[ilo[l] - 1, l] / 2.0
                uv, duv, _, A, B = ow(ei, float(l))
                trx = 1.0 / math.sqrt(ri(A, B, A, B))
                plo[l], dplo[l] = trx * uv, trx * duv
                A, B = trx * A, trx * B
                pi12lo[l] = ri(A1[l], B1[l], A, B)
                pe12lo[l] = ri(AE1[l], BE1[l], A, B)
                A1LO[l], B1LO[l] = A, B
        alo, blo, clo = (np.zeros((NLOAT, LOMAX + 1)) for _ in range(3))
        rmt = at.rmt
        for l in range(LOMAX + 1):
            for jlo in range(1, ilo[l] + 1):
                _abc(l, jlo, bool(lapw[l]), rmt, p, dp, pe, dpe, pei, plo, dplo, pi12lo, pe12lo, alo, blo, clo)
        rad = AtomRadial(e=e, p=p, dp=dp, pe=pe, dpe=dpe, pei=pei, nodes=nodes, lapw=lapw, ilo=ilo, loor=loor,
                         elo=elo, alo=alo, blo=blo, clo=clo, plo=plo, dplo=dplo, pi12lo=pi12lo, pe12lo=pe12lo,
                         searched=searched)
        if vns is not None:
            _nonspherical(rad, at, vns.lm[ja], vns.vlm[ja], lnsmax, ri, A1, B1, AE1, BE1, A1LO, B1LO)
        out.append(rad)
    return out


def _abc(l, jlo, lapw, rmt, p, dp, pe, dpe, pei, plo, dplo, pi12lo, pe12lo, alo, blo, clo):
    """LO coefficients A, B, C (abc.f:35-63)."""
    if lapw:
        xac = plo[l] * dpe[l] - dplo[l] * pe[l]
        xac = xac * rmt * rmt
        xbc = plo[l] * dp[l] - dplo[l] * p[l]
        xbc = -xbc * rmt * rmt
        c = xac * (xac + 2.0 * pi12lo[l]) + xbc * (xbc * pei[l] + 2.0 * pe12lo[l]) + 1.0
        c = 1.0 / math.sqrt(c)
        c = min(c, 200.0)
        clo[jlo - 1, l] = c
        alo[jlo - 1, l] = c * xac
        blo[jlo - 1, l] = c * xbc
    elif jlo == 1:
        alonorm = math.sqrt(1.0 + (p[l] / pe[l]) ** 2 * pei[l])
        alo[0, l] = 1.0 / alonorm
        blo[0, l] = -p[l] / pe[l] / alonorm
        clo[0, l] = 0.0
    else:
        xbc = -p[l] / plo[l]
        xac = math.sqrt(1 + xbc ** 2 + 2 * xbc * pi12lo[l])
        alo[jlo - 1, l] = 1.0 / xac
        blo[jlo - 1, l] = 0.0
        clo[jlo - 1, l] = xbc / xac


def _nonspherical(rad, at, lm_all, vlm_all, lnsmax, ri, A1, B1, AE1, BE1, A1LO, B1LO):
    """Gaunt list and radial integrals of the non-spherical potential
    (atpar.f:331-480)."""
    lm, vlm = [], []
    for (L, M), v in zip(lm_all, vlm_all):
        if abs(L) <= lnsmax * 2:
            lm.append((L, M))
            vlm.append(np.array(v, dtype=np.float64))
    gl = []
    for l0 in range(lnsmax + 1):
        for lp in range(lnsmax + 1):
            for lmx, (lll, mm0) in enumerate(lm, start=1):
                ll = abs(lll)
                if (l0 + lp + ll) % 2 == 1 or l0 + lp - ll < 0 or l0 - lp + ll < 0 or lp - l0 + ll < 0:
                    continue
                mm = mm0
                while True:
                    for m in range(-l0, l0 + 1):
                        for mp in range(-lp, lp + 1):
                            if -m + mm + mp != 0:
                                continue
                            g = complex(gaunt(l0, ll, lp, m, mm, mp), 0.0)
                            if at.iatnr > 0:
                                if ll in (3, 7, 9):
                                    g = -g * 1j if mm < 0 else g * 1j
                            elif mm != 0:
                                minu, imag1 = 1, 1.0 + 0j
                                if lll < 0:
                                    imag1, minu = -1j, -1
                                if mm % 2 == 1:
                                    imag1, minu = -imag1, -minu
                                if mm > 0:
                                    minu = 1
                                g = g * imag1 * float(minu) / math.sqrt(2.0)
                            gl.append((l0, ll, lp, lmx, m, mp, g))
                    if mm > 0:
                        mm = -mm
                        continue
                    break
    if at.iatnr > 0 and len(lm_all) > 1:
        cbcomb(lm, vlm)
    vns, vnslo = {}, {}
    prev = None
    for (l0, ll, lp, lm1, m, mp, g) in gl:
        key = (l0, ll, lp, lm1)
        if key == prev:
            continue
        v = vlm[lm1 - 1]
        A, B, AE, BE = A1[l0] * v, B1[l0] * v, AE1[l0] * v, BE1[l0] * v
        vns[(l0, lm1, lp)] = (ri(A, B, A1[lp], B1[lp]), ri(AE, BE, AE1[lp], BE1[lp]), ri(A, B, AE1[lp], BE1[lp]))
        if l0 <= LOMAX and rad.loor[l0]:
            A, B = A1LO[l0] * v, B1LO[l0] * v
            lolo = 0.0
            if lp <= LOMAX and rad.loor[lp]:
                lolo = ri(A, B, A1LO[lp], B1LO[lp])
            vnslo[(l0, lm1, lp)] = (ri(A, B, A1[lp], B1[lp]), ri(A, B, AE1[lp], BE1[lp]), lolo)
        prev = key
    rad.lm, rad.gaunts, rad.vns, rad.vnslo = lm, gl, vns, vnslo


def tns_arrays(rads: List[AtomRadial], lnsmax: int):
    """The gaunt list and radial integrals in the reference's module layout
    (LQIND, LQNS, GFAC, VNS1..3, VNS1LO..3LO) for lapw1gpu_tns_from_gaunt."""
    nat = len(rads)
    ngau = max(1, max(len(r.gaunts) for r in rads))
    lmmx = max(1, max(len(r.lm) for r in rads))
    lqind = np.array([len(r.gaunts) for r in rads], dtype=np.int32)
    lqns = np.zeros((nat, ngau, 6), dtype=np.int32)
    gfac = np.zeros((nat, ngau), dtype=np.complex128)
    v = [np.zeros((nat, NSLMAX, lmmx, NSLMAX)) for _ in range(3)]
    vlo = [np.zeros((nat, NSLMAX, lmmx, LOMAX + 1)) for _ in range(3)]
    loor = np.zeros((nat, LOMAX + 1), dtype=np.int32)
    for a, r in enumerate(rads):
        loor[a] = r.loor
        for i, (l0, ll, lp, lmx, m, mp, g) in enumerate(r.gaunts):
            lqns[a, i] = (l0 + 1, ll, lp + 1, lmx, m, mp)
            gfac[a, i] = g
        for (l0, lm1, lp), vals in r.vns.items():
            for q in range(3):
                v[q][a, lp, lm1 - 1, l0] = vals[q]            # VNSq(L0+1, LM1, LP+1)
        for (l0, lm1, lp), vals in r.vnslo.items():
            vlo[0][a, lp, lm1 - 1, l0] = vals[0]              # VNS1LO(L0+1, LM1, LP+1)
            vlo[1][a, lp, lm1 - 1, l0] = vals[1]
            if lp <= LOMAX:
                vlo[2][a, lp, lm1 - 1, l0] = vals[2]
    return lqind, lqns, gfac, v, vlo, loor


# ----------------------------------------------------------------- symmetry
def rotdef(struct: Struct) -> np.ndarray:
    """ROTIJ of every atom (rotdef.f): the first symmetry operation that
    maps the type's first atom onto it, as the C view [col][row] of
    ROTIJ(3,3) (i.e. the operation's lines as case.struct writes them)."""
    toler = 1.0e-7
    toler2 = 1.5 * toler
    lat = struct.lattic.upper()
    out = []
    for at in struct.atoms:
        p1 = at.pos[0]
        for pm in at.pos:
            found = None
            for i in range(len(struct.imat)):
                x = struct.imat[i] @ p1 + struct.tau[i]
                x1 = np.mod(np.abs(x - pm) + toler, 1.0) - toler
                if np.max(np.abs(x1)) < toler2:
                    found = i
                    break
                if lat[0] == "B":
                    y = np.mod(x1 + 0.5 + toler, 1.0) - toler
                    if np.max(np.abs(y)) < toler2:
                        found = i
                        break
                if lat[0] == "F" or lat[:3] == "CXY":
                    x1[:2] = np.mod(x1[:2] + 0.5 + toler, 1.0) - toler
                    if np.max(np.abs(x1)) < toler2:
                        found = i
                        break
                    x1[:2] = np.mod(x1[:2] + 0.5, 1.0)
                if lat[0] == "F" or lat[:3] == "CXZ":
                    x1[0] = math.fmod(x1[0] + 0.5 + toler, 1.0) - toler
                    x1[2] = math.fmod(x1[2] + 0.5 + toler, 1.0) - toler
                    if np.max(np.abs(x1)) < toler2:
                        found = i
                        break
                    x1[0] = math.fmod(x1[0] + 0.5, 1.0)
                    x1[2] = math.fmod(x1[2] + 0.5, 1.0)
                if lat[0] == "F" or lat[:3] == "CYZ":
                    x1[1:] = np.mod(x1[1:] + 0.5 + toler, 1.0) - toler
                    if np.max(np.abs(x1)) < toler2:
                        found = i
                        break
            if found is None:
                raise ValueError("ROTDEF: no symmetry operation found")
            out.append(np.array(struct.imat[found], dtype=np.float64))
    return np.stack(out)


def _matmm(a, b):
    return np.asarray(a) @ np.asarray(b)


def locdef(rotij_c: np.ndarray, br2: np.ndarray) -> np.ndarray:
    """ROTIJ of a non-orthogonal lattice in Cartesian form (latgen.f:
    GBAS = BR2 / 2 pi, RBAS = GBAS^-1 (gbass.f), ROTIJ := GBAS ROTIJ RBAS;
    locdef.f), in and out as the C view [col][row]."""
    gbas = np.asarray(br2, dtype=np.float64) / (2.0 * math.pi)
    rbas = np.linalg.inv(gbas)
    out = []
    for rc in rotij_c:
        R = np.asarray(rc).T                     # R[row, col] = ROTIJ(row, col)
        out.append((_matmm(_matmm(gbas, R), rbas)).T)
    return np.stack(out)


# ----------------------------------------------------------------- the problem
def problem_from_case(struct: Struct, in1: In1, vsp, vns: Optional[Vns], k, rads=None, tns=None,
                      name: str = "") -> Problem:
    """One k-point's Problem from the case files: k as SETKPT stores it
    (ISX/IDV, ISY/IDV, ISZ/IDV).  rads / tns (ATPAR's results and the T
    blocks) may be passed to reuse them across k-points."""
    from . import lapw1gpu
    lt = struct.lattic
    br2, ortho, pia = lattice.latgen(lt, *struct.abc, *struct.angles)
    ltop = min(in1.lmax + 1, LDL)
    lnsmax = in1.lnsmax if in1.lnsmax > 0 else 2
    lnsmax = min(lnsmax, NSLMAX - 1)
    if rads is None:
        rads = atpar(struct, in1, vsp, vns, ltop, lnsmax)
    nat = len(struct.atoms)
    mult = np.array([a.mult for a in struct.atoms], dtype=np.int32)
    rmt = np.array([a.rmt for a in struct.atoms])
    pos = np.concatenate([a.pos for a in struct.atoms]).astype(np.float64)
    rotij = rotdef(struct)
    if not ortho and not lt.upper().startswith("CXZ"):
        rotij = locdef(rotij, br2)
    rotloc = np.stack([a.rotloc for a in struct.atoms])
    omega = (2.0 * math.pi) ** 3 / abs(np.linalg.det(br2))
    vi = 1.0 / omega
    v = 4.0 * math.pi * vi * rmt ** 3 / 3.0
    ilo = np.stack([r.ilo for r in rads])
    loor = np.stack([r.loor for r in rads])
    lapw = np.stack([r.lapw for r in rads])
    rkm = in1.rkmax / float(rmt.min())
    nv, kzz, xk, yk, zk, rk = lattice.basis(rkm, np.asarray(k, dtype=np.float64), br2, ortho, pia, lt, mult, ilo,
                                            pos, rotij, rotloc)
    nlo = int(sum((2 * l + 1) * mult[a] * ilo[a, l] for a in range(nat) for l in range(LOMAX + 1)))
    ins = 0 if vns is not None else 1
    if ins == 0:
        imat, tau = warp.symops_from_struct([{"imat": m.tolist(), "tau": t.tolist()}
                                             for m, t in zip(struct.imat, struct.tau)])
        wtab, _, _ = warp.setwar(vns.potk, imat, tau)
        if tns is None:
            lqind, lqns, gfac, vv, vlo, lo_ = tns_arrays(rads, lnsmax)
            tns = lapw1gpu.tns_from_gaunt(nat, lnsmax, lqind, lqns, gfac, vv[0], vv[1], vv[2], vlo[0], vlo[1],
                                          vlo[2], lo_)
    else:
        wtab = np.zeros((1, 1, 1), dtype=np.complex128)
        tns = np.zeros((nat, 9, 25, 25), dtype=np.complex128)
    st = lambda f: np.stack([getattr(r, f) for r in rads])  # noqa: E731
    prob = Problem(nv=nv, nlo=nlo, ltop=ltop, lnsmax=lnsmax, vi=vi, mult=mult, rmt=rmt, v=v, pos=pos,
                   rotij=rotij, rotloc=rotloc, kzz=kzz, xk=xk, yk=yk, zk=zk, rk=rk,
                   p=st("p"), pe=st("pe"), dp=st("dp"), dpe=st("dpe"), pei=st("pei"), e=st("e"), lapw=lapw,
                   ilo=ilo, loor=loor, alo=st("alo"), blo=st("blo"), clo=st("clo"), elo=st("elo"),
                   pi12lo=st("pi12lo"), pe12lo=st("pe12lo"), dplo=st("dplo"),
                   warp=wtab, tns=tns, ins=ins, nohns=0 if ins == 0 else 1, name=name,
                   bkzz=lattice.kzz_matrix(br2, ortho, pia, lt),
                   meta=dict(k=tuple(float(x) for x in k), rkmax=in1.rkmax, omega=omega, br2=br2, lattic=lt,
                             abc=struct.abc, emin=in1.emin, emax=in1.emax))
    prob.validate()
    return prob
