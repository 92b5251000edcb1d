"""Seeded synthetic inputs for the H/S setup.

The reference's inputs come from lapw0 (potential) and ATPAR (radial
solution); neither runs here, so each workload draws them from a seeded
generator with the distributions the benchmark definitions give:

  u(R), u'(R), udot(R), udot'(R), |udot|^2 ~ U[0.2, 1.5]; E_l ~ U[-0.5, 1.0] Ry
  non-spherical T blocks ~ N(0, 0.01 Ry), Hermitian over (u, udot, lo) x (l,m)
  interstitial V(G), |G| <= 12 1/bohr: N(0,1)/(1+|G|^2), V(-G) = conj V(G)
  LO coefficients A, B, C, u_lo'(R) like the radial values, E_lo like E_l;
  the overlap integrals PI12LO, PE12LO ~ U[0.05, 0.4] (x |udot| for PE12LO)
  so that the (u, udot, u_lo) Gram matrix stays positive definite and S is
  an overlap matrix (Cholesky in the eigen-solve succeeds).

Workloads (seed = 1000 + index, numpy default_rng):
  c0  fcc, a=7.65, 1 atom, Rmt 2.5, RKmax 7 (~40 PW), lmax 10, lmax_ns 4,
      k = (0.1, 0.2, 0.3) 2pi/a
  c1  2x2x2 cubic ABO3 supercell a=14.8, Rmt 2.2/1.9/1.6, RKmax 7
      (~4600 PW) + one LO per atom for l<=2, one general k
  c2  c1 at 64 seeded k-points in the irreducible wedge
  c3  100 atoms, 20x20x20 bohr box, random positions (min separation
      3.8 bohr), Rmt 1.8-2.3 (shrunk so spheres never overlap), RKmax 6,
      LO for l<=2
  c4  c3's cell at RKmax 8, 16 k-points
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Sequence

import numpy as np

from .lattice import basis, kzz_matrix, latgen
from .problem import LOMAX, NLOAT, NSL2, NTNS, Problem

LDL = 13  # LMAX of lapw1's param.inc: leading dimension of per-l arrays


@dataclass
class Cell:
    lattic: str
    abc: tuple
    angles: tuple
    types: list          # per type: dict(pos=[[x,y,z],...], rmt=float)


def _rand_rot(rng):
    q, r = np.linalg.qr(rng.standard_normal((3, 3)))
    q = q * np.sign(np.diag(r))
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    return q


def make_warp(rng, br2, gmax=12.0):
    """V(G) on the integer box of |BR2 n| <= gmax, V(-n) = conj V(n)."""
    binv = np.linalg.inv(br2)
    w = [int(math.floor(np.linalg.norm(binv[i]) * gmax)) + 1 for i in range(3)]
    n1 = np.arange(-w[0], w[0] + 1)
    n2 = np.arange(-w[1], w[1] + 1)
    n3 = np.arange(-w[2], w[2] + 1)
    N3, N2, N1 = np.meshgrid(n3, n2, n1, indexing="ij")
    g = np.stack([N1, N2, N3], axis=-1) @ br2.T
    gl = np.linalg.norm(g, axis=-1)
    vals = (rng.standard_normal(gl.shape) + 1j * rng.standard_normal(gl.shape)) / (1.0 + gl ** 2)
    vals[gl > gmax] = 0.0
    # Hermitian in G: table[z,y,x] <-> table[-z,-y,-x]
    flipped = np.conj(vals[::-1, ::-1, ::-1])
    vals = 0.5 * (vals + flipped)
    c = tuple(x // 2 for x in vals.shape)
    vals[c] = vals[c].real
    return np.ascontiguousarray(vals)


def make_tns(rng, nat, lnsmax, loor, scale=0.01):
    """T blocks [nat, 9, 25, 25] from a Hermitian (u,udot,lo)x(l,m) matrix."""
    K = NSL2
    nsl2 = (lnsmax + 1) ** 2
    tns = np.zeros((nat, NTNS, K, K), dtype=np.complex128)
    lm_l = np.array([l for l in range(5) for _ in range(2 * l + 1)])
    for a in range(nat):
        M = scale * (rng.standard_normal((3 * K, 3 * K)) + 1j * rng.standard_normal((3 * K, 3 * K)))
        M = 0.5 * (M + M.conj().T)
        mask = np.zeros(3 * K, dtype=bool)
        for r in range(3):
            for lm in range(nsl2):
                l = lm_l[lm]
                if r < 2 or (l <= LOMAX and loor[a][l]):
                    mask[r * K + lm] = True
        M[~mask, :] = 0
        M[:, ~mask] = 0
        blk = 0
        for r0 in range(3):
            for rp in range(3):
                tns[a, blk] = M[r0 * K:(r0 + 1) * K, rp * K:(rp + 1) * K]
                blk += 1
    return tns


def _radial(rng, nat, ltop):
    u = lambda: rng.uniform(0.2, 1.5, size=(nat, LDL))
    p, pe, dp, dpe, pei = u(), u(), u(), u(), u()
    e = rng.uniform(-0.5, 1.0, size=(nat, LDL))
    return p, pe, dp, dpe, pei, e


def synth_problem(cell: Cell, rkmax: float, k, *, lmax=10, lnsmax=4, lo_l: Sequence[int] = (),
                  apw_l: Sequence[int] = (), seed=0, ins=0, rotate_local=False,
                  orb: Sequence[tuple] = (), gmax=12.0, name="", rng=None, params=None) -> Problem:
    """One k-point problem on `cell`.

    lo_l   l values carrying one LAPW-type LO (LOOR) on every atom type
    apw_l  l values treated as APW+lo (LAPW flag off, one 'lo' each)
    orb    HORB atoms: tuples (atom type 1-based, (l,...))
    params reuse of the radial/potential draws of another k-point (dict)
    """
    rng = rng if rng is not None else np.random.default_rng(seed)
    br2, ortho, pia = latgen(cell.lattic, *cell.abc, *cell.angles)
    nat = len(cell.types)
    mult = np.array([len(t["pos"]) for t in cell.types], dtype=np.int32)
    rmt = np.array([t["rmt"] for t in cell.types], dtype=np.float64)
    pos = np.array([p for t in cell.types for p in t["pos"]], dtype=np.float64)
    ndf = int(mult.sum())
    # unit-cell volume from the reciprocal basis: Omega = (2pi)^3 / det(BR2)
    omega = (2 * math.pi) ** 3 / abs(np.linalg.det(br2))
    vi = 1.0 / omega
    v = 4.0 * math.pi * vi * rmt ** 3 / 3.0
    ltop = lmax + 1

    if params is None:
        params = {}
        if rotate_local:
            params["rotloc"] = np.stack([_rand_rot(rng).T for _ in range(nat)])
            params["rotij"] = np.stack([_rand_rot(rng).T for _ in range(ndf)])
        else:
            params["rotloc"] = np.stack([np.eye(3)] * nat)
            params["rotij"] = np.stack([np.eye(3)] * ndf)
        params["radial"] = _radial(rng, nat, ltop)
        lapw = np.ones((nat, LDL), dtype=np.int32)
        ilo = np.zeros((nat, LOMAX + 1), dtype=np.int32)
        loor = np.zeros((nat, LOMAX + 1), dtype=np.int32)
        for l in apw_l:
            lapw[:, l] = 0
            ilo[:, l] += 1
        for l in lo_l:
            ilo[:, l] += 1
            loor[:, l] = 1
        sh = (nat, NLOAT, LOMAX + 1)
        alo = rng.uniform(0.2, 1.5, size=sh)
        blo = rng.uniform(0.2, 1.5, size=sh)
        clo = rng.uniform(0.2, 1.5, size=sh)
        elo = rng.uniform(-0.5, 1.0, size=sh)
        for a in range(nat):
            for l in apw_l:
                clo[a, 0, l] = 0.0        # APW+lo 'lo': C = 0 (abc.f:51-55)
        pei = params["radial"][4]
        pi12lo = rng.uniform(0.05, 0.4, size=(nat, LOMAX + 1))
        pe12lo = rng.uniform(0.05, 0.4, size=(nat, LOMAX + 1)) * np.sqrt(pei[:, :LOMAX + 1])
        dplo = rng.uniform(0.2, 1.5, size=(nat, LOMAX + 1))
        params["lo"] = (lapw, ilo, loor, alo, blo, clo, elo, pi12lo, pe12lo, dplo)
        params["warp"] = make_warp(rng, br2, gmax)
        params["tns"] = make_tns(rng, nat, lnsmax, loor)
        if orb:
            iatom = np.array([o[0] for o in orb], dtype=np.int32)
            nlorb = np.array([len(o[1]) for o in orb], dtype=np.int32)
            lorb = np.zeros((len(orb), 3), dtype=np.int32)
            vorb = np.zeros((len(orb), 4, 7, 7), dtype=np.complex128)
            for i, o in enumerate(orb):
                for j, l in enumerate(o[1]):
                    lorb[i, j] = l
                    m = 0.01 * (rng.standard_normal((2 * l + 1, 2 * l + 1)) + 1j * rng.standard_normal((2 * l + 1, 2 * l + 1)))
                    m = 0.5 * (m + m.conj().T)
                    vorb[i, l, 3 - l:4 + l, 3 - l:4 + l] = m
            params["orb"] = (iatom, nlorb, lorb, vorb)
    lapw, ilo, loor, alo, blo, clo, elo, pi12lo, pe12lo, dplo = params["lo"]
    p, pe, dp, dpe, pei, e = params["radial"]
    rkm = rkmax / float(rmt.min())
    nlo = int(sum((2 * l + 1) * mult[a] * ilo[a, l] for a in range(nat) for l in range(LOMAX + 1)))
    nv, kzz, xk, yk, zk, rk = basis(rkm, np.asarray(k, dtype=np.float64), br2, ortho, pia, cell.lattic,
                                    mult, ilo, pos, params["rotij"], params["rotloc"])
    kw = {}
    if "orb" in params:
        iatom, nlorb, lorb, vorb = params["orb"]
        kw = dict(iatom=iatom, nlorb=nlorb, lorb=lorb, vorb=vorb)
    prob = Problem(nv=nv, nlo=nlo, ltop=ltop, lnsmax=lnsmax, vi=vi, mult=mult, rmt=rmt, v=v, pos=pos,
                   rotij=params["rotij"], rotloc=params["rotloc"], kzz=kzz, xk=xk, yk=yk, zk=zk, rk=rk,
                   p=p, pe=pe, dp=dp, dpe=dpe, pei=pei, e=e, lapw=lapw, ilo=ilo, loor=loor,
                   alo=alo, blo=blo, clo=clo, elo=elo, pi12lo=pi12lo, pe12lo=pe12lo, dplo=dplo,
                   warp=params["warp"], tns=params["tns"], ins=ins, name=name,
                   bkzz=kzz_matrix(br2, ortho, pia, cell.lattic),
                   meta=dict(k=tuple(float(x) for x in k), rkmax=rkmax, omega=omega, br2=br2,
                             lattic=cell.lattic, abc=cell.abc), **kw)
    prob.validate()
    prob._params = params
    return prob


# ---------------------------------------------------------------- cells
def cell_fcc1():
    return Cell("F", (7.65, 7.65, 7.65), (90.0, 90.0, 90.0), [dict(pos=[[0.0, 0.0, 0.0]], rmt=2.5)])


def cell_abo3_222(a=14.8, rmt=(2.2, 1.9, 1.6)):
    types = []
    half = 0.5
    for i in range(2):
        for j in range(2):
            for k in range(2):
                types.append(dict(pos=[[i * half, j * half, k * half]], rmt=rmt[0]))
    for i in range(2):
        for j in range(2):
            for k in range(2):
                types.append(dict(pos=[[(i + .5) * half, (j + .5) * half, (k + .5) * half]], rmt=rmt[1]))
    for i in range(2):
        for j in range(2):
            for k in range(2):
                for f in ((.5, .5, 0.), (.5, 0., .5), (0., .5, .5)):
                    types.append(dict(pos=[[(i + f[0]) * half, (j + f[1]) * half, (k + f[2]) * half]], rmt=rmt[2]))
    return Cell("P", (a, a, a), (90.0, 90.0, 90.0), types)


def cell_random100(seed=1003, natom=100, box=20.0, dmin=3.8, rlo=1.8, rhi=2.3):
    rng = np.random.default_rng(seed)
    pts = []
    while len(pts) < natom:
        c = rng.uniform(0, box, size=3)
        ok = True
        for q in pts:
            d = c - q
            d -= box * np.round(d / box)
            if np.linalg.norm(d) < dmin:
                ok = False
                break
        if ok:
            pts.append(c)
    pts = np.array(pts)
    dd = pts[:, None, :] - pts[None, :, :]
    dd -= box * np.round(dd / box)
    dist = np.linalg.norm(dd, axis=-1) + np.eye(natom) * 1e9
    dnn = dist.min(axis=1)
    rmt = np.minimum(rng.uniform(rlo, rhi, size=natom), 0.98 * dnn / 2.0)
    types = [dict(pos=[list(pts[i] / box)], rmt=float(rmt[i])) for i in range(natom)]
    return Cell("P", (box, box, box), (90.0, 90.0, 90.0), types)


def wedge_kpoints(rng, nk):
    """k in the irreducible wedge of the simple-cubic zone, 0 <= kx <= ky <= kz <= 0.5 (2pi/a)."""
    out = []
    while len(out) < nk:
        k = np.sort(rng.uniform(0.0, 0.5, size=3))
        out.append(k)
    return out


def config(name: str, nk: int | None = None, kofs: int = 0) -> List[Problem]:
    """Workloads c0..c4 (see module docstring) and small test cases.

    For the k-point lists (c2, c4) the k-points come from their own seeded
    stream, apart from the crystal's draws: k-points kofs .. kofs+nk-1 of
    that stream, on the same crystal for every kofs (a k-point shard of one
    run, as lapw1para splits a k-list)."""
    if name == "c0":
        rng = np.random.default_rng(1000)
        return [synth_problem(cell_fcc1(), 7.0, (0.1, 0.2, 0.3), rng=rng, name="c0")]
    if name == "c1":
        rng = np.random.default_rng(1001)
        return [synth_problem(cell_abo3_222(), 7.0, wedge_kpoints(rng, 1)[0], lo_l=(0, 1, 2), rng=rng, name="c1k0")]
    if name == "c3":
        rng = np.random.default_rng(1003)
        k = rng.uniform(0.0, 0.5, size=3)
        return [synth_problem(cell_random100(), 6.0, k, lo_l=(0, 1, 2), rng=rng, name="c3k0")]
    if name in ("c2", "c4"):
        idx = 2 if name == "c2" else 4
        rng = np.random.default_rng(1000 + idx)
        rng_k = np.random.default_rng([1000 + idx, 1])
        nkk = nk or (64 if name == "c2" else 16)
        if name == "c2":
            cell, rkmax = cell_abo3_222(), 7.0
            ks = wedge_kpoints(rng_k, kofs + nkk)[kofs:]
        else:
            cell, rkmax = cell_random100(), 8.0
            ks = [rng_k.uniform(0.0, 0.5, size=3) for _ in range(kofs + nkk)][kofs:]
        out, params = [], None
        for i, k in enumerate(ks):
            pr = synth_problem(cell, rkmax, k, lo_l=(0, 1, 2), rng=rng, params=params, name=f"{name}k{kofs + i}")
            params = pr._params
            out.append(pr)
        return out
    raise ValueError(name)


# ---------------------------------------------------------------- small test cells
def cell_small_mixed():
    """P orthorhombic cell with a MULT=2 type and a MULT=1 type."""
    return Cell("P", (6.1, 6.6, 7.2), (90.0, 90.0, 90.0), [
        dict(pos=[[0.0, 0.0, 0.0], [0.5, 0.5, 0.5]], rmt=2.0),
        dict(pos=[[0.5, 0.0, 0.25]], rmt=1.7),
    ])


def cell_many_equiv():
    """P cubic cell (10.5 bohr) on a 3 x 3 x 3 grid of sites 3.5 bohr apart:
    one type of MULT 17 (more equivalent atoms than one staged chunk of the
    force kernel holds) and five one-atom types, Rmt 1.1 everywhere."""
    sites = [[(i + 0.5) / 3.0, (j + 0.5) / 3.0, (k + 0.5) / 3.0] for i in range(3) for j in range(3) for k in range(3)]
    types = [dict(pos=sites[:17], rmt=1.1)] + [dict(pos=[sites[17 + 2 * t]], rmt=1.1) for t in range(5)]
    return Cell("P", (10.5, 10.5, 10.5), (90.0, 90.0, 90.0), types)


def small_case(kind: str = "lo", seed: int = 7, rkmax: float = 5.0) -> Problem:
    """Small problems that exercise every branch: LOs with MULT>1, APW+lo,
    local rotations, HORB, INS != 0."""
    cell = cell_small_mixed()
    k = (0.13, 0.27, 0.41)
    if kind == "plain":
        return synth_problem(cell, rkmax, k, seed=seed, name="small-plain")
    if kind == "lo":
        return synth_problem(cell, rkmax, k, seed=seed, lo_l=(0, 1, 2), rotate_local=True, name="small-lo")
    if kind == "apw":
        return synth_problem(cell, rkmax, k, seed=seed, apw_l=(0, 1), lo_l=(1,), rotate_local=True,
                             name="small-apw")
    if kind == "ins":
        return synth_problem(cell, rkmax, k, seed=seed, lo_l=(0,), ins=1, name="small-ins")
    if kind == "orb":
        return synth_problem(cell, rkmax, k, seed=seed, lo_l=(2,), apw_l=(0,), rotate_local=True,
                             orb=((1, (2,)), (2, (1, 2))), name="small-orb")
    if kind == "multilo":
        return synth_problem(cell, rkmax, k, seed=seed, lo_l=(1, 1), apw_l=(1,), rotate_local=True,
                             name="small-multilo")
    if kind == "gamma":
        return synth_problem(cell, rkmax, (0.0, 0.0, 0.0), seed=seed, lo_l=(0, 1), name="small-gamma")
    if kind == "manyeq":
        return synth_problem(cell_many_equiv(), rkmax, k, seed=seed, name="small-manyeq")
    raise ValueError(kind)
