"""The algebra behind the adjoint's spherical projections (forces.cuh:
frc_zlm, k_force_rsph, k_force_pre), restated in numpy on seeded inputs.

  * the real harmonics of frc_zlm's recursion (Q_mm = (2m-1)!!, the
    three-term recursion in l, sqrt((2l+1)(l-m)!/(l+m)!), sqrt 2 and
    Re/Im (ux + i uy)^m for m != 0) satisfy sum_m Z_lm(u) Z_lm(v) =
    (2l+1) P_l(u.v) for l <= 10;
  * the pair sum of k_force_sph over J < I (the Legendre recursion with
    hamilt.F's UTOP branch, the H and S coefficient forms, the phases and
    -4 pi (KZZ_I - KZZ_J)) equals the blocked form: block projections
    against the running sum of the earlier blocks plus the pairs inside
    each block, with mAB != mBA (no symmetric shortcut) and a zero
    k-vector row.
The GPU tests check the kernels themselves against the FP64 adjoint.
"""
from math import factorial

import numpy as np

LT = 11


def zlm(u, L=LT):
    """Z_lm(u) for lm = l l + l + m, the recursion of frc_zlm."""
    ux, uy, uz = u
    out = np.zeros(L * L)
    for l in range(L):
        for m in range(-l, l + 1):
            am = abs(m)
            q0 = 1.0
            for k in range(1, am + 1):
                q0 *= 2 * k - 1
            q = q0
            if l > am:
                qm2, qm1 = q0, (2 * am + 1) * uz * q0
                for ll in range(am + 2, l + 1):
                    qm2, qm1 = qm1, ((2 * ll - 1) * uz * qm1 - (ll + am - 1) * qm2) / (ll - am)
                q = qm1
            nrm = np.sqrt((2 * l + 1) * factorial(l - am) / factorial(l + am))
            if am == 0:
                v = nrm * q
            else:
                c = (ux + 1j * uy) ** am
                v = np.sqrt(2.0) * nrm * q * (c.real if m > 0 else c.imag)
            out[l * l + l + m] = v
    return out


def legendre_weights(x):
    """(2l+1) P_l(x) as k_force_sph forms them (UTOP branch for |x| >= 0.9999999)."""
    w = np.zeros(LT)
    pm2, pm1 = 1.0, x
    w[0], w[1] = 1.0, 3.0 * x
    top = not abs(x) < 0.9999999
    for l in range(2, LT):
        pplx = x * pm1
        pl = x * pm1 if top else pplx + (l - 1) / l * (pplx - pm2)
        pm2, pm1 = pm1, pl
        w[l] = (2 * l + 1) * pl
    return w


def test_addition_theorem_of_the_harmonics():
    rng = np.random.default_rng(7)
    for _ in range(20):
        u, v = rng.normal(size=3), rng.normal(size=3)
        u, v = u / np.linalg.norm(u), v / np.linalg.norm(v)
        zu, zv = zlm(u), zlm(v)
        s = np.array([np.sum((zu * zv)[l * l:(l + 1) ** 2]) for l in range(LT)])
        x = float(u @ v)
        exact = np.array([(2 * l + 1) * np.polynomial.legendre.legval(x, [0] * l + [1]) for l in range(LT)])
        assert np.abs(s - exact).max() <= 1e-12 * max(1.0, np.abs(exact).max())
    # the pole: only m = 0 survives
    zp = zlm(np.array([0.0, 0.0, 1.0]))
    for l in range(LT):
        assert abs(zp[l * l + l] - np.sqrt(2 * l + 1)) < 1e-12
        assert np.abs(np.delete(zp[l * l:(l + 1) ** 2], l)).max(initial=0.0) == 0.0


def _case(rng, n=96, nb=5, mult=(1, 2)):
    ntyp = len(mult)
    ndf = sum(mult)
    kv = rng.normal(size=(n, 3))
    kv[3] = 0.0
    al = rng.normal(size=(ntyp, LT, n))
    bl = rng.normal(size=(ntyp, LT, n))
    al[:, 1:, 3] = bl[:, 1:, 3] = 0.0  # l > 0 vanish at k = 0
    coef = {k: rng.normal(size=(ntyp, LT)) for k in ("vif", "chn", "mAA", "mAB", "mBA", "mBB")}
    kzz = rng.integers(-4, 5, size=(n, 3))
    pos = rng.random(size=(ndf, 3))
    phase = np.exp(2j * np.pi * kzz @ pos.T).T
    C = rng.normal(size=(n, nb)) + 1j * rng.normal(size=(n, nb))
    f, eps = rng.random(nb), rng.normal(size=nb)
    tof = np.repeat(np.arange(ntyp), mult)
    return dict(n=n, nb=nb, ndf=ndf, kv=kv, al=al, bl=bl, coef=coef, kzz=kzz, phase=phase, C=C, f=f, eps=eps,
                tof=tof)


def _pair_sum(c, pairs):
    """dE/dr over the given pairs (J < I), as k_force_sph forms it."""
    kv, al, bl, cf, kzz, ph = c["kv"], c["al"], c["bl"], c["coef"], c["kzz"], c["phase"]
    rk = np.linalg.norm(kv, axis=1)
    rho = (c["C"] * c["f"]) @ c["C"].conj().T
    rhoe = (c["C"] * (c["f"] * c["eps"])) @ c["C"].conj().T
    F = np.zeros((c["ndf"], 3))
    for I, J in pairs:
        x = kv[I] @ kv[J]
        den = rk[I] * rk[J]
        if den > 1e-8:
            x /= den
        w = legendre_weights(x)
        for a in range(c["ndf"]):
            t = c["tof"][a]
            v = cf["vif"][t]
            tS = np.sum(w * v * (al[t, :, J] * al[t, :, I] + cf["chn"][t] * bl[t, :, J] * bl[t, :, I]))
            tH = np.sum(w * v * (al[t, :, J] * (cf["mAA"][t] * al[t, :, I] + cf["mAB"][t] * bl[t, :, I])
                                 + bl[t, :, J] * (cf["mBA"][t] * al[t, :, I] + cf["mBB"][t] * bl[t, :, I])))
            cP = np.conj(ph[a, J]) * ph[a, I]
            g = tH * np.imag(cP * rho[J, I]) - tS * np.imag(cP * rhoe[J, I])
            F[a] += g * (-4.0 * np.pi) * (kzz[I] - kzz[J])
    return F


def _projections(c, rows):
    """Y[a, alpha, lm, g, b] over `rows`: the product of k_force_rsph's operand with (G c)^T."""
    kv = c["kv"]
    rk = np.linalg.norm(kv, axis=1)
    Z = np.array([zlm(kv[i] / rk[i] if rk[i] > 0 else np.array([0.0, 0.0, 1.0])) for i in rows])
    lofm = np.concatenate([[l] * (2 * l + 1) for l in range(LT)])
    G = np.concatenate([c["C"][rows][None], (2 * np.pi * c["kzz"][rows]).T[:, :, None] * c["C"][rows][None]])
    Y = np.zeros((c["ndf"], 2, LT * LT, 4, c["nb"]), complex)
    for a in range(c["ndf"]):
        t = c["tof"][a]
        for alpha, A in enumerate((c["al"], c["bl"])):
            L = A[t][lofm][:, rows] * Z.T * np.conj(c["phase"][a, rows])[None, :]
            Y[a, alpha] = np.einsum("kr,grb->kgb", L, G)
    return Y


def _contract(c, Pre, Y):
    """k_force_pre's sum for one block against the prefix."""
    cf = c["coef"]
    lofm = np.concatenate([[l] * (2 * l + 1) for l in range(LT)])
    F = np.zeros((c["ndf"], 3))
    for a in range(c["ndf"]):
        t = c["tof"][a]
        v = cf["vif"][t][lofm]
        MH = np.stack([np.stack([cf["mAA"][t][lofm], cf["mAB"][t][lofm]], -1),
                       np.stack([cf["mBA"][t][lofm], cf["mBB"][t][lofm]], -1)], 1) * v[:, None, None]
        MS = np.zeros_like(MH)
        MS[:, 0, 0], MS[:, 1, 1] = v, v * cf["chn"][t][lofm]
        for comp in range(3):
            X = np.imag(Pre[a][:, None, :, 0] * np.conj(Y[a][None, :, :, comp + 1])
                        - Pre[a][:, None, :, comp + 1] * np.conj(Y[a][None, :, :, 0]))
            tH = np.einsum("kab,abkx,x->", MH, X, c["f"])
            tS = np.einsum("kab,abkx,x->", MS, X, c["f"] * c["eps"])
            F[a, comp] = -2.0 * (tH - tS)
    return F


def test_blocked_projections_equal_the_pair_sum():
    c = _case(np.random.default_rng(3))
    n, B = c["n"], 32
    direct = _pair_sum(c, [(I, J) for I in range(n) for J in range(I)])
    blocks = [list(range(r, min(n, r + B))) for r in range(0, n, B)]
    F = np.zeros_like(direct)
    Pre = None
    for rows in blocks:
        Y = _projections(c, rows)
        if Pre is None:
            Pre = Y
        else:
            F += _contract(c, Pre, Y)
            Pre = Pre + Y
        F += _pair_sum(c, [(I, J) for I in rows for J in rows if J < I])
    assert np.abs(direct).max() > 0
    assert np.abs(F - direct).max() <= 1e-11 * np.abs(direct).max()
