"""Reference band-energy gradients from the oracle (test infrastructure).

Two independent routes to dE/dPOS for E = sum_b occ_b eps_b of the packed
H/S that the oracle builds:
  * `hf_gradient`: Hellmann-Feynman, sum_b occ_b x_b^H (dH - eps_b dS) x_b,
    with dH, dS the fourth-order central differences of the oracle's H, S
    (the elements are trigonometric functions of POS: with h = 1e-5 the
    truncation and rounding errors are both ~1e-11 relative);
  * `fd_band_energy`: central differences of E itself.
"""
from __future__ import annotations

import numpy as np
import scipy.linalg

from hack_wein2k_b200.problem import hermitian_from_packed
from oracle import oracle as O


def hs_of(prob, pos):
    hs, hsd = O.setup(prob.copy(pos=pos))
    return hermitian_from_packed(hs, hsd)


def eigh(prob, pos=None):
    H, S = hs_of(prob, prob.pos if pos is None else pos)
    return scipy.linalg.eigh(H, S)


def gapped_nb(w, lo=4, hi=None):
    """An occupied-band count with a clear gap above it (degenerate sets whole)."""
    hi = hi or max(lo + 1, len(w) // 3)
    gaps = np.diff(w[:hi + 1])
    nb = int(np.argmax(gaps[lo - 1:hi])) + lo
    return nb, float(gaps[nb - 1])


def hf_gradient(prob, nb, occ=None, atoms=None, h=1.0e-5):
    w, X = eigh(prob)
    occ = np.ones(nb) if occ is None else np.asarray(occ)
    Xb, wb = X[:, :nb], w[:nb]
    atoms = range(prob.ndf) if atoms is None else atoms
    g = np.zeros((prob.ndf, 3))
    for a in atoms:
        for c in range(3):
            mats = []
            for step in (2.0, 1.0, -1.0, -2.0):
                q = np.array(prob.pos, dtype=np.float64, copy=True)
                q[a, c] += step * h
                mats.append(hs_of(prob, q))
            (H2, S2), (H1, S1), (Hm1, Sm1), (Hm2, Sm2) = mats
            dH = (-H2 + 8.0 * H1 - 8.0 * Hm1 + Hm2) / (12.0 * h)
            dS = (-S2 + 8.0 * S1 - 8.0 * Sm1 + Sm2) / (12.0 * h)
            t = np.einsum("ib,ij,jb->b", Xb.conj(), dH, Xb) - wb * np.einsum("ib,ij,jb->b", Xb.conj(), dS, Xb)
            g[a, c] = float(np.sum(occ * t.real))
    return g


def fd_band_energy(prob, nb, a, c, h=1.0e-5, occ=None):
    occ = np.ones(nb) if occ is None else np.asarray(occ)
    vals = []
    for sgn in (1.0, -1.0):
        pos = np.array(prob.pos, dtype=np.float64, copy=True)
        pos[a, c] += sgn * h
        w, _ = eigh(prob, pos)
        vals.append(float(np.sum(occ * w[:nb])))
    return (vals[0] - vals[1]) / (2 * h)
