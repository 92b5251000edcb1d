"""Generalized eigen-solve of the packed H,S on the GPU (SECLR4's role).

SECLR4 (seclr4.F:158-345) conjugates HS/HSDIAG, factors the upper triangle
(ZPOTRF 'U', which ZHCGST takes as the factor of S**T), reduces H from the
lower triangle to the standard problem (ZHCGST), solves it (ZHEEVX2, energy window EL..EU) and
back-transforms the eigenvectors (ZTRSM).  This module does the same on
the device with the cuSOLVER routines torch.linalg exposes (Cholesky,
triangular solves, Hermitian eigen-decomposition); it is the consumer of
the setup, used by the force adjoint and by eigenvalue checks.
"""
from __future__ import annotations

from typing import Optional, Tuple

import torch


def hermitian_from_packed_device(hs: torch.Tensor, hsdiag: torch.Tensor) -> Tuple[torch.Tensor, torch.Tensor]:
    """H and S (complex128, n x n, row-major torch layout of the math
    matrices) from the packed state on the device.  `hs` is the caller's
    column-major HS viewed as a torch tensor of shape [n(col)][n(row)]
    complex (i.e. hs[c, r] = HS(r, c)); `hsdiag` is HSDIAG.  H comes from
    the lower triangle; S is the transpose of the Hermitian matrix the upper
    triangle stores (ZHCGST factors S**T, zhcgst.f:34-42), so
    S(i,j) = conj(HS(j,i)) for i > j."""
    m = hs.transpose(0, 1).conj()              # m[r, c] = conj(HS(r, c))
    low = torch.tril(m, -1)
    up = torch.triu(m, 1).transpose(0, 1)      # up[i, j] = conj(HS(j, i)), i > j
    H = low + low.conj().transpose(0, 1) + torch.diag(torch.diagonal(m).real.to(m.dtype))
    S = up + up.conj().transpose(0, 1) + torch.diag(hsdiag.conj().real.to(m.dtype))
    return H, S


def solve(H: torch.Tensor, S: torch.Tensor, el: float = -1e70, eu: float = 1e70,
          nmax: Optional[int] = None) -> Tuple[torch.Tensor, torch.Tensor]:
    """Eigenvalues (ascending, within [el, eu], at most nmax) and
    S-orthonormal eigenvectors (columns) of H x = e S x."""
    L = torch.linalg.cholesky(S)                       # S = L L^H (L = U^H)
    Y = torch.linalg.solve_triangular(L, H, upper=False)
    A = torch.linalg.solve_triangular(L, Y.conj().transpose(0, 1), upper=False)   # L^-1 H L^-H
    A = 0.5 * (A + A.conj().transpose(0, 1))
    w, V = torch.linalg.eigh(A)
    sel = (w >= el) & (w <= eu)
    w, V = w[sel], V[:, sel]
    if nmax is not None:
        w, V = w[:nmax], V[:, :nmax]
    X = torch.linalg.solve_triangular(L.conj().transpose(0, 1), V, upper=True)    # back-transform
    return w, X


def eigenvalues(H: torch.Tensor, S: torch.Tensor, nmax: Optional[int] = None) -> torch.Tensor:
    """The ascending eigenvalues of H x = e S x (the lowest nmax), without
    eigenvectors: the same reduction as `solve`, then the eigenvalue-only
    Hermitian solver."""
    L = torch.linalg.cholesky(S)
    Y = torch.linalg.solve_triangular(L, H, upper=False)
    A = torch.linalg.solve_triangular(L, Y.conj().transpose(0, 1), upper=False)
    A = 0.5 * (A + A.conj().transpose(0, 1))
    w = torch.linalg.eigvalsh(A)
    return w if nmax is None else w[:nmax]
