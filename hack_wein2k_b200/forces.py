"""Band-energy gradients with respect to the atom positions (adjoint of the setup).

E(POS) = sum_b occ[b] eps_b, with eps_b the lowest eigenvalues of the
generalized problem H x = eps S x built from the packed HS/HSDIAG exactly
as SECLR4 reads it (seclr4.F:158-345).  `BandEnergy` is a
`torch.autograd.Function`: the forward pass runs the setup
(lapw1gpu_kpoint_run) and the device eigen-solve (`seclr.solve`), the
backward pass calls lapw1gpu_forces, the Hellmann-Feynman adjoint of the
setup (hack_wein2k_b200/csrc/forces.cuh).  lapw1 itself has no derivative
code; WIEN2k's forces are computed later by lapw2 (SRC_lapw2/fomai1.f,
l2main.F:630-634) from the eigenvectors, on a different formulation, so the
gradient is checked against central finite differences of E.

Positions are POS in lattice coordinates (the `Problem.pos` rows); Cartesian
forces are -(1/2pi) BKZZ dE/dPOS per atom (`cartesian_forces`).
"""
from __future__ import annotations

import dataclasses
from typing import Optional

import numpy as np
import torch

from . import lapw1gpu
from .problem import Problem
from .seclr import hermitian_from_packed_device, solve


def _setup_device(gctx: "lapw1gpu.Context", prob: Problem):
    n = prob.n
    dev = torch.device("cuda", gctx.device)
    kp = gctx.upload(prob)
    hs = torch.zeros((n, n), dtype=torch.complex128, device=dev)   # hs[c, r] = HS(r, c)
    hd = torch.zeros(n, dtype=torch.complex128, device=dev)
    torch.cuda.synchronize(dev)
    kp.run(hs.data_ptr(), n, hd.data_ptr(), stages=7, stats=True)   # stats: returns synchronised
    return kp, hs, hd


def band_energy(gctx: "lapw1gpu.Context", prob: Problem, occ: torch.Tensor):
    """(E, eps, X, kp): band energy of the lowest len(occ) states."""
    kp, hs, hd = _setup_device(gctx, prob)
    H, S = hermitian_from_packed_device(hs, hd)
    nb = occ.shape[0]
    w, X = solve(H, S, nmax=nb)
    return (occ * w).sum(), w, X, kp


def gradient(gctx: "lapw1gpu.Context", kp: "lapw1gpu.KPoint", X: torch.Tensor, occ: torch.Tensor,
             eps: torch.Tensor) -> torch.Tensor:
    """dE/dPOS ([ndf, 3], float64, on the device) for eigenvectors X
    (n x nb columns, S-normalised), occupations and eigenvalues."""
    n, nb = X.shape
    Xc = X.transpose(0, 1).contiguous()          # column-major n x nb, ldc = n
    occ = occ.to(dtype=torch.float64).contiguous()
    eps = eps.to(dtype=torch.float64).contiguous()
    grad = torch.empty((kp.prob.ndf, 3), dtype=torch.float64, device=X.device)
    torch.cuda.synchronize(X.device)             # the library runs on its own stream
    kp.forces(Xc.data_ptr(), n, nb, occ.data_ptr(), eps.data_ptr(), grad.data_ptr())
    return grad


class BandEnergy(torch.autograd.Function):
    """E(pos) = sum occ * eps; pos is a [ndf, 3] float64 CPU tensor (POS)."""

    @staticmethod
    def forward(ctx, pos: torch.Tensor, gctx, prob: Problem, occ: torch.Tensor):
        p2 = dataclasses.replace(prob, pos=pos.detach().cpu().numpy().astype(np.float64).copy())
        dev = torch.device("cuda", gctx.device)
        occ_d = occ.to(device=dev, dtype=torch.float64)
        E, w, X, kp = band_energy(gctx, p2, occ_d)
        ctx.save_for_backward(X, w, occ_d)
        ctx.kp, ctx.gctx = kp, gctx
        return E.detach().cpu()

    @staticmethod
    def backward(ctx, gE):
        X, w, occ_d = ctx.saved_tensors
        g = gradient(ctx.gctx, ctx.kp, X, occ_d, w)
        ctx.kp.free()
        return gE * g.cpu(), None, None, None


def cartesian_forces(prob: Problem, grad: np.ndarray) -> np.ndarray:
    """Forces -dE/dR (Cartesian, Ry/bohr) from dE/dPOS: R = 2 pi BKZZ^-T POS."""
    bk = np.asarray(prob.bkzz, dtype=np.float64).reshape(3, 3)
    return -(np.asarray(grad) @ bk.T) / (2.0 * np.pi)


def finite_difference(gctx: "lapw1gpu.Context", prob: Problem, occ: torch.Tensor, atom: int, comp: int,
                      h: float = 1.0e-5) -> float:
    """Central difference of E along POS[atom, comp] (lattice units)."""
    dev = torch.device("cuda", gctx.device)
    occ_d = occ.to(device=dev, dtype=torch.float64)
    vals = []
    for sgn in (+1.0, -1.0):
        pos = np.array(prob.pos, dtype=np.float64, copy=True)
        pos[atom, comp] += sgn * h
        E, _, _, kp = band_energy(gctx, dataclasses.replace(prob, pos=pos), occ_d)
        kp.free()
        vals.append(float(E))
    return (vals[0] - vals[1]) / (2.0 * h)


def _main() -> None:
    """Time the adjoint on a seeded workload: one setup, the device
    eigen-solve for the lowest `--bands` states, then `--repeat` calls of
    lapw1gpu_forces timed with CUDA events on the current stream.  Prints
    one JSON line."""
    import argparse
    import json

    from . import synth
    ap = argparse.ArgumentParser(prog="python -m hack_wein2k_b200.forces")
    ap.add_argument("--case", default="c3", help="synthetic workload name (c0..c4)")
    ap.add_argument("--prec", choices=["fp64", "split"], default="split")
    ap.add_argument("--bands", type=int, default=400)
    ap.add_argument("--repeat", type=int, default=3)
    a = ap.parse_args()
    dev = torch.device("cuda", 0)
    gctx = lapw1gpu.Context(0)
    if a.prec == "split":
        gctx.set_precision(lapw1gpu.PREC_SPLIT, 5)
        gctx.set_slices(5, 4)
    prob = synth.config(a.case)[0]
    occ = torch.ones(a.bands, dtype=torch.float64, device=dev)
    kp, hs, hd = _setup_device(gctx, prob)
    H, S = hermitian_from_packed_device(hs, hd)
    del hs, hd
    w, X = solve(H, S, nmax=a.bands)
    del H, S
    torch.cuda.empty_cache()
    ms = []
    for _ in range(a.repeat):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        g = gradient(gctx, kp, X, occ, w)
        e1.record()
        torch.cuda.synchronize(dev)
        ms.append(e0.elapsed_time(e1))
    print(json.dumps({"case": a.case, "n": prob.n, "prec": a.prec, "bands": a.bands, "forces_ms": ms,
                      "max_abs_grad": float(g.abs().max())}))
    kp.free()
    gctx.close()


if __name__ == "__main__":
    _main()
