"""Band-energy gradients on the GPU (lapw1gpu_forces, the adjoint of the setup).

lapw1 has no force code and the reference's forces (lapw2 fomai1.f) use a
different formulation, so the adjoint is pinned by
  * the Hellmann-Feynman sum over the ORACLE's dH/dPOS, dS/dPOS (central
    differences of the oracle's matrices, exact to rounding): relative
    tolerance 1e-8 of the largest component;
  * central differences of E itself through the GPU setup and the device
    eigen-solve (the torch.autograd path): 2e-6 of the largest component.
"""
import numpy as np
import pytest
import torch

from hack_wein2k_b200 import forces as FO
from hack_wein2k_b200 import lapw1gpu, synth
from tests import force_ref as FR

# "multilo" is left out: its seeded overlap is indefinite (no eigen-solve)
KINDS = ["plain", "lo", "apw", "ins", "gamma"]
TOL_HF = 1e-8
TOL_FD = 2e-6


def _occ(p, nb):
    return torch.ones(nb, dtype=torch.float64)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", KINDS)
def test_adjoint_matches_oracle_hellmann_feynman(ctx, kind):
    p = synth.small_case(kind)
    w, _ = FR.eigh(p)
    nb, gap = FR.gapped_nb(w)
    ref = FR.hf_gradient(p, nb)
    dev = torch.device("cuda", ctx.device)
    occ = _occ(p, nb).to(dev)
    E, eps, X, kp = FO.band_energy(ctx, p, occ)
    g = FO.gradient(ctx, kp, X, occ, eps).cpu().numpy()
    kp.free()
    assert np.abs(eps.cpu().numpy() - w[:nb]).max() <= 1e-9
    scale = np.abs(ref).max()
    assert np.abs(g - ref).max() <= TOL_HF * scale, (g, ref)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", KINDS)
def test_split_density_matrices_match_fp64(ctx, kind):
    """In split precision lapw1gpu_forces forms rho and rhoE as int8 slice
    products (5 slices); for the same eigenvectors the gradient agrees with
    the FP64 one (ZHERKX density matrices) to 1e-8 of its largest component."""
    p = synth.small_case(kind)
    w, _ = FR.eigh(p)
    nb, _ = FR.gapped_nb(w)
    dev = torch.device("cuda", ctx.device)
    occ = _occ(p, nb).to(dev)
    E, eps, X, kp = FO.band_energy(ctx, p, occ)
    g64 = FO.gradient(ctx, kp, X, occ, eps).cpu().numpy()
    ctx.set_precision(lapw1gpu.PREC_SPLIT, 5)
    try:
        gs = FO.gradient(ctx, kp, X, occ, eps).cpu().numpy()
    finally:
        ctx.set_precision(lapw1gpu.PREC_FP64)
    kp.free()
    scale = np.abs(g64).max()
    assert scale > 0
    assert np.abs(gs - g64).max() <= 1e-8 * scale, (gs, g64)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", KINDS + ["manyeq"])
def test_spherical_projections_match_fp64(ctx, kind):
    """lapw1gpu_set_force_projection: the spherical pairs of two different
    64-row blocks as int8 slice projections (6 slices) against the running
    sum of the earlier blocks, the pairs inside a block on the FP64 pair
    kernel.  Same eigenvectors: the gradient agrees with the FP64 adjoint
    to 1e-8 of its largest component ("gamma" has a zero k-vector row,
    "apw" rows without bl, "manyeq" 17 equivalent atoms of one type)."""
    p = synth.small_case(kind, rkmax=2.5) if kind == "manyeq" else synth.small_case(kind)
    w, _ = FR.eigh(p)
    nb, _ = FR.gapped_nb(w)
    dev = torch.device("cuda", ctx.device)
    occ = _occ(p, nb).to(dev)
    E, eps, X, kp = FO.band_energy(ctx, p, occ)
    g64 = FO.gradient(ctx, kp, X, occ, eps).cpu().numpy()
    ctx.set_precision(lapw1gpu.PREC_SPLIT, 5)
    ctx.set_force_projection(6, 64)
    try:
        gp = FO.gradient(ctx, kp, X, occ, eps).cpu().numpy()
    finally:
        ctx.set_force_projection(-1, 1024)
        ctx.set_precision(lapw1gpu.PREC_FP64)
    kp.free()
    scale = np.abs(g64).max()
    assert scale > 0
    assert np.abs(gp - g64).max() <= 1e-8 * scale, (gp, g64)


@pytest.mark.gpu
def test_force_projection_arguments(ctx):
    """The block must be a multiple of 32 rows, at least 64; slices -1, 0 or 4..8."""
    for bad in [(6, 48), (6, 100), (3, 1024), (9, 1024), (-2, 1024)]:
        with pytest.raises(lapw1gpu.Lapw1GpuError) as e:
            ctx.set_force_projection(*bad)
        assert e.value.code == 7  # LAPW1GPU_ERR_RANGE
    ctx.set_force_projection(-1, 1024)


@pytest.fixture(scope="module")
def manyeq_ref():
    p = synth.small_case("manyeq", rkmax=2.5)
    w, _ = FR.eigh(p)
    nb, _ = FR.gapped_nb(w)
    return p, nb, w, FR.hf_gradient(p, nb)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64", "split"])
def test_adjoint_many_equivalent_atoms(ctx, manyeq_ref, prec):
    """One type of 17 equivalent atoms (more than a staged chunk of the
    spherical force kernel holds: its phases are read from global memory)
    and five one-atom types (the path that forms one type's force terms
    beside the next type's l sums): the gradient of all 22 atoms matches
    the oracle's Hellmann-Feynman sum (split: density matrices as int8
    slice products, 1e-7 of the largest component)."""
    p, nb, w, ref = manyeq_ref
    dev = torch.device("cuda", ctx.device)
    occ = _occ(p, nb).to(dev)
    E, eps, X, kp = FO.band_energy(ctx, p, occ)
    if prec == "split":
        ctx.set_precision(lapw1gpu.PREC_SPLIT, 5)
    try:
        g = FO.gradient(ctx, kp, X, occ, eps).cpu().numpy()
    finally:
        ctx.set_precision(lapw1gpu.PREC_FP64)
        kp.free()
    assert np.abs(eps.cpu().numpy() - w[:nb]).max() <= 1e-9
    scale = np.abs(ref).max()
    assert scale > 0
    assert np.abs(g - ref).max() <= (TOL_HF if prec == "fp64" else 1e-7) * scale, (g, ref)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["lo", "ins"])
def test_autograd_matches_band_energy_fd(ctx, kind):
    p = synth.small_case(kind)
    w, _ = FR.eigh(p)
    nb, _ = FR.gapped_nb(w)
    occ = _occ(p, nb)
    pos = torch.tensor(p.pos, dtype=torch.float64, requires_grad=True)
    E = FO.BandEnergy.apply(pos, ctx, p, occ)
    E.backward()
    g = pos.grad.numpy()
    scale = np.abs(g).max()
    for a, c in [(0, 0), (1, 1), (2, 2)]:
        fd = FO.finite_difference(ctx, p, occ, a, c)
        assert abs(fd - g[a, c]) <= TOL_FD * scale, (a, c, fd, g[a, c])


@pytest.mark.gpu
def test_adjoint_on_the_40_atom_cell(ctx):
    """The 40-atom ABO3 supercell (n = 4953): two components against FD of E."""
    p = synth.config("c1")[0]
    dev = torch.device("cuda", ctx.device)
    E, eps, X, kp = FO.band_energy(ctx, p, torch.ones(p.n // 4, dtype=torch.float64, device=dev))
    w = eps.cpu().numpy()
    nb, gap = FR.gapped_nb(w, lo=8, hi=len(w) - 1)
    kp.free()
    occ = torch.ones(nb, dtype=torch.float64, device=dev)
    E, eps, X, kp = FO.band_energy(ctx, p, occ)
    g = FO.gradient(ctx, kp, X, occ, eps).cpu().numpy()
    kp.free()
    scale = np.abs(g).max()
    assert scale > 0
    for a, c in [(0, 0), (p.ndf - 1, 2)]:
        fd = FO.finite_difference(ctx, p, occ.cpu(), a, c)
        assert abs(fd - g[a, c]) <= TOL_FD * scale, (a, c, fd, g[a, c])


@pytest.mark.gpu
def test_horb_problems_are_rejected(ctx):
    p = synth.small_case("orb")
    dev = torch.device("cuda", ctx.device)
    occ = torch.ones(4, dtype=torch.float64, device=dev)
    E, eps, X, kp = FO.band_energy(ctx, p, occ)
    with pytest.raises(lapw1gpu.Lapw1GpuError) as ei:
        FO.gradient(ctx, kp, X, occ, eps)
    kp.free()
    assert ei.value.code == 1


@pytest.mark.gpu
def test_forces_timing_entry_point(ctx, monkeypatch, capsys):
    """`python -m hack_wein2k_b200.forces` on the one-atom c0 case prints one
    JSON line with finite timings and a finite gradient."""
    import json
    import sys
    monkeypatch.setattr(sys, "argv", ["forces", "--case", "c0", "--bands", "4", "--repeat", "2"])
    FO._main()
    out = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert out["case"] == "c0" and len(out["forces_ms"]) == 2
    assert all(np.isfinite(out["forces_ms"])) and np.isfinite(out["max_abs_grad"])
