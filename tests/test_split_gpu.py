"""Split-precision path (Ozaki int8 slices on tcgen05) against the FP64 oracle.

The spherical muffin-tin contraction (S slices 4..7; FP64 otherwise) and
the HNS contraction run as exact int32 products of S int8 slices per
operand; the per-matrix relative errors of H and S therefore fall as
~2^(-7S) (S is the slice count).  Tolerances per S are written below; the
path is also checked through the generalized eigenvalues (SECLR4's
problem) against the bound of 1e-6 Ry for the split path.
"""
import numpy as np
import pytest
import scipy.linalg as sl

from hack_wein2k_b200 import lapw1gpu, synth
from hack_wein2k_b200.problem import hermitian_from_packed
from oracle import oracle as O
from tests.conftest import gpu_available
from tests.helpers import rel_errors

# relative max-norm error bound of H and of S per slice count
TOL_H = {4: 2e-7, 5: 2e-9, 6: 2e-11, 7: 1e-12, 8: 1e-12}


@pytest.fixture(scope="module")
def sctx():
    if not gpu_available():
        pytest.skip("no CUDA device")
    c = lapw1gpu.Context(0, prec=lapw1gpu.PREC_SPLIT, slices=7)
    yield c
    c.close()


@pytest.mark.gpu
@pytest.mark.parametrize("slices", [4, 5, 6, 7, 8])
@pytest.mark.parametrize("kind", ["lo", "apw", "multilo", "manyeq"])
def test_split_small(sctx, kind, slices):
    sctx.set_precision(lapw1gpu.PREC_SPLIT, slices)
    p = synth.small_case(kind)
    hs, hsd = sctx.setup(p)
    hs_o, hsd_o = O.setup(p)
    err = rel_errors(hs, hsd, hs_o, hsd_o)
    assert err["S"] <= TOL_H[slices], err
    assert err["H"] <= TOL_H[slices], err


@pytest.mark.gpu
@pytest.mark.parametrize("slices", [5, 7])
def test_split_c1(sctx, slices):
    sctx.set_precision(lapw1gpu.PREC_SPLIT, slices)
    p = synth.config("c1")[0]
    hs, hsd = sctx.setup(p)
    hs_o, hsd_o = O.setup(p)
    err = rel_errors(hs, hsd, hs_o, hsd_o)
    assert err["S"] <= TOL_H[slices] and err["H"] <= TOL_H[slices], err


# SECLR4 solves inside the energy window EL..EU of case.in1 (seclr4.F:150-155);
# the window here is [-10, 10] Ry
EWIN = (-10.0, 10.0)


def _window_eigs(hs, hsd):
    w = sl.eigh(*hermitian_from_packed(hs, hsd), eigvals_only=True)
    return w


@pytest.mark.gpu
@pytest.mark.parametrize("slices", [5, 6, 7])
@pytest.mark.parametrize("case", ["lo6", "c0"])
def test_split_eigenvalues(sctx, slices, case):
    """Generalized eigenvalues of the split-path H,S inside the energy window
    within 1e-6 Ry of the FP64 oracle's (S = 5 is the default)."""
    sctx.set_precision(lapw1gpu.PREC_SPLIT, slices)
    p = synth.small_case("lo", rkmax=6.0) if case == "lo6" else synth.config("c0")[0]
    hs, hsd = sctx.setup(p)
    hs_o, hsd_o = O.setup(p)
    w, wo = _window_eigs(hs, hsd), _window_eigs(hs_o, hsd_o)
    win = (wo > EWIN[0]) & (wo < EWIN[1])
    assert win.sum() >= 0.9 * len(wo)
    assert np.max(np.abs(w - wo)[win]) <= 1e-6, np.max(np.abs(w - wo)[win])


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["lo6", "c0"])
def test_fp64_eigenvalues(ctx, case):
    """The plain FP64 GPU path: window eigenvalues within 1e-8 Ry of the
    oracle's (host LAPACK solve of both)."""
    ctx.set_precision(lapw1gpu.PREC_FP64)
    p = synth.small_case("lo", rkmax=6.0) if case == "lo6" else synth.config("c0")[0]
    hs, hsd = ctx.setup(p)
    hs_o, hsd_o = O.setup(p)
    w, wo = _window_eigs(hs, hsd), _window_eigs(hs_o, hsd_o)
    win = (wo > EWIN[0]) & (wo < EWIN[1])
    assert np.max(np.abs(w - wo)[win]) <= 1e-8, np.max(np.abs(w - wo)[win])


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["lo6", "c0"])
def test_mixed_slices_eigenvalues(sctx, case):
    """Spherical part with 5 slices, HNS with 4: window eigenvalues within
    1e-6 Ry of the FP64 oracle's."""
    sctx.set_precision(lapw1gpu.PREC_SPLIT, 5)
    sctx.set_slices(5, 4)
    p = synth.small_case("lo", rkmax=6.0) if case == "lo6" else synth.config("c0")[0]
    hs, hsd = sctx.setup(p)
    hs_o, hsd_o = O.setup(p)
    w, wo = _window_eigs(hs, hsd), _window_eigs(hs_o, hsd_o)
    win = (wo > EWIN[0]) & (wo < EWIN[1])
    assert np.max(np.abs(w - wo)[win]) <= 1e-6, np.max(np.abs(w - wo)[win])
    sctx.set_precision(lapw1gpu.PREC_SPLIT, 5)


@pytest.mark.gpu
def test_split_matches_fp64_gpu_path(sctx):
    """S=8 split (HNS sliced, spherical part FP64) and the FP64 GPU path
    agree to FP64 rounding on c0."""
    p = synth.config("c0")[0]
    sctx.set_precision(lapw1gpu.PREC_SPLIT, 8)
    a = sctx.setup(p)
    sctx.set_precision(lapw1gpu.PREC_FP64)
    b = sctx.setup(p)
    err = rel_errors(a[0], a[1], b[0], b[1])
    assert err["H"] <= 1e-12 and err["S"] == 0.0, err


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64", "split"])
def test_nonfinite_element_is_reported(ctx, prec):
    """A NaN energy parameter (planted in the host inputs) makes H elements
    non-finite: both paths end with the non-finite status (the FP64 path by
    its scan of HS, the split path in the kernels that write HS)."""
    import dataclasses

    import torch
    p = synth.small_case("lo")
    e = np.array(p.e, dtype=np.float64, copy=True)
    e.flat[0] = np.nan
    p = dataclasses.replace(p, e=e)
    if prec == "split":
        ctx.set_precision(lapw1gpu.PREC_SPLIT, 5)
    kp = None
    try:
        kp = ctx.upload(p)
        dev = torch.device("cuda", ctx.device)
        hs = torch.zeros((p.n, p.n), dtype=torch.complex128, device=dev)
        hd = torch.zeros(p.n, dtype=torch.complex128, device=dev)
        kp.run(hs.data_ptr(), p.n, hd.data_ptr())  # asynchronous: status read on request
        async_status = ctx.last_status()
        with pytest.raises(lapw1gpu.Lapw1GpuError) as ei:
            kp.run(hs.data_ptr(), p.n, hd.data_ptr(), stats=True)
    finally:
        if kp is not None:
            kp.free()
        ctx.set_precision(lapw1gpu.PREC_FP64)
    assert async_status & 2
    assert ei.value.code == 4
    assert ctx.last_status() & 2


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["lo", "multilo"])
def test_split_stages_compose(sctx, kind):
    """HAMILT then HNS as two separate runs on the same device HS equals one
    run of both, bit for bit (the HNS operands are prepared on their own
    stream and joined before the products in both cases)."""
    import torch
    sctx.set_precision(lapw1gpu.PREC_SPLIT, 5)
    sctx.set_slices(5, 4)
    p = synth.small_case(kind)
    dev = torch.device("cuda", sctx.device)
    kp = sctx.upload(p)
    try:
        a = torch.zeros((p.n, p.n), dtype=torch.complex128, device=dev)
        ad = torch.zeros(p.n, dtype=torch.complex128, device=dev)
        kp.run(a.data_ptr(), p.n, ad.data_ptr(), stages=3, stats=True)
        b = torch.zeros_like(a)
        bd = torch.zeros_like(ad)
        kp.run(b.data_ptr(), p.n, bd.data_ptr(), stages=1, stats=True)
        kp.run(b.data_ptr(), p.n, bd.data_ptr(), stages=2, stats=True)
        assert torch.equal(a, b) and torch.equal(ad, bd)
    finally:
        kp.free()
        sctx.set_precision(lapw1gpu.PREC_SPLIT, 7)


@pytest.mark.gpu
@pytest.mark.parametrize("slices", [4, 5])
@pytest.mark.parametrize("case", ["lo", "manyeq", "c1"])
def test_sph_tc_kblock_shapes_agree(sctx, slices, case):
    """k_sph_tc with 128-byte K blocks (two-stage ring, the default) against
    64-byte ones (four-stage ring): the level sums are exact int32 sums, so
    the two tile shapes give the same bits; both within the slice count's
    bound of the oracle."""
    sctx.set_precision(lapw1gpu.PREC_SPLIT, slices)
    p = synth.config("c1")[0] if case == "c1" else synth.small_case(case)
    kb0 = sctx.tuning()["sph_kblock"]
    try:
        sctx.set_tuning(sph_kblock=64)
        hs64, hsd64 = sctx.setup(p)
        sctx.set_tuning(sph_kblock=128)
        hs128, hsd128 = sctx.setup(p)
    finally:
        sctx.set_tuning(sph_kblock=kb0)
    assert np.array_equal(hs64, hs128) and np.array_equal(hsd64, hsd128)
    hs_o, hsd_o = O.setup(p)
    err = rel_errors(hs128, hsd128, hs_o, hsd_o)
    assert err["S"] <= TOL_H[slices] and err["H"] <= TOL_H[slices], err


@pytest.mark.gpu
def test_second_context_keeps_kernel_limits(sctx):
    """A kernel's dynamic shared-memory limit belongs to the kernel on the
    device: a second context that runs a small problem after the first ran
    a large one must not lower it under what the first context's next,
    medium problem needs (the split slicer's shared memory grows with the
    atom count)."""
    sctx.set_precision(lapw1gpu.PREC_SPLIT, 5)
    other = lapw1gpu.Context(0, prec=lapw1gpu.PREC_SPLIT, slices=5)
    try:
        sctx.setup(synth.config("c1")[0])
        other.setup(synth.small_case("lo"))
        p = synth.small_case("manyeq")
        hs, hsd = sctx.setup(p)
    finally:
        other.close()
    hs_o, hsd_o = O.setup(p)
    err = rel_errors(hs, hsd, hs_o, hsd_o)
    assert err["S"] <= TOL_H[5] and err["H"] <= TOL_H[5], err
