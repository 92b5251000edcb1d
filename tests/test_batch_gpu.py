"""k-point batches (one captured CUDA graph, concurrent k-point chains) and
the autotuner.

A batch runs the same kernels as single k-points, so its HS/HSDIAG must be
bitwise equal to lapw1gpu_kpoint_run's on every k-point, on the first call
(capture) and on replays; k-points of uneven size share the graph.  The
oracle pins two of them at the FP64 parity bar (1e-12).
"""
import numpy as np
import pytest
import torch

from hack_wein2k_b200 import lapw1gpu, synth
from oracle import oracle as O
from tests.helpers import rel_errors

TOL_FP64 = 1e-12


def _small_batch():
    """Uneven k-points of the small mixed cell, every branch kind."""
    return [synth.small_case(k) for k in ("lo", "apw", "ins", "gamma", "plain", "multilo")]


def _alloc(probs, dev):
    hs = [torch.zeros((p.n, p.n), dtype=torch.complex128, device=dev) for p in probs]
    hd = [torch.zeros(p.n, dtype=torch.complex128, device=dev) for p in probs]
    return hs, hd


def _host(t):
    """device HS viewed [col][row] -> Fortran-ordered numpy HS(row, col)"""
    return t.cpu().numpy().T


def _single(ctx, probs, dev):
    out = []
    for p in probs:
        kp = ctx.upload(p)
        hs, hd = _alloc([p], dev)
        kp.run(hs[0].data_ptr(), p.n, hd[0].data_ptr(), stats=True)
        out.append((_host(hs[0]), hd[0].cpu().numpy()))
        kp.free()
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("prec,slices", [(lapw1gpu.PREC_FP64, 6), (lapw1gpu.PREC_SPLIT, 5)])
@pytest.mark.parametrize("sets", [1, 2, 3])
def test_batch_equals_single_runs(ctx, prec, slices, sets):
    dev = torch.device("cuda", ctx.device)
    ctx.set_precision(prec, slices)
    ctx.set_tuning(batch_sets=sets)
    probs = _small_batch()
    ref = _single(ctx, probs, dev)
    kps = [ctx.upload(p) for p in probs]
    hs, hd = _alloc(probs, dev)
    for call in range(2):  # capture, then replay
        for t in hs + hd:
            t.zero_()
        st = ctx.setup_batch(kps, [h.data_ptr() for h in hs], [p.n for p in probs], [d.data_ptr() for d in hd])
        assert st["ms_total"] > 0 and st["kernel_launches"] > 0
        for i, p in enumerate(probs):
            assert np.array_equal(_host(hs[i]), ref[i][0]), (call, i)
            assert np.array_equal(hd[i].cpu().numpy(), ref[i][1]), (call, i)
    for k in kps:
        k.free()
    ctx.set_tuning(batch_sets=2)
    ctx.set_precision(lapw1gpu.PREC_FP64)


@pytest.mark.gpu
def test_batch_against_oracle(ctx):
    dev = torch.device("cuda", ctx.device)
    ctx.set_precision(lapw1gpu.PREC_FP64)
    probs = [synth.small_case("lo"), synth.small_case("gamma")]
    kps = [ctx.upload(p) for p in probs]
    hs, hd = _alloc(probs, dev)
    ctx.setup_batch(kps, [h.data_ptr() for h in hs], [p.n for p in probs], [d.data_ptr() for d in hd])
    for i, p in enumerate(probs):
        hs_o, hd_o = O.setup(p)
        err = rel_errors(_host(hs[i]), hd[i].cpu().numpy(), hs_o, hd_o)
        assert err["H"] <= TOL_FP64 and err["S"] <= TOL_FP64, err
    for k in kps:
        k.free()


@pytest.mark.gpu
def test_batch_of_uneven_c2_kpoints(ctx):
    """Four k-points of the 40-atom cell's wedge (uneven N) in one graph."""
    dev = torch.device("cuda", ctx.device)
    ctx.set_precision(lapw1gpu.PREC_SPLIT, 6)
    probs = synth.config("c2", nk=4)
    assert len({p.n for p in probs}) > 1
    ref = _single(ctx, probs, dev)
    kps = [ctx.upload(p) for p in probs]
    hs, hd = _alloc(probs, dev)
    ctx.setup_batch(kps, [h.data_ptr() for h in hs], [p.n for p in probs], [d.data_ptr() for d in hd])
    for i in range(len(probs)):
        assert np.array_equal(_host(hs[i]), ref[i][0])
    for k in kps:
        k.free()
    ctx.set_precision(lapw1gpu.PREC_FP64)


@pytest.mark.gpu
@pytest.mark.parametrize("prec,slices", [(lapw1gpu.PREC_FP64, 6), (lapw1gpu.PREC_SPLIT, 6)])
def test_autotune_keeps_results_exact(ctx, prec, slices):
    """The tuner only picks among equivalent schedules: results after tuning
    still meet the parity bar of the precision."""
    dev = torch.device("cuda", ctx.device)
    ctx.set_precision(prec, slices)
    p = synth.small_case("lo", rkmax=6.0)
    kp = ctx.upload(p)
    hs, hd = _alloc([p], dev)
    t = ctx.autotune(kp, hs[0].data_ptr(), p.n, hd[0].data_ptr())
    assert t["hns_diag_b"] in (256, 512, 1024, 2048)
    assert t["split_group"] in (4, 8, 16, 32) and t["sph_tc"] in (0, 1) and t["ms_best"] > 0
    assert t["sph_kblock"] in (64, 128)
    kp.run(hs[0].data_ptr(), p.n, hd[0].data_ptr(), stats=True)
    hs_o, hd_o = O.setup(p)
    err = rel_errors(_host(hs[0]), hd[0].cpu().numpy(), hs_o, hd_o)
    tol = TOL_FP64 if prec == lapw1gpu.PREC_FP64 else 2e-11
    assert err["H"] <= tol and err["S"] <= tol, err
    kp.free()
    ctx.set_tuning(hns_diag_b=512, split_group=16, sph_tc=1)
    ctx.set_precision(lapw1gpu.PREC_FP64)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [lapw1gpu.PREC_FP64, lapw1gpu.PREC_SPLIT])
def test_forces_batch_equals_single_calls(ctx, prec):
    """lapw1gpu_forces_batch queues the adjoint of uneven k-points back to
    back; every gradient is the single call's to 1e-12 of its largest
    component (the force kernels sum over pair tiles with atomic adds, whose
    order varies from run to run)."""
    from hack_wein2k_b200 import forces as FO
    dev = torch.device("cuda", ctx.device)
    probs = [synth.small_case(k) for k in ("lo", "apw", "ins", "gamma")]
    nb = 6
    occ = torch.ones(nb, dtype=torch.float64, device=dev)
    setup = [FO.band_energy(ctx, p, occ) for p in probs]  # (E, eps, X, kp), FP64 setup
    ctx.set_precision(prec, 5)
    try:
        ref = [FO.gradient(ctx, kp, X, occ, w).cpu().numpy() for (_, w, X, kp) in setup]
        xs = [X.transpose(0, 1).contiguous() for (_, _, X, _) in setup]
        ws = [w.contiguous() for (_, w, _, _) in setup]
        gs = [torch.full((p.ndf, 3), np.nan, dtype=torch.float64, device=dev) for p in probs]
        torch.cuda.synchronize()
        ms = ctx.forces_batch([kp for (_, _, _, kp) in setup], [x.data_ptr() for x in xs], [p.n for p in probs],
                              nb, occ.data_ptr(), [w.data_ptr() for w in ws], [g.data_ptr() for g in gs])
    finally:
        ctx.set_precision(lapw1gpu.PREC_FP64)
        for (_, _, _, kp) in setup:
            kp.free()
    assert ms > 0
    for g, r in zip(gs, ref):
        assert np.abs(g.cpu().numpy() - r).max() <= 1e-12 * np.abs(r).max()


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [lapw1gpu.PREC_FP64, lapw1gpu.PREC_SPLIT])
def test_setup_async_with_forces_in_between(ctx, prec):
    """lapw1gpu_setup_async, then lapw1gpu_forces of another, resident
    k-point while the HS copies run, then lapw1gpu_setup_wait: the host HS
    and HSDIAG equal the synchronous setup's bit for bit, and the forces
    equal a call made alone (up to the order of their atomic sums)."""
    from hack_wein2k_b200 import forces as FO
    dev = torch.device("cuda", ctx.device)
    ctx.set_precision(prec, 5)
    try:
        occ = torch.ones(8, dtype=torch.float64, device=dev)
        _, w, X, kp = FO.band_energy(ctx, synth.small_case("lo"), occ)
        g_alone = FO.gradient(ctx, kp, X, occ, w).cpu().numpy()
        p = synth.config("c0")[0]
        hs_s, hd_s = ctx.setup(p)
        n = p.n
        hs = np.zeros((n, n), dtype=np.complex128, order="F")
        hd = np.zeros(n, dtype=np.complex128)
        Xc = X.transpose(0, 1).contiguous()
        g = torch.empty_like(torch.from_numpy(g_alone)).to(dev)
        torch.cuda.synchronize(dev)
        ctx.setup_async(p, hs, hd)
        kp.forces(Xc.data_ptr(), X.shape[0], X.shape[1], occ.data_ptr(), w.contiguous().data_ptr(), g.data_ptr())
        hs_a, hd_a = ctx.setup_wait()
        kp.free()
    finally:
        ctx.set_precision(lapw1gpu.PREC_FP64)
    assert hs_a is hs and hd_a is hd
    assert np.array_equal(hs, hs_s) and np.array_equal(hd, hd_s)
    g = g.cpu().numpy()
    assert np.abs(g - g_alone).max() <= 1e-12 * np.abs(g_alone).max()
