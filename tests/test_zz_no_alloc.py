"""The allocation-free HNS entry point (lapw1gpu_hns_noalloc) against the
regular HNS stage (lapw1gpu_setup_stages with stage 2).

lapw1gpu_hns_noalloc exists for callers that cannot let the library
allocate device memory (a host whose device memory is reserved by its
eigen-solver library or owned by a framework's caching allocator): its
scratch is one fixed 64 MiB device array inside the library.  This file
runs last so that a failure here leaves every other test already run; it
passes alone in a fresh process and after the other tests (the array keeps
the previous call's contents, which must not leak into the result).
"""
import numpy as np
import pytest

from hack_wein2k_b200 import lapw1gpu, synth
from tests.conftest import gpu_available
from tests.helpers import rel_errors

TOL_FP64 = 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["lo", "multilo", "plain"])
def test_hns_noalloc_matches_hns_stage_twice(kind):
    if not gpu_available():
        pytest.skip("no CUDA device")
    import torch

    p = synth.small_case(kind)
    n = p.n
    rng = np.random.default_rng(11)
    base = np.asfortranarray(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    based = rng.standard_normal(n) + 1j * rng.standard_normal(n)

    # existing entry point: HNS stage on host buffers
    with lapw1gpu.Context(0) as ctx:
        ref, refd = ctx.setup(p, stages=2, hs=base.copy(order="F"), hsdiag=based.copy())

    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    status = torch.full((1,), -1, dtype=torch.int32, device=dev)  # the call clears it
    for call in range(2):
        d_hs = torch.from_numpy(base.reshape(-1, order="F").view(np.float64).copy()).to(dev)
        lapw1gpu.hns_noalloc(p, d_hs.data_ptr(), n, stream.cuda_stream, status.data_ptr())
        torch.cuda.synchronize(dev)
        out = d_hs.cpu().numpy().view(np.complex128).reshape((n, n), order="F")
        err = rel_errors(out, based, ref, refd)
        assert err["H"] <= TOL_FP64 and err["S"] == 0.0, (call, err)
        assert np.array_equal(np.triu(out, 1), np.triu(base, 1)), call
        assert int(status.item()) == 0, call


@pytest.mark.gpu
def test_hns_noalloc_rejects_problems_beyond_its_array():
    if not gpu_available():
        pytest.skip("no CUDA device")
    import torch

    p = synth.config("c1")[0]  # HNS operands alone exceed the 64 MiB array
    d_hs = torch.zeros(p.n * p.n * 2, dtype=torch.float64, device="cuda")
    with pytest.raises(lapw1gpu.Lapw1GpuError) as e:
        lapw1gpu.hns_noalloc(p, d_hs.data_ptr(), p.n, 0)
    assert e.value.code == 7  # LAPW1GPU_ERR_RANGE


def _oversized_rmt(p):
    """The problem with type 0's RMT stretched so that RMT |k+G| reaches 25,
    beyond SPHBES's start table (sphbes.f:60-64)."""
    import dataclasses
    rmt = np.array(p.rmt, dtype=np.float64, copy=True)
    rmt[0] = 25.0 / float(np.max(p.rk[: p.nv]))
    return dataclasses.replace(p, rmt=rmt)


@pytest.mark.gpu
def test_hns_noalloc_reports_sphbes_range_like_the_hns_stage():
    """An RMT that puts RMT |k+G| beyond SPHBES's range: the HNS stage
    returns LAPW1GPU_ERR_RANGE from its device status word, and the
    allocation-free entry point returns the same code from its host check,
    before any device work (the caller's HS is left untouched)."""
    if not gpu_available():
        pytest.skip("no CUDA device")
    import torch

    p = _oversized_rmt(synth.small_case("lo"))
    n = p.n
    with lapw1gpu.Context(0) as ctx:
        with pytest.raises(lapw1gpu.Lapw1GpuError) as e:
            ctx.setup(p, stages=2, hs=np.zeros((n, n), dtype=np.complex128, order="F"))
        assert e.value.code == 7
    d_hs = torch.zeros(n * n * 2, dtype=torch.float64, device="cuda")
    with pytest.raises(lapw1gpu.Lapw1GpuError) as e:
        lapw1gpu.hns_noalloc(p, d_hs.data_ptr(), n, 0)
    assert e.value.code == 7
    torch.cuda.synchronize()
    assert float(d_hs.abs().max()) == 0.0


@pytest.mark.gpu
def test_hns_noalloc_status_word_reports_nonfinite():
    """A non-finite T entry: the HNS stage returns LAPW1GPU_ERR_NONFINITE, and
    the allocation-free entry point leaves bit 2 (non-finite) in the caller's
    status word; a clean call afterwards clears it again."""
    if not gpu_available():
        pytest.skip("no CUDA device")
    import dataclasses

    import torch

    p = synth.small_case("lo")
    tns = np.array(p.tns, copy=True)
    tns[0, 0, 0, 0] = np.nan
    bad = dataclasses.replace(p, tns=tns)
    n = p.n
    with lapw1gpu.Context(0) as ctx:
        with pytest.raises(lapw1gpu.Lapw1GpuError) as e:
            ctx.setup(bad, stages=2, hs=np.zeros((n, n), dtype=np.complex128, order="F"))
        assert e.value.code == 4
    dev = torch.device("cuda", 0)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    d_hs = torch.zeros(n * n * 2, dtype=torch.float64, device=dev)
    lapw1gpu.hns_noalloc(bad, d_hs.data_ptr(), n, 0, status.data_ptr())
    torch.cuda.synchronize(dev)
    assert int(status.item()) & 2
    d_hs.zero_()
    lapw1gpu.hns_noalloc(p, d_hs.data_ptr(), n, 0, status.data_ptr())
    torch.cuda.synchronize(dev)
    assert int(status.item()) == 0
