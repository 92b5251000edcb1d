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
    for call in range(2):
        d_hs = torch.from_numpy(base.reshape(-1, order="F").view(np.float64).copy()).to(dev)
        lapw1gpu.hns_noalloc(p, d_hs.data_ptr(), n, stream.cuda_stream)
        torch.cuda.synchronize(dev)
        out = d_hs.cpu().numpy().view(np.complex128).reshape((n, n), order="F")
        err = rel_errors(out, based, ref, refd)
        assert err["H"] <= TOL_FP64 and err["S"] == 0.0, (call, err)
        assert np.array_equal(np.triu(out, 1), np.triu(base, 1)), call


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
