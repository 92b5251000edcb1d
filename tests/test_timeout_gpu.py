"""Bounded device waits: a wait that runs out ends the run with
LAPW1GPU_ERR_TIMEOUT and leaves the context usable.

The test hook lapw1gpu_test_wait_timeout makes the MMA issuer of the
split-precision spherical kernel wait on a barrier that nothing arrives at
(bounded to about half a millisecond); every other wait of the kernel keeps
its full bound, so the producer drains its copies in flight and TMEM is
freed before the kernel returns.  A clean run on the same context follows.
"""
import pytest

from hack_wein2k_b200 import lapw1gpu, synth
from oracle import oracle as O
from tests.helpers import rel_errors


@pytest.mark.gpu
def test_timeout_status_then_clean_run(ctx):
    p = synth.small_case("lo")
    hs_o, hsd_o = O.setup(p)
    saved = ctx.tuning()
    ctx.set_precision(lapw1gpu.PREC_SPLIT, 5)
    ctx.set_tuning(sph_tc=1)
    try:
        ctx.test_wait_timeout(True)
        with pytest.raises(lapw1gpu.Lapw1GpuError) as e:
            ctx.setup(p)
        assert e.value.code == 5  # LAPW1GPU_ERR_TIMEOUT
        ctx.test_wait_timeout(False)
        for _ in range(2):
            hs, hsd = ctx.setup(p)
            err = rel_errors(hs, hsd, hs_o, hsd_o)
            assert err["H"] <= 2e-9 and err["S"] <= 2e-9, err
    finally:
        ctx.test_wait_timeout(False)
        ctx.set_tuning(sph_tc=saved["sph_tc"])
        ctx.set_precision(lapw1gpu.PREC_FP64)
