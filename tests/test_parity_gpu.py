"""GPU path (C ABI) against the CPU oracle on identical seeded inputs.

Tolerance: per-matrix relative error max|HS_gpu - HS_oracle| / max|HS_oracle|
<= 1e-12 for H and for S (the FP64 path's parity bar), with H the lower
triangle plus diagonal of HS and S the strict upper triangle plus HSDIAG.
"""
import numpy as np
import pytest

from hack_wein2k_b200 import synth
from oracle import oracle as O
from tests.helpers import rel_errors

TOL_FP64 = 1e-12

SMALL = ["plain", "lo", "apw", "ins", "orb", "multilo", "gamma", "manyeq"]


@pytest.mark.gpu
@pytest.mark.parametrize("kind", SMALL)
def test_small_cases_full_setup(ctx, kind):
    p = synth.small_case(kind)
    hs, hsd = ctx.setup(p)
    hs_o, hsd_o = O.setup(p)
    err = rel_errors(hs, hsd, hs_o, hsd_o)
    assert err["H"] <= TOL_FP64 and err["S"] <= TOL_FP64, err


@pytest.mark.gpu
@pytest.mark.parametrize("stages", [1, 3])
@pytest.mark.parametrize("kind", ["lo", "apw", "multilo"])
def test_stages(ctx, kind, stages):
    """HAMILT(+ZSWAP) alone, then with HNS: each reference routine checked."""
    p = synth.small_case(kind)
    hs, hsd = ctx.setup(p, stages=stages)
    hs_o, hsd_o = O.setup(p, stages=stages)
    err = rel_errors(hs, hsd, hs_o, hsd_o)
    assert err["H"] <= TOL_FP64 and err["S"] <= TOL_FP64, err


@pytest.mark.gpu
def test_hns_alone_adds_to_callers_matrix(ctx):
    """HNS stage on a caller-provided HS only adds to its lower triangle."""
    p = synth.small_case("lo")
    rng = np.random.default_rng(1)
    n = p.n
    base = np.asfortranarray(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    based = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    hs, hsd = ctx.setup(p, stages=2, hs=base.copy(order="F"), hsdiag=based.copy())
    hs_o = base.copy(order="F")
    O.lib()  # oracle HNS on the same start
    import ctypes as C
    cp = p.to_c()
    rc = O.lib().oracle_hns(C.byref(cp), hs_o.reshape(-1, order="F").view(np.float64).ctypes.data_as(
        C.POINTER(C.c_double)), n)
    assert rc == 0
    err = rel_errors(hs, hsd, hs_o, based)
    assert err["H"] <= TOL_FP64 and err["S"] == 0.0, err
    assert np.array_equal(np.triu(hs, 1), np.triu(base, 1))


@pytest.mark.gpu
def test_config_c0(ctx):
    p = synth.config("c0")[0]
    hs, hsd = ctx.setup(p)
    hs_o, hsd_o = O.setup(p)
    err = rel_errors(hs, hsd, hs_o, hsd_o)
    assert err["H"] <= TOL_FP64 and err["S"] <= TOL_FP64, err


@pytest.mark.gpu
def test_config_c1_full_size(ctx):
    """40-atom ABO3 supercell, N ~ 4950, one general k: the benchmark workload."""
    p = synth.config("c1")[0]
    assert 4800 < p.n < 5100
    hs, hsd, st = ctx.setup(p, stats=True)
    hs_o, hsd_o = O.setup(p)
    err = rel_errors(hs, hsd, hs_o, hsd_o)
    assert err["H"] <= TOL_FP64 and err["S"] <= TOL_FP64, err
    assert st["ms_total"] > 0


@pytest.mark.gpu
def test_repeat_is_deterministic(ctx):
    p = synth.small_case("lo")
    a = ctx.setup(p)
    b = ctx.setup(p)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


@pytest.mark.gpu
def test_ldhs_larger_than_n(ctx):
    """HS with a leading dimension above HSROWS: rows beyond n untouched."""
    p = synth.small_case("apw")
    n = p.n
    big = np.full((n + 7, n), 3.0 + 1j, dtype=np.complex128, order="F")
    hs, hsd = ctx.setup(p, hs=big)
    hs_o, hsd_o = O.setup(p)
    err = rel_errors(hs[:n], hsd, hs_o, hsd_o)
    assert err["H"] <= TOL_FP64 and err["S"] <= TOL_FP64
    assert np.all(hs[n:] == 3.0 + 1j)
