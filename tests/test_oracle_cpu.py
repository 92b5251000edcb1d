"""The oracle's building blocks against independent implementations, and
the host-side helpers of the product against the oracle (CPU only)."""
import numpy as np
import pytest
import scipy.special as sp

from hack_wein2k_b200 import lapw1gpu, lattice, synth
from hack_wein2k_b200.problem import hermitian_from_packed
from oracle import oracle as O


@pytest.mark.parametrize("x", [0.0, 1e-6, 0.05, 0.1, 0.1000001, 0.7, 2.5, 7.3, 9.6, 12.0, 14.9])
def test_sphbes_against_scipy(x):
    n = 12
    fj = O.sphbes(n, x)
    ref = sp.spherical_jn(np.arange(n + 1), x)
    # the series branch (x <= 0.1) keeps two terms: truncation error ~x^4
    tol = 1e-12 if x > 0.1 else 1e-6 * max(x, 1e-3) ** 2
    assert np.allclose(fj, ref, rtol=0, atol=tol), (fj - ref)


def test_ylm_against_scipy():
    rng = np.random.default_rng(3)
    for v in list(rng.standard_normal((20, 3))) + [np.array([0, 0, 1.0]), np.array([0, 0, -2.0]),
                                                    np.array([1.0, 0, 0]), np.array([0, 0, 0.0])]:
        y = O.ylm(v, 10)
        r = np.linalg.norm(v)
        th = np.arccos(v[2] / r) if r > 0 else 0.0
        ph = np.arctan2(v[1], v[0]) if r > 0 else 0.0
        for l in range(11):
            for m in range(-l, l + 1):
                ref = sp.sph_harm_y(l, m, th, ph)
                assert abs(y[l * l + l + m] - ref) < 1e-12, (l, m, v)


def test_numpy_ylm_matches_oracle():
    rng = np.random.default_rng(4)
    vs = rng.standard_normal((50, 3))
    yn = lattice.ylm(vs, 6)
    for i, v in enumerate(vs):
        assert np.max(np.abs(yn[i] - O.ylm(v, 6))) < 1e-14


def test_tns_from_gaunt_product_equals_oracle():
    """lapw1gpu_tns_from_gaunt (host-side, product) and the oracle's LMSORT
    grouping agree, repeated (l0,m0,l',m',LM) tuples included."""
    import ctypes as C
    rng = np.random.default_rng(5)
    nat, ngau, lmmx, lnsmax = 2, 60, 6, 4
    lqind = np.array([55, 40], dtype=np.int32)
    lqns = np.zeros((nat, ngau, 6), dtype=np.int32)
    for a in range(nat):
        for i in range(lqind[a]):
            l0, lp = rng.integers(0, 5, 2)
            lqns[a, i] = [lp + 1, 0, l0 + 1, rng.integers(1, lmmx + 1), rng.integers(-lp, lp + 1),
                          rng.integers(-l0, l0 + 1)]
        lqns[a, 5] = lqns[a, 2]  # a repeated tuple
    gfac = rng.standard_normal((nat, ngau)) + 1j * rng.standard_normal((nat, ngau))
    v = [rng.standard_normal((nat, 5, lmmx, 5)) for _ in range(3)]
    vl = [rng.standard_normal((nat, 5, lmmx, 4)) for _ in range(3)]
    loor = np.array([[1, 1, 0, 0], [0, 1, 1, 0]], dtype=np.int32)
    t_prod = lapw1gpu.tns_from_gaunt(nat, lnsmax, lqind, lqns, gfac, *v, *vl, loor)
    t_ora = np.zeros_like(t_prod)
    L = O.lib()
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))
    g = np.ascontiguousarray(gfac)
    arrs = [np.ascontiguousarray(a) for a in v + vl]
    L.oracle_tns_from_gaunt(nat, lnsmax, ngau, lmmx, ip(lqind), ip(lqns), dp(g.view(np.float64)),
                            *[dp(a) for a in arrs], ip(loor), dp(t_ora.view(np.float64)))
    assert np.array_equal(t_prod, t_ora)
    assert np.count_nonzero(t_prod) > 0


@pytest.mark.parametrize("kind", ["plain", "lo", "apw", "ins", "orb", "gamma"])
def test_oracle_overlap_is_hermitian_positive(kind):
    p = synth.small_case(kind)
    hs, hsd = O.setup(p)
    H, S = hermitian_from_packed(hs, hsd)
    assert np.all(np.isfinite(hs)) and np.all(np.isfinite(hsd))
    w = np.linalg.eigvalsh(S)
    assert w.min() > 0, w.min()
