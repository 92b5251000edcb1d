"""ctypes front end of the CPU oracle (oracle/lapw1_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke check and the
benchmark's CPU-baseline leg, never by the product package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "liblapw1_oracle.so")
_lib = None


def build(force: bool = False) -> str:
    srcs = [os.path.join(_HERE, "lapw1_oracle.c"), os.path.join(_HERE, "..", "include", "lapw1gpu.h")]
    if force or not os.path.exists(_SO) or any(os.path.getmtime(_SO) < os.path.getmtime(s) for s in srcs):
        subprocess.check_call(["make", "-s", "-C", _HERE])
    return _SO


_NATIVE_SO = os.path.join(_HERE, "liblapw1_oracle_native.so")
_native = None


def _bind(lib):
    dp = C.POINTER(C.c_double)
    lib.oracle_sphbes.argtypes = [C.c_int, C.c_double, dp]
    lib.oracle_ylm.argtypes = [dp, C.c_int, dp]
    lib.oracle_albl.argtypes = [C.c_void_p, dp, dp]
    for f in ("oracle_setup", "oracle_hamilt"):
        getattr(lib, f).argtypes = [C.c_void_p, dp, C.c_int, dp]
    lib.oracle_hamilt_range.argtypes = [C.c_void_p, dp, C.c_int, dp, C.c_int, C.c_int, C.c_int]
    lib.oracle_swapdiag.argtypes = [C.c_void_p, dp, C.c_int, dp]
    lib.oracle_hns.argtypes = [C.c_void_p, dp, C.c_int]
    lib.oracle_hns_range.argtypes = [C.c_void_p, dp, C.c_int, C.c_int, C.c_int]
    lib.oracle_horb.argtypes = [C.c_void_p, dp, C.c_int]
    lib.oracle_use_blas.argtypes = [C.c_char_p, C.c_char_p]
    return lib


def openblas_path():
    """The LP64 OpenBLAS that ships with scipy (its CBLAS symbols carry the
    scipy_ prefix), or None."""
    try:
        import glob
        import scipy
        d = os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs")
        hits = sorted(glob.glob(os.path.join(d, "libscipy_openblas*.so")))
        return hits[0] if hits else None
    except Exception:
        return None


def baseline_lib():
    """The oracle built for the timed CPU baseline: -O3 -march=native on the
    machine that runs it (the portable build if that compile fails), with
    the ZHER2M blocks on OpenBLAS zgemm when scipy's OpenBLAS is found.
    Returns (library, description)."""
    global _native
    if _native is None:
        try:
            subprocess.check_call(["make", "-s", "-C", _HERE, "native"], stdout=subprocess.DEVNULL,
                                  stderr=subprocess.DEVNULL)
            lib_, flags = _bind(C.CDLL(_NATIVE_SO)), "gcc -O3 -march=native -fopenmp"
        except Exception:
            lib_, flags = lib(), "gcc -O3 -march=x86-64-v3 -fopenmp"
        blas = openblas_path()
        if blas and lib_.oracle_use_blas(blas.encode(), b"scipy_cblas_zgemm") == 0:
            flags += ", ZHER2M blocks on OpenBLAS zgemm (" + os.path.basename(blas) + ")"
        else:
            flags += ", ZHER2M as plain loops (no OpenBLAS found)"
        _native = (lib_, flags)
    return _native


class blas_zgemm:
    """Context manager: the portable oracle's ZHER2M blocks on OpenBLAS
    zgemm (the loops otherwise).  Same sums in another order: for checks of
    large problems that the loops make slow."""

    def __enter__(self):
        path = openblas_path()
        self.on = bool(path) and lib().oracle_use_blas(path.encode(), b"scipy_cblas_zgemm") == 0
        return self

    def __exit__(self, *a):
        lib().oracle_use_blas(None, None)


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = _bind(C.CDLL(_SO))
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def sphbes(n: int, x: float) -> np.ndarray:
    out = np.zeros(n + 2)
    rc = lib().oracle_sphbes(n, float(x), _dp(out))
    if rc:
        raise ValueError(f"sphbes failed ({rc})")
    return out[: n + 1]


def ylm(v, lmax: int) -> np.ndarray:
    v = np.ascontiguousarray(v, dtype=np.float64)
    out = np.zeros((lmax + 1) ** 2, dtype=np.complex128)
    lib().oracle_ylm(_dp(v), lmax, _dp(out.view(np.float64)))
    return out


def albl(prob):
    cp = prob.to_c()
    al = np.zeros((prob.nat, prob.ltop, prob.nv))
    bl = np.zeros_like(al)
    rc = lib().oracle_albl(C.byref(cp), _dp(al), _dp(bl))
    if rc:
        raise RuntimeError("oracle_albl failed")
    return al, bl


def setup(prob, stages: int = 7):
    """HS (n x n, Fortran order) and HSDIAG after the selected stages:
    1 HAMILT+ZSWAP, 2 HNS, 4 HORB (matching lapw1gpu_setup_stages)."""
    cp = prob.to_c()
    n = prob.n
    hs = np.zeros((n, n), dtype=np.complex128, order="F")
    hsd = np.zeros(n, dtype=np.complex128)
    L = lib()
    hsv = hs.reshape(-1, order="F").view(np.float64)
    hdv = hsd.view(np.float64)
    if stages & 1:
        rc = L.oracle_hamilt(C.byref(cp), _dp(hsv), n, _dp(hdv))
        if rc:
            raise RuntimeError(f"oracle_hamilt failed ({rc})")
        L.oracle_swapdiag(C.byref(cp), _dp(hsv), n, _dp(hdv))
    if stages & 2 and not prob.nohns:
        rc = L.oracle_hns(C.byref(cp), _dp(hsv), n)
        if rc:
            raise RuntimeError(f"oracle_hns failed ({rc})")
    if stages & 4 and prob.natorb > 0:
        rc = L.oracle_horb(C.byref(cp), _dp(hsv), n)
        if rc:
            raise RuntimeError(f"oracle_horb failed ({rc})")
    return hs, hsd


def hamilt_sample(prob, col_lo: int, col_hi: int, L=None):
    """HAMILT over PW columns col_lo..col_hi only (a bounded CPU sample)."""
    cp = prob.to_c()
    n = prob.n
    hs = np.zeros((n, n), dtype=np.complex128, order="F")
    hsd = np.zeros(n, dtype=np.complex128)
    rc = (L or lib()).oracle_hamilt_range(C.byref(cp), _dp(hs.reshape(-1, order="F").view(np.float64)), n,
                                   _dp(hsd.view(np.float64)), col_lo, col_hi, 0)
    if rc:
        raise RuntimeError("oracle_hamilt_range failed")
    return hs, hsd


def hns_sample(prob, atom_lo: int, atom_hi: int, L=None):
    """HNS over equivalent atoms atom_lo..atom_hi only (a bounded CPU sample)."""
    cp = prob.to_c()
    n = prob.n
    hs = np.zeros((n, n), dtype=np.complex128, order="F")
    rc = (L or lib()).oracle_hns_range(C.byref(cp), _dp(hs.reshape(-1, order="F").view(np.float64)), n,
                                atom_lo, atom_hi)
    if rc:
        raise RuntimeError("oracle_hns_range failed")
    return hs
