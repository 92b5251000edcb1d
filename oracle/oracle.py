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


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(_SO)
        dp = C.POINTER(C.c_double)
        _lib.oracle_sphbes.argtypes = [C.c_int, C.c_double, dp]
        _lib.oracle_ylm.argtypes = [dp, C.c_int, dp]
        _lib.oracle_albl.argtypes = [C.c_void_p, dp, dp]
        for f in ("oracle_setup", "oracle_hamilt"):
            getattr(_lib, f).argtypes = [C.c_void_p, dp, C.c_int, dp]
        _lib.oracle_hamilt_range.argtypes = [C.c_void_p, dp, C.c_int, dp, C.c_int, C.c_int, C.c_int]
        _lib.oracle_swapdiag.argtypes = [C.c_void_p, dp, C.c_int, dp]
        _lib.oracle_hns.argtypes = [C.c_void_p, dp, C.c_int]
        _lib.oracle_hns_range.argtypes = [C.c_void_p, dp, C.c_int, C.c_int, C.c_int]
        _lib.oracle_horb.argtypes = [C.c_void_p, dp, C.c_int]
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


def hamilt_sample(prob, col_lo: int, col_hi: int):
    """HAMILT over PW columns col_lo..col_hi only (a bounded CPU sample)."""
    cp = prob.to_c()
    n = prob.n
    hs = np.zeros((n, n), dtype=np.complex128, order="F")
    hsd = np.zeros(n, dtype=np.complex128)
    rc = lib().oracle_hamilt_range(C.byref(cp), _dp(hs.reshape(-1, order="F").view(np.float64)), n,
                                   _dp(hsd.view(np.float64)), col_lo, col_hi, 0)
    if rc:
        raise RuntimeError("oracle_hamilt_range failed")
    return hs, hsd


def hns_sample(prob, atom_lo: int, atom_hi: int):
    cp = prob.to_c()
    n = prob.n
    hs = np.zeros((n, n), dtype=np.complex128, order="F")
    rc = lib().oracle_hns_range(C.byref(cp), _dp(hs.reshape(-1, order="F").view(np.float64)), n,
                                atom_lo, atom_hi)
    if rc:
        raise RuntimeError("oracle_hns_range failed")
    return hs
