"""ctypes binding of liblapw1gpu.so (the C ABI of include/lapw1gpu.h).

This is the Python side of the drop-in boundary: the same entry points a
Fortran caller binds with ISO_C_BINDING.  The library must be present:
there is no CPU fallback, and every call fails loudly if the CUDA
extension is missing or the device is unusable.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Tuple

import numpy as np

from .problem import CProblem, CStats, Problem

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblapw1gpu.so")

PREC_FP64 = 0
PREC_SPLIT = 1

STATUS = {
    0: "ok", 1: "bad argument", 2: "device out of memory", 3: "CUDA error",
    4: "non-finite matrix element", 5: "device wait timed out", 6: "no sm_100 device",
    7: "size beyond a documented limit",
}

# every symbol include/lapw1gpu.h declares
EXPORTS = [
    "lapw1gpu_init", "lapw1gpu_finalize", "lapw1gpu_set_precision", "lapw1gpu_kpoint_upload",
    "lapw1gpu_kpoint_free", "lapw1gpu_kpoint_run", "lapw1gpu_setup", "lapw1gpu_setup_stages",
    "lapw1gpu_stream", "lapw1gpu_last_status", "lapw1gpu_tns_from_gaunt", "lapw1gpu_version", "lapw1gpu_last_error",
    "lapw1gpu_setup_async", "lapw1gpu_setup_wait",
    "lapw1gpu_hns_noalloc", "lapw1gpu_forces", "lapw1gpu_setup_batch", "lapw1gpu_get_tuning",
    "lapw1gpu_set_tuning", "lapw1gpu_autotune", "lapw1gpu_set_slices", "lapw1gpu_test_wait_timeout",
    "lapw1gpu_last_launches", "lapw1gpu_host_register", "lapw1gpu_host_unregister", "lapw1gpu_forces_stats",
    "lapw1gpu_forces_batch", "lapw1gpu_set_force_slices", "lapw1gpu_set_force_projection",
    "lapw1gpu_seclr4",
]

_lib = None


class Tuning(C.Structure):
    """ctypes mirror of `lapw1gpu_tuning`."""

    _fields_ = [("hns_diag_b", C.c_int), ("split_group", C.c_int), ("sph_tc", C.c_int),
                ("batch_sets", C.c_int), ("sph_kblock", C.c_int), ("ms_best", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Lapw1GpuError(RuntimeError):
    def __init__(self, where: str, code: int):
        super().__init__(f"{where}: {STATUS.get(code, 'error')} (status {code})")
        self.code = code


def load(path: Optional[str] = None):
    """Load the library (built by hack_wein2k_b200.build); raise if absent."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python -m hack_wein2k_b200.build`")
    lib = C.CDLL(path)
    vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int)
    lib.lapw1gpu_init.argtypes = [C.c_int, C.POINTER(vp)]
    lib.lapw1gpu_finalize.argtypes = [vp]
    lib.lapw1gpu_set_precision.argtypes = [vp, C.c_int, C.c_int]
    lib.lapw1gpu_set_slices.argtypes = [vp, C.c_int, C.c_int]
    lib.lapw1gpu_set_force_slices.argtypes = [vp, C.c_int, C.c_int]
    lib.lapw1gpu_set_force_projection.argtypes = [vp, C.c_int, C.c_int]
    lib.lapw1gpu_seclr4.argtypes = [vp, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_int,
                                    C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_int)]
    lib.lapw1gpu_kpoint_upload.argtypes = [vp, C.POINTER(CProblem), C.POINTER(vp)]
    lib.lapw1gpu_kpoint_free.argtypes = [vp]
    lib.lapw1gpu_kpoint_run.argtypes = [vp, vp, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.POINTER(CStats)]
    lib.lapw1gpu_setup.argtypes = [vp, C.POINTER(CProblem), dp, C.c_int, dp, C.POINTER(CStats)]
    lib.lapw1gpu_setup_stages.argtypes = [vp, C.POINTER(CProblem), C.c_int, dp, C.c_int, dp,
                                          C.POINTER(CStats)]
    lib.lapw1gpu_stream.argtypes = [vp]
    lib.lapw1gpu_stream.restype = vp
    lib.lapw1gpu_last_status.argtypes = [vp]
    lib.lapw1gpu_version.restype = C.c_char_p
    lib.lapw1gpu_setup_async.argtypes = [vp, C.POINTER(CProblem), C.c_void_p, C.c_int, C.c_void_p]
    lib.lapw1gpu_setup_wait.argtypes = [vp, C.POINTER(CStats)]
    lib.lapw1gpu_last_error.restype = C.c_char_p
    lib.lapw1gpu_tns_from_gaunt.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, ip, ip, dp, dp, dp, dp,
                                            dp, dp, dp, ip, dp]
    lib.lapw1gpu_hns_noalloc.argtypes = [C.POINTER(CProblem), C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    lib.lapw1gpu_forces.argtypes = [vp, vp, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.lapw1gpu_setup_batch.argtypes = [vp, C.POINTER(vp), C.c_int, C.c_int, C.POINTER(C.c_void_p),
                                         C.POINTER(C.c_int), C.POINTER(C.c_void_p), C.POINTER(CStats)]
    lib.lapw1gpu_get_tuning.argtypes = [vp, C.POINTER(Tuning)]
    lib.lapw1gpu_set_tuning.argtypes = [vp, C.POINTER(Tuning)]
    lib.lapw1gpu_autotune.argtypes = [vp, vp, C.c_void_p, C.c_int, C.c_void_p, C.POINTER(Tuning)]
    lib.lapw1gpu_test_wait_timeout.argtypes = [vp, C.c_int]
    lib.lapw1gpu_last_launches.argtypes = [vp]
    lib.lapw1gpu_forces_stats.argtypes = [vp, C.POINTER(CStats)]
    lib.lapw1gpu_forces_batch.argtypes = [vp, C.POINTER(vp), C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_int),
                                          C.c_int, C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                          C.POINTER(C.c_double)]
    lib.lapw1gpu_host_register.argtypes = [vp, C.c_void_p, C.c_size_t]
    lib.lapw1gpu_host_unregister.argtypes = [vp, C.c_void_p]
    _lib = lib
    return lib


def _check(where: str, rc: int):
    if rc != 0:
        err = Lapw1GpuError(where, rc)
        if rc == 3 and _lib is not None:  # the failing CUDA call, for the message
            err.args = (f"{err.args[0]} [{_lib.lapw1gpu_last_error().decode()}]",)
        raise err


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class KPoint:
    """One k-point's inputs resident on the device (lapw1gpu_kpoint)."""

    def __init__(self, ctx: "Context", prob: Problem):
        self.ctx, self.prob = ctx, prob
        self._cp = prob.to_c()
        h = C.c_void_p()
        _check("lapw1gpu_kpoint_upload", ctx.lib.lapw1gpu_kpoint_upload(ctx.h, C.byref(self._cp), C.byref(h)))
        self.h = h

    def run(self, d_hs_ptr: int, ldhs: int, d_hsdiag_ptr: int, stages: int = 7, stats: bool = False):
        st = CStats() if stats else None
        rc = self.ctx.lib.lapw1gpu_kpoint_run(self.ctx.h, self.h, stages, C.c_void_p(d_hs_ptr), ldhs,
                                              C.c_void_p(d_hsdiag_ptr), C.byref(st) if st is not None else None)
        _check("lapw1gpu_kpoint_run", rc)
        return st.as_dict() if st is not None else None

    def forces(self, d_c_ptr: int, ldc: int, nb: int, d_occ_ptr: int, d_eps_ptr: int, d_grad_ptr: int) -> None:
        """dE/dPOS of E = sum occ*eps into the device array at d_grad_ptr
        (ndf x 3 doubles); eigenvectors column-major n x nb on the device."""
        rc = self.ctx.lib.lapw1gpu_forces(self.ctx.h, self.h, C.c_void_p(d_c_ptr), ldc, nb, C.c_void_p(d_occ_ptr),
                                          C.c_void_p(d_eps_ptr), C.c_void_p(d_grad_ptr))
        _check("lapw1gpu_forces", rc)

    def free(self):
        # a k-point outliving its context (closed first) is not freed: the
        # context's finalize released the device and its handle is gone
        if self.h and self.ctx.h:
            self.ctx.lib.lapw1gpu_kpoint_free(self.h)
        self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Context:
    """A lapw1gpu context on one CUDA device."""

    def __init__(self, device: int = 0, prec: int = PREC_FP64, slices: int = 5):
        self.lib = load()
        h = C.c_void_p()
        _check("lapw1gpu_init", self.lib.lapw1gpu_init(device, C.byref(h)))
        self.h = h
        self.device = device
        self.set_precision(prec, slices)

    def set_precision(self, prec: int, slices: int = 5):
        _check("lapw1gpu_set_precision", self.lib.lapw1gpu_set_precision(self.h, prec, slices))
        self.prec, self.slices = prec, slices

    def set_slices(self, slices_sph: int, slices_hns: int):
        """split precision with separate slice counts (lapw1gpu_set_slices)"""
        _check("lapw1gpu_set_slices", self.lib.lapw1gpu_set_slices(self.h, slices_sph, slices_hns))

    def set_force_slices(self, slices: int, slices_projection: Optional[int] = None):
        """int8 slices of the adjoint's density matrices and of its HNS
        projections in split precision (lapw1gpu_set_force_slices)"""
        sp = slices if slices_projection is None else slices_projection
        _check("lapw1gpu_set_force_slices", self.lib.lapw1gpu_set_force_slices(self.h, slices, sp))

    def set_force_projection(self, slices: int, block_rows: int = 1024):
        """split precision: the adjoint's spherical pairs of different blocks
        of block_rows PW rows as int8 slice projections (slices 4..8; 0: the
        FP64 pair kernel for every pair; -1: 6 slices from 6 blocks of rows)
        (lapw1gpu_set_force_projection)"""
        _check("lapw1gpu_set_force_projection",
               self.lib.lapw1gpu_set_force_projection(self.h, slices, block_rows))

    @property
    def stream_handle(self) -> int:
        return int(self.lib.lapw1gpu_stream(self.h) or 0)

    def last_status(self) -> int:
        return int(self.lib.lapw1gpu_last_status(self.h))

    def host_register(self, arr: np.ndarray) -> None:
        """page-lock a host array for the context's lifetime (lapw1gpu_host_register)"""
        _check("lapw1gpu_host_register", self.lib.lapw1gpu_host_register(self.h, C.c_void_p(arr.ctypes.data),
                                                                         arr.nbytes))

    def host_unregister(self, arr: np.ndarray) -> None:
        _check("lapw1gpu_host_unregister", self.lib.lapw1gpu_host_unregister(self.h, C.c_void_p(arr.ctypes.data)))

    def forces_stats(self) -> dict:
        """device times of the last forces call (lapw1gpu_forces_stats)"""
        st = CStats()
        _check("lapw1gpu_forces_stats", self.lib.lapw1gpu_forces_stats(self.h, C.byref(st)))
        return st.as_dict()

    def last_launches(self) -> int:
        """kernels the last setup, batch or forces call launched"""
        return int(self.lib.lapw1gpu_last_launches(self.h))

    def test_wait_timeout(self, on: bool) -> None:
        """Test hook (lapw1gpu_test_wait_timeout): make the spherical tensor
        kernel's consumer wait run out on later split-precision runs."""
        _check("lapw1gpu_test_wait_timeout", self.lib.lapw1gpu_test_wait_timeout(self.h, 1 if on else 0))

    def setup(self, prob: Problem, stages: int = 7, hs: Optional[np.ndarray] = None,
              hsdiag: Optional[np.ndarray] = None, stats: bool = False):
        """calkpt.F:153-185 on host buffers.  Returns (HS, HSDIAG[, stats]);
        HS is n x n complex128 in Fortran order (the reference's HS)."""
        n = prob.n
        if hs is None:
            hs = np.zeros((n, n), dtype=np.complex128, order="F")
        if hsdiag is None:
            hsdiag = np.zeros(n, dtype=np.complex128)
        assert hs.flags.f_contiguous and hs.dtype == np.complex128 and hs.shape[0] >= n
        cp = prob.to_c()
        st = CStats()
        rc = self.lib.lapw1gpu_setup_stages(self.h, C.byref(cp), stages,
                                            _dp(hs.reshape(-1, order="F").view(np.float64)), hs.shape[0],
                                            _dp(hsdiag.view(np.float64)), C.byref(st))
        _check("lapw1gpu_setup", rc)
        if stats:
            return hs, hsdiag, st.as_dict()
        return hs, hsdiag

    def setup_async(self, prob: Problem, hs: np.ndarray, hsdiag: np.ndarray) -> None:
        """lapw1gpu_setup_async into host buffers (HS Fortran-ordered); the
        problem's arrays and the buffers are held until setup_wait."""
        n = prob.n
        assert hs.flags.f_contiguous and hs.dtype == np.complex128 and hs.shape[0] >= n
        cp = prob.to_c()
        rc = self.lib.lapw1gpu_setup_async(self.h, C.byref(cp), hs.ctypes.data, hs.shape[0], hsdiag.ctypes.data)
        _check("lapw1gpu_setup_async", rc)
        self._async_keep = (cp, hs, hsdiag)

    def setup_wait(self, stats: bool = False):
        """lapw1gpu_setup_wait: (HS, HSDIAG[, stats]) of the queued setup."""
        st = CStats()
        rc = self.lib.lapw1gpu_setup_wait(self.h, C.byref(st))
        keep, self._async_keep = getattr(self, "_async_keep", None), None
        _check("lapw1gpu_setup_wait", rc)
        hs, hsdiag = keep[1], keep[2]
        return (hs, hsdiag, st.as_dict()) if stats else (hs, hsdiag)

    def upload(self, prob: Problem) -> KPoint:
        return KPoint(self, prob)

    def setup_batch(self, kps, d_hs_ptrs, ldhs, d_hsdiag_ptrs, stages: int = 7) -> dict:
        """lapw1gpu_setup_batch over resident k-points into device buffers;
        returns the batch stats (ms_total of the whole batch)."""
        nk = len(kps)
        karr = (C.c_void_p * nk)(*[k.h.value if isinstance(k.h, C.c_void_p) else k.h for k in kps])
        harr = (C.c_void_p * nk)(*d_hs_ptrs)
        larr = (C.c_int * nk)(*ldhs)
        darr = (C.c_void_p * nk)(*d_hsdiag_ptrs)
        st = CStats()
        _check("lapw1gpu_setup_batch",
               self.lib.lapw1gpu_setup_batch(self.h, karr, nk, stages, harr, larr, darr, C.byref(st)))
        return st.as_dict()

    def forces_batch(self, kps, d_c_ptrs, ldc, nb: int, d_occ_ptr: int, d_eps_ptrs, d_grad_ptrs) -> float:
        """lapw1gpu_forces_batch over resident k-points; returns the device
        time of the whole list (ms)."""
        nk = len(kps)
        karr = (C.c_void_p * nk)(*[k.h.value if isinstance(k.h, C.c_void_p) else k.h for k in kps])
        ms = C.c_double()
        _check("lapw1gpu_forces_batch",
               self.lib.lapw1gpu_forces_batch(self.h, karr, nk, (C.c_void_p * nk)(*d_c_ptrs), (C.c_int * nk)(*ldc),
                                              nb, C.c_void_p(d_occ_ptr), (C.c_void_p * nk)(*d_eps_ptrs),
                                              (C.c_void_p * nk)(*d_grad_ptrs), C.byref(ms)))
        return ms.value

    def seclr4(self, d_hs_ptr: int, ldhs: int, d_hsdiag_ptr: int, n: int, el: float, eu: float, nmax: int,
               d_eig_ptr: int, d_vec_ptr: int = 0, ldv: int = 0) -> int:
        """lapw1gpu_seclr4: eigenvalues (and eigenvectors) of the packed
        state on the device; returns how many were found."""
        nf = C.c_int()
        _check("lapw1gpu_seclr4",
               self.lib.lapw1gpu_seclr4(self.h, C.c_void_p(d_hs_ptr), ldhs, C.c_void_p(d_hsdiag_ptr), n, el, eu, nmax,
                                        C.c_void_p(d_eig_ptr), C.c_void_p(d_vec_ptr) if d_vec_ptr else None,
                                        ldv or n, C.byref(nf)))
        return nf.value

    def tuning(self) -> dict:
        t = Tuning()
        _check("lapw1gpu_get_tuning", self.lib.lapw1gpu_get_tuning(self.h, C.byref(t)))
        return t.as_dict()

    def set_tuning(self, **kw) -> None:
        t = Tuning()
        _check("lapw1gpu_get_tuning", self.lib.lapw1gpu_get_tuning(self.h, C.byref(t)))
        for k, v in kw.items():
            setattr(t, k, v)
        _check("lapw1gpu_set_tuning", self.lib.lapw1gpu_set_tuning(self.h, C.byref(t)))

    def autotune(self, kp: KPoint, d_hs_ptr: int, ldhs: int, d_hsdiag_ptr: int) -> dict:
        t = Tuning()
        _check("lapw1gpu_autotune", self.lib.lapw1gpu_autotune(self.h, kp.h, C.c_void_p(d_hs_ptr), ldhs,
                                                               C.c_void_p(d_hsdiag_ptr), C.byref(t)))
        return t.as_dict()

    def close(self):
        if self.h:
            self.lib.lapw1gpu_finalize(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def version() -> str:
    return load().lapw1gpu_version().decode()


def hns_noalloc(prob: Problem, d_hs_ptr: int, ldhs: int, stream: int = 0, d_status_ptr: int = 0) -> None:
    """lapw1gpu_hns_noalloc: add the HNS update into a caller-owned device
    HS without any allocation by the library (see include/lapw1gpu.h).
    d_status_ptr (optional): a device int that receives the call's status
    bits once the stream has run the call."""
    cp = prob.to_c()
    _check("lapw1gpu_hns_noalloc",
           load().lapw1gpu_hns_noalloc(C.byref(cp), C.c_void_p(d_hs_ptr), ldhs, C.c_void_p(stream),
                                       C.c_void_p(d_status_ptr) if d_status_ptr else None))


def tns_from_gaunt(nat, lnsmax, lqind, lqns, gfac, vns1, vns2, vns3, vnslo1, vnslo2, vnslo3, loor):
    """Product-side gaunt-list -> T-block builder (lapw1gpu_tns_from_gaunt)."""
    lib = load()
    lqns = np.ascontiguousarray(lqns, dtype=np.int32)
    ngau = lqns.shape[1]
    lmmx = np.asarray(vns1).shape[2]
    out = np.zeros((nat, 9, 25, 25), dtype=np.complex128)
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (vns1, vns2, vns3, vnslo1, vnslo2, vnslo3)]
    g = np.ascontiguousarray(gfac, dtype=np.complex128)
    li = np.ascontiguousarray(lqind, dtype=np.int32)
    lo = np.ascontiguousarray(loor, dtype=np.int32)
    rc = lib.lapw1gpu_tns_from_gaunt(nat, lnsmax, ngau, lmmx, li.ctypes.data_as(C.POINTER(C.c_int)),
                                     lqns.ctypes.data_as(C.POINTER(C.c_int)), _dp(g.view(np.float64)),
                                     *[_dp(a) for a in arrs], lo.ctypes.data_as(C.POINTER(C.c_int)),
                                     _dp(out.view(np.float64)))
    _check("lapw1gpu_tns_from_gaunt", rc)
    return out
