"""Python binding of libskgemm (the C ABI in include/skgemm.h) over ctypes.

The host-side classes mirror the reference's static C++ entry points, with the
same names, argument order and meaning, so that checks read like the
reference's own drivers:

* ``gemm.compute_test(M, N, K, A, B, D, alpha, gamma)``     gemm_opt.cpp:376
* ``gemm.compute_packed(M, N, K, Ap, Bp, D, alpha, gamma)`` gemm_opt.cpp:314
* ``gemm.compute_streamk_packed(...)``                      gemm_crsp.cpp:316
* ``sme_syrk.compute(K, M, Ap, C, alpha, beta)``            sme_syrk.hpp:137
* ``sme_gemm_trp_3d.compute(Nd, nb, A, B, D)``              sme_trp_3d.hpp:194

They take host numpy float64 arrays and block, like the reference. Where the
reference silently returns (bad shapes, no error channel) these raise
``SkgemmError`` carrying the C status code.

The ``*_dev`` functions take CUDA device pointers (or torch tensors) and a
stream, and are asynchronous. There is no CPU fallback: without the built
library or an sm_100 device every call raises.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(HERE), "libskgemm.so")

OK = 0
ERR_INVALID_ARG = -1
ERR_OOM = -2
ERR_CUDA = -3
ERR_DEVICE_TIMEOUT = -4
ERR_NO_DEVICE = -5
ERR_UNSUPPORTED = -6

PREC_NATIVE = 0
PREC_OZAKI_I8 = 1
PREC_AUTO = 2  # batched plans: per problem, the faster path
PREC_OZAKI_BF16 = 3  # Ozaki with BF16 residues (results equal PREC_OZAKI_I8)


class SkgemmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"skgemm status {code}: {msg}")
        self.code = code


class Options(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("slices", ctypes.c_int),
                ("err_bound_out", ctypes.c_double), ("slices_used_out", ctypes.c_int)]


OP_GEMM_PACKED = 0
OP_SYRK_PACKED = 1
OP_ROT = 2


class BatchItem(ctypes.Structure):
    """skgemm_batch_item_t: one problem of a grouped launch."""
    _fields_ = [("op", ctypes.c_int), ("M", ctypes.c_int64), ("N", ctypes.c_int64),
                ("K", ctypes.c_int64), ("A", ctypes.c_void_p), ("B", ctypes.c_void_p),
                ("D", ctypes.c_void_p), ("ldd", ctypes.c_int64), ("alpha", ctypes.c_double),
                ("beta", ctypes.c_double)]


class PlanOptions(ctypes.Structure):
    """skgemm_plan_options_t."""
    _fields_ = [("tile", ctypes.c_int), ("grid", ctypes.c_int), ("order", ctypes.c_int),
                ("no_tune", ctypes.c_int), ("no_graph", ctypes.c_int),
                ("precision", ctypes.c_int), ("slices", ctypes.c_int),
                ("ozaki_problems_out", ctypes.c_int), ("tile_out", ctypes.c_int), ("grid_out", ctypes.c_int),
                ("order_out", ctypes.c_int), ("candidates_timed_out", ctypes.c_int),
                ("tuned_ms_out", ctypes.c_double), ("model_efficiency_out", ctypes.c_double),
                ("graph_kernels_out", ctypes.c_int)]


class ServeRequest(ctypes.Structure):
    """skgemm_serve_request_t."""
    _fields_ = [("Ng", ctypes.c_int64), ("nb", ctypes.c_int64), ("arrival_s", ctypes.c_double),
                ("seed", ctypes.c_uint64), ("S_out", ctypes.c_void_p), ("Hs_out", ctypes.c_void_p),
                ("Psi_out", ctypes.c_void_p), ("Psi_in_out", ctypes.c_void_p),
                ("HPsi_in_out", ctypes.c_void_p), ("Q_in_out", ctypes.c_void_p),
                ("admit_s", ctypes.c_double), ("done_s", ctypes.c_double)]


class ServeOptions(ctypes.Structure):
    """skgemm_serve_options_t."""
    _fields_ = [("precision", ctypes.c_int), ("slices", ctypes.c_int),
                ("hbm_budget_bytes", ctypes.c_double), ("max_inflight", ctypes.c_int),
                ("ozaki_streams", ctypes.c_int), ("max_batch_tflop", ctypes.c_double),
                ("realtime", ctypes.c_int), ("policy", ctypes.c_int), ("aging_s", ctypes.c_double),
                ("sim_native_tflops", ctypes.c_double),
                ("sim_ozaki_tflops", ctypes.c_double), ("sim_gen_gbs", ctypes.c_double),
                ("makespan_s", ctypes.c_double), ("flop", ctypes.c_double),
                ("batches", ctypes.c_int), ("mean_batch_problems", ctypes.c_double),
                ("peak_admitted_bytes", ctypes.c_double), ("scratch_bytes", ctypes.c_double)]


_i64 = ctypes.c_int64
_vp = ctypes.c_void_p
_d = ctypes.c_double
_lib: Optional[ctypes.CDLL] = None

# name -> argtypes (all return int status except the two string getters)
_SIGS = {
    "skgemm_stream_status": [_vp],
    "skgemm_probe_fp64_peak": [ctypes.POINTER(ctypes.c_double)],
    "skgemm_diag_expire_wait": [ctypes.c_double, _vp],
    "skgemm_kernel_timing": [ctypes.c_int],
    "skgemm_kernel_timing_report": [ctypes.c_char_p, _i64],
    "skgemm_diag_expire_fixup_wait": [ctypes.c_double, _vp],
    "skgemm_probe_i8_peak": [ctypes.POINTER(ctypes.c_double)],
    "skgemm_igemm_s8_dev": [_i64, _i64, _i64, _vp, _i64, _vp, _i64, _vp, _i64, _vp],
    "skgemm_dgemm": [_i64, _i64, _i64, _vp, _vp, _vp, _d, _d],
    "skgemm_dgemm_packed": [_i64, _i64, _i64, _vp, _vp, _vp, _d, _d],
    "skgemm_dgemm_dev": [_i64, _i64, _i64, _vp, _i64, _vp, _i64, _vp, _i64, _d, _d, _vp],
    "skgemm_dgemm_packed_dev": [_i64, _i64, _i64, _vp, _vp, _vp, _i64, _d, _d, _vp],
    "skgemm_dgemm_packed_dev_noalloc": [_i64, _i64, _i64, _vp, _vp, _vp, _i64, _d, _d, _vp],
    "skgemm_dgemm_packed_dev_opt": [_i64, _i64, _i64, _vp, _vp, _vp, _i64, _d, _d,
                                    ctypes.POINTER(Options), _vp],
    "skgemm_dsyrk_packed": [_i64, _i64, _vp, _vp, _d, _d],
    "skgemm_dsyrk_packed_dev": [_i64, _i64, _vp, _vp, _i64, _d, _d, _vp],
    "skgemm_dsyrk_packed_dev_opt": [_i64, _i64, _vp, _vp, _i64, _d, _d,
                                    ctypes.POINTER(Options), _vp],
    "skgemm_dsubspace_packed_dev": [_i64, _i64, _vp, _vp, _vp, _i64, _vp, _i64,
                                    ctypes.POINTER(Options), _vp],
    "skgemm_drot": [_i64, _i64, _vp, _vp, _vp],
    "skgemm_drot_opt": [_i64, _i64, _vp, _vp, _vp, ctypes.POINTER(Options)],
    "skgemm_dgemm_packed_opt": [_i64, _i64, _i64, _vp, _vp, _vp, _d, _d,
                                ctypes.POINTER(Options)],
    "skgemm_dsyrk_packed_opt": [_i64, _i64, _vp, _vp, _d, _d, ctypes.POINTER(Options)],
    "skgemm_drot_dev": [_i64, _i64, _vp, _vp, _vp, _vp],
    "skgemm_drot_dev_opt": [_i64, _i64, _vp, _vp, _vp, ctypes.POINTER(Options), _vp],
    "skgemm_drot_band_dev": [_i64, _i64, _vp, _vp, _vp, _vp],
    "skgemm_drot_band_dev_opt": [_i64, _i64, _vp, _vp, _vp, ctypes.POINTER(Options), _vp],
    "skgemm_pack_dev": [_i64, _i64, _vp, _i64, _i64, ctypes.c_int, _vp, _vp],
    "skgemm_unpack_dev": [_i64, _i64, _vp, ctypes.c_int, _vp, _i64, _i64, _vp],
    "skgemm_pack_c16_dev": [_i64, _i64, _vp, _vp, _vp],
    "skgemm_pack_r16_dev": [_i64, _i64, _vp, _vp, _vp],
    "skgemm_unpack_c16_dev": [_i64, _i64, _vp, _vp, _vp],
    "skgemm_unpack_r16_dev": [_i64, _i64, _vp, _vp, _vp],
    "skgemm_stencil_ext_dev": [_i64, _i64, _i64, _i64, ctypes.c_int, _vp, _vp,
                               ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                               ctypes.POINTER(ctypes.c_double), ctypes.c_double, _vp,
                               ctypes.c_int, _vp],
    "skgemm_halo_periodic_dev": [_i64, _i64, _i64, _i64, ctypes.c_int, _vp, _vp, _vp],
    "skgemm_nloc_create": [_i64, ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32),
                           ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_uint32),
                           ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_double),
                           ctypes.POINTER(ctypes.c_double), _i64, ctypes.POINTER(ctypes.c_void_p)],
    "skgemm_nloc_apply_dev": [_vp, _i64, ctypes.c_double, _vp, _vp, ctypes.c_int, _vp],
    "skgemm_band_to_grid_dev": [_i64, _i64, _vp, _vp, _vp],
    "skgemm_grid_to_band_dev": [_i64, _i64, _vp, _vp, _vp],
    "skgemm_plan_create": [ctypes.POINTER(BatchItem), ctypes.c_int,
                           ctypes.POINTER(PlanOptions), _vp, ctypes.POINTER(_vp)],
    "skgemm_plan_run": [_vp, _vp],
    "skgemm_plan_status": [_vp, _vp],
    "skgemm_plan_precisions": [_vp, ctypes.POINTER(ctypes.c_int), ctypes.c_int],
    "skgemm_batch_dev": [ctypes.POINTER(BatchItem), ctypes.c_int, _vp],
    "skgemm_serve_run": [ctypes.POINTER(ServeRequest), ctypes.c_int,
                         ctypes.POINTER(ServeOptions)],
    "skgemm_serve_simulate": [ctypes.POINTER(ServeRequest), ctypes.c_int,
                              ctypes.POINTER(ServeOptions)],
    "skgemm_stream_release": [_vp],
    "skgemm_debug_fill": [],
    "skgemm_tune_cache_save": [ctypes.c_char_p],
    "skgemm_tune_cache_load": [ctypes.c_char_p],
    "skgemm_tune_cache_clear": [],
    "skgemm_batch_schedule": [ctypes.POINTER(BatchItem), ctypes.c_int, ctypes.c_int,
                              ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                              ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_double)],
}


# The reference's own extern "C" converter names (include/sme_pack.hpp:316-352):
# void f(int Nd, int nb, const double* src, double* dst), host pointers.
LINALG = ("linalg_pack_c16_f64", "linalg_pack_r16_f64", "linalg_unpack_c16_f64",
          "linalg_unpack_r16_f64")


def lib() -> ctypes.CDLL:
    """Loads libskgemm.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise SkgemmError(ERR_UNSUPPORTED,
                              f"{LIB_PATH} not built (python stream-k-gemm_b200/build.py)")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = ctypes.c_int
        L.skgemm_version.restype = ctypes.c_char_p
        L.skgemm_version.argtypes = []
        L.skgemm_last_error.restype = ctypes.c_char_p
        L.skgemm_last_error.argtypes = []
        L.skgemm_plan_destroy.restype = None
        L.skgemm_nloc_destroy.restype = None
        L.skgemm_nloc_destroy.argtypes = [ctypes.c_void_p]
        L.skgemm_plan_destroy.argtypes = [_vp]
        for name in LINALG:
            f = getattr(L, name)
            f.argtypes = [ctypes.c_int, ctypes.c_int, _vp, _vp]
            f.restype = None
        _lib = L
    return _lib


def exported_symbols() -> list:
    return ["skgemm_version", "skgemm_last_error", "skgemm_plan_destroy",
            "skgemm_nloc_destroy"] + list(_SIGS) + list(LINALG)


def version() -> str:
    return lib().skgemm_version().decode()


def _check(code: int) -> int:
    if code != OK:
        msg = lib().skgemm_last_error().decode(errors="replace")
        raise SkgemmError(code, msg)
    return code


def _hptr(a: np.ndarray, writable: bool = False):
    if not isinstance(a, np.ndarray) or a.dtype != np.float64 or not a.flags.c_contiguous:
        raise SkgemmError(ERR_INVALID_ARG, "host arrays must be C-contiguous float64 numpy arrays")
    if writable and not a.flags.writeable:
        raise SkgemmError(ERR_INVALID_ARG, "output array is read-only")
    return a.ctypes.data


def _dptr(x) -> int:
    """Device address of a torch tensor, or an int address as given."""
    if x is None:
        return 0
    if isinstance(x, int):
        return x
    return int(x.data_ptr())


def _stream(s) -> int:
    if s is None:
        return 0
    if isinstance(s, int):
        return s
    return int(s.cuda_stream)  # torch.cuda.Stream


# ------------------------------------------------------- reference mirror
class gemm:
    """Mirror of the reference's ``gemm<double>`` (gemm_opt.cpp:55 /
    gemm_crsp.cpp:57): D = alpha*A*B + gamma."""

    @staticmethod
    def compute_test(M, N, K, A_colmajor, B_rowmajor, D, alpha=1.0, gamma=0.0):
        _check(lib().skgemm_dgemm(M, N, K, _hptr(A_colmajor), _hptr(B_rowmajor),
                                  _hptr(D, True), alpha, gamma))

    @staticmethod
    def compute_packed(M, N, K, A_packed, B_packed, D, alpha=1.0, gamma=0.0, precision=None,
                       slices=0):
        """``precision`` (an addition, default native) routes the host call
        through the Ozaki split; returns the options (moduli used, bound)."""
        o = _opts(precision, slices)
        if o is None:
            _check(lib().skgemm_dgemm_packed(M, N, K, _hptr(A_packed), _hptr(B_packed),
                                             _hptr(D, True), alpha, gamma))
            return None
        _check(lib().skgemm_dgemm_packed_opt(M, N, K, _hptr(A_packed), _hptr(B_packed),
                                             _hptr(D, True), alpha, gamma, ctypes.byref(o)))
        return o

    compute_streamk_packed = compute_packed


class sme_syrk:
    """Mirror of ``sme_syrk<double>`` (include/sme_syrk.hpp:22, syrk_crsp.cpp:51):
    C = alpha*A^T*A + beta*C, upper triangle, column-major C."""

    @staticmethod
    def compute(K, M, A_packed, C, alpha=1.0, beta=0.0, precision=None, slices=0):
        o = _opts(precision, slices)
        if o is None:
            _check(lib().skgemm_dsyrk_packed(K, M, _hptr(A_packed), _hptr(C, True), alpha, beta))
            return None
        _check(lib().skgemm_dsyrk_packed_opt(K, M, _hptr(A_packed), _hptr(C, True), alpha, beta,
                                             ctypes.byref(o)))
        return o


class sme_gemm_trp_3d:
    """Mirror of ``sme_gemm_trp_3d<double>`` (include/sme_trp_3d.hpp:48): D = A*B
    with A grid-packed, B row-major, D band-packed."""

    @staticmethod
    def compute(Nd, nb, A_grid, B, D_band, precision=None, slices=0):
        o = _opts(precision, slices)
        if o is None:
            _check(lib().skgemm_drot(Nd, nb, _hptr(A_grid), _hptr(B), _hptr(D_band, True)))
            return None
        _check(lib().skgemm_drot_opt(Nd, nb, _hptr(A_grid), _hptr(B), _hptr(D_band, True),
                                     ctypes.byref(o)))
        return o


sme_gemm_trp = sme_gemm_trp_3d


# --------------------------------------------------------- device entries
def _opts(precision, slices):
    if precision is None or precision == PREC_NATIVE:
        return None
    o = Options()
    o.precision = precision
    o.slices = slices or 0
    return o


def dgemm_packed_dev(M, N, K, A_packed, B_packed, D, ldd=None, alpha=1.0, gamma=0.0,
                     stream=None, precision=None, slices=0):
    o = _opts(precision, slices)
    if o is None:
        _check(lib().skgemm_dgemm_packed_dev(M, N, K, _dptr(A_packed), _dptr(B_packed),
                                             _dptr(D), ldd or N, alpha, gamma, _stream(stream)))
        return None
    _check(lib().skgemm_dgemm_packed_dev_opt(M, N, K, _dptr(A_packed), _dptr(B_packed),
                                             _dptr(D), ldd or N, alpha, gamma,
                                             ctypes.byref(o), _stream(stream)))
    return o


def dgemm_packed_dev_noalloc(M, N, K, A_packed, B_packed, D, ldd=None, alpha=1.0, gamma=0.0,
                             stream=None):
    """Allocation-free packed GEMM (static device scratch; blocks until done)."""
    _check(lib().skgemm_dgemm_packed_dev_noalloc(M, N, K, _dptr(A_packed), _dptr(B_packed),
                                                 _dptr(D), ldd or N, alpha, gamma,
                                                 _stream(stream)))


def dgemm_dev(M, N, K, A_colmajor, lda, B_rowmajor, ldb, D, ldd, alpha=1.0, gamma=0.0,
              stream=None):
    _check(lib().skgemm_dgemm_dev(M, N, K, _dptr(A_colmajor), lda, _dptr(B_rowmajor), ldb,
                                  _dptr(D), ldd, alpha, gamma, _stream(stream)))


def dsyrk_packed_dev(K, M, A_packed, C, ldc=None, alpha=1.0, beta=0.0, stream=None,
                     precision=None, slices=0):
    o = _opts(precision, slices)
    if o is None:
        _check(lib().skgemm_dsyrk_packed_dev(K, M, _dptr(A_packed), _dptr(C), ldc or M, alpha,
                                             beta, _stream(stream)))
        return None
    _check(lib().skgemm_dsyrk_packed_dev_opt(K, M, _dptr(A_packed), _dptr(C), ldc or M, alpha,
                                             beta, ctypes.byref(o), _stream(stream)))
    return o


def dsubspace_packed_dev(K, M, Psi_packed16, HPsi_packed32, S, Hs, lds=None, ldh=None,
                         stream=None, precision=None, slices=0):
    """S = Psi^T Psi (upper, column-major) and Hs = Psi^T HPsi (row-major) in one
    call; with the Ozaki precision Psi is split once for both products."""
    o = _opts(precision, slices)
    _check(lib().skgemm_dsubspace_packed_dev(K, M, _dptr(Psi_packed16), _dptr(HPsi_packed32),
                                             _dptr(S), lds or M, _dptr(Hs), ldh or M,
                                             ctypes.byref(o) if o is not None else None,
                                             _stream(stream)))
    return o


def drot_dev(Nd, nb, A_grid, Q, D_band, stream=None, precision=None, slices=0):
    o = _opts(precision, slices)
    if o is None:
        _check(lib().skgemm_drot_dev(Nd, nb, _dptr(A_grid), _dptr(Q), _dptr(D_band),
                                     _stream(stream)))
        return None
    _check(lib().skgemm_drot_dev_opt(Nd, nb, _dptr(A_grid), _dptr(Q), _dptr(D_band),
                                     ctypes.byref(o), _stream(stream)))
    return o


def drot_band_dev(Nd, nb, A_band, Q, D_band, stream=None, precision=None, slices=0):
    """The rotation on band-packed Psi (the layout SYRK and GEMM read); equals
    drot_dev on the grid-packed copy, bit for bit."""
    o = _opts(precision, slices)
    if o is None:
        _check(lib().skgemm_drot_band_dev(Nd, nb, _dptr(A_band), _dptr(Q), _dptr(D_band),
                                          _stream(stream)))
        return None
    _check(lib().skgemm_drot_band_dev_opt(Nd, nb, _dptr(A_band), _dptr(Q), _dptr(D_band),
                                          ctypes.byref(o), _stream(stream)))
    return o


def pack_dev(R, K, X, sr, sk, T, X_packed, stream=None):
    _check(lib().skgemm_pack_dev(R, K, _dptr(X), sr, sk, T, _dptr(X_packed), _stream(stream)))


def unpack_dev(R, K, X_packed, T, X, sr, sk, stream=None):
    """Packed-T panels -> strided dense X[r*sr + k*sk] (rows r < R)."""
    _check(lib().skgemm_unpack_dev(R, K, _dptr(X_packed), T, _dptr(X), sr, sk, _stream(stream)))


class sme_pack:
    """The reference's C converters by their own names (sme_pack.hpp:316-352),
    host numpy arrays, blocking: ``pack_c16(Nd, nb, src, dst)`` etc. Like the
    reference they convert the first 16 * (Nd // 16) grid points; a refused
    call raises here (the C functions return nothing and leave the reason in
    skgemm_last_error)."""

    @staticmethod
    def _call(name, Nd, nb, src, dst):
        getattr(lib(), name)(Nd, nb, _hptr(src), _hptr(dst, True))
        msg = lib().skgemm_last_error().decode(errors="replace")
        if msg:
            raise SkgemmError(ERR_INVALID_ARG, msg)

    @staticmethod
    def pack_c16(Nd, nb, src, dst):
        sme_pack._call("linalg_pack_c16_f64", Nd, nb, src, dst)

    @staticmethod
    def pack_r16(Nd, nb, src, dst):
        sme_pack._call("linalg_pack_r16_f64", Nd, nb, src, dst)

    @staticmethod
    def unpack_c16(Nd, nb, src, dst):
        sme_pack._call("linalg_unpack_c16_f64", Nd, nb, src, dst)

    @staticmethod
    def unpack_r16(Nd, nb, src, dst):
        sme_pack._call("linalg_unpack_r16_f64", Nd, nb, src, dst)


def pack_c16_dev(Nd, nb, src, dst, stream=None):
    """linalg_pack_c16_f64 (sme_pack.hpp:319): column-major [Nd, nb] -> grid-packed."""
    _check(lib().skgemm_pack_c16_dev(Nd, nb, _dptr(src), _dptr(dst), _stream(stream)))


def pack_r16_dev(Nd, nb, src, dst, stream=None):
    """linalg_pack_r16_f64 (sme_pack.hpp:322): row-major [nb, Nd] -> grid-packed."""
    _check(lib().skgemm_pack_r16_dev(Nd, nb, _dptr(src), _dptr(dst), _stream(stream)))


def unpack_c16_dev(Nd, nb, src, dst, stream=None):
    """linalg_unpack_c16_f64 (sme_pack.hpp:325): grid-packed -> column-major [Nd, nb]."""
    _check(lib().skgemm_unpack_c16_dev(Nd, nb, _dptr(src), _dptr(dst), _stream(stream)))


def unpack_r16_dev(Nd, nb, src, dst, stream=None):
    """linalg_unpack_r16_f64 (sme_pack.hpp:328): grid-packed -> row-major [nb, Nd]."""
    _check(lib().skgemm_unpack_r16_dev(Nd, nb, _dptr(src), _dptr(dst), _stream(stream)))


def _coef(c, n):
    """The first n stencil coefficients (index 0 .. FDn) as a C array."""
    if len(c) < n:
        raise SkgemmError(ERR_INVALID_ARG, f"stencil coefficients need {n} values (0 .. FDn)")
    return (ctypes.c_double * n)(*[float(x) for x in c[:n]])


def stencil_ext_dev(ni, nj, nk, nb, ext16, A_diag, coef_x, coef_y, coef_z, coef_0, out,
                    out_tile=32, FDn=6, stream=None):
    """H Psi = stencil(extended band-packed Psi) into 32- (or 16-) band-packed
    out (calc_laplacian_extended_packed_16to32 / _16to16)."""
    _check(lib().skgemm_stencil_ext_dev(ni, nj, nk, nb, FDn, _dptr(ext16), _dptr(A_diag),
                                        _coef(coef_x, max(FDn + 1, 0)),
                                        _coef(coef_y, max(FDn + 1, 0)),
                                        _coef(coef_z, max(FDn + 1, 0)),
                                        float(coef_0), _dptr(out), out_tile, _stream(stream)))


def halo_periodic_dev(ni, nj, nk, nb, local16, ext16, FDn=6, stream=None):
    """Single-rank periodic extension of band-packed Psi (halo_packed.hpp)."""
    _check(lib().skgemm_halo_periodic_dev(ni, nj, nk, nb, FDn, _dptr(local16), _dptr(ext16),
                                          _stream(stream)))


class NlocProjector:
    """A nonlocal projector set on the device (skgemm_nloc_create): the
    reference's Effective_potential_nloc. Arrays as numpy (host); `apply`
    adds V_nloc psi into out (16- or 32-band-packed, device tensors)."""

    def __init__(self, nrow, ncol, atom, offsets, index, chi, gamma, K):
        arr = lambda a, t: np.ascontiguousarray(a, dtype=t)
        self._keep = [arr(nrow, np.uint32), arr(ncol, np.uint32), arr(atom, np.int32),
                      arr(offsets, np.uint32), arr(index, np.uint32), arr(chi, np.float64),
                      arr(gamma, np.float64)]
        nr, nc, at, off, idx, ch, gm = self._keep
        P = len(nr)
        if len(nc) != P or len(at) != P or len(off) != P + 1:
            raise SkgemmError(ERR_INVALID_ARG, "ncol and atom take one entry per projector, "
                                               "offsets one more")
        if (len(idx) < int(nr.sum(dtype=np.int64))
                or len(ch) < int((nr.astype(np.int64) * nc).sum())
                or len(gm) < int(nc.sum(dtype=np.int64))):
            raise SkgemmError(ERR_INVALID_ARG, "index, chi or gamma shorter than the projectors")
        c = ctypes
        h = c.c_void_p()
        _check(lib().skgemm_nloc_create(
            len(nr), nr.ctypes.data_as(c.POINTER(c.c_uint32)),
            nc.ctypes.data_as(c.POINTER(c.c_uint32)), at.ctypes.data_as(c.POINTER(c.c_int32)),
            off.ctypes.data_as(c.POINTER(c.c_uint32)), idx.ctypes.data_as(c.POINTER(c.c_uint32)),
            ch.ctypes.data_as(c.POINTER(c.c_double)), gm.ctypes.data_as(c.POINTER(c.c_double)),
            K, c.byref(h)))
        self._h = h

    def apply(self, nb, dv, psi16, out, out_tile=32, stream=None):
        _check(lib().skgemm_nloc_apply_dev(self._h, nb, float(dv), _dptr(psi16), _dptr(out),
                                           out_tile, _stream(stream)))

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().skgemm_nloc_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def band_to_grid_dev(Nd, nb, src, dst, stream=None):
    _check(lib().skgemm_band_to_grid_dev(Nd, nb, _dptr(src), _dptr(dst), _stream(stream)))


def grid_to_band_dev(Nd, nb, src, dst, stream=None):
    _check(lib().skgemm_grid_to_band_dev(Nd, nb, _dptr(src), _dptr(dst), _stream(stream)))


def stream_status(stream=None) -> None:
    """Synchronise ``stream``; raise if a device-side wait ran out of budget."""
    _check(lib().skgemm_stream_status(_stream(stream)))


def igemm_s8_dev(M, N, K, A, lda, B, ldb, C, ldc, stream=None):
    """Exact int8 x int8 -> int32 GEMM, both operands K-major (device)."""
    _check(lib().skgemm_igemm_s8_dev(M, N, K, _dptr(A), lda, _dptr(B), ldb, _dptr(C), ldc,
                                     _stream(stream)))


def diag_expire_wait(budget_ms, stream=None) -> None:
    """Enqueue one bounded device wait that runs out after budget_ms; the next
    stream_status(stream) raises SkgemmError(ERR_DEVICE_TIMEOUT)."""
    _check(lib().skgemm_diag_expire_wait(float(budget_ms), _stream(stream)))


def diag_expire_fixup_wait(budget_ms, stream=None) -> None:
    """Enqueue the Stream-K fixup's flag wait on a flag nothing sets, with
    budget_ms; the next stream_status(stream) raises ERR_DEVICE_TIMEOUT."""
    _check(lib().skgemm_diag_expire_fixup_wait(float(budget_ms), _stream(stream)))


def kernel_timing(enable: bool) -> None:
    """Start (clearing the record) or stop per-kernel event timing."""
    _check(lib().skgemm_kernel_timing(1 if enable else 0))


def kernel_timing_report() -> dict:
    """{kernel name: (launches, total ms)} recorded since kernel_timing(True)
    (synchronises; clears the record)."""
    buf = ctypes.create_string_buffer(1 << 16)
    n = lib().skgemm_kernel_timing_report(buf, len(buf))
    if n < 0:
        _check(n)
    out = {}
    for line in buf.value.decode().splitlines():
        name, cnt, ms = line.split()
        out[name] = (int(cnt), float(ms))
    return out


def probe_i8_peak() -> float:
    v = ctypes.c_double(0.0)
    _check(lib().skgemm_probe_i8_peak(ctypes.byref(v)))
    return v.value


def probe_fp64_peak() -> float:
    v = ctypes.c_double(0.0)
    _check(lib().skgemm_probe_fp64_peak(ctypes.byref(v)))
    return v.value


# ------------------------------------------------------------------ batched
def batch_item(op, M, N, K, A, B, D, ldd=0, alpha=1.0, beta=0.0) -> BatchItem:
    """One problem of a grouped launch (device buffers: torch tensors or addresses)."""
    return BatchItem(op, M, N, K, _dptr(A), _dptr(B), _dptr(D), ldd, alpha, beta)


def _item_array(items):
    arr = (BatchItem * max(1, len(items)))()
    for i, it in enumerate(items):
        arr[i] = it
    return arr


class Plan:
    """A tuned, graph-captured grouped launch of a fixed set of problems
    (skgemm_plan_create / _run / _status / _destroy)."""

    def __init__(self, items, tile=0, grid=0, order=0, tune=True, graph=True, stream=None,
                 precision=PREC_NATIVE, slices=0):
        self.options = PlanOptions(tile, grid, order, 0 if tune else 1, 0 if graph else 1,
                                   precision, slices)
        self._items = _item_array(items)
        self._n = len(items)
        h = ctypes.c_void_p(0)
        _check(lib().skgemm_plan_create(self._items, len(items), ctypes.byref(self.options),
                                        _stream(stream), ctypes.byref(h)))
        self._h = h

    def run(self, stream=None) -> None:
        _check(lib().skgemm_plan_run(self._h, _stream(stream)))

    def status(self, stream=None) -> None:
        _check(lib().skgemm_plan_status(self._h, _stream(stream)))

    @property
    def config(self) -> dict:
        o = self.options
        return {"tile": o.tile_out, "grid": o.grid_out, "order": o.order_out,
                "ozaki_problems": o.ozaki_problems_out,
                "candidates_timed": o.candidates_timed_out, "tuned_ms": o.tuned_ms_out,
                "model_efficiency": o.model_efficiency_out,
                "graph_kernels": o.graph_kernels_out}

    def precisions(self) -> list:
        """Per item: PREC_NATIVE, PREC_OZAKI_I8 or PREC_OZAKI_BF16 (the path the
        plan runs it on)."""
        n = self._n
        out = (ctypes.c_int * max(1, n))()
        _check(lib().skgemm_plan_precisions(self._h, out, n))
        return list(out)[:n]

    def close(self) -> None:
        if self._h and self._h.value:
            lib().skgemm_plan_destroy(self._h)
            self._h = ctypes.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def debug_fill() -> bool:
    """True when the library runs in debug fill mode (SKGEMM_DEBUG_FILL=1)."""
    return bool(lib().skgemm_debug_fill())


def tune_cache_save(path) -> int:
    """Write this process's tuned plan choices to `path` (JSON); returns the
    entry count."""
    n = lib().skgemm_tune_cache_save(os.fsencode(path))
    return _check(n) if n < 0 else n


def tune_cache_load(path) -> int:
    """Load tuned plan choices from `path`; returns the entry count."""
    n = lib().skgemm_tune_cache_load(os.fsencode(path))
    return _check(n) if n < 0 else n


def tune_cache_clear() -> None:
    _check(lib().skgemm_tune_cache_clear())


def batch_dev(items, stream=None) -> None:
    """One-shot grouped launch (cost-model configuration, no graph)."""
    _check(lib().skgemm_batch_dev(_item_array(items), len(items), _stream(stream)))


def batch_schedule(items, tile=128, order=1):
    """Host-only grouped schedule: (perm, iter_begin, useful/issued MAC ratio)."""
    n = len(items)
    perm = (ctypes.c_int * max(1, n))()
    ib = (ctypes.c_int64 * (n + 1))()
    eff = ctypes.c_double(0.0)
    _check(lib().skgemm_batch_schedule(_item_array(items), n, tile, order, perm, ib,
                                       ctypes.byref(eff)))
    return list(perm)[:n], list(ib), eff.value


# ------------------------------------------------------------------ serving
def serve_trace(n, rate=200.0, ng_range=(1e4, 4e5), nb_range=(32, 2048), seed=0):
    """Poisson arrivals (rate per second) of subspace requests with Ng and nb
    log-uniform in the given ranges, rounded to multiples of 16 (the packed
    layouts' granule); returns a list of (arrival_s, Ng, nb, seed)."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=n))
    ng = np.exp(rng.uniform(np.log(ng_range[0]), np.log(ng_range[1]), size=n))
    nb = np.exp(rng.uniform(np.log(nb_range[0]), np.log(nb_range[1]), size=n))
    ng = np.maximum(16, np.round(ng / 16) * 16).astype(np.int64)
    nb = np.maximum(16, np.round(nb / 16) * 16).astype(np.int64)
    return [(float(t[i]), int(ng[i]), int(nb[i]), int(seed * 1000003 + i)) for i in range(n)]


SERVE_FIFO = 0
SERVE_SMALLEST = 1  # least work first among waiting requests, aged
SERVE_RATIO = 2  # highest response ratio next (largest wait / work)


def serve(trace, precision=PREC_NATIVE, slices=0, hbm_budget=150e9, max_inflight=0,
          ozaki_streams=0, max_batch_tflop=0.0, realtime=True, simulate=False, keep=None,
          sim=(0.0, 0.0, 0.0), policy=SERVE_FIFO, aging_s=0.0):
    """Runs (or simulates) a request trace; returns (per-request rows, options).

    ``keep``: optional dict index -> dict of host numpy buffers to fill
    (keys S, Hs, Psi, Psi_in, HPsi_in, Q)."""
    n = len(trace)
    reqs = (ServeRequest * max(1, n))()
    hold = []
    for i, (t, ng, nb, sd) in enumerate(trace):
        r = reqs[i]
        r.Ng, r.nb, r.arrival_s, r.seed = ng, nb, t, sd
        if keep and i in keep:
            k = keep[i]
            for key, field in (("S", "S_out"), ("Hs", "Hs_out"), ("Psi", "Psi_out"),
                               ("Psi_in", "Psi_in_out"), ("HPsi_in", "HPsi_in_out"),
                               ("Q", "Q_in_out")):
                if key in k:
                    setattr(r, field, _hptr(k[key], True))
                    hold.append(k[key])
    o = ServeOptions()
    o.precision, o.slices, o.hbm_budget_bytes = precision, slices, hbm_budget
    o.max_inflight, o.ozaki_streams, o.max_batch_tflop = max_inflight, ozaki_streams, max_batch_tflop
    o.realtime = 1 if realtime else 0
    o.policy, o.aging_s = policy, aging_s
    o.sim_native_tflops, o.sim_ozaki_tflops, o.sim_gen_gbs = sim
    f = lib().skgemm_serve_simulate if simulate else lib().skgemm_serve_run
    _check(f(reqs, n, ctypes.byref(o)))
    rows = [(trace[i][0] if realtime else 0.0, reqs[i].admit_s, reqs[i].done_s) for i in range(n)]
    return rows, o


def stream_release(stream=None) -> None:
    _check(lib().skgemm_stream_release(_stream(stream)))
