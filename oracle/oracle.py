"""TEST INFRASTRUCTURE ONLY: Python access to the oracle.

* liboracle.so (built from tca_oracle.c): the CPU restatement of the
  reference path -- smtx parsing, dense<->CSR, FP64 / FP32 SpMM, compare_mat,
  and the host build of the tile format.
* _ref/libtcaref.so (built from the reference sources by the Makefile, when
  the reference tree was present at build time): the reference's own
  functions, used to make the golden fixtures and, on a GPU, as the
  reference TCA kernel / cuSPARSE / cuBLAS comparators.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline and
reference legs may import this module.
"""
from __future__ import annotations

import ctypes
import os
import pathlib

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
REF_PATH = HERE / "_ref" / "libtcaref.so"

_P, _I = ctypes.c_void_p, ctypes.c_int


class OrcPlan(ctypes.Structure):
    _fields_ = [("M", _I), ("K", _I), ("nnz", _I), ("n_windows", _I), ("n_tc", _I), ("n_cc", _I),
                ("n_tc_chunks", _I), ("tc_nnz", ctypes.c_longlong),
                ("perm", _P), ("p_row_ptr", _P), ("p_col", _P), ("src", _P), ("p_val", _P),
                ("tc_windows", _P), ("cc_windows", _P), ("tile_first", _P), ("win_cols", _P),
                ("tile_ptr", _P), ("tile_src", _P), ("tile_entries", _P),
                ("n_images", _I), ("img_idx", _P), ("images", _P),
                ("n_cc_items", _I), ("n_all_items", _I), ("cc_items", _P), ("all_items", _P),
                ("n_pairs", _I), ("tc_pairs", _P)]


_lib = None
_ref = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} missing: run `make -C oracle`")
        L = ctypes.CDLL(str(LIB_PATH))
        L.orc_h2f.argtypes = [ctypes.c_uint16]; L.orc_h2f.restype = ctypes.c_float
        L.orc_f2h.argtypes = [ctypes.c_float]; L.orc_f2h.restype = ctypes.c_uint16
        L.orc_smtx_parse.argtypes = [ctypes.c_char_p, ctypes.c_long, _P, _P, _P, _P, _P]
        L.orc_smtx_parse.restype = _I
        L.orc_pattern_to_dense.argtypes = [_I, _I, _P, _P, _P]; L.orc_pattern_to_dense.restype = None
        L.orc_dense_to_csr.argtypes = [_P, _I, _I, _P, _P, _P]; L.orc_dense_to_csr.restype = ctypes.c_long
        L.orc_csr_to_dense.argtypes = [_I, _I, _P, _P, _P, _P]; L.orc_csr_to_dense.restype = None
        L.orc_spmm_f64.argtypes = [_I, _I, _P, _P, _P, _P, _I, _P, _I, _I]; L.orc_spmm_f64.restype = None
        L.orc_spmm_f32.argtypes = [_I, _I, _P, _P, _P, _P, _I, _P, _I, _I, _I]; L.orc_spmm_f32.restype = None
        L.orc_gemm_f32.argtypes = [_I, _I, _I, _P, _P, _P]; L.orc_gemm_f32.restype = None
        L.orc_compare_mat.argtypes = [_P, _P, ctypes.c_long, ctypes.c_float]; L.orc_compare_mat.restype = ctypes.c_long
        L.orc_ref_warp_demand.argtypes = [_I, _P, _I, _I, _P]; L.orc_ref_warp_demand.restype = None
        L.orc_plan_build.argtypes = [_P, _P, _P, _I, _I, _I, _I, ctypes.c_float, _I, ctypes.POINTER(OrcPlan)]
        L.orc_plan_build.restype = _I
        L.orc_plan_free.argtypes = [ctypes.POINTER(OrcPlan)]; L.orc_plan_free.restype = None
        L.orc_mtx_parse.argtypes = [ctypes.c_char_p, ctypes.c_long, _I, _I, ctypes.c_float, _P, _P,
                                    ctypes.POINTER(ctypes.POINTER(_I)), ctypes.POINTER(ctypes.POINTER(_I)),
                                    ctypes.POINTER(ctypes.POINTER(ctypes.c_uint16))]
        L.orc_mtx_parse.restype = ctypes.c_long
        L.orc_f32_to_e4m3.argtypes = [ctypes.c_float]; L.orc_f32_to_e4m3.restype = ctypes.c_uint8
        L.orc_e4m3_to_f32.argtypes = [ctypes.c_uint8]; L.orc_e4m3_to_f32.restype = ctypes.c_float
        L.orc_quant_rows.argtypes = [_I, _P, _P, _P, _P]; L.orc_quant_rows.restype = None
        L.orc_quant_cols.argtypes = [_I, _I, _P, _I, _P, _I, _P]; L.orc_quant_cols.restype = None
        _lib = L
    return _lib


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def f16_bits(a) -> np.ndarray:
    return _c(a, np.float16).view(np.uint16)


# ---------------------------------------------------------------- parsing
def smtx_parse(text: bytes):
    """Returns (M, K, nnz, row_ptr, col_idx) or raises ValueError."""
    L = lib()
    M, K, nnz = _I(), _I(), _I()
    if L.orc_smtx_parse(text, len(text), ctypes.byref(M), ctypes.byref(K), ctypes.byref(nnz), None, None):
        raise ValueError("malformed smtx header")
    rp = np.zeros(M.value + 1, np.int32)
    ci = np.zeros(max(nnz.value, 1), np.int32)
    if L.orc_smtx_parse(text, len(text), ctypes.byref(M), ctypes.byref(K), ctypes.byref(nnz),
                        rp.ctypes.data, ci.ctypes.data):
        raise ValueError("malformed smtx body")
    return M.value, K.value, nnz.value, rp, ci[: nnz.value]


def pattern_to_dense(M, K, row_ptr, col_idx) -> np.ndarray:
    out = np.empty((M, K), np.uint16)
    rp, ci = _c(row_ptr, np.int32), _c(col_idx, np.int32)
    lib().orc_pattern_to_dense(M, K, rp.ctypes.data, ci.ctypes.data, out.ctypes.data)
    return out.view(np.float16)


def dense_to_csr(A):
    Ab = f16_bits(A)
    M, K = Ab.shape
    L = lib()
    nnz = L.orc_dense_to_csr(Ab.ctypes.data, M, K, None, None, None)
    rp = np.zeros(M + 1, np.int32)
    ci = np.zeros(max(nnz, 1), np.int32)
    v = np.zeros(max(nnz, 1), np.uint16)
    L.orc_dense_to_csr(Ab.ctypes.data, M, K, rp.ctypes.data, ci.ctypes.data, v.ctypes.data)
    return rp, ci[:nnz], v[:nnz].view(np.float16)


def csr_to_dense(M, K, row_ptr, col_idx, vals) -> np.ndarray:
    out = np.empty((M, K), np.uint16)
    rp, ci, vb = _c(row_ptr, np.int32), _c(col_idx, np.int32), f16_bits(vals)
    lib().orc_csr_to_dense(M, K, rp.ctypes.data, ci.ctypes.data, vb.ctypes.data, out.ctypes.data)
    return out.view(np.float16)


# ---------------------------------------------------------------- SpMM
def spmm_f64(row_ptr, col_idx, vals, B, C=None, keep_empty=False) -> np.ndarray:
    """FP64 CSR x dense (the error reference)."""
    M = row_ptr.size - 1
    Bb = f16_bits(B)
    N = Bb.shape[1]
    out = np.zeros((M, N), np.float64) if C is None else _c(C, np.float64).copy()
    rp, ci, vb = _c(row_ptr, np.int32), _c(col_idx, np.int32), f16_bits(vals)
    lib().orc_spmm_f64(M, N, rp.ctypes.data, ci.ctypes.data, vb.ctypes.data, Bb.ctypes.data, N,
                       out.ctypes.data, N, 1 if keep_empty else 0)
    return out


def spmm_f32(row_ptr, col_idx, vals, B, C=None, keep_empty=False, nthreads=0) -> np.ndarray:
    """FP32 accumulation in CSR order (bit-identical to the reference naive_gemm
    for sorted columns); OpenMP over rows, nthreads <= 0 uses all cores."""
    M = row_ptr.size - 1
    Bb = f16_bits(B)
    N = Bb.shape[1]
    out = np.zeros((M, N), np.float32) if C is None else _c(C, np.float32).copy()
    rp, ci, vb = _c(row_ptr, np.int32), _c(col_idx, np.int32), f16_bits(vals)
    lib().orc_spmm_f32(M, N, rp.ctypes.data, ci.ctypes.data, vb.ctypes.data, Bb.ctypes.data, N,
                       out.ctypes.data, N, 1 if keep_empty else 0, nthreads)
    return out


def gemm_f32(A, B) -> np.ndarray:
    Ab, Bb = f16_bits(A), f16_bits(B)
    M, K = Ab.shape
    N = Bb.shape[1]
    out = np.empty((M, N), np.float32)
    lib().orc_gemm_f32(M, N, K, Ab.ctypes.data, Bb.ctypes.data, out.ctypes.data)
    return out


def compare_mat(gold, x, tol=1e-3) -> int:
    """Number of elements compare_mat (src/general.cuh:71-123) would flag."""
    g, y = _c(gold, np.float32).ravel(), _c(x, np.float32).ravel()
    return int(lib().orc_compare_mat(g.ctypes.data, y.ctypes.data, g.size, tol))


def ref_warp_demand(row_ptr, N, warps_per_tb=8) -> np.ndarray:
    rp = _c(row_ptr, np.int32)
    out = np.empty(rp.size - 1, np.int32)
    lib().orc_ref_warp_demand(rp.size - 1, rp.ctypes.data, N, warps_per_tb, out.ctypes.data)
    return out


# ---------------------------------------------------------------- tile format
def build_plan(row_ptr, col_idx, vals, K, sort_rows=True, tc_min_density=0.01, path=0) -> dict:
    """Host build of the tile format; same arrays as tca_plan_export."""
    L = lib()
    rp, ci, vb = _c(row_ptr, np.int32), _c(col_idx, np.int32), f16_bits(vals)
    M = rp.size - 1
    p = OrcPlan()
    rc = L.orc_plan_build(rp.ctypes.data, ci.ctypes.data, vb.ctypes.data, M, K, ci.size,
                          1 if sort_rows else 0, tc_min_density, path, ctypes.byref(p))
    if rc != 0:
        raise ValueError("malformed CSR")

    def arr(ptr, n, dt):
        if n <= 0 or not ptr:
            return np.zeros(0, dt)
        return np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(np.ctypeslib.as_ctypes_type(dt))),
                                     shape=(n,)).copy()

    out = dict(
        n_windows=p.n_windows, n_tc=p.n_tc, n_cc=p.n_cc, n_tc_chunks=p.n_tc_chunks, tc_nnz=p.tc_nnz,
        perm=arr(p.perm, M, np.int32), p_row_ptr=arr(p.p_row_ptr, M + 1 if M > 0 else 0, np.int32),
        p_col=arr(p.p_col, p.nnz, np.int32), p_val=arr(p.p_val, p.nnz, np.uint16),
        src=arr(p.src, p.nnz, np.int32), tc_windows=arr(p.tc_windows, p.n_tc, np.int32),
        cc_windows=arr(p.cc_windows, p.n_cc, np.int32),
        tile_first=arr(p.tile_first, p.n_tc + 1 if M > 0 else 0, np.int32),
        win_cols=arr(p.win_cols, p.n_tc_chunks * 64, np.int32),
        tile_ptr=arr(p.tile_ptr, p.n_tc_chunks + 1 if M > 0 else 0, np.int32),
        tile_entries=arr(p.tile_entries, p.tc_nnz, np.uint32),
        tile_src=arr(p.tile_src, p.tc_nnz, np.int32),
        n_images=p.n_images, tile_image_idx=arr(p.img_idx, p.n_tc_chunks, np.int32),
        tile_images=arr(p.images, p.n_images * 8192, np.uint16),
        cc_items=arr(p.cc_items, 2 * p.n_cc_items, np.int32),
        all_items=arr(p.all_items, 2 * p.n_all_items, np.int32),
        tc_pairs=arr(p.tc_pairs, 2 * p.n_pairs, np.int32),
    )
    L.orc_plan_free(ctypes.byref(p))
    return out


# ---------------------------------------------------------------- reference library
def mtx_parse(text: bytes, zero_based=True, pattern_only=False, missing=0.0):
    """(M, K, row_ptr, col, vals fp16) of MatrixMarket text (orc_mtx_parse), or None if malformed."""
    L = lib()
    M, K = ctypes.c_int(), ctypes.c_int()
    rp, ci = ctypes.POINTER(ctypes.c_int)(), ctypes.POINTER(ctypes.c_int)()
    va = ctypes.POINTER(ctypes.c_uint16)()
    n = L.orc_mtx_parse(text, len(text), int(zero_based), int(pattern_only), missing, ctypes.byref(M),
                        ctypes.byref(K), ctypes.byref(rp), ctypes.byref(ci), ctypes.byref(va))
    if n < 0:
        return None
    libc = ctypes.CDLL(None)
    out = (M.value, K.value, np.ctypeslib.as_array(rp, (M.value + 1,)).copy(),
           np.ctypeslib.as_array(ci, (max(n, 1),))[:n].copy(),
           np.ctypeslib.as_array(va, (max(n, 1),))[:n].copy().view(np.float16))
    for ptr in (rp, ci, va):
        libc.free(ptr)
    return out


def e4m3_table() -> np.ndarray:
    """The FP32 value of every E4M3 code (orc_e4m3_to_f32); NaN codes are NaN."""
    L = lib()
    return np.array([L.orc_e4m3_to_f32(q) for q in range(256)], dtype=np.float32)


def f32_to_e4m3(x) -> np.ndarray:
    """Elementwise E4M3 encoding, round to nearest even, saturating (orc_f32_to_e4m3)."""
    L = lib()
    x = np.asarray(x, dtype=np.float32)
    return np.array([L.orc_f32_to_e4m3(float(v)) for v in x.ravel()], dtype=np.uint8).reshape(x.shape)


def quant_rows(row_ptr, vals):
    """(scale[M] float32, q[nnz] uint8): per-row E4M3 quantization of CSR values (orc_quant_rows)."""
    rp = _c(row_ptr, np.int32)
    v = f16_bits(vals)
    M = rp.size - 1
    scale = np.empty(M, np.float32)
    q = np.empty(v.size, np.uint8)
    lib().orc_quant_rows(M, rp.ctypes.data, v.ctypes.data, scale.ctypes.data, q.ctypes.data)
    return scale, q


def quant_cols(B, ldq=None):
    """(q[K, ldq] uint8, scale[N] float32): per-column E4M3 quantization of B (orc_quant_cols)."""
    b = f16_bits(B)
    K, N = b.shape
    ldq = ldq or N
    q = np.zeros((K, ldq), np.uint8)
    scale = np.empty(N, np.float32)
    lib().orc_quant_cols(K, N, b.ctypes.data, N, q.ctypes.data, ldq, scale.ctypes.data)
    return q, scale


def spmm_fp8_f64(row_ptr, col_idx, vals, B):
    """FP64 product of the dequantized operands: (s_a[r] q_a) (s_b[n] q_b) summed in FP64 --
    what the E4M3 forward computes, up to FP32 accumulation."""
    tab = e4m3_table().astype(np.float64)
    sa, qa = quant_rows(row_ptr, vals)
    qb, sb = quant_cols(B)
    import scipy.sparse as sp
    rp = np.asarray(row_ptr)
    M = rp.size - 1
    rows = np.repeat(np.arange(M), np.diff(rp))
    a = tab[qa] * sa.astype(np.float64)[rows]
    b = tab[qb] * sb.astype(np.float64)[None, :]
    A = sp.csr_matrix((a, np.asarray(col_idx), rp), shape=(M, b.shape[0]))
    return np.asarray(A @ b)


def ref_available() -> bool:
    return REF_PATH.exists()


def ref() -> ctypes.CDLL:
    """The reference's own functions (oracle/_ref/libtcaref.so)."""
    global _ref
    if _ref is None:
        if not REF_PATH.exists():
            raise RuntimeError(f"{REF_PATH} missing: run `make -C oracle ref` where the reference tree exists")
        R = ctypes.CDLL(str(REF_PATH))
        D = ctypes.POINTER(ctypes.c_double)
        R.ref_free.argtypes = [_P]; R.ref_free.restype = None
        R.ref_smtx_to_dense.argtypes = [ctypes.c_char_p, _P, _P, _P, ctypes.POINTER(ctypes.POINTER(ctypes.c_uint16))]
        R.ref_smtx_to_dense.restype = _I
        R.ref_dense_to_csr.argtypes = [_P, _I, _I, _P, ctypes.POINTER(ctypes.POINTER(_I)),
                                       ctypes.POINTER(ctypes.POINTER(_I)), ctypes.POINTER(ctypes.POINTER(ctypes.c_uint16))]
        R.ref_dense_to_csr.restype = _I
        R.ref_csr_to_dense.argtypes = [_I, _I, _I, _P, _P, _P, ctypes.POINTER(ctypes.POINTER(ctypes.c_uint16))]
        R.ref_csr_to_dense.restype = _I
        R.ref_mtx_to_csr.argtypes = [ctypes.c_char_p, _I, _I, _P, _P, _P, ctypes.POINTER(ctypes.POINTER(_I)),
                                     ctypes.POINTER(ctypes.POINTER(_I)), ctypes.POINTER(ctypes.POINTER(ctypes.c_uint16))]
        R.ref_mtx_to_csr.restype = ctypes.c_int
        R.ref_mtx_to_dense.argtypes = [ctypes.c_char_p, _I, _P, _P, ctypes.POINTER(ctypes.POINTER(ctypes.c_uint16))]
        R.ref_mtx_to_dense.restype = ctypes.c_int
        R.ref_naive_gemm.argtypes = [_P, _P, _P, _I, _I, _I]; R.ref_naive_gemm.restype = None
        R.ref_our_spmm_balanced.argtypes = [_I, _I, _I, _I, _P, _P, _P, _P, _P, _I, D]
        R.ref_our_spmm_balanced.restype = None
        R.ref_cusparse_spmm.argtypes = [_P, _P, _P, _I, _I, _I, _I, D]; R.ref_cusparse_spmm.restype = None
        R.ref_cusparse_blockspmm.argtypes = [_P, _P, _P, _I, _I, _I, _I, _I, D]
        R.ref_cusparse_blockspmm.restype = None
        R.ref_gemmex.argtypes = [_P, _P, _P, _I, _I, _I, _I, D]; R.ref_gemmex.restype = None
        R.ref_cusparselt_24.argtypes = [_P, _P, _P, _I, _I, _I, _I, D]; R.ref_cusparselt_24.restype = None
        R.ref_tca_schedule.argtypes = [_I, _I, _I, _I, _P]; R.ref_tca_schedule.restype = _P
        R.ref_tca_launch.argtypes = [_P, _P, _P, _P, _P, _P, _P]; R.ref_tca_launch.restype = _I
        R.ref_tca_free.argtypes = [_P]; R.ref_tca_free.restype = None
        R.ref_cusparse_setup.argtypes = [_I, _I, _I, _I, _P, _P, _P, _P, _P]; R.ref_cusparse_setup.restype = _P
        R.ref_cusparse_run.argtypes = [_P, _P]; R.ref_cusparse_run.restype = _I
        R.ref_cusparse_free.argtypes = [_P]; R.ref_cusparse_free.restype = None
        _ref = R
    return _ref


def _take(ptr, n, dt):
    a = np.ctypeslib.as_array(ptr, shape=(n,)).copy() if n > 0 else np.zeros(0, dt)
    ref().ref_free(ctypes.cast(ptr, ctypes.c_void_p))
    return a.astype(dt, copy=False)


def ref_smtx_to_dense(path: str):
    M, K, nnz = _I(), _I(), _I()
    p = ctypes.POINTER(ctypes.c_uint16)()
    if ref().ref_smtx_to_dense(str(path).encode(), ctypes.byref(M), ctypes.byref(K), ctypes.byref(nnz),
                               ctypes.byref(p)):
        raise OSError(path)
    A = _take(p, M.value * K.value, np.uint16).view(np.float16).reshape(M.value, K.value)
    return A, nnz.value


def ref_dense_to_csr(A):
    Ab = f16_bits(A)
    M, K = Ab.shape
    nnz = _I()
    rp, ci = ctypes.POINTER(_I)(), ctypes.POINTER(_I)()
    v = ctypes.POINTER(ctypes.c_uint16)()
    ref().ref_dense_to_csr(Ab.ctypes.data, M, K, ctypes.byref(nnz), ctypes.byref(rp), ctypes.byref(ci), ctypes.byref(v))
    n = nnz.value
    return _take(rp, M + 1, np.int32), _take(ci, n, np.int32), _take(v, n, np.uint16).view(np.float16)


def ref_mtx_to_csr(path: str, zero_based=True, pattern_only=False):
    """The reference's mtx_input_to_CSR on a file: (M, K, row_ptr, col, vals fp16)."""
    R = ref()
    M, K, nnz = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    rp, ci = ctypes.POINTER(_I)(), ctypes.POINTER(_I)()
    va = ctypes.POINTER(ctypes.c_uint16)()
    rc = R.ref_mtx_to_csr(path.encode(), int(zero_based), int(pattern_only), ctypes.byref(M), ctypes.byref(K),
                          ctypes.byref(nnz), ctypes.byref(rp), ctypes.byref(ci), ctypes.byref(va))
    if rc != 0:
        raise OSError(path)
    n = nnz.value
    return (M.value, K.value, _take(rp, M.value + 1, np.int32), _take(ci, n, np.int32),
            _take(va, n, np.uint16).view(np.float16))


def ref_mtx_to_dense(path: str, zero_based=True):
    """The reference's mtx_input_to_Dense on a file: M x K fp16."""
    R = ref()
    M, K = ctypes.c_int(), ctypes.c_int()
    mat = ctypes.POINTER(ctypes.c_uint16)()
    rc = R.ref_mtx_to_dense(path.encode(), int(zero_based), ctypes.byref(M), ctypes.byref(K), ctypes.byref(mat))
    if rc != 0:
        raise OSError(path)
    return _take(mat, M.value * K.value, np.uint16).view(np.float16).reshape(M.value, K.value)


def ref_csr_to_dense(M, K, row_ptr, col_idx, vals):
    rp, ci, vb = _c(row_ptr, np.int32), _c(col_idx, np.int32), f16_bits(vals)
    p = ctypes.POINTER(ctypes.c_uint16)()
    ref().ref_csr_to_dense(M, K, ci.size, rp.ctypes.data, ci.ctypes.data, vb.ctypes.data, ctypes.byref(p))
    return _take(p, M * K, np.uint16).view(np.float16).reshape(M, K)


def ref_naive_gemm(A, B):
    Ab, Bb = f16_bits(A), f16_bits(B)
    M, K = Ab.shape
    N = Bb.shape[1]
    C = np.empty((M, N), np.float32)
    ref().ref_naive_gemm(Ab.ctypes.data, Bb.ctypes.data, C.ctypes.data, M, N, K)
    return C


def ref_our_spmm_balanced(row_ptr, col_idx, vals, K, B, C=None, n_iter=1):
    """The reference TCA kernel through its own host API (needs a GPU).
    Returns (C float32, ms per iteration as the reference reports it)."""
    rp, ci, vb, Bb = _c(row_ptr, np.int32), _c(col_idx, np.int32), f16_bits(vals), f16_bits(B)
    M = rp.size - 1
    N = Bb.shape[1]
    out = np.zeros((M, N), np.float32) if C is None else _c(C, np.float32).copy()
    ms = ctypes.c_double(-1.0)
    ref().ref_our_spmm_balanced(M, N, K, ci.size, rp.ctypes.data, ci.ctypes.data, vb.ctypes.data,
                                Bb.ctypes.data, out.ctypes.data, n_iter, ctypes.byref(ms))
    return out, ms.value


def ref_cusparse_spmm(A, B, C=None, n_iter=1):
    Ab, Bb = f16_bits(A), f16_bits(B)
    M, K = Ab.shape
    N = Bb.shape[1]
    out = np.zeros((M, N), np.float32) if C is None else _c(C, np.float32).copy()
    ms = ctypes.c_double(-1.0)
    ref().ref_cusparse_spmm(Ab.ctypes.data, Bb.ctypes.data, out.ctypes.data, M, N, K, n_iter, ctypes.byref(ms))
    return out, ms.value


def ref_cusparse_blockspmm(A, B, bs, C=None, n_iter=1):
    """The reference's Blocked-ELL comparator (shapes must be multiples of bs:
    the reference reads its host buffers with the padded strides otherwise)."""
    Ab, Bb = f16_bits(A), f16_bits(B)
    M, K = Ab.shape
    N = Bb.shape[1]
    out = np.zeros((M, N), np.float32) if C is None else _c(C, np.float32).copy()
    ms = ctypes.c_double(-1.0)
    ref().ref_cusparse_blockspmm(Ab.ctypes.data, Bb.ctypes.data, out.ctypes.data, M, N, K, n_iter, bs,
                                 ctypes.byref(ms))
    return out, ms.value


def ref_cusparselt_24(A, B, n_iter=1):
    """The reference's cuSPARSELt 2:4 comparator: (C, ms) for A pruned by
    cuSPARSELt times B."""
    Ab, Bb = f16_bits(A), f16_bits(B)
    M, K = Ab.shape
    N = Bb.shape[1]
    out = np.zeros((M, N), np.float32)
    ms = ctypes.c_double(-1.0)
    ref().ref_cusparselt_24(Ab.ctypes.data, Bb.ctypes.data, out.ctypes.data, M, N, K, n_iter, ctypes.byref(ms))
    return out, ms.value


def prune_24_rows(A):
    """2:4 pruning along the rows of a dense matrix (K a multiple of 4): in
    every group of four consecutive elements of a row the two of largest
    magnitude stay, the other two become zero (cuSPARSELt's STRIP pruning,
    src/spmm_cusparse.cu:83; ties between equal magnitudes are not resolved
    here -- callers use data without them)."""
    A = np.asarray(A)
    M, K = A.shape
    g = A.reshape(M, K // 4, 4)
    order = np.argsort(-np.abs(g.astype(np.float32)), axis=2, kind="stable")
    keep = np.zeros(g.shape, bool)
    np.put_along_axis(keep, order[:, :, :2], True, axis=2)
    return np.where(keep, g, np.zeros_like(g)).reshape(M, K)


def ref_gemmex(A, B, C=None, n_iter=1):
    Ab, Bb = f16_bits(A), f16_bits(B)
    M, K = Ab.shape
    N = Bb.shape[1]
    out = np.zeros((M, N), np.float32) if C is None else _c(C, np.float32).copy()
    ms = ctypes.c_double(-1.0)
    ref().ref_gemmex(Ab.ctypes.data, Bb.ctypes.data, out.ctypes.data, M, N, K, n_iter, ctypes.byref(ms))
    return out, ms.value


class RefTcaKernel:
    """The reference TCA kernel (kernel_our_spmm_balanced<64>) on device
    buffers with the schedule its own host code builds (workload_manager):
    launch() issues one forward on the given CUDA stream, C (FP32) = A B.
    Device pointers are plain integers (e.g. torch's data_ptr())."""

    def __init__(self, M, N, K, row_ptr_host, d_val, d_row_ptr, d_col, d_B, d_C):
        rp = _c(row_ptr_host, np.int32)
        self._R = ref()
        with quiet_stdout():
            self._h = self._R.ref_tca_schedule(M, N, K, int(rp[-1]), rp.ctypes.data)
        self._args = (d_val, d_row_ptr, d_col, d_B, d_C)

    def launch(self, stream):
        rc = self._R.ref_tca_launch(self._h, *self._args, stream)
        if rc != 0:
            raise RuntimeError(f"reference kernel launch failed: CUDA error {rc}")

    def close(self):
        if self._h:
            self._R.ref_tca_free(self._h)
            self._h = None


class RefCusparse:
    """The reference comparator's cusparseSpMM call (CSR 32I, FP16 A/B, FP32
    C and compute, ALG_DEFAULT) on device buffers: launch() issues one
    forward on the given CUDA stream."""

    def __init__(self, M, N, K, nnz, d_row_ptr, d_col, d_val, d_B, d_C):
        self._R = ref()
        self._h = self._R.ref_cusparse_setup(M, N, K, nnz, d_row_ptr, d_col, d_val, d_B, d_C)
        if not self._h:
            raise RuntimeError("cuSPARSE set-up failed")

    def launch(self, stream):
        rc = self._R.ref_cusparse_run(self._h, stream)
        if rc != 0:
            raise RuntimeError(f"cusparseSpMM failed: status {rc}")

    def close(self):
        if self._h:
            self._R.ref_cusparse_free(self._h)
            self._h = None


class quiet_stdout:
    """Silences the C stdout of the reference functions (they print timings)."""

    def __enter__(self):
        import sys
        sys.stdout.flush()
        self._fd = os.dup(1)
        self._null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self._null, 1)
        return self

    def __exit__(self, *exc):
        ctypes.CDLL(None).fflush(None)
        os.dup2(self._fd, 1)
        os.close(self._fd)
        os.close(self._null)
        return False
