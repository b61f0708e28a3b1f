"""Python bindings of libtca_spmm.so (the B200 TCA-SpMM library).

The library is called through its C ABI (include/tca_spmm.h) with ctypes;
torch is used only to own device memory and streams. Nothing here computes
on the CPU: when the shared library is missing the import of any compute
function raises, so a missing build can never be masked by a fallback.

Reference counterparts (paths within the reference project):
  spmm / Plan.spmm     kernel_our_spmm_balanced   src/our_spmm.cu:290-346
  Plan                 workload_manager           src/our_spmm.cu:347-471
  spmm_host            our_spmm_balanced          src/our_spmm.cu:472-588
"""
from __future__ import annotations

import ctypes
import os
import pathlib

import numpy as np

_PKG_ROOT = pathlib.Path(__file__).resolve().parents[2]
LIB_PATH = pathlib.Path(os.environ.get("TCA_SPMM_LIB", _PKG_ROOT / "lib" / "libtca_spmm.so"))

DTYPE_F16, DTYPE_F32, DTYPE_E4M3 = 0, 1, 2
FLAG_KEEP_EMPTY_ROWS = 1

# tca_plan_array_t
ARR_ROW_PERM, ARR_P_ROW_PTR, ARR_P_COL, ARR_P_VAL, ARR_SRC = 0, 1, 2, 3, 4
ARR_TC_WINDOWS, ARR_CC_WINDOWS, ARR_TILE_FIRST, ARR_WIN_COLS = 5, 6, 7, 8
ARR_TILE_PTR, ARR_TILE_ENTRIES, ARR_TILE_SRC = 9, 10, 11
ARR_TILE_IMAGE_IDX, ARR_TILE_IMAGES = 12, 13
ARR_CC_ITEMS, ARR_ALL_ITEMS = 14, 15
ARR_ROW_SCALE, ARR_P_VAL_F8, ARR_TILE_ENTRIES_F8, ARR_TILE_IMAGES_F8 = 16, 17, 18, 19
ARR_TC_PAIRS = 20
_ARR_DTYPE = {ARR_P_VAL: np.uint16, ARR_TILE_ENTRIES: np.uint32, ARR_TILE_IMAGES: np.uint16,
              ARR_ROW_SCALE: np.float32, ARR_P_VAL_F8: np.uint8, ARR_TILE_ENTRIES_F8: np.uint32,
              ARR_TILE_IMAGES_F8: np.uint8}

STATUS = {
    0: "TCA_OK", 1: "TCA_ERR_INVALID_ARG", 2: "TCA_ERR_CUDA", 3: "TCA_ERR_ALLOC",
    4: "TCA_ERR_UNSUPPORTED", 5: "TCA_ERR_TIMEOUT", 6: "TCA_ERR_FORMAT", 7: "TCA_ERR_IO",
}


class TcaError(RuntimeError):
    """A libtca_spmm entry point returned a non-zero tca_status_t."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


class PlanOpts(ctypes.Structure):
    _fields_ = [("sort_rows", ctypes.c_int), ("tc_min_density", ctypes.c_float),
                ("path", ctypes.c_int), ("pair_windows", ctypes.c_int), ("reserved", ctypes.c_int * 4)]


class PlanInfo(ctypes.Structure):
    _fields_ = [("M", ctypes.c_int), ("K", ctypes.c_int), ("nnz", ctypes.c_int),
                ("n_windows", ctypes.c_int), ("n_tc_windows", ctypes.c_int),
                ("n_cc_windows", ctypes.c_int), ("n_tc_chunks", ctypes.c_int),
                ("n_images", ctypes.c_int), ("tc_nnz", ctypes.c_longlong),
                ("format_bytes", ctypes.c_longlong)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class BatchItem(ctypes.Structure):
    _fields_ = [("plan", ctypes.c_void_p), ("d_B_f16", ctypes.c_void_p), ("ldb", ctypes.c_int),
                ("N", ctypes.c_int), ("d_C", ctypes.c_void_p), ("ldc", ctypes.c_int), ("n_tile", ctypes.c_int),
                ("cc_cols", ctypes.c_int)]


_lib = None

_P, _I, _F, _U, _VP = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_uint, ctypes.c_void_p
_SIGS = {
    "tca_version": ([], ctypes.c_char_p),
    "tca_last_error_string": ([], ctypes.c_char_p),
    "tca_status_string": ([_I], ctypes.c_char_p),
    "tca_spmm_csr": ([_P, _P, _P, _I, _I, _I, _P, _I, _I, _P, _I, _I, _F, _F, _U, _VP], _I),
    "tca_spmm_csr_f64": ([_P, _P, _P, _I, _I, _I, _P, _I, _I, _P, _I, ctypes.c_double, ctypes.c_double, _U,
                          _VP], _I),
    "tca_plan_opts_default": ([ctypes.POINTER(PlanOpts)], None),
    "tca_plan_create": ([_P, _P, _P, _I, _I, _I, ctypes.POINTER(PlanOpts), _VP, ctypes.POINTER(_VP)], _I),
    "tca_plan_update_values": ([_VP, _P, _VP], _I),
    "tca_plan_info": ([_VP, ctypes.POINTER(PlanInfo)], _I),
    "tca_plan_export": ([_VP, _I, _P, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)], _I),
    "tca_plan_status": ([_VP], _I),
    "tca_plan_destroy": ([_VP], _I),
    "tca_spmm": ([_VP, _P, _I, _I, _P, _I, _I, _F, _F, _U, _VP], _I),
    "tca_spmm_events": ([_VP, _P, _I, _I, _P, _I, _I, _F, _F, _U, _VP, ctypes.POINTER(_VP)], _I),
    "tca_plan_launch_counts": ([_VP, _I, ctypes.POINTER(_I), ctypes.POINTER(_I)], _I),
    "tca_spmm_batched": ([ctypes.POINTER(BatchItem), _I, _I, _F, _F, _U, _VP, ctypes.POINTER(_VP)], _I),
    "tca_sddmm": ([_VP, _P, _I, _P, _I, _I, _P, _I, _F, _VP], _I),
    "tca_spmm_t": ([_VP, _P, _I, _I, _P, _I, _I, _F, _F, _VP], _I),
    "tca_plan_build_transpose": ([_VP, _VP], _I),
    "tca_plan_quantize_fp8": ([_VP, _VP], _I),
    "tca_quantize_b_fp8": ([_P, _I, _I, _I, _P, _I, _P, _VP], _I),
    "tca_spmm_fp8": ([_VP, _P, _I, _I, _P, _I, _I, _F, _F, _U, _VP], _I),
    "tca_spmm_fp8_static": ([_VP, _P, _I, _I, _P, _I, _I, _F, _F, _U, _VP], _I),
    "tca_spmm_fp8_batched": ([ctypes.POINTER(BatchItem), _I, _I, _F, _F, _U, _VP, ctypes.POINTER(_VP)], _I),
    "tca_batch_graph_create": ([ctypes.POINTER(BatchItem), _I, _I, _F, _F, _U, _I, ctypes.POINTER(_VP)], _I),
    "tca_batch_graph_create_events": ([ctypes.POINTER(BatchItem), _I, _I, _F, _F, _U, _I, ctypes.POINTER(_VP),
                                       ctypes.POINTER(_VP)], _I),
    "tca_batch_graph_launch": ([_VP, _VP], _I),
    "tca_batch_graph_destroy": ([_VP], _I),
    "tca_batch_autotune": ([ctypes.POINTER(BatchItem), _I, _I, _I, _I, _VP], _I),
    "tca_mtx_parse": ([ctypes.c_char_p, ctypes.c_size_t, _I, _I, _F, ctypes.POINTER(_I), ctypes.POINTER(_I),
                       ctypes.POINTER(_I), ctypes.POINTER(_VP), ctypes.POINTER(_VP), ctypes.POINTER(_VP)], _I),
    "tca_mtx_read": ([ctypes.c_char_p, _I, _I, _F, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_I),
                      ctypes.POINTER(_VP), ctypes.POINTER(_VP), ctypes.POINTER(_VP)], _I),
    "tca_free": ([_VP], None),
    "tca_spmm_host": ([_P, _P, _P, _I, _I, _I, _P, _I, _P, _I, _U, _I, ctypes.POINTER(ctypes.c_double)], _I),
    "tca_pool_stats": ([_I, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t),
                        ctypes.POINTER(ctypes.c_size_t)], _I),
}


def exported_symbols() -> list[str]:
    """Names of the C-ABI entry points this module binds."""
    return list(_SIGS)


def lib() -> ctypes.CDLL:
    """Loads libtca_spmm.so once; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C tca-spmm_b200` "
                               "(or __graft_entry__.build()); there is no CPU fallback")
        handle = ctypes.CDLL(str(LIB_PATH))
        for name, (args, res) in _SIGS.items():
            fn = getattr(handle, name)
            fn.argtypes = args
            fn.restype = res
        _lib = handle
    return _lib


def pool_stats(reset_high: bool = False) -> dict:
    """The library's device memory pool on the current device (tca_pool_stats):
    bytes reserved, in use, and the highest use since the last reset."""
    r, u, h = ctypes.c_size_t(), ctypes.c_size_t(), ctypes.c_size_t()
    _check(lib().tca_pool_stats(1 if reset_high else 0, ctypes.byref(r), ctypes.byref(u), ctypes.byref(h)))
    return {"reserved": r.value, "used": u.value, "used_high": h.value}


def _check(rc: int) -> None:
    if rc != 0:
        raise TcaError(rc, lib().tca_last_error_string().decode())


def version() -> str:
    return lib().tca_version().decode()


def _torch():
    import torch
    return torch


def _stream_handle(stream=None) -> int:
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def _ptr(t) -> int:
    return t.data_ptr() if t is not None and t.numel() > 0 else 0


def _out_code(dtype) -> int:
    torch = _torch()
    if dtype == torch.float16:
        return DTYPE_F16
    if dtype == torch.float32:
        return DTYPE_F32
    raise ValueError(f"output dtype {dtype} is not float16 or float32")


def _check_dev(name, t, dtype):
    torch = _torch()
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    if t.dtype != dtype:
        raise ValueError(f"{name} must be {dtype}, got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    del torch


def _prepare_dense(B, out, M, out_dtype):
    torch = _torch()
    if B.dim() != 2 or B.dtype != torch.float16 or not B.is_cuda or B.stride(1) != 1:
        raise ValueError("B must be a 2-D CUDA float16 tensor with unit column stride")
    N = B.shape[1]
    if out is None:
        out = torch.empty((M, N), dtype=out_dtype, device=B.device)
    if out.dim() != 2 or out.shape[0] != M or out.shape[1] != N or out.stride(1) != 1 or not out.is_cuda:
        raise ValueError("out must be a CUDA M x N tensor with unit column stride")
    return N, out


def spmm_csr(row_ptr, col_idx, vals, B, K=None, out=None, out_dtype=None, alpha=1.0, beta=0.0,
             keep_empty_rows=False, stream=None):
    """Plan-free CUDA-core forward: out = alpha * A @ B + beta * out (tca_spmm_csr)."""
    torch = _torch()
    _check_dev("row_ptr", row_ptr, torch.int32)
    _check_dev("col_idx", col_idx, torch.int32)
    _check_dev("vals", vals, torch.float16)
    M = row_ptr.numel() - 1
    K = B.shape[0] if K is None else K
    out_dtype = out_dtype or (out.dtype if out is not None else torch.float16)
    N, out = _prepare_dense(B, out, M, out_dtype)
    flags = FLAG_KEEP_EMPTY_ROWS if keep_empty_rows else 0
    _check(lib().tca_spmm_csr(_ptr(row_ptr), _ptr(col_idx), _ptr(vals), M, K, vals.numel(),
                              _ptr(B), B.stride(0), N, _ptr(out), out.stride(0), _out_code(out.dtype),
                              alpha, beta, flags, _stream_handle(stream)))
    return out


PATHS = {"auto": 0, "cuda_core": 1, "tensor_core": 2}


class Plan:
    """The row-window, column-condensed tile format of one sparsity pattern,
    built on the GPU by tca_plan_create (replaces workload_manager,
    src/our_spmm.cu:347-471)."""

    def __init__(self, row_ptr, col_idx, vals, K, sort_rows=True, tc_min_density=None,
                 path="auto", pair_windows=False, stream=None):
        torch = _torch()
        _check_dev("row_ptr", row_ptr, torch.int32)
        _check_dev("col_idx", col_idx, torch.int32)
        _check_dev("vals", vals, torch.float16)
        self._lib = lib()
        opts = PlanOpts()
        self._lib.tca_plan_opts_default(ctypes.byref(opts))
        opts.sort_rows = 1 if sort_rows else 0
        if tc_min_density is not None:
            opts.tc_min_density = float(tc_min_density)
        opts.path = PATHS[path]
        opts.pair_windows = 1 if pair_windows else 0
        self.M = row_ptr.numel() - 1
        self.K = int(K)
        self.nnz = col_idx.numel()
        h = _VP()
        _check(self._lib.tca_plan_create(_ptr(row_ptr), _ptr(col_idx), _ptr(vals), self.M, self.K,
                                         self.nnz, ctypes.byref(opts), _stream_handle(stream),
                                         ctypes.byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    def info(self) -> dict:
        inf = PlanInfo()
        _check(self._lib.tca_plan_info(self._h, ctypes.byref(inf)))
        return inf.as_dict()

    def export(self, which: int) -> np.ndarray:
        n = ctypes.c_size_t()
        _check(self._lib.tca_plan_export(self._h, which, None, 0, ctypes.byref(n)))
        dt = _ARR_DTYPE.get(which, np.int32)
        arr = np.empty(n.value // np.dtype(dt).itemsize, dtype=dt)
        if n.value:
            _check(self._lib.tca_plan_export(self._h, which, arr.ctypes.data, n.value, ctypes.byref(n)))
        return arr

    def update_values(self, vals, stream=None):
        _check(self._lib.tca_plan_update_values(self._h, _ptr(vals), _stream_handle(stream)))

    def status(self):
        _check(self._lib.tca_plan_status(self._h))

    def spmm(self, B, out=None, out_dtype=None, alpha=1.0, beta=0.0, keep_empty_rows=False, stream=None):
        """out = alpha * A @ B + beta * out through the plan (tca_spmm)."""
        torch = _torch()
        out_dtype = out_dtype or (out.dtype if out is not None else torch.float16)
        N, out = _prepare_dense(B, out, self.M, out_dtype)
        flags = FLAG_KEEP_EMPTY_ROWS if keep_empty_rows else 0
        _check(self._lib.tca_spmm(self._h, _ptr(B), B.stride(0), N, _ptr(out), out.stride(0),
                                  _out_code(out.dtype), alpha, beta, flags, _stream_handle(stream)))
        return out

    def spmm_events(self, B, out, events, alpha=1.0, beta=0.0, keep_empty_rows=False, stream=None):
        """Plan.spmm recording 4 torch.cuda.Event objects (or None) around the
        tensor-core and CUDA-core kernels (tca_spmm_events)."""
        N, out = _prepare_dense(B, out, self.M, out.dtype)
        arr = (_VP * 4)(*[(e.cuda_event if e is not None else None) for e in events])
        flags = FLAG_KEEP_EMPTY_ROWS if keep_empty_rows else 0
        _check(self._lib.tca_spmm_events(self._h, _ptr(B), B.stride(0), N, _ptr(out), out.stride(0),
                                         _out_code(out.dtype), alpha, beta, flags, _stream_handle(stream), arr))
        return out

    def sddmm(self, dY, B, out=None, out_dtype=None, alpha=1.0, stream=None):
        """dA on the plan's pattern: out[j] = alpha * dot(dY[row_j], B[col_j]) in
        the caller's nonzero order (tca_sddmm)."""
        torch = _torch()
        if dY.dim() != 2 or dY.dtype != torch.float16 or dY.stride(1) != 1 or dY.shape[0] != self.M:
            raise ValueError("dY must be an M x N float16 tensor with unit column stride")
        if B.dim() != 2 or B.dtype != torch.float16 or B.stride(1) != 1 or B.shape[1] != dY.shape[1]:
            raise ValueError("B must be a K x N float16 tensor with unit column stride")
        out_dtype = out_dtype or (out.dtype if out is not None else torch.float32)
        if out is None:
            out = torch.empty(self.nnz, dtype=out_dtype, device=dY.device)
        _check(self._lib.tca_sddmm(self._h, _ptr(dY), dY.stride(0), _ptr(B), B.stride(0), dY.shape[1], _ptr(out),
                                   _out_code(out.dtype), alpha, _stream_handle(stream)))
        return out

    def spmm_t(self, dY, out=None, out_dtype=None, alpha=1.0, beta=0.0, stream=None):
        """dB = alpha * A^T dY + beta * out (tca_spmm_t)."""
        torch = _torch()
        if dY.dim() != 2 or dY.dtype != torch.float16 or dY.stride(1) != 1 or dY.shape[0] != self.M:
            raise ValueError("dY must be an M x N float16 tensor with unit column stride")
        out_dtype = out_dtype or (out.dtype if out is not None else torch.float32)
        N = dY.shape[1]
        if out is None:
            out = torch.empty((self.K, N), dtype=out_dtype, device=dY.device)
        _check(self._lib.tca_spmm_t(self._h, _ptr(dY), dY.stride(0), N, _ptr(out), out.stride(0),
                                    _out_code(out.dtype), alpha, beta, _stream_handle(stream)))
        return out

    def quantize_fp8(self, stream=None):
        """Builds / refreshes the plan's E4M3 form of A (tca_plan_quantize_fp8)."""
        _check(self._lib.tca_plan_quantize_fp8(self._h, _stream_handle(stream)))

    def spmm_fp8(self, B, out=None, out_dtype=None, alpha=1.0, beta=0.0, keep_empty_rows=False, stream=None):
        """E4M3 forward: A per-row and B per-column quantized, FP32 accumulation
        (tca_spmm_fp8). B is float16; it is quantized per call."""
        torch = _torch()
        out_dtype = out_dtype or (out.dtype if out is not None else torch.float16)
        N, out = _prepare_dense(B, out, self.M, out_dtype)
        flags = FLAG_KEEP_EMPTY_ROWS if keep_empty_rows else 0
        _check(self._lib.tca_spmm_fp8(self._h, _ptr(B), B.stride(0), N, _ptr(out), out.stride(0),
                                      _out_code(out.dtype), alpha, beta, flags, _stream_handle(stream)))
        return out

    def build_transpose(self, stream=None):
        _check(self._lib.tca_plan_build_transpose(self._h, _stream_handle(stream)))

    def launch_counts(self, N: int) -> tuple[int, int]:
        a, b = _I(), _I()
        _check(self._lib.tca_plan_launch_counts(self._h, N, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def close(self):
        if getattr(self, "_h", None):
            self._lib.tca_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def spmm_batched(plans, Bs, outs, alpha=1.0, beta=0.0, keep_empty_rows=False, n_tile=0, events=None,
                 stream=None, cc_cols=0):
    """Forwards of many plans in a few launches (tca_spmm_batched). `outs`
    must all have the same dtype (float16 or float32). cc_cols picks the
    CUDA-core kernel of every item (CC_COLS_*; 0 = by N)."""
    n = len(plans)
    arr = (BatchItem * max(n, 1))()
    for i, (p, B, C) in enumerate(zip(plans, Bs, outs)):
        N, _ = _prepare_dense(B, C, p.M, C.dtype)
        arr[i] = BatchItem(p.handle, _ptr(B), B.stride(0), N, _ptr(C), C.stride(0), n_tile, cc_cols)
    code = _out_code(outs[0].dtype) if n else DTYPE_F16
    ev = None
    if events is not None:
        ev = (_VP * 4)(*[(e.cuda_event if e is not None else None) for e in events])
    flags = FLAG_KEEP_EMPTY_ROWS if keep_empty_rows else 0
    _check(lib().tca_spmm_batched(arr, n, code, alpha, beta, flags, _stream_handle(stream), ev))
    return outs


def spmm_fp8_batched(plans, Bs, outs, alpha=1.0, beta=0.0, keep_empty_rows=False, n_tile=0, events=None,
                     stream=None):
    """E4M3 forwards of many plans in a few launches (tca_spmm_fp8_batched);
    every plan at most once."""
    n = len(plans)
    arr = (BatchItem * max(n, 1))()
    for i, (p, B, C) in enumerate(zip(plans, Bs, outs)):
        N, _ = _prepare_dense(B, C, p.M, C.dtype)
        arr[i] = BatchItem(p.handle, _ptr(B), B.stride(0), N, _ptr(C), C.stride(0), n_tile)
    code = _out_code(outs[0].dtype) if n else DTYPE_F16
    ev = None
    if events is not None:
        ev = (_VP * 4)(*[(e.cuda_event if e is not None else None) for e in events])
    flags = FLAG_KEEP_EMPTY_ROWS if keep_empty_rows else 0
    _check(lib().tca_spmm_fp8_batched(arr, n, code, alpha, beta, flags, _stream_handle(stream), ev))
    return outs


PRECISION_F16, PRECISION_E4M3 = 0, 1
# cc_cols values: the CUDA-core stream kernel with 2, 4 or 8 output columns
# per lane, or the FP16 tensor-core item kernel (mma.sync)
CC_COLS_2, CC_COLS_4, CC_COLS_8, CC_COLS_MMA = 2, 4, 8, 16
_PRECISIONS = {"f16": PRECISION_F16, "fp16": PRECISION_F16, "e4m3": PRECISION_E4M3, "fp8": PRECISION_E4M3}


def _batch_items(plans, Bs, outs, n_tiles=None, cc_cols=None):
    n = len(plans)
    arr = (BatchItem * max(n, 1))()
    for i, (p, B, C) in enumerate(zip(plans, Bs, outs)):
        N, _ = _prepare_dense(B, C, p.M, C.dtype)
        arr[i] = BatchItem(p.handle, _ptr(B), B.stride(0), N, _ptr(C), C.stride(0),
                           (n_tiles[i] if n_tiles else 0), (cc_cols[i] if cc_cols else 0))
    return arr


def autotune(plans, Bs, outs, precision="f16", reps=5, stream=None):
    """The fastest (n_tile, cc_cols) per item (tca_batch_autotune): every
    candidate timed on the item alone, then those picks timed as one batch
    against each uniform configuration for all items. Overwrites `outs`."""
    arr = _batch_items(plans, Bs, outs)
    code = _out_code(outs[0].dtype) if plans else DTYPE_F16
    _check(lib().tca_batch_autotune(arr, len(plans), code, _PRECISIONS[precision], reps, _stream_handle(stream)))
    return [(arr[i].n_tile, arr[i].cc_cols) for i in range(len(plans))]


class BatchGraph:
    """A batch of forwards (many layers) captured once as a CUDA graph
    (tca_batch_graph_create) and replayed with launch(). Holds references to
    the plans and tensors, whose addresses the graph keeps."""

    def __init__(self, plans, Bs, outs, alpha=1.0, beta=0.0, keep_empty_rows=False, precision="f16",
                 n_tiles=None, cc_cols=None, events=None):
        """events: 4 torch.cuda.Event (or None) recorded inside the graph around
        the tensor-core and the CUDA-core launches of every replay."""
        self._keep = (list(plans), list(Bs), list(outs), events)
        self._lib = lib()
        arr = _batch_items(plans, Bs, outs, n_tiles, cc_cols)
        code = _out_code(outs[0].dtype) if plans else DTYPE_F16
        flags = FLAG_KEEP_EMPTY_ROWS if keep_empty_rows else 0
        h = _VP()
        if events is None:
            _check(self._lib.tca_batch_graph_create(arr, len(plans), code, alpha, beta, flags,
                                                    _PRECISIONS[precision], ctypes.byref(h)))
        else:
            ev = (_VP * 4)(*[(e.cuda_event if e is not None else None) for e in events])
            _check(self._lib.tca_batch_graph_create_events(arr, len(plans), code, alpha, beta, flags,
                                                           _PRECISIONS[precision], ev, ctypes.byref(h)))
        self._h = h

    def launch(self, stream=None):
        _check(self._lib.tca_batch_graph_launch(self._h, _stream_handle(stream)))

    def close(self):
        if getattr(self, "_h", None):
            self._lib.tca_batch_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def quantize_b_fp8(B, stream=None):
    """B (K x N float16, CUDA) -> (Bq uint8 K x ldq, scale float32 N) with
    ldq = N rounded up to 16 (tca_quantize_b_fp8)."""
    torch = _torch()
    if B.dim() != 2 or B.dtype != torch.float16 or B.stride(1) != 1:
        raise ValueError("B must be a K x N float16 tensor with unit column stride")
    K, N = B.shape
    ldq = (N + 15) // 16 * 16
    Bq = torch.zeros((K, ldq), dtype=torch.uint8, device=B.device)
    scale = torch.empty(N, dtype=torch.float32, device=B.device)
    _check(lib().tca_quantize_b_fp8(_ptr(B), B.stride(0), K, N, _ptr(Bq), ldq, _ptr(scale), _stream_handle(stream)))
    return Bq, scale


def mtx_read(path, zero_based=False, pattern_only=False, missing_value=0.0):
    """A MatrixMarket coordinate file as host CSR (tca_mtx_read): (M, K,
    row_ptr int32, col_idx int32, vals float16), rows in order, file order
    within a row, as the reference's mtx_input_to_CSR reads it."""
    L = lib()
    M, K, nnz = _I(), _I(), _I()
    rp, ci, v = _VP(), _VP(), _VP()
    _check(L.tca_mtx_read(str(path).encode(), int(zero_based), int(pattern_only), missing_value, ctypes.byref(M),
                          ctypes.byref(K), ctypes.byref(nnz), ctypes.byref(rp), ctypes.byref(ci), ctypes.byref(v)))

    def take(ptr, n, dt):
        a = np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(np.ctypeslib.as_ctypes_type(dt))),
                                  shape=(max(n, 1),))[:n].copy()
        L.tca_free(ptr)
        return a

    n = nnz.value
    return (M.value, K.value, take(rp, M.value + 1, np.int32), take(ci, n, np.int32),
            take(v, n, np.uint16).view(np.float16))


def spmm_csr_f64(row_ptr, col_idx, vals, B, K=None, out=None, alpha=1.0, beta=0.0, keep_empty_rows=False,
                 stream=None):
    """FP64 forward from CSR on CUDA cores (tca_spmm_csr_f64): float64 values,
    B and output."""
    torch = _torch()
    if B.dim() != 2 or B.dtype != torch.float64 or not B.is_cuda or B.stride(1) != 1:
        raise ValueError("B must be a 2-D CUDA float64 tensor with unit column stride")
    M = row_ptr.numel() - 1
    N = B.shape[1]
    if out is None:
        out = torch.empty((M, N), dtype=torch.float64, device=B.device)
    K = B.shape[0] if K is None else K
    flags = FLAG_KEEP_EMPTY_ROWS if keep_empty_rows else 0
    _check(lib().tca_spmm_csr_f64(_ptr(row_ptr), _ptr(col_idx), _ptr(vals), M, K, col_idx.numel(), _ptr(B),
                                  B.stride(0), N, _ptr(out), out.stride(0), alpha, beta, flags,
                                  _stream_handle(stream)))
    return out


def spmm_host(row_ptr: np.ndarray, col_idx: np.ndarray, vals: np.ndarray, K: int, B: np.ndarray,
              C: np.ndarray | None = None, keep_empty_rows=True, n_iter=1):
    """Host-buffer forward with the reference's convention (tca_spmm_host ->
    our_spmm_balanced semantics): numpy in, numpy out, C float32 or float16.
    Returns (C, mean device ms of one forward)."""
    M = row_ptr.size - 1
    N = B.shape[1]
    if C is None:
        C = np.zeros((M, N), dtype=np.float32)
    code = DTYPE_F32 if C.dtype == np.float32 else DTYPE_F16
    rp = np.ascontiguousarray(row_ptr, dtype=np.int32)
    ci = np.ascontiguousarray(col_idx, dtype=np.int32)
    v = np.ascontiguousarray(vals, dtype=np.float16)
    Bc = np.ascontiguousarray(B, dtype=np.float16)
    ms = ctypes.c_double()
    flags = FLAG_KEEP_EMPTY_ROWS if keep_empty_rows else 0
    _check(lib().tca_spmm_host(rp.ctypes.data, ci.ctypes.data, v.ctypes.data, M, K, ci.size,
                               Bc.ctypes.data, N, C.ctypes.data, code, flags, n_iter, ctypes.byref(ms)))
    return C, ms.value
