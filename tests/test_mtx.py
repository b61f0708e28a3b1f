"""MatrixMarket input (the reference's mtx_input_to_CSR / mtx_input_to_Dense,
src/file_input.cu:8-134) on the CPU: the oracle's restatement, the C ABI
(tca_mtx_parse / tca_mtx_read) and the C++ drop-ins (compiled against
include/tca_spmm_compat.h and run) against the reference's own outputs in
tests/golden/golden.npz, bit for bit; malformed text is a format error."""
import ctypes
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from oracle import oracle
import tca_spmm

GOLD = ROOT / "tests" / "golden"
PKG = ROOT / "tca-spmm_b200"
CASES = [  # (one_based, pattern_only), as tests/golden/make_golden.py wrote them
    (True, False), (True, True), (False, False)]
TCA_ERR_FORMAT = 6


def lib():
    L = tca_spmm.lib()
    PI = ctypes.POINTER(ctypes.c_int)
    PP = ctypes.POINTER(ctypes.c_void_p)
    L.tca_mtx_parse.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                PI, PI, PI, PP, PP, PP]
    L.tca_mtx_read.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_float, PI, PI, PI, PP, PP, PP]
    L.tca_free.argtypes = [ctypes.c_void_p]
    L.tca_free.restype = None
    return L


def take(L, ptr, n, dt):
    out = np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(np.ctypeslib.as_ctypes_type(dt))),
                                shape=(max(n, 1),))[:n].copy()
    L.tca_free(ptr)
    return out


def mtx(text=None, path=None, zero_based=True, pattern_only=False, missing=0.0):
    L = lib()
    M, K, nnz = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    rp, ci, v = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
    args = (int(zero_based), int(pattern_only), missing, ctypes.byref(M), ctypes.byref(K), ctypes.byref(nnz),
            ctypes.byref(rp), ctypes.byref(ci), ctypes.byref(v))
    rc = L.tca_mtx_read(str(path).encode(), *args) if path is not None else L.tca_mtx_parse(text, len(text), *args)
    if rc:
        return rc, None
    n = nnz.value
    return 0, (M.value, K.value, take(L, rp, M.value + 1, np.int32), take(L, ci, n, np.int32),
               take(L, v, n, np.uint16).view(np.float16))


def dense_of(M, K, rp, ci, v):
    return oracle.csr_to_dense(M, K, rp, ci, v)


@pytest.mark.parametrize("i", range(len(CASES)))
def test_oracle_and_library_match_the_reference(golden, i):
    one_based, pattern = CASES[i]
    path = GOLD / f"mtx_{i}.mtx"
    text = path.read_bytes()
    shape = tuple(golden[f"mtx_{i}_csr_shape"])
    want = (golden[f"mtx_{i}_csr_row_ptr"], golden[f"mtx_{i}_csr_col"], golden[f"mtx_{i}_csr_val"].view(np.uint16))
    orc = oracle.mtx_parse(text, zero_based=not one_based, pattern_only=pattern, missing=0.0)
    rc, ours = mtx(path=path, zero_based=not one_based, pattern_only=pattern)
    assert rc == 0
    for got in (orc, ours):
        assert (got[0], got[1]) == shape
        np.testing.assert_array_equal(got[2], want[0])
        np.testing.assert_array_equal(got[3], want[1])
        np.testing.assert_array_equal(got[4].view(np.uint16), want[2])
    # the dense reader: missing values are 1.0, later duplicates win
    rc, d = mtx(text=text, zero_based=not one_based, missing=1.0)
    np.testing.assert_array_equal(dense_of(*d).view(np.uint16), golden[f"mtx_{i}_dense"].view(np.uint16))


@pytest.mark.parametrize("text", [
    b"% only a comment\n",                       # no header
    b"3 3 2\n1 1 1.0\n",                          # fewer entries than announced
    b"3 3 1\n1 1 1.0\n2 2 2.0\n",                 # more entries than announced
    b"3 3 1\n4 1 1.0\n",                          # row out of range (1-based)
    b"3 3 1\n1 0 1.0\n",                          # column 0 in a 1-based file
    b"3 3 1\nx 1 1.0\n",                          # not "r c [v]"
])
def test_malformed_text_is_a_format_error(text):
    rc, _ = mtx(text=text, zero_based=False)
    assert rc == TCA_ERR_FORMAT
    assert oracle.mtx_parse(text, zero_based=False) is None


def test_blank_lines_and_late_comments_are_skipped():
    rc, got = mtx(text=b"%%MatrixMarket\n\n2 3 2\n\n1 3 0.5\n% late comment\n2 1\n", zero_based=False)
    assert rc == 0
    M, K, rp, ci, v = got
    assert (M, K) == (2, 3) and list(rp) == [0, 1, 2] and list(ci) == [2, 0]
    assert list(v.astype(np.float32)) == [0.5, 0.0]  # a missing value is 0.0 in the CSR reader


DRIVER = r"""
#include <cstdio>
#include <fstream>
#include "tca_spmm_compat.h"
int main(int argc, char **argv)
{
    Arguments arg;
    arg.input_is_zero_based = argv[2][0] == '0';
    arg.pattern_only = argv[3][0] == '1';
    std::ifstream f1(argv[1]);
    CSR *c = nullptr;
    mtx_input_to_CSR(f1, &c, &arg);
    std::ifstream f2(argv[1]);
    half *d = nullptr;
    mtx_input_to_Dense(f2, &d, &arg);
    printf("%d %d %d\n", c->nRow, c->nCol, c->nnz);
    for (int i = 0; i <= c->nRow; i++) printf("%d ", c->row_offset[i]);
    printf("\n");
    for (int i = 0; i < c->nnz; i++) printf("%d:%04x ", c->col_idx[i], (unsigned)__half_as_ushort(c->value[i]));
    printf("\n");
    for (int i = 0; i < c->nRow * c->nCol; i++) printf("%04x ", (unsigned)__half_as_ushort(d[i]));
    printf("\n");
    destroy_csr(c);
    free(d);
    return 0;
}
"""


def test_cpp_drop_ins_match_the_reference(golden, tmp_path):
    src = tmp_path / "mtx_driver.cu"
    src.write_text(DRIVER)
    exe = tmp_path / "mtx_driver"
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    r = subprocess.run([nvcc, "-std=c++17", "-I", str(ROOT / "include"), str(src), "-L", str(PKG / "lib"),
                        "-ltca_spmm", "-Xlinker", f"-rpath,{PKG / 'lib'}", "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    for i, (one_based, pattern) in enumerate(CASES):
        out = subprocess.run([str(exe), str(GOLD / f"mtx_{i}.mtx"), "1" if one_based else "0",
                              "1" if pattern else "0"], capture_output=True, text=True, check=True).stdout.split("\n")
        M, K, n = map(int, out[0].split())
        assert (M, K) == tuple(golden[f"mtx_{i}_csr_shape"])
        np.testing.assert_array_equal(np.array(out[1].split(), np.int32), golden[f"mtx_{i}_csr_row_ptr"])
        pairs = [t.split(":") for t in out[2].split()]
        np.testing.assert_array_equal(np.array([int(a) for a, _ in pairs], np.int32), golden[f"mtx_{i}_csr_col"])
        np.testing.assert_array_equal(np.array([int(b, 16) for _, b in pairs], np.uint16),
                                      golden[f"mtx_{i}_csr_val"].view(np.uint16))
        dense = np.array([int(x, 16) for x in out[3].split()], np.uint16).reshape(M, K)
        np.testing.assert_array_equal(dense, golden[f"mtx_{i}_dense"].view(np.uint16))


@pytest.mark.gpu
@pytest.mark.parametrize("i", range(len(CASES)))
def test_forward_from_a_matrix_market_file(cuda, i):
    """File -> tca_spmm.mtx_read -> plan -> forward, against the FP64 oracle on
    the same CSR (rows keep their file order, so some windows are ineligible
    for the tensor cores and run on CUDA cores)."""
    torch = pytest.importorskip("torch")
    one_based, pattern = CASES[i]
    M, K, rp, ci, v = tca_spmm.mtx_read(GOLD / f"mtx_{i}.mtx", zero_based=not one_based, pattern_only=pattern)
    B = np.random.default_rng(i).uniform(-1, 1, (K, 64)).astype(np.float16)
    plan = tca_spmm.Plan(*(torch.from_numpy(x).to(cuda) for x in (rp, ci, v)), K)
    C = plan.spmm(torch.from_numpy(B).to(cuda), out_dtype=torch.float32).cpu().numpy()
    ref = oracle.spmm_f64(rp, ci, v, B)
    assert np.linalg.norm(C - ref) <= 1e-5 * max(np.linalg.norm(ref), 1e-30)
