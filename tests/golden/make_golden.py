"""Generates the golden fixtures in this directory by running the reference's
own CPU functions, compiled from the reference sources into
oracle/_ref/libtcaref.so (`make -C oracle ref`):

  smtx_*.smtx            seeded synthetic smtx files (written by this script)
  golden.npz             for each case, the reference's outputs:
    smtx_<i>_coords      smtx_input_to_Dense (src/file_input.cu:135-193) on
                         smtx_<i>.smtx, stored as the (row, col) pairs of its
                         nonzeros (all values are 1.0) plus the shape
    d2c_<i>_*            convert_dense_to_csr (src/miscalleneous.cu:29-65) on a
                         seeded dense FP16 matrix with -0.0, subnormals and
                         repeated values
    c2d_<i>_dense        convert_csr_to_dense (src/miscalleneous.cu:66-81)
    gemm_<i>_*           naive_gemm (src/miscalleneous.cu:114-134) on a seeded
                         sparse A (dense storage) and B
  mtx_*.mtx              seeded MatrixMarket files (written by this script)
    mtx_<i>_csr_*        mtx_input_to_CSR (src/file_input.cu:63-134) on mtx_<i>.mtx
    mtx_<i>_dense        mtx_input_to_Dense (src/file_input.cu:8-62) on mtx_<i>.mtx
  body_decoder_layer_2_ffn_conv1.smtx
                         the reference's only data fixture (data/ in the
                         reference project), copied unchanged
    fixture_shape, fixture_coords
                         smtx_input_to_Dense on it, stored as for smtx_<i>
    args_<i>             the fields of the reference's Arguments(argc, argv)
                         (src/arg_parse.h:33-133) for the argv ARGS_CASES[i],
                         printed by a small driver compiled against the
                         reference's own header

The reference project is located by the environment variable
TCA_REFERENCE_ROOT. Run from the repository root:
    TCA_REFERENCE_ROOT=<reference project> python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import pathlib
import shutil
import subprocess
import sys
import tempfile

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import oracle  # noqa: E402

OUT = pathlib.Path(__file__).resolve().parent


def write_smtx(path, M, K, row_ptr, col):
    """Same layout as the reference fixture: header, row_ptr line, col line,
    single spaces with a trailing space."""
    with open(path, "w") as f:
        f.write(f"{M}, {K}, {int(row_ptr[-1])}\n")
        f.write("".join(f"{x} " for x in row_ptr) + "\n")
        f.write("".join(f"{x} " for x in col) + "\n")


def smtx_cases(rng):
    cases = []
    # mostly-empty rows with one row above 64 nnz (both reference kernel paths)
    M, K = 2048, 512
    nz_rows = rng.choice(M, 28, replace=False)
    row_nnz = np.zeros(M, np.int64)
    row_nnz[nz_rows] = rng.integers(1, 60, size=28)
    row_nnz[nz_rows[0]] = 65
    cases.append((M, K, row_nnz))
    # small dense-ish and ragged cases
    cases.append((37, 53, rng.binomial(53, 0.3, size=37)))
    cases.append((64, 1024, np.where(rng.random(64) < 0.2, 0, rng.integers(1, 1024, size=64))))
    out = []
    for M, K, row_nnz in cases:
        row_ptr = np.zeros(M + 1, np.int32)
        np.cumsum(row_nnz, out=row_ptr[1:])
        cols = [np.sort(rng.choice(K, int(n), replace=False)) for n in row_nnz]
        col = np.concatenate(cols).astype(np.int32) if cols else np.zeros(0, np.int32)
        out.append((M, K, row_ptr, col))
    return out


def dense_case(rng, M, K, density):
    A = (rng.standard_normal((M, K)) * 0.5).astype(np.float16)
    A[rng.random((M, K)) >= density] = 0
    bits = A.view(np.uint16)
    neg0 = rng.random((M, K)) < 0.02
    bits[neg0] = 0x8000                       # -0.0 is not a nonzero
    sub = rng.random((M, K)) < 0.01
    bits[sub] = rng.integers(1, 0x3ff, size=int(sub.sum()), dtype=np.uint16)  # subnormals are
    return A


def write_mtx(path, rng, M, K, n, one_based, with_values, missing_every=0):
    """Coordinate MatrixMarket text: a banner and a comment, "M K n", then n
    entries in random order (rows and columns unsorted, some duplicates), a
    value on each line unless with_values is False or the line is one of every
    missing_every lines."""
    rows = rng.integers(0, M, n)
    cols = rng.integers(0, K, n)
    if n > 4:
        rows[1], cols[1] = rows[0], cols[0]  # a duplicate entry
    vals = rng.standard_normal(n) * rng.choice([1e-3, 1.0, 300.0], n)
    b = 1 if one_based else 0
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate " + ("real" if with_values else "pattern") + " general\n")
        f.write("% generated by make_golden.py\n")
        f.write(f"{M} {K} {n}\n")
        for i in range(n):
            line = f"{rows[i] + b} {cols[i] + b}"
            if with_values and not (missing_every and i % missing_every == 0):
                line += f" {vals[i]:.7g}"
            f.write(line + "\n")


MTX_CASES = [  # (M, K, n, one_based, with_values, missing_every, pattern_only)
    (40, 30, 120, True, True, 7, False),
    (25, 50, 60, True, False, 0, True),
    (64, 16, 90, False, True, 0, False),
]


# argv of Arguments(argc, argv) cases (argv[0] is the program name). Option
# -f, whose copy the reference makes one byte short of its terminator, is
# checked against known answers in the tests instead.
ARGS_CASES = [
    [],
    ["-m", "2048", "-n", "256", "-k", "512", "-i", "20", "-t", "0.01", "-s", "0.95", "-p", "1", "-b", "1",
     "-e", "16", "-d", "2"],
    ["-d", "0", "-p", "0", "-b", "0", "-s", "1e-1", "-t", "2.5e-4"],
    ["-m", "12abc", "-n", " 64", "-q", "-k", "-7"],
]

# Prints the fields of Arguments(argc, argv); compiled against the
# reference's src/arg_parse.h (USE_REFERENCE) or this project's
# include/tca_spmm_compat.h (the tests).
ARGS_DRIVER = r'''
#ifdef USE_REFERENCE
#include "arg_parse.h"
#else
#include "tca_spmm_compat.h"
#endif
#include <cstdio>
int main(int argc, char **argv)
{
    Arguments a(argc, argv);
    std::printf("%d %d %d %d %d %d %d %a %a %d %d %d %d\n", a.M, a.N, a.K, a.num_iter, (int)a.pattern_only,
                (int)a.input_is_zero_based, (int)a.input_file_exists, (double)a.target_sparsity,
                (double)a.tolerance, (int)a.a_type, (int)a.b_type, (int)a.c_type, a.ell_block_size);
    return 0;
}
'''


def reference_args(ref_src):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    with tempfile.TemporaryDirectory() as d:
        src = pathlib.Path(d) / "args_ref.cu"
        src.write_text(ARGS_DRIVER)
        exe = pathlib.Path(d) / "args_ref"
        subprocess.run([nvcc, "-std=c++17", "-DUSE_REFERENCE", "-I", str(ROOT / "oracle" / "stub"), "-I",
                        str(ref_src), str(src), "-o", str(exe)], check=True)
        return [subprocess.run([str(exe)] + argv, capture_output=True, text=True, check=True).stdout.strip()
                for argv in ARGS_CASES]


def main():
    ref_root = os.environ.get("TCA_REFERENCE_ROOT")
    if not ref_root:
        sys.exit("set TCA_REFERENCE_ROOT to the reference project's directory")
    ref_root = pathlib.Path(ref_root)
    subprocess.run(["make", "-C", str(ROOT / "oracle"), "all", "ref", f"REF_SRC={ref_root / 'src'}"], check=True)
    rng = np.random.default_rng(20240601)
    g = {}
    for i, (M, K, row_ptr, col) in enumerate(smtx_cases(rng)):
        path = OUT / f"smtx_{i}.smtx"
        write_smtx(path, M, K, row_ptr, col)
        A, nnz = oracle.ref_smtx_to_dense(path)
        r, c = np.nonzero(A.view(np.uint16))
        assert np.all(A[r, c] == 1.0)
        g[f"smtx_{i}_shape"] = np.array([A.shape[0], A.shape[1], nnz], np.int64)
        g[f"smtx_{i}_coords"] = np.stack([r, c]).astype(np.int32)
    for i, (M, K, d) in enumerate([(33, 47, 0.3), (128, 64, 0.05), (7, 300, 0.6)]):
        A = dense_case(rng, M, K, d)
        rp, ci, v = oracle.ref_dense_to_csr(A)
        g[f"d2c_{i}_A"] = A
        g[f"d2c_{i}_row_ptr"], g[f"d2c_{i}_col"], g[f"d2c_{i}_val"] = rp, ci, v
        g[f"c2d_{i}_dense"] = oracle.ref_csr_to_dense(M, K, rp, ci, v)
    for i, (M, K, N, d) in enumerate([(64, 96, 40, 0.2), (128, 256, 64, 0.05), (30, 70, 24, 0.9)]):
        A = (rng.standard_normal((M, K)) * 0.3).astype(np.float16)
        A[rng.random((M, K)) >= d] = 0
        B = rng.uniform(-1, 1, size=(K, N)).astype(np.float16)
        g[f"gemm_{i}_A"], g[f"gemm_{i}_B"] = A, B
        g[f"gemm_{i}_C"] = oracle.ref_naive_gemm(A, B)
    mrng = np.random.default_rng(20250301)
    for i, (M, K, n, one_based, with_values, missing_every, pattern_only) in enumerate(MTX_CASES):
        path = OUT / f"mtx_{i}.mtx"
        write_mtx(path, mrng, M, K, n, one_based, with_values, missing_every)
        with oracle.quiet_stdout():
            m, k, rp, ci, v = oracle.ref_mtx_to_csr(str(path), zero_based=not one_based, pattern_only=pattern_only)
            D = oracle.ref_mtx_to_dense(str(path), zero_based=not one_based)
        g[f"mtx_{i}_csr_shape"] = np.array([m, k], np.int64)
        g[f"mtx_{i}_csr_row_ptr"], g[f"mtx_{i}_csr_col"], g[f"mtx_{i}_csr_val"] = rp, ci, v
        g[f"mtx_{i}_dense"] = D
    fixture = next((ref_root / "data").glob("*.smtx"))
    shutil.copyfile(fixture, OUT / fixture.name)
    A, nnz = oracle.ref_smtx_to_dense(OUT / fixture.name)
    r, c = np.nonzero(A.view(np.uint16))
    g["fixture_shape"] = np.array([A.shape[0], A.shape[1], nnz], np.int64)
    g["fixture_coords"] = np.stack([r, c]).astype(np.int32)
    for i, line in enumerate(reference_args(ref_root / "src")):
        g[f"args_{i}"] = np.array(line)
    np.savez_compressed(OUT / "golden.npz", **g)
    print("wrote", OUT / "golden.npz", len(g), "arrays")


if __name__ == "__main__":
    main()
