"""The reference's run options class, Arguments(argc, argv)
(src/arg_parse.h:33-133), through the C++ drop-in header: field by field
against the reference's own parse of the same argv (tests/golden/golden.npz,
made by make_golden.py from a driver compiled against the reference header),
plus the option the golden run leaves out (-f) and the error paths. Also the
reference-style call smtx_input_to_CSR(fin, &csr, NULL), which must compile
(one overload) and read the reference's data fixture."""
import pathlib
import shutil
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT

sys.path.insert(0, str(ROOT / "tests" / "golden"))
from make_golden import ARGS_CASES, ARGS_DRIVER  # noqa: E402

PKG = ROOT / "tca-spmm_b200"
GOLD = ROOT / "tests" / "golden"
FIXTURE = GOLD / "body_decoder_layer_2_ffn_conv1.smtx"

EXTRA = r"""
#include <cstdio>
#include <cstring>
#include <fstream>
#include "tca_spmm_compat.h"
int main(int argc, char **argv)
{
    if (argc > 1 && std::strcmp(argv[1], "smtx") == 0) {
        std::ifstream fin(argv[2]);
        CSR *c = nullptr;
        smtx_input_to_CSR(fin, &c, NULL); // the reference's call shape
        if (!c) return 3;
        std::printf("%d %d %d %d\n", c->nRow, c->nCol, c->nnz, c->row_offset[c->nRow]);
        destroy_csr(c);
        return 0;
    }
    if (argc > 1 && std::strcmp(argv[1], "noexit") == 0) {
        tca_compat_set_exit_on_error(0);
        argv[1] = argv[0];
        Arguments a(argc - 1, argv + 1);
        std::printf("%d %d %d %s\n", (int)a.input_file_exists, (int)a.a_type, (int)a.c_type,
                    a.input_fname ? a.input_fname : "-");
        std::printf("%s\n", tca_last_error_string());
        return 0;
    }
    Arguments a(argc, argv);
    std::printf("%d %s %d\n", (int)a.input_file_exists, a.input_fname ? a.input_fname : "-", a.M);
    Arguments b(argc, argv); // a second parse in one process sees its argv from the start
    std::printf("%d %d\n", (int)b.input_file_exists, b.M);
    return 0;
}
"""


def _compile(tmp_path, name, text):
    src = tmp_path / f"{name}.cu"
    src.write_text(text)
    exe = tmp_path / name
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    r = subprocess.run([nvcc, "-std=c++17", "-I", str(ROOT / "include"), str(src), "-L", str(PKG / "lib"),
                        "-ltca_spmm", "-Xlinker", f"-rpath,{PKG / 'lib'}", "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


@pytest.fixture(scope="module")
def drivers(tmp_path_factory):
    d = tmp_path_factory.mktemp("args")
    return _compile(d, "args_ours", ARGS_DRIVER), _compile(d, "args_extra", EXTRA)


@pytest.mark.parametrize("i", range(len(ARGS_CASES)))
def test_arguments_match_the_reference(golden, drivers, i):
    out = subprocess.run([str(drivers[0])] + ARGS_CASES[i], capture_output=True, text=True, check=True)
    assert out.stdout.strip() == str(golden[f"args_{i}"])


def test_input_file_option(drivers):
    out = subprocess.run([str(drivers[1]), "-m", "77", "-f", str(FIXTURE)], capture_output=True, text=True,
                         check=True).stdout.split("\n")
    assert out[0] == f"1 {FIXTURE} 77"
    assert out[1] == "1 77"


def test_missing_input_file_exits_like_the_reference(drivers, tmp_path):
    r = subprocess.run([str(drivers[0]), "-f", str(tmp_path / "absent.smtx")], capture_output=True, text=True)
    assert r.returncode == 1  # EXIT_FAILURE, as src/arg_parse.h:121-124
    assert "Input file not exists" in r.stderr


def test_unsupported_dtype_exits_like_the_reference(drivers):
    r = subprocess.run([str(drivers[0]), "-d", "1"], capture_output=True, text=True)
    assert r.returncode == 1  # src/arg_parse.h:110-114
    assert "Not Implemented" in r.stderr


def test_errors_return_when_exit_is_off(drivers, tmp_path):
    r = subprocess.run([str(drivers[1]), "noexit", "-d", "1", "-f", str(tmp_path / "absent.smtx")],
                       capture_output=True, text=True, check=True).stdout.split("\n")
    fields = r[0].split()
    assert fields[:3] == ["0", "0", "1"]  # file flag off, dtype left at its default (FP16 A, FP32 C)
    assert fields[3] == str(tmp_path / "absent.smtx")
    assert "Input file not exists" in r[1]


def test_smtx_input_to_csr_with_null_arguments(golden, drivers):
    out = subprocess.run([str(drivers[1]), "smtx", str(FIXTURE)], capture_output=True, text=True, check=True)
    M, K, nnz, last = map(int, out.stdout.split())
    assert (M, K, nnz) == tuple(golden["fixture_shape"])
    assert last == nnz
