"""The C-ABI library loads and exports every entry point include/*.h declares;
argument checks that fail before any device work behave as documented.
No call here reaches the GPU."""
import ctypes
import re

import numpy as np
import pytest

from conftest import ROOT
import tca_spmm


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        for m in re.finditer(r"TCA_API[^;(]*?\b(tca_\w+)\s*\(", h.read_text()):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "tca_spmm" in names and "tca_plan_create" in names and "tca_spmm_csr" in names


@pytest.mark.parametrize("name", declared_symbols())
def test_library_exports_symbol(name):
    L = tca_spmm.lib()
    assert hasattr(L, name), f"{name} declared in include/ but not exported"


def test_python_binds_exported_symbols():
    L = tca_spmm.lib()
    for name in tca_spmm.exported_symbols():
        assert hasattr(L, name)


def test_version_and_status_strings():
    assert "sm_100a" in tca_spmm.version()
    L = tca_spmm.lib()
    assert L.tca_status_string(0) == b"TCA_OK"
    assert L.tca_status_string(6) == b"TCA_ERR_FORMAT"
    assert L.tca_status_string(99) == b"TCA_ERR_UNKNOWN"


def test_invalid_arguments_rejected_before_device_work():
    L = tca_spmm.lib()
    # bad output dtype
    rc = L.tca_spmm_csr(None, None, None, 4, 4, 0, None, 4, 4, None, 4, 7, 1.0, 0.0, 0, None)
    assert rc == 1 and b"c_dtype" in L.tca_last_error_string()
    # ldb < N
    rc = L.tca_spmm_csr(None, None, None, 4, 4, 0, 1, 2, 4, 1, 4, 0, 1.0, 0.0, 0, None)
    assert rc == 1 and b"ldb" in L.tca_last_error_string()
    # empty problem is a no-op success
    assert L.tca_spmm_csr(None, None, None, 0, 4, 0, None, 4, 4, None, 4, 0, 1.0, 0.0, 0, None) == 0
    # plan: NULL output handle, negative sizes, bad options
    assert L.tca_plan_create(None, None, None, 1, 1, 0, None, None, None) == 1
    h = ctypes.c_void_p()
    assert L.tca_plan_create(None, None, None, -1, 1, 0, None, None, ctypes.byref(h)) == 1
    opts = tca_spmm.PlanOpts()
    L.tca_plan_opts_default(ctypes.byref(opts))
    assert opts.sort_rows == 1 and opts.path == 0 and abs(opts.tc_min_density - 0.01) < 1e-7
    opts.path = 5
    assert L.tca_plan_create(1, 1, 1, 1, 1, 1, ctypes.byref(opts), None, ctypes.byref(h)) == 1
    # an M == 0 plan needs no device memory and behaves as an empty problem
    assert L.tca_plan_create(None, None, None, 0, 8, 0, None, None, ctypes.byref(h)) == 0
    info = tca_spmm.PlanInfo()
    assert L.tca_plan_info(h, ctypes.byref(info)) == 0 and info.M == 0 and info.n_windows == 0
    assert L.tca_spmm(h, None, 8, 8, None, 8, 0, 1.0, 0.0, 0, None) == 0
    assert L.tca_plan_destroy(h) == 0
    # spmm_host: bad CSR pointers
    assert L.tca_spmm_host(None, None, None, 2, 2, 1, None, 2, None, 1, 0, 1, None) == 1


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(tca_spmm, "LIB_PATH", tmp_path / "nope.so")
    monkeypatch.setattr(tca_spmm, "_lib", None)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        tca_spmm.lib()
