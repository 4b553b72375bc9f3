"""The C-ABI library loads without a GPU and exports every entry point the
public header declares; argument validation runs on the host and reports
through sw100_last_error()."""
import ctypes
import os
import re

import pytest

from conftest import REPO

from solweig_project_b200 import _native as N
from solweig_project_b200 import build


@pytest.fixture(scope="module")
def lib():
    build.build()
    return N.load()


def declared_symbols():
    text = open(os.path.join(REPO, "include", "solweig_b200.h")).read()
    return set(re.findall(r"^\s*(?:const\s+)?[\w\s\*]*?\b(sw100_\w+)\s*\(", text, flags=re.M))


def test_header_declares_the_bound_symbols():
    assert declared_symbols() == set(N.SYMBOLS)


def test_library_exports_every_declared_symbol(lib):
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_abi_version(lib):
    assert lib.sw100_abi_version() == N.ABI_VERSION == 3


def test_workspace_queries(lib):
    assert N.workspace_bytes("sw100_svf_workspace_bytes", 500, 500, 18000) >= 500 * 500 * 16 + 18000 * 4
    assert N.workspace_bytes("sw100_time_loop_workspace_bytes", 100, 100, 14) >= 15 * 100 * 100 * 16
    assert N.workspace_bytes("sw100_sun_march_workspace_bytes", 7, 9) >= 7 * 9 * 16


@pytest.mark.parametrize("rows,cols", [(0, 5), (5, -1), (70000, 70000)])
def test_bad_grid_is_refused(lib, rows, cols):
    out = ctypes.c_int64(0)
    rc = lib.sw100_svf_workspace_bytes(rows, cols, 10, ctypes.byref(out))
    assert rc == 1002  # SW100_E_SIZE
    assert b"grid" in lib.sw100_last_error()


def test_null_site_is_refused_before_any_launch(lib):
    before = lib.sw100_launch_count()
    rc = lib.sw100_svf_sweep(None, 8, 8, None, None, 0, None, None, None, 0, None)
    assert rc == 1001  # SW100_E_ARG
    assert b"site" in lib.sw100_last_error()
    with pytest.raises(N.NativeError):
        N.call("sw100_time_loop", None, 8, 8, None, None, 1, None, None, 0, None)
    assert lib.sw100_launch_count() == before


def test_missing_library_fails_loudly(tmp_path, monkeypatch):
    monkeypatch.setattr(N, "_LIB", None)
    with pytest.raises(N.NativeUnavailable):
        N.load(str(tmp_path / "nope.so"))
