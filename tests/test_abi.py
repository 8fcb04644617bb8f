"""The C-ABI library loads and exports every function include/cardiotrust_cuda.h declares.

CPU-only: no compute call is made. Functions that need a device are called only
where the CUDA runtime reports no device, to check they fail with a status
instead of crashing.
"""

import ctypes
import pathlib
import re

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]


def declared_functions():
    text = (ROOT / "include" / "cardiotrust_cuda.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|const char\s*\*)\s+(ct_\w+)\s*\(", text, flags=re.M)))


@pytest.fixture(scope="module")
def lib():
    from cardiotrust_b200 import build as b

    b.build()
    from cardiotrust_b200 import _lib

    return _lib.lib()


def test_header_declares_entry_points():
    names = declared_functions()
    assert "ct_run_epoch" in names and "ct_scenario_create" in names
    assert len(names) >= 15


def test_every_declared_symbol_is_exported(lib):
    from cardiotrust_b200 import _lib

    names = declared_functions()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(_lib.EXPORTED) == names


def test_version_and_status_strings(lib):
    assert lib.ct_version() == 1
    assert lib.ct_status_string(0) == b"ok"
    assert lib.ct_status_string(-4) == b"device-side wait timed out"


def test_null_arguments_are_rejected(lib):
    from cardiotrust_b200 import _lib

    assert lib.ct_ctx_create(0, None, None) == _lib.CT_ERR_INVALID_ARGUMENT
    assert lib.ct_run_epoch(None, None, None, 0, 0) == _lib.CT_ERR_INVALID_ARGUMENT
    assert lib.ct_run_epoch_host(None, None, None, 0, 0, None, None, None, None, None) == _lib.CT_ERR_INVALID_ARGUMENT
    assert lib.ct_sync(None) == _lib.CT_ERR_INVALID_ARGUMENT
    buf = ctypes.create_string_buffer(256)
    assert lib.ct_last_error(buf, len(buf)) == 0
    assert b"NULL" in buf.value


def test_struct_layouts_match_header(lib):
    from cardiotrust_b200 import _lib

    # ct_algorithm: 4 x i32, i64, 6 x f32 -> 48 bytes with natural alignment
    assert ctypes.sizeof(_lib.CtAlgorithm) == 48
    # ct_scenario_desc: 5 x i64 + 9 pointers
    assert ctypes.sizeof(_lib.CtScenarioDesc) == 5 * 8 + 9 * 8


def test_context_without_device_fails_cleanly(lib):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    h = ctypes.c_void_p()
    rc = lib.ct_ctx_create(0, None, ctypes.byref(h))
    assert rc in (-1, -2)  # no device: invalid device index or CUDA error, never a crash
