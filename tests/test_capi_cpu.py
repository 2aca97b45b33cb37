"""The C ABI library: it loads, exports every entry point the header declares,
and reports errors instead of aborting (no GPU needed)."""
import ctypes
import os
import re

import pytest

from caustic_b200 import build, capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    with open(os.path.join(ROOT, "include", "causticot.h")) as f:
        text = f.read()
    return re.findall(r"COT_API\s+int\s+(cot_\w+)\s*\(", text)


@pytest.fixture(scope="module")
def lib():
    build.build_lib()
    return ctypes.CDLL(capi.LIB_PATH)


def test_header_declares_the_surface():
    names = declared()
    for n in ("cot_create", "cot_destroy", "cot_set_problem", "cot_eval", "cot_cells", "cot_solve",
              "cot_centroids", "cot_source_masses", "cot_last_error", "cot_version"):
        assert n in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_every_export():
    assert set(declared()) <= set(capi.EXPORTED)


def test_version(lib):
    assert capi.version() == (0, 1, 0)


def test_errors_are_codes_not_aborts(lib):
    L = capi.load()
    # NULL handle / NULL output
    assert L.cot_create(None, None) == capi.COT_EINVAL
    buf = ctypes.create_string_buffer(256)
    assert L.cot_last_error(None, buf, 256) == capi.COT_OK
    assert b"NULL" in buf.value
    assert L.cot_eval(None, None, None, None, None, None, 0) == capi.COT_EINVAL
    assert L.cot_solve(None, None, None, None, 0) == capi.COT_EINVAL


def test_create_without_gpu_reports_cuda_error():
    from tests.conftest import has_gpu

    if has_gpu():
        pytest.skip("a GPU is present")
    with pytest.raises(capi.CotError) as e:
        capi.Solver()
    assert e.value.code == capi.COT_ECUDA
