"""The bounds-checked debug build (libbcn_b200_check.so, -DBCN_CHECK)
compiles, loads and exports the same C ABI plus its check entry points;
the release build reports that it has no guards. CPU only: no kernel runs."""
import ctypes
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def check_lib():
    import importlib.util
    spec = importlib.util.spec_from_file_location("_bcn_build", os.path.join(ROOT, "block_compression_b200", "build.py"))
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    return ctypes.CDLL(b.build(check=True))


def test_check_build_exports_the_abi_and_reports_enabled(bcn, check_lib):
    from test_capi_cpu import _declared_functions
    for n in _declared_functions():
        getattr(check_lib, n)
    check_lib.bc_check_enabled.restype = ctypes.c_int
    assert check_lib.bc_check_enabled() == 1
    assert bcn.lib.bc_check_enabled() == 0
    # argument checks run before any CUDA work
    check_lib.bc_check_read.argtypes = [ctypes.c_void_p]
    assert check_lib.bc_check_read(None) == -6
    assert check_lib.bc_compress_rgba8(0, None, None, 0, None, 0, 6, 8, 24) == -1
