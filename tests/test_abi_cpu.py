"""Host-side checks that need no GPU: the C-ABI library loads and exports every
entry point the public header declares, and fails cleanly without a device."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "dayflower_cuda.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(dfc_\w+)\s*\(", text, re.M)))


def test_header_declares_the_binding_table(cuda_lib):
    from dayflower_b200 import _native
    bound = {name for name, _, _ in _native.SIGNATURES}
    assert set(declared_symbols()) == bound


def test_library_exports_every_declared_symbol(cuda_lib):
    for name in declared_symbols():
        assert hasattr(cuda_lib, name), name


def test_create_reports_missing_device_or_bad_index(cuda_lib):
    h = ctypes.c_void_p()
    rc = cuda_lib.dfc_create(10_000, ctypes.byref(h))
    assert rc != 0 and not h.value
    assert cuda_lib.dfc_create(0, None) == 1  # DFC_E_INVALID_ARG for a null out-pointer


def test_null_handle_calls_are_rejected(cuda_lib):
    assert cuda_lib.dfc_set_maximum_bounce(None, 5) == 1
    assert cuda_lib.dfc_render(None, 1, None) == 1
    assert cuda_lib.dfc_destroy(None) == 1
    assert cuda_lib.dfc_last_error(None) == b"null handle"


def test_library_is_built_for_sm100a():
    from dayflower_b200 import build
    assert "arch=compute_100a,code=sm_100a" in " ".join(build.GENCODE)
    assert os.path.exists(build.cuda_lib_path())
