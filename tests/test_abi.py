"""C ABI checks that need no GPU: the library loads and exports every symbol
that include/ehgp.h declares; status names are stable."""
import ctypes

import ehgp


def test_library_exports_every_declared_symbol():
    lib = ehgp.load()
    declared = ehgp.declared_symbols()
    assert "ehgp_lbvh_build" in declared and "ehgp_ctx_create" in declared
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing


def test_status_strings():
    lib = ehgp.load()
    for code, name in ehgp.STATUS.items():
        assert lib.ehgp_status_string(code).decode() == name
    assert lib.ehgp_status_string(999).decode() == "EHGP_ERR_UNKNOWN"


def test_create_rejects_bad_limits_without_gpu_work():
    lib = ehgp.load()
    h = ctypes.c_void_p()
    assert lib.ehgp_ctx_create(0, None, ctypes.byref(h)) == 1
    lim = ehgp.Limits(0, 0.8)
    assert lib.ehgp_ctx_create(0, ctypes.byref(lim), ctypes.byref(h)) == 1
    assert lib.ehgp_last_error(None).decode() == ""
    assert lib.ehgp_ctx_destroy(None) == 0
