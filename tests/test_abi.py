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


def test_server_arguments_checked_before_any_device_call():
    """ehgp_server_create refuses bad limits without touching a device (no GPU needed)."""
    import ctypes as C
    lib = ehgp.load()
    h = C.c_void_p()
    for lim in (ehgp.ServerLimits(0, 1000, 0.8), ehgp.ServerLimits(4, 0, 0.8), ehgp.ServerLimits(4, 1000, 0.0),
                ehgp.ServerLimits(4, 1000, 1.5), ehgp.ServerLimits(65, 1000, 0.8)):
        assert lib.ehgp_server_create(0, C.byref(lim), C.byref(h)) == 1
    assert lib.ehgp_server_destroy(None) == 0
    assert lib.ehgp_cloud_submit(None, None, None) == 1
