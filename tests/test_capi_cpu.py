"""C ABI checks that need no GPU: the in-tree library loads, exports every
function include/viss.h declares, and rejects bad arguments with a status
(the reference's CHECK macro, error.cuh:4-19, would exit(1) instead)."""
import ctypes as C

import pytest


def test_library_exports_every_declared_symbol(viss):
    from viss_optimize_3d_b200 import _capi
    names = _capi.declared_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(_capi.lib, n)]
    assert not missing, f"declared in viss.h but not exported: {missing}"


def test_version_and_status_strings(viss):
    from viss_optimize_3d_b200 import _capi
    assert _capi.lib.viss_version() >= 1
    for st in (0, -1, -2, -3, -4, -5, -6, -7):
        assert _capi.lib.viss_status_string(st)
    assert b"unknown" in _capi.lib.viss_status_string(-99)


@pytest.mark.parametrize("call", [
    lambda L: L.viss_pix2ang(0, 0, 0, 1, None, None, None, None),        # nside 0
    lambda L: L.viss_pix2ang(4, 7, 0, 1, None, None, None, None),        # bad scheme
    lambda L: L.viss_pix2ang(4, 0, 190, 5, None, None, None, None),      # past npix
    lambda L: L.viss_pix_convert(4, 0, 1, None, None),                   # null output
    lambda L: L.viss_plan_create(None),
    lambda L: L.viss_forward(None, None, None, 0, None),
    lambda L: L.viss_adjoint(None, None, None, 1.0, 0, None),
    lambda L: L.viss_adjoint_gridded(None, None, None, 1.0, 0, 0, None),
    lambda L: L.viss_plan_gridded_info(None, None, None, None),
    lambda L: L.viss_dcf(10, None, 5, 1, None, None, None, None),
    lambda L: L.viss_dcf(10, C.c_void_p(16), 0, 1, None, None, C.c_void_p(16), None),  # nr 0
    lambda L: L.viss_occulters(3, C.c_void_p(16), -1.0, 0, 0.0, C.c_void_p(16), None),
    lambda L: L.viss_occulters(3, C.c_void_p(16), 1.0, 0, 0.0, C.c_void_p(24), None),  # misaligned
])
def test_bad_arguments_return_status(viss, call):
    from viss_optimize_3d_b200 import _capi
    st = call(_capi.lib)
    assert st == _capi.VISS_ERR_ARG
    assert _capi.last_error()


def test_cone_threshold_is_host_only(viss):
    from viss_optimize_3d_b200 import _capi
    import math
    thr = _capi.lib.viss_cone_threshold(1737.1e3, 300e3)
    assert abs(thr + math.sqrt(1 - (1737.1e3 / 2037.1e3) ** 2)) < 1e-6
