"""ctypes binding of libviss.so (include/viss.h).

Loads the in-tree library built by ``viss_optimize_3d_b200._build``.  There
is no fallback: if the library is missing, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
import os
import re

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libviss.so")
HEADER = os.path.join(os.path.dirname(PKG), "include", "viss.h")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is missing: build it with `python -m viss_optimize_3d_b200._build` "
        "(the CUDA library has no CPU fallback)")

lib = C.CDLL(LIB_PATH)

_v = C.c_void_p
_i = C.c_int
_i64 = C.c_int64
_d = C.c_double
_f = C.c_float

VISS_OK = 0
VISS_ERR_ARG = -1
VISS_ERR_CUDA = -2
VISS_ERR_ALLOC = -3
VISS_ERR_TIMEOUT = -4
VISS_ERR_NOTFINITE = -5
VISS_ERR_IO = -6
VISS_ERR_STATE = -7
VISS_FP64 = 0x1
VISS_NO_MASK = 0x2
VISS_NO_OFFSET = 0x4
VISS_ACCUMULATE = 0x8
VISS_RING = 0
VISS_NESTED = 1

_SIGS = {
    "viss_version": (_i, []),
    "viss_status_string": (C.c_char_p, [_i]),
    "viss_last_error": (C.c_size_t, [C.c_char_p, C.c_size_t]),
    "viss_mk_pix2xy": (_i, [_v, _v, _v]),
    "viss_pix2ang": (_i, [_i, _i, _i64, _i64, _v, _v, _v, _v]),
    "viss_pix_convert": (_i, [_i, _i, _i, _v, _v]),
    "viss_pix2lmn": (_i, [_i, _i, _v, _v]),
    "viss_sky_pre": (_i, [_i64, _v, _v, _v, _f, _v, _v, _v]),
    "viss_occulters": (_i, [_i64, _v, _d, _i, _d, _v, _v]),
    "viss_cone_threshold": (_d, [_f, _f]),
    "viss_mask_bits": (_i, [_i64, _i64, _v, _v, _v, _v, _v]),
    "viss_plan_create": (_i, [C.POINTER(_v)]),
    "viss_plan_destroy": (_i, [_v]),
    "viss_plan_set_pixels": (_i, [_v, _i64, _v, _v]),
    "viss_plan_set_samples": (_i, [_v, _i64, _v, _v, _v, _i64, _v, _v]),
    "viss_forward": (_i, [_v, _v, _v, _i, _v]),
    "viss_adjoint": (_i, [_v, _v, _v, _f, _i, _v]),
    "viss_adjoint_gridded": (_i, [_v, _v, _v, _f, _i, _i64, _v]),
    "viss_plan_gridded_info": (_i, [_v, _v, _v, _v]),
    "viss_plan_last_counts": (_i, [_v, C.POINTER(_i64), C.POINTER(_i64)]),
    "viss_plan_tune": (_i, [_v, _v, _v, _v, _v, _i, C.POINTER(_i), C.POINTER(_i), _v]),
    "viss_plan_set_shapes": (_i, [_v, _i, _i]),
    "viss_plan_debug_drop_copy": (_i, [_v, _i]),
    "viss_plan_set_formation": (_i, [_v, _i64, _i, _v, _v, _v, _v, _v]),
    "viss_plan_set_formation_channels": (_i, [_v, _i]),
    "viss_forward_formation": (_i, [_v, _v, _v, _i, _v]),
    "viss_adjoint_formation": (_i, [_v, _v, _v, _f, _i, _v]),
    "viss_plan_set_channels": (_i, [_v, _i]),
    "viss_plan_last_stats": (_i, [_v, C.POINTER(_i64), C.POINTER(_i64), C.POINTER(_i64)]),
    "viss_forward_noalloc": (_i, [_i64, _v, _v, _i64, _v, _v, _v, _i64, _v, _v, _v]),
    "viss_dcf": (_i, [_i64, _v, _i, _i, _v, _v, _v, _v]),
    "viss_weights": (_i, [_i64, _v, _v, _v, _v, _i, _v, _v, _v]),
    "viss_wrot": (_i, [_i64, _v, _v, _v]),
    "viss_conj_mirror": (_i, [_i64, _v, _v]),
    "viss_scale_coef": (_i, [_i64, _v, _v, _v, _v]),
    "viss_stage_day_rows": (_i, [_i64, _v, _v, _v, _v, _v, _v, _v, _v, _v]),
    "viss_accumulate_image": (_i, [_i64, _v, _v, _v]),
}

for _name, (_res, _args) in _SIGS.items():
    _fn = getattr(lib, _name)
    _fn.restype = _res
    _fn.argtypes = _args


class VissError(RuntimeError):
    """A libviss entry point returned a non-zero status."""

    def __init__(self, status: int, where: str):
        self.status = status
        msg = last_error()
        super().__init__(f"{where}: {lib.viss_status_string(status).decode()} ({status}): {msg}")


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    lib.viss_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(status: int, where: str) -> None:
    if status != VISS_OK:
        raise VissError(status, where)


def declared_symbols() -> list[str]:
    """Every function name declared in include/viss.h."""
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(viss_[a-z0-9_]+)\s*\(", text)))
