"""B200-native (sm_100a) direct-sum visibility generation and density-
compensated imaging on HEALPix grids -- the hot path of
SSshuishui/viss_optimize_3d behind a C ABI (include/viss.h).

The GPU entry points load the in-tree CUDA library (libviss.so) on first use
and raise ImportError if it is missing; there is no CPU fallback.  The
generator (``synth``) is plain numpy and loads nothing.
"""
import importlib

_API = ("Plan", "cone_threshold", "conj_mirror_", "dcf", "healpix_moonback_pre", "mask_bits",
        "mk_pix2xy", "occulters", "pix2ang", "pix2lmn", "pix_convert", "scale_coef", "weights",
        "wrot_")

__all__ = list(_API)


def __getattr__(name):
    if name in _API:
        return getattr(importlib.import_module(".api", __name__), name)
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")
