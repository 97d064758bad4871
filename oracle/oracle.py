"""ctypes wrapper around oracle/liboracle.so, the FP64 CPU restatement of the
viss_optimize_3d hot path.

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of bench.py, to check results and to time the CPU path.  The product
(``viss_optimize_3d_b200``) never imports it.

Each wrapper names the reference lines its C function restates (see the
header of viss_oracle.c).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int32)
_up = C.POINTER(C.c_uint32)
_i64 = C.c_int64


def build(force: bool = False) -> str:
    """Compile liboracle.so with the Makefile beside this file."""
    if force or not os.path.exists(_LIB_PATH) or (
        os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "viss_oracle.c"))
    ):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.orc_pix2ang.argtypes = [C.c_int, C.c_int, _i64, _i64, _dp, _dp, _dp]
        L.orc_pix2ang.restype = C.c_int
        L.orc_nest2ring.argtypes = [C.c_int, _i64]
        L.orc_nest2ring.restype = _i64
        L.orc_ring2nest.argtypes = [C.c_int, _i64]
        L.orc_ring2nest.restype = _i64
        L.orc_vec2pix.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double]
        L.orc_vec2pix.restype = _i64
        L.orc_pix2ring.argtypes = [C.c_int, C.c_int, _i64, C.POINTER(_i64), C.POINTER(_i64)]
        L.orc_mk_pix2xy.argtypes = [_ip, _ip]
        L.orc_lmn_from_xyz.argtypes = [_i64, _dp, _dp]
        L.orc_sky_pre_f32.argtypes = [_i64, _fp, _fp, _fp, C.c_float, _dp, _fp]
        L.orc_cone_threshold.argtypes = [C.c_float, C.c_float]
        L.orc_cone_threshold.restype = C.c_double
        L.orc_occulters.argtypes = [_i64, _dp, C.c_double, C.c_int, C.c_double, _dp]
        L.orc_mask_bits.argtypes = [_i64, _i64, _dp, _ip, _dp, _up]
        L.orc_dots.argtypes = [_i64, _dp, _dp, _dp]
        L.orc_forward.argtypes = [_i64, _dp, _dp, _i64, _dp, _dp, _ip, _dp, _dp, C.c_int]
        L.orc_forward_dphase.argtypes = [_i64, _dp, _dp, _i64, _dp, _dp, _ip, _dp, _dp, C.c_int]
        L.orc_dcf.argtypes = [_i64, _fp, C.c_int, C.c_int, _ip, _up, _fp]
        L.orc_gamma_dg.argtypes = [_i64, _fp, _fp, _fp]
        L.orc_weights.argtypes = [_i64, _ip, _fp, _fp, C.c_int, _fp]
        L.orc_wrot.argtypes = [_i64, _dp, _dp]
        L.orc_adjoint.argtypes = [_i64, _dp, _dp, _dp, _i64, _dp, _ip, _dp, _dp, C.c_int]
        L.orc_max_threads.restype = C.c_int
        _lib = L
    return _lib


def _ptr(a, ct):
    if a is None:
        return None
    return a.ctypes.data_as(ct)


def _c(a, dtype):
    return None if a is None else np.ascontiguousarray(a, dtype=dtype)


# ---------------------------------------------------------------- HEALPix
def pix2ang(nside: int, nest: bool = False, first: int = 0, count: int | None = None):
    """theta, phi, xyz (FP64, rounded from long double) -- pix2ang.cu:92-160,
    following the published HEALPix formulas."""
    npix = 12 * nside * nside
    if count is None:
        count = npix - first
    th = np.empty(count)
    ph = np.empty(count)
    xyz = np.empty((count, 3))
    rc = lib().orc_pix2ang(nside, 1 if nest else 0, first, count, _ptr(th, _dp), _ptr(ph, _dp),
                           _ptr(xyz, _dp))
    if rc != 0:
        raise ValueError("orc_pix2ang: bad arguments")
    return th, ph, xyz


def nest2ring(nside: int, p) -> np.ndarray:
    return np.array([lib().orc_nest2ring(nside, int(x)) for x in np.atleast_1d(p)], dtype=np.int64)


def ring2nest(nside: int, p) -> np.ndarray:
    return np.array([lib().orc_ring2nest(nside, int(x)) for x in np.atleast_1d(p)], dtype=np.int64)


def vec2pix(nside: int, xyz, nest: bool = False) -> np.ndarray:
    xyz = np.atleast_2d(xyz)
    return np.array([lib().orc_vec2pix(nside, 1 if nest else 0, *map(float, v)) for v in xyz],
                    dtype=np.int64)


def pix2ring(nside: int, p, nest: bool = False):
    a, b = _i64(), _i64()
    lib().orc_pix2ring(nside, 1 if nest else 0, int(p), C.byref(a), C.byref(b))
    return a.value, b.value


def mk_pix2xy():
    x = np.empty(1024, np.int32)
    y = np.empty(1024, np.int32)
    lib().orc_mk_pix2xy(_ptr(x, _ip), _ptr(y, _ip))
    return x, y


# ---------------------------------------------------------------- sky convention
def lmn_from_xyz(xyz) -> np.ndarray:
    """vissgen3d_blockage.cu:53-74: (l, m, n) = (x, -y, z)."""
    xyz = _c(xyz, np.float64)
    out = np.empty_like(xyz)
    lib().orc_lmn_from_xyz(xyz.shape[0], _ptr(xyz, _dp), _ptr(out, _dp))
    return out


def sky_pre_f32(theta, phi, B, s):
    theta = _c(theta, np.float32)
    phi = _c(phi, np.float32)
    B = _c(B, np.float32)
    n = theta.shape[0]
    lmn = np.empty((n, 3))
    Bo = np.empty(n, np.float32)
    lib().orc_sky_pre_f32(n, _ptr(theta, _fp), _ptr(phi, _fp), _ptr(B, _fp), float(s),
                          _ptr(lmn, _dp), _ptr(Bo, _fp))
    return lmn, Bo


# ---------------------------------------------------------------- occultation
def cone_threshold(R: float = 1737.1e3, h: float = 300e3) -> float:
    """vissgen3d_blockage.cu:249-252 threshold cos(phi)."""
    return lib().orc_cone_threshold(R, h)


def occulters(P, R: float, mode: int = 0, fixed_thr: float = 0.0) -> np.ndarray:
    P = _c(P, np.float64)
    occ = np.empty((P.shape[0], 4))
    lib().orc_occulters(P.shape[0], _ptr(P, _dp), float(R), int(mode), float(fixed_thr),
                        _ptr(occ, _dp))
    return occ


def dots(lmn, q4) -> np.ndarray:
    """fma(s2, q2, fma(s1, q1, s0*q0)) per pixel: the predicate's dot product."""
    lmn = _c(lmn, np.float64)
    q4 = _c(q4, np.float64)
    out = np.empty(lmn.shape[0])
    lib().orc_dots(lmn.shape[0], _ptr(lmn, _dp), _ptr(q4, _dp), _ptr(out, _dp))
    return out


def mask_bits(lmn, refs, occ) -> np.ndarray:
    lmn = _c(lmn, np.float64)
    refs = _c(refs, np.int32)
    occ = _c(occ, np.float64)
    K, J = refs.shape[0], lmn.shape[0]
    bits = np.empty((K, (J + 31) // 32), np.uint32)
    lib().orc_mask_bits(K, J, _ptr(lmn, _dp), _ptr(refs, _ip), _ptr(occ, _dp), _ptr(bits, _up))
    return bits


# ---------------------------------------------------------------- forward / adjoint
def forward(uvw, lmn, I, refs=None, occ=None, off=None, nthreads: int = 0) -> np.ndarray:
    """vissgen3d_blockage.cu:76-102 in FP64: complex128 V[K]."""
    uvw = _c(uvw, np.float64)
    lmn = _c(lmn, np.float64)
    I = _c(I, np.float64)
    refs = _c(refs, np.int32)
    occ = _c(occ, np.float64) if occ is not None else np.zeros((1, 4))
    off = _c(off, np.float64)
    K, J = uvw.shape[0], lmn.shape[0]
    V = np.empty((K, 2))
    lib().orc_forward(K, _ptr(uvw, _dp), _ptr(off, _dp), J, _ptr(lmn, _dp), _ptr(I, _dp),
                      _ptr(refs, _ip), _ptr(occ, _dp), _ptr(V, _dp), int(nthreads))
    return V[:, 0] + 1j * V[:, 1]


def forward_dphase(uvw, lmn, I, refs=None, occ=None, off=None, nthreads: int = 0) -> np.ndarray:
    """sum_j I_j vis s_j exp(-2 pi i phase): complex128 D[K, 3]."""
    uvw = _c(uvw, np.float64)
    lmn = _c(lmn, np.float64)
    I = _c(I, np.float64)
    refs = _c(refs, np.int32)
    occ = _c(occ, np.float64) if occ is not None else np.zeros((1, 4))
    off = _c(off, np.float64)
    K, J = uvw.shape[0], lmn.shape[0]
    D = np.empty((K, 3, 2))
    lib().orc_forward_dphase(K, _ptr(uvw, _dp), _ptr(off, _dp), J, _ptr(lmn, _dp),
                             _ptr(I, _dp), _ptr(refs, _ip), _ptr(occ, _dp), _ptr(D, _dp),
                             int(nthreads))
    return D[..., 0] + 1j * D[..., 1]


def adjoint(uvw, a, lmn, refs=None, occ=None, off=None, nthreads: int = 0) -> np.ndarray:
    """vissgen3d_blockage.cu:167-192 in FP64: C_j = sum_k Re(a_k e^{+2 pi i phase})."""
    uvw = _c(uvw, np.float64)
    lmn = _c(lmn, np.float64)
    a = np.ascontiguousarray(np.stack([np.real(a), np.imag(a)], axis=-1), dtype=np.float64)
    refs = _c(refs, np.int32)
    occ = _c(occ, np.float64) if occ is not None else np.zeros((1, 4))
    off = _c(off, np.float64)
    K, J = uvw.shape[0], lmn.shape[0]
    Cj = np.empty(J)
    lib().orc_adjoint(K, _ptr(uvw, _dp), _ptr(off, _dp), _ptr(a, _dp), J, _ptr(lmn, _dp),
                      _ptr(refs, _ip), _ptr(occ, _dp), _ptr(Cj, _dp), int(nthreads))
    return Cj


# ---------------------------------------------------------------- DCF / gamma
def dcf(bll, nr: int, multiplicity: int = 1):
    """vissgen3d_blockage.cu:105-130 + vissgen3d_noblockage.cu:132-141."""
    bll = _c(bll, np.float32)
    n = bll.shape[0]
    gs = np.empty(n, np.int32)
    counts = np.empty(max(nr, 1), np.uint32)
    d = np.empty(nr + 1, np.float32)
    rc = lib().orc_dcf(n, _ptr(bll, _fp), int(nr), int(multiplicity), _ptr(gs, _ip), _ptr(counts, _up), _ptr(d, _fp))
    if rc != 0:
        raise MemoryError
    return gs, counts[:nr], d


def gamma_dg(w, bll) -> np.ndarray:
    """vissgen3d_blockage.cu:153-162."""
    w = _c(w, np.float32)
    bll = _c(bll, np.float32)
    dg = np.empty(w.shape[0], np.float32)
    lib().orc_gamma_dg(w.shape[0], _ptr(w, _fp), _ptr(bll, _fp), _ptr(dg, _fp))
    return dg


def weights(gs, dg, dcf_table, nr: int) -> np.ndarray:
    """vissgen3d_blockage.cu:178,187: min(dcf[gs] * dg, 1/8) in FP32."""
    gs = _c(gs, np.int32)
    dg = _c(dg, np.float32)
    dcf_table = _c(dcf_table, np.float32)
    wt = np.empty(gs.shape[0], np.float32)
    lib().orc_weights(gs.shape[0], _ptr(gs, _ip), _ptr(dg, _fp), _ptr(dcf_table, _fp), int(nr),
                      _ptr(wt, _fp))
    return wt


def wrot(w, V) -> np.ndarray:
    """vissgen3d_blockage.cu:150-151: V exp(-2 pi i w) in FP64."""
    w = _c(w, np.float64)
    Vr = np.ascontiguousarray(np.stack([np.real(V), np.imag(V)], axis=-1), dtype=np.float64)
    lib().orc_wrot(w.shape[0], _ptr(w, _dp), _ptr(Vr, _dp))
    return Vr[:, 0] + 1j * Vr[:, 1]


def max_threads() -> int:
    return lib().orc_max_threads()
