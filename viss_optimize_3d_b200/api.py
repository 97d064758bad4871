"""Torch-facing API over the C ABI (include/viss.h).

All tensors live on a CUDA device; every call is asynchronous on torch's
current stream of that device.  Each function names the reference kernel or
host stage it replaces (SSshuishui/viss_optimize_3d).
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _capi as capi
from ._capi import check, lib

_SCHEMES = {"ring": capi.VISS_RING, "nest": capi.VISS_NESTED, "nested": capi.VISS_NESTED,
            0: capi.VISS_RING, 1: capi.VISS_NESTED}


def _stream(t: torch.Tensor | None = None):
    dev = t.device if t is not None else torch.device("cuda", torch.cuda.current_device())
    return C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _cuda(t, dtype, device=None, shape_last=None):
    if t is None:
        return None
    if not isinstance(t, torch.Tensor):
        t = torch.as_tensor(t)
    dev = device if device is not None else (t.device if t.is_cuda else torch.device("cuda"))
    t = t.to(device=dev, dtype=dtype).contiguous()
    if shape_last is not None and (t.dim() != 2 or t.shape[1] != shape_last):
        raise ValueError(f"expected an (n, {shape_last}) array, got {tuple(t.shape)}")
    return t


def _scheme(s) -> int:
    try:
        return _SCHEMES[s]
    except KeyError:
        raise ValueError(f"unknown HEALPix scheme {s!r}") from None


# ------------------------------------------------------------------ HEALPix
def mk_pix2xy(device=None):
    """pix2ang.cu:61-88 (mk_pix2xy): 1024-entry bit de-interleave tables."""
    dev = device or torch.device("cuda")
    x = torch.empty(1024, dtype=torch.int32, device=dev)
    y = torch.empty(1024, dtype=torch.int32, device=dev)
    check(lib.viss_mk_pix2xy(_p(x), _p(y), _stream(x)), "viss_mk_pix2xy")
    return x, y


def pix2ang(nside: int, scheme="ring", first: int = 0, count: int | None = None, device=None):
    """pix2ang.cu:92-160 (f_pix2and_nest): FP64 (theta, phi, xyz) of HEALPix
    pixel centres [first, first+count) in RING or NESTED order."""
    npix = 12 * nside * nside
    count = npix - first if count is None else count
    dev = device or torch.device("cuda")
    th = torch.empty(count, dtype=torch.float64, device=dev)
    ph = torch.empty(count, dtype=torch.float64, device=dev)
    xyz = torch.empty((count, 3), dtype=torch.float64, device=dev)
    check(lib.viss_pix2ang(nside, _scheme(scheme), first, count, _p(th), _p(ph), _p(xyz),
                           _stream(th)), "viss_pix2ang")
    return th, ph, xyz


def pix_convert(nside: int, from_scheme, to_scheme, device=None) -> torch.Tensor:
    """out[p] = index in `to_scheme` of pixel p of `from_scheme`."""
    dev = device or torch.device("cuda")
    out = torch.empty(12 * nside * nside, dtype=torch.int64, device=dev)
    check(lib.viss_pix_convert(nside, _scheme(from_scheme), _scheme(to_scheme), _p(out),
                               _stream(out)), "viss_pix_convert")
    return out


def pix2lmn(nside: int, scheme="ring", device=None) -> torch.Tensor:
    """Sky directions (l, m, n) of all pixels (vissgen3d_blockage.cu:53-74)."""
    dev = device or torch.device("cuda")
    lmn = torch.empty((12 * nside * nside, 3), dtype=torch.float64, device=dev)
    check(lib.viss_pix2lmn(nside, _scheme(scheme), _p(lmn), _stream(lmn)), "viss_pix2lmn")
    return lmn


def healpix_moonback_pre(theta, phi, B, s: float):
    """vissgen3d_blockage.cu:53-74 for FP32 (theta, phi, B): returns (lmn FP64
    (npix, 3), B*s FP32)."""
    theta = _cuda(theta, torch.float32)
    phi = _cuda(phi, torch.float32, theta.device)
    B = _cuda(B, torch.float32, theta.device)
    n = theta.shape[0]
    lmn = torch.empty((n, 3), dtype=torch.float64, device=theta.device)
    Bo = torch.empty_like(B)
    check(lib.viss_sky_pre(n, _p(theta), _p(phi), _p(B), float(s), _p(lmn), _p(Bo),
                           _stream(theta)), "viss_sky_pre")
    return lmn, Bo


# --------------------------------------------------------------- occultation
def cone_threshold(R: float = 1737.1e3, h: float = 300e3) -> float:
    """cos(phi), phi = pi - asinf(R/(R+h)) (vissgen3d_blockage.cu:249-252)."""
    return float(lib.viss_cone_threshold(R, h))


def occulters(P, R: float = 1737.4e3, mode: int = 0, fixed_thr: float = 0.0) -> torch.Tensor:
    """Occulter rows (q, thr) from satellite positions P (n, 3) in metres:
    mode 0 ray-sphere against radius R, mode 1 fixed threshold."""
    P = _cuda(P, torch.float64, shape_last=3)
    occ = torch.empty((P.shape[0], 4), dtype=torch.float64, device=P.device)
    check(lib.viss_occulters(P.shape[0], _p(P), float(R), int(mode), float(fixed_thr), _p(occ),
                             _stream(P)), "viss_occulters")
    return occ


def mask_bits(lmn, refs, occ) -> torch.Tensor:
    """Visibility bits: bit j of row k is (sample k, pixel j) visible."""
    lmn = _cuda(lmn, torch.float64, shape_last=3)
    refs = _cuda(refs, torch.int32, lmn.device, shape_last=3)
    occ = _cuda(occ, torch.float64, lmn.device, shape_last=4)
    K, J = refs.shape[0], lmn.shape[0]
    bits = torch.empty((K, (J + 31) // 32), dtype=torch.int32, device=lmn.device)
    check(lib.viss_mask_bits(K, J, _p(lmn), _p(refs), _p(occ), _p(bits), _stream(lmn)),
          "viss_mask_bits")
    return bits


# --------------------------------------------------------------------- plan
class Plan:
    """Geometry of one observation (pixels x samples) in the kernels' layout.

    lmn  (J, 3) FP64 sky directions
    uvw  (K, 3) FP64 baselines in wavelengths
    off  (K,)   FP64 per-sample phase offset in turns (None = 0); the
                reference's forward uses off = -w (its w(n-1) convention)
    refs (K, 3) int32 occulter rows per sample (-1 unused); None = no mask
    occ  (G, 4) FP64 occulter table
    """

    def __init__(self, lmn, uvw=None, off=None, refs=None, occ=None, channels: int = 1):
        self._h = C.c_void_p()
        check(lib.viss_plan_create(C.byref(self._h)), "viss_plan_create")
        lmn = _cuda(lmn, torch.float64, shape_last=3)
        self.device = lmn.device
        self.J = lmn.shape[0]
        self.K = 0
        self.channels = 1
        self.masked = False
        self.form_T = self.form_S = self.form_B = 0   # formation mode (set_formation)
        self.form_C = 1
        check(lib.viss_plan_set_pixels(self._h, self.J, _p(lmn), _stream(lmn)), "viss_plan_set_pixels")
        if uvw is not None:
            self.set_samples(uvw, off, refs, occ)
        if channels != 1:
            self.set_channels(channels)

    def set_samples(self, uvw, off=None, refs=None, occ=None):
        """(Re)stage the samples; resets the plan to one channel.  Synchronises
        the stream once (it checks the phase bound of the split path)."""
        uvw = _cuda(uvw, torch.float64, self.device, shape_last=3)
        off = _cuda(off, torch.float64, self.device)
        refs = _cuda(refs, torch.int32, self.device, shape_last=3)
        occ = _cuda(occ, torch.float64, self.device, shape_last=4) if refs is not None else None
        K = uvw.shape[0]
        check(lib.viss_plan_set_samples(self._h, K, _p(uvw), _p(off), _p(refs),
                                        0 if occ is None else occ.shape[0], _p(occ), _stream(uvw)),
              "viss_plan_set_samples")
        self.K = K
        self.masked = refs is not None
        self.channels = 1

    def set_channels(self, channels: int):
        """Split the samples into `channels` consecutive equal blocks, one per
        frequency; sky and image become (channels, J)."""
        check(lib.viss_plan_set_channels(self._h, int(channels)), "viss_plan_set_channels")
        self.channels = int(channels)

    @staticmethod
    def _flags(fp64, mask, use_offset, accumulate=False):
        f = 0
        if fp64:
            f |= capi.VISS_FP64
        if not mask:
            f |= capi.VISS_NO_MASK
        if not use_offset:
            f |= capi.VISS_NO_OFFSET
        if accumulate:
            f |= capi.VISS_ACCUMULATE
        return f

    def forward(self, sky, fp64: bool = False, mask: bool = True, use_offset: bool = True,
                out: torch.Tensor | None = None) -> torch.Tensor:
        """healpix_moonback_viss (vissgen3d_blockage.cu:76-102):
        V_k = sum_j sky_j vis_kj exp(-2 pi i (u_k.s_j + off_k)), complex64.
        Asynchronous; a bounded device-side wait that gave up inside the
        kernel is raised by the next last_stats() / last_counts()."""
        sky = _cuda(sky, torch.float32, self.device)
        if sky.numel() != self.channels * self.J:
            raise ValueError(f"sky must hold {self.channels} x {self.J} values")
        if out is None:
            out = torch.empty(self.K, dtype=torch.complex64, device=self.device)
        elif (out.dtype != torch.complex64 or not out.is_contiguous() or out.numel() != self.K
              or out.device != self.device):
            raise ValueError(f"out must be a contiguous complex64 tensor of {self.K} values on {self.device}")
        check(lib.viss_forward(self._h, _p(sky), _p(out), self._flags(fp64, mask, use_offset),
                               _stream(sky)), "viss_forward")
        return out

    def adjoint(self, coef, scale: float = 1.0, fp64: bool = False, mask: bool = True,
                use_offset: bool = True, out: torch.Tensor | None = None) -> torch.Tensor:
        """computeC (vissgen3d_blockage.cu:167-192):
        img_j = scale * sum_k Re(coef_k exp(+2 pi i (u_k.s_j + off_k))) vis_kj.
        Asynchronous, like forward (a timed-out wait surfaces in last_stats())."""
        coef = _cuda(coef, torch.complex64, self.device)
        if coef.shape != (self.K,):
            raise ValueError(f"coef must have shape ({self.K},)")
        if out is None:
            shape = (self.J,) if self.channels == 1 else (self.channels, self.J)
            out = torch.empty(shape, dtype=torch.float32, device=self.device)
        elif (out.dtype != torch.float32 or not out.is_contiguous()
              or out.numel() != self.channels * self.J or out.device != self.device):
            raise ValueError(f"out must be a contiguous float32 tensor of {self.channels} x {self.J} "
                             f"values on {self.device}")
        check(lib.viss_adjoint(self._h, _p(coef), _p(out), float(scale),
                               self._flags(fp64, mask, use_offset), _stream(coef)), "viss_adjoint")
        return out

    def adjoint_gridded(self, coef, scale: float = 1.0, mask: bool = True, use_offset: bool = True,
                        facet_pixels: int = 0, out: torch.Tensor | None = None,
                        accumulate: bool = False) -> torch.Tensor:
        """The imaging adjoint through per-facet type-3 NUFFTs
        (viss_adjoint_gridded): the image of adjoint(coef, scale, mask=mask)
        to ~1e-6 relative.  Unmasked (or a plan without occulter refs): computeC
        of the noblockage programs (vissgen3d_noblockage.cu:167-182), all
        gridded.  Occulted: computeC of the blockage programs
        (vissgen3d_blockage.cu:167-192), the pairs whose facet the sample sees
        wholly gridded and the rest through the direct kernel.  facet_pixels
        = 0 lets the library choose (occulted: a multiple of 256); with
        accumulate the image is added to `out`."""
        coef = _cuda(coef, torch.complex64, self.device)
        if coef.shape != (self.K,):
            raise ValueError(f"coef must have shape ({self.K},)")
        if self.channels != 1:
            raise ValueError("the gridded adjoint takes one channel")
        if out is None:
            out = torch.empty(self.J, dtype=torch.float32, device=self.device)
        elif (out.dtype != torch.float32 or not out.is_contiguous() or out.numel() != self.J
              or out.device != self.device):
            raise ValueError(f"out must be a contiguous float32 tensor of {self.J} values on {self.device}")
        flags = self._flags(False, mask, use_offset, accumulate)
        check(lib.viss_adjoint_gridded(self._h, _p(coef), _p(out), float(scale), flags, int(facet_pixels),
                                       _stream(coef)), "viss_adjoint_gridded")
        return out

    def gridded_info(self) -> dict:
        """What the last adjoint_gridded used: facet size, grid dimensions and
        the spreading blocks that did not fit one shared-memory box."""
        fp, hbm = C.c_int64(), C.c_int64()
        dims = (C.c_int32 * 3)()
        check(lib.viss_plan_gridded_info(self._h, C.byref(fp), dims, C.byref(hbm)), "viss_plan_gridded_info")
        return {"facet_pixels": fp.value, "grid": tuple(dims), "hbm_blocks": hbm.value}

    # ---------------------------------------------------- formation mode
    def set_formation(self, U, off=None, occ_sat=None, occ_snap=None):
        """Samples of a satellite formation (viss_plan_set_formation): U is
        (T, S, 3) FP64 satellite vectors in wavelengths; sample k = t * B + pair
        for the B = S(S-1)/2 pairs a < b in lexicographic order, u = U_a - U_b.
        off (T, B) turns, occ_sat (T, S, 4) and occ_snap (T, 4) occulter rows,
        each optional.  Kept beside the plan's ordinary samples.

        U of shape (C, T, S, 3) gives C frequency channels of the same
        snapshots (viss_plan_set_formation_channels): the occulter rows (T, ...)
        are shared by the channels, off is (C, T, B); sky and image are then
        C x J and V / coef C x T x B."""
        U = torch.as_tensor(U) if not isinstance(U, torch.Tensor) else U
        C = 1
        if U.dim() == 4:
            C = int(U.shape[0])
            U = U.reshape(-1, U.shape[2], U.shape[3])
        if U.dim() != 3 or U.shape[2] != 3:
            raise ValueError("U must be (T, S, 3) or (C, T, S, 3)")
        T, S = int(U.shape[0]), int(U.shape[1])
        B = S * (S - 1) // 2
        U = _cuda(U.reshape(T * S, 3), torch.float64, self.device, shape_last=3)
        off = _cuda(None if off is None else torch.as_tensor(off).reshape(T * B), torch.float64, self.device)

        def rows(r, width):
            if r is None:
                return None
            r = torch.as_tensor(r).reshape(-1, 4)
            if C > 1:
                r = _cuda(r, torch.float64, self.device, shape_last=4).repeat(C, 1)
            if r.shape[0] != T * width:
                raise ValueError(f"occulter rows must cover {T // C} snapshots x {width}")
            return _cuda(r, torch.float64, self.device, shape_last=4)

        occ_sat, occ_snap = rows(occ_sat, S), rows(occ_snap, 1)
        check(lib.viss_plan_set_formation(self._h, T, S, _p(U), _p(off), _p(occ_sat), _p(occ_snap),
                                          _stream(U)), "viss_plan_set_formation")
        self.form_T, self.form_S, self.form_B, self.form_C = T, S, B, C
        if C > 1:
            check(lib.viss_plan_set_formation_channels(self._h, C), "viss_plan_set_formation_channels")

    def forward_formation(self, sky, mask: bool = True, use_offset: bool = True,
                          out: torch.Tensor | None = None, accumulate: bool = False):
        """V (T * B complex64) of the formation's samples (channel-major with
        channels: sky then holds C x J values)."""
        sky = _cuda(sky, torch.float32, self.device)
        if sky.numel() != self.form_C * self.J:
            raise ValueError(f"sky must hold {self.form_C * self.J} values")
        n = self.form_T * self.form_B
        if out is None:
            out = torch.empty(n, dtype=torch.complex64, device=self.device)
        elif (out.dtype != torch.complex64 or not out.is_contiguous() or out.numel() != n
              or out.device != self.device):
            raise ValueError(f"out must be a contiguous complex64 tensor of {n} values on {self.device}")
        check(lib.viss_forward_formation(self._h, _p(sky), _p(out), self._flags(False, mask, use_offset, accumulate),
                                         _stream(sky)), "viss_forward_formation")
        return out

    def adjoint_formation(self, coef, scale: float = 1.0, mask: bool = True, use_offset: bool = True,
                          out: torch.Tensor | None = None, accumulate: bool = False):
        """img (J FP32, or C x J with channels) = scale * the adjoint of the
        formation's samples."""
        n = self.form_T * self.form_B
        nimg = self.form_C * self.J
        coef = _cuda(coef, torch.complex64, self.device).reshape(-1)
        if coef.shape != (n,):
            raise ValueError(f"coef must hold {n} values")
        if out is None:
            out = torch.empty(nimg if self.form_C == 1 else (self.form_C, self.J), dtype=torch.float32,
                              device=self.device)
        elif (out.dtype != torch.float32 or not out.is_contiguous() or out.numel() != nimg
              or out.device != self.device):
            raise ValueError(f"out must be a contiguous float32 tensor of {nimg} values on {self.device}")
        check(lib.viss_adjoint_formation(self._h, _p(coef), _p(out), float(scale),
                                         self._flags(False, mask, use_offset, accumulate), _stream(coef)),
              "viss_adjoint_formation")
        return out

    def last_counts(self):
        """(exponentials evaluated, K*J) of the last forward/adjoint (syncs)."""
        ev, tot = C.c_int64(), C.c_int64()
        check(lib.viss_plan_last_counts(self._h, C.byref(ev), C.byref(tot)), "viss_plan_last_counts")
        return ev.value, tot.value

    def tune(self, sky, coef=None, mask: bool = True, use_offset: bool = True):
        """Time every launch shape on this problem and keep the fastest
        (synchronous); returns (forward shape, adjoint shape)."""
        sky = _cuda(sky, torch.float32, self.device)
        if coef is None:
            coef = torch.ones(self.K, dtype=torch.complex64, device=self.device)
        coef = _cuda(coef, torch.complex64, self.device)
        if sky.numel() != self.channels * self.J or coef.numel() != self.K:
            raise ValueError("tune: sky must hold channels x J values and coef K values")
        V = torch.empty(self.K, dtype=torch.complex64, device=self.device)
        img = torch.empty(self.channels * self.J, dtype=torch.float32, device=self.device)
        fs, as_ = C.c_int(), C.c_int()
        check(lib.viss_plan_tune(self._h, _p(sky), _p(coef), _p(V), _p(img),
                                 self._flags(False, mask, use_offset), C.byref(fs), C.byref(as_),
                                 _stream(sky)), "viss_plan_tune")
        return fs.value, as_.value

    def set_shapes(self, fwd_shape: int, adj_shape: int):
        check(lib.viss_plan_set_shapes(self._h, int(fwd_shape), int(adj_shape)),
              "viss_plan_set_shapes")

    def last_stats(self):
        """(evaluated, evaluated in mixed tiles, K*J) of the last call (syncs)."""
        ev, mx, tot = C.c_int64(), C.c_int64(), C.c_int64()
        check(lib.viss_plan_last_stats(self._h, C.byref(ev), C.byref(mx), C.byref(tot)),
              "viss_plan_last_stats")
        return ev.value, mx.value, tot.value

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib.viss_plan_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------- DCF etc.
def dcf(bll, nr: int, multiplicity: int = 1):
    """ceilAndScale + countOccurrences + calculateR + calculateDcf
    (vissgen3d_blockage.cu:105-141, un-shifted formula of
    vissgen3d_noblockage.cu:132-141): returns (gs int32, counts int32 view of
    uint32, dcf FP32[nr+1])."""
    bll = _cuda(bll, torch.float32)
    n = bll.shape[0]
    gs = torch.empty(n, dtype=torch.int32, device=bll.device)
    counts = torch.empty(nr, dtype=torch.int32, device=bll.device)
    d = torch.empty(nr + 1, dtype=torch.float32, device=bll.device)
    check(lib.viss_dcf(n, _p(bll), int(nr), int(multiplicity), _p(gs), _p(counts), _p(d),
                       _stream(bll)), "viss_dcf")
    return gs, counts, d


def weights(w, bll, gs, dcf_table, nr: int):
    """viss_gamma_trans dg (vissgen3d_blockage.cu:153-162) and the imaging
    weight min(dcf[gs] dg, 1/8) (:178, :187)."""
    w = _cuda(w, torch.float32)
    bll = _cuda(bll, torch.float32, w.device)
    gs = _cuda(gs, torch.int32, w.device)
    dcf_table = _cuda(dcf_table, torch.float32, w.device)
    n = w.shape[0]
    dg = torch.empty(n, dtype=torch.float32, device=w.device)
    wt = torch.empty(n, dtype=torch.float32, device=w.device)
    check(lib.viss_weights(n, _p(w), _p(bll), _p(gs), _p(dcf_table), int(nr), _p(dg), _p(wt),
                           _stream(w)), "viss_weights")
    return dg, wt


def wrot_(w, V: torch.Tensor) -> torch.Tensor:
    """V <- V exp(-2 pi i w) in place (vissgen3d_blockage.cu:150-151)."""
    w = _cuda(w, torch.float32, V.device)
    if V.dtype != torch.complex64 or not V.is_contiguous():
        raise ValueError("V must be a contiguous complex64 tensor")
    check(lib.viss_wrot(V.shape[0], _p(w), _p(V), _stream(V)), "viss_wrot")
    return V


def conj_mirror_(V: torch.Tensor, mirror: int) -> torch.Tensor:
    """V[mirror:2 mirror] = conj(V[:mirror]) in place (vissgen3d_blockage.cu:100)."""
    if V.dtype != torch.complex64 or not V.is_contiguous() or V.shape[0] < 2 * mirror:
        raise ValueError("V must be contiguous complex64 with at least 2*mirror rows")
    check(lib.viss_conj_mirror(mirror, _p(V), _stream(V)), "viss_conj_mirror")
    return V


def scale_coef(wt, V: torch.Tensor) -> torch.Tensor:
    wt = _cuda(wt, torch.float32, V.device)
    out = torch.empty_like(V)
    check(lib.viss_scale_coef(V.shape[0], _p(wt), _p(V), _p(out), _stream(V)), "viss_scale_coef")
    return out


def accumulate_image(total: torch.Tensor, img: torch.Tensor) -> torch.Tensor:
    """total += img in FP64 with non-finite pixels counted as 0, on the device
    (viss_accumulate_image): the day sum the reference's notebooks form on the
    host (healpix3d_blockage.ipynb:103-116)."""
    if total.dtype != torch.float64 or not total.is_contiguous() or not total.is_cuda:
        raise ValueError("total must be a contiguous float64 CUDA tensor")
    img = _cuda(img, torch.float32, total.device)
    if img.numel() != total.numel():
        raise ValueError("img and total must hold the same number of pixels")
    check(lib.viss_accumulate_image(total.numel(), _p(img), _p(total), _stream(total)),
          "viss_accumulate_image")
    return total
