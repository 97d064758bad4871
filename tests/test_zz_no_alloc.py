"""The allocation-free forward entry point (viss_forward_noalloc).

Callers that cannot allocate device memory -- a host application that
controls the whole device-memory budget through its own pool allocator, or a
pipeline that must not allocate after start-up -- use this entry point; its
intermediates live in a fixed __device__ array inside the library.  These
tests call it through the C ABI and check its output against the plan-based
viss_forward within the split path's tolerance (rel-L2 <= 1e-5): two calls in
a row with different skies (so a stale scratch would show), a phase offset,
no occultation, pixels in NESTED order, the argument checks, and a bounded
wait that gives up (reported by the same call, after which the next call is
right again).  The file is collected last and passes alone in a fresh process
as well as after the other tests.
"""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _rel(a, b):
    return (torch.linalg.norm(a - b) / torch.linalg.norm(b)).item()


@pytest.fixture(scope="module")
def obs_c2_small(viss, cuda_device):
    from viss_optimize_3d_b200 import pipeline, synth
    cfg = synth.scaled(synth.CONFIGS["c2"], nside=32, n_snap=360)   # 12,288 px, 10,080 samples
    obs = synth.make_observation(cfg)
    return obs, pipeline.upload(obs, cfg.freqs_hz[0], device=cuda_device)


def _noalloc(lmn, sky, uvw, off, refs, occ, V, dev):
    from viss_optimize_3d_b200 import _capi
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    return _capi.lib.viss_forward_noalloc(lmn.shape[0], _p(lmn), _p(sky), uvw.shape[0], _p(uvw), _p(off),
                                          _p(refs), 0 if occ is None else occ.shape[0], _p(occ), _p(V),
                                          stream)


def test_forward_noalloc_matches_viss_forward(obs_c2_small, cuda_device):
    from viss_optimize_3d_b200 import _capi
    _obs, g = obs_c2_small
    rng = np.random.default_rng(3)
    for call in range(2):
        sky = g.sky if call == 0 else torch.as_tensor(
            rng.uniform(0.0, 2.0, g.plan.J).astype(np.float32), device=cuda_device)
        V_ref = g.plan.forward(sky)
        V = torch.full_like(V_ref, float("nan"))
        st = _noalloc(g.lmn, sky, g.uvw, None, g.refs, g.occ, V, cuda_device)
        assert st == _capi.VISS_OK, _capi.last_error()
        torch.cuda.synchronize()
        err = _rel(V, V_ref)
        assert err <= TOL, (call, err)


def test_forward_noalloc_offset_unmasked_and_nested(obs_c2_small, viss, cuda_device):
    """A per-sample phase offset (against a plan with the same offset), no
    occulter refs (against the plan's unmasked forward), and the pixels in
    NESTED order (tiles as compact as the plan's own sorted ones)."""
    from viss_optimize_3d_b200 import _capi, api
    obs, g = obs_c2_small
    gen = torch.Generator(device=cuda_device).manual_seed(5)
    off = torch.rand(g.plan.K, dtype=torch.float64, device=cuda_device, generator=gen) * 8 - 4
    plan_off = api.Plan(g.lmn, g.uvw, off, g.refs, g.occ)
    V_ref = plan_off.forward(g.sky)
    V = torch.full_like(V_ref, float("nan"))
    assert _noalloc(g.lmn, g.sky, g.uvw, off, g.refs, g.occ, V, cuda_device) == _capi.VISS_OK, _capi.last_error()
    torch.cuda.synchronize()
    assert _rel(V, V_ref) <= TOL
    # no occultation
    V_ref = g.plan.forward(g.sky, mask=False)
    assert _noalloc(g.lmn, g.sky, g.uvw, None, None, None, V, cuda_device) == _capi.VISS_OK, _capi.last_error()
    torch.cuda.synchronize()
    assert _rel(V, V_ref) <= TOL
    # the same sky in NESTED order gives the same visibilities
    nest2ring = viss.pix_convert(obs.cfg.nside, "nest", "ring", device=cuda_device)
    lmn_n = g.lmn[nest2ring].contiguous()
    sky_n = g.sky[nest2ring].contiguous()
    V_ref = g.plan.forward(g.sky)
    assert _noalloc(lmn_n, sky_n, g.uvw, None, g.refs, g.occ, V, cuda_device) == _capi.VISS_OK, _capi.last_error()
    torch.cuda.synchronize()
    assert _rel(V, V_ref) <= TOL


def test_forward_noalloc_rejects_bad_inputs(obs_c2_small, cuda_device):
    """Sizes past the fixed scratch, an occulter ref equal to the table size,
    and a baseline whose phase exceeds the split path's 2^28-turn bound are
    refused with VISS_ERR_ARG before anything is computed."""
    from viss_optimize_3d_b200 import _capi
    _obs, g = obs_c2_small
    dummy = torch.zeros(8, dtype=torch.float64, device=cuda_device)
    st = _capi.lib.viss_forward_noalloc(1000, _p(dummy), _p(dummy), 40000, _p(dummy), None, None, 0,
                                        None, _p(dummy), None)
    assert st == _capi.VISS_ERR_ARG
    assert "exceeds the fixed scratch" in _capi.last_error()
    V = torch.empty(g.plan.K, dtype=torch.complex64, device=cuda_device)
    refs = g.refs.clone()
    refs[17, 1] = g.occ.shape[0]
    assert _noalloc(g.lmn, g.sky, g.uvw, None, refs, g.occ, V, cuda_device) == _capi.VISS_ERR_ARG
    assert "outside" in _capi.last_error()
    uvw = g.uvw.clone()
    uvw[3, 0] = 3e8
    assert _noalloc(g.lmn, g.sky, uvw, None, g.refs, g.occ, V, cuda_device) == _capi.VISS_ERR_ARG
    assert "2^28" in _capi.last_error()


def test_forward_noalloc_reports_a_lost_copy(obs_c2_small, cuda_device):
    """A bounded staging wait that gives up is returned by the call itself:
    viss_plan_debug_drop_copy(NULL, 1) makes the next call's first block skip
    one staging copy (no fault, no trap); the call returns VISS_ERR_TIMEOUT
    after about a second, and the next call is right again."""
    from viss_optimize_3d_b200 import _capi
    _obs, g = obs_c2_small
    V_ref = g.plan.forward(g.sky)
    V = torch.empty_like(V_ref)
    assert _capi.lib.viss_plan_debug_drop_copy(None, 1) == _capi.VISS_OK
    st = _noalloc(g.lmn, g.sky, g.uvw, None, g.refs, g.occ, V, cuda_device)
    assert st == _capi.VISS_ERR_TIMEOUT, (st, _capi.last_error())
    assert "incomplete" in _capi.last_error()
    st = _noalloc(g.lmn, g.sky, g.uvw, None, g.refs, g.occ, V, cuda_device)
    assert st == _capi.VISS_OK, _capi.last_error()
    torch.cuda.synchronize()
    assert _rel(V, V_ref) <= TOL
