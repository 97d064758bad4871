"""The allocation-free forward entry point (viss_forward_noalloc).

Callers that cannot allocate device memory -- a host application that
controls the whole device-memory budget through its own pool allocator, or a
pipeline that must not allocate after start-up -- use this entry point; its
intermediates live in a fixed __device__ array inside the library.  This test
calls it through the C ABI twice in a row (with different skies, so a stale
scratch would show) and checks each output against the plan-based
viss_forward within the split path's tolerance (rel-L2 <= 1e-5).  It lives in
its own file, collected last, and passes alone in a fresh process as well as
after the other tests.
"""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _p(t):
    return C.c_void_p(t.data_ptr())


def test_forward_noalloc_matches_viss_forward(viss, cuda_device):
    from viss_optimize_3d_b200 import _capi, pipeline, synth

    cfg = synth.scaled(synth.CONFIGS["c2"], nside=32, n_snap=360)   # 12,288 px, 10,080 samples
    obs = synth.make_observation(cfg)
    g = pipeline.upload(obs, cfg.freqs_hz[0], device=cuda_device)
    stream = C.c_void_p(torch.cuda.current_stream(cuda_device).cuda_stream)
    rng = np.random.default_rng(3)
    for call in range(2):
        sky = g.sky if call == 0 else torch.as_tensor(
            rng.uniform(0.0, 2.0, g.plan.J).astype(np.float32), device=cuda_device)
        V_ref = g.plan.forward(sky)
        V = torch.full_like(V_ref, float("nan"))
        st = _capi.lib.viss_forward_noalloc(g.plan.J, _p(g.lmn), _p(sky), g.plan.K, _p(g.uvw), None,
                                            _p(g.refs), g.occ.shape[0], _p(g.occ), _p(V), stream)
        assert st == _capi.VISS_OK, _capi.last_error()
        torch.cuda.synchronize()
        err = (torch.linalg.norm(V - V_ref) / torch.linalg.norm(V_ref)).item()
        assert err <= TOL, (call, err)


def test_forward_noalloc_rejects_sizes_past_its_scratch(viss, cuda_device):
    from viss_optimize_3d_b200 import _capi
    dummy = torch.zeros(8, dtype=torch.float64, device=cuda_device)
    st = _capi.lib.viss_forward_noalloc(1000, _p(dummy), _p(dummy), 40000, _p(dummy), None, None, 0,
                                        None, _p(dummy), None)
    assert st == _capi.VISS_ERR_ARG
    assert "exceeds the fixed scratch" in _capi.last_error()
