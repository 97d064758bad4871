"""The tile classification is conservative.  Occulter rows whose limb runs
exactly through chosen pixels (threshold = the exact FP64 dot product of the
occultation predicate, vissgen3d_blockage.cu:88-94, or one ulp either side)
leave those pixels to the exact per-pixel test, whatever the FP32 tile and
sub-tile cones and the FP32 classification rows say about the rest; the GPU
forward and adjoint then match the FP64 oracle sample by sample and pixel by
pixel (a single wrong mask bit moves a value by one whole sky or coefficient
unit, ~0.5 here, against tolerances of 1e-2).  Also rows that are not unit
vectors (the classification normalises them) and rows every pixel passes or
fails."""
import numpy as np
import pytest
import torch

from viss_optimize_3d_b200 import api

pytestmark = pytest.mark.gpu


def _grazing_case(oracle, lmn, K=1536, seed=5):
    rng = np.random.default_rng(seed)
    J = lmn.shape[0]
    G = 2 * K
    occ = np.empty((G, 4))
    q = rng.standard_normal((G, 3))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    scale = np.where(np.arange(G) % 5 == 4, 3.7, 1.0)          # some rows not unit length
    q *= scale[:, None]
    px = rng.integers(0, J, G)
    for g in range(G):
        thr = oracle.dots(lmn[px[g]][None], np.array([*q[g], 0.0]))[0]
        if g % 3 == 1:
            thr = np.nextafter(thr, np.inf)      # the chosen pixel just hidden
        elif g % 3 == 2:
            thr = np.nextafter(thr, -np.inf)     # just visible
        occ[g] = (*q[g], thr)
    occ[7] = (0.0, 0.0, 1.0, -4.0)               # every pixel passes
    occ[11] = (0.0, 0.0, 1.0, 4.0)               # every pixel fails
    refs = np.stack([np.arange(K), K + np.arange(K), np.full(K, -1)], axis=1).astype(np.int32)
    refs[::9, 1] = -1
    uvw = rng.uniform(-40.0, 40.0, (K, 3))
    sky = rng.uniform(0.5, 1.5, J)
    return uvw, sky, refs, occ


@pytest.fixture(scope="module")
def case(viss, cuda_device, oracle):
    lmn_d = api.pix2lmn(16, "ring", device=cuda_device)
    lmn = lmn_d.cpu().numpy()
    uvw, sky, refs, occ = _grazing_case(oracle, lmn)
    dev = cuda_device
    plan = api.Plan(lmn_d, torch.as_tensor(uvw, device=dev), None,
                    torch.as_tensor(refs, device=dev), torch.as_tensor(occ, device=dev))
    return lmn, uvw, sky, refs, occ, plan


def test_grazing_rows_forward(case, oracle, cuda_device):
    lmn, uvw, sky, refs, occ, plan = case
    Vo = oracle.forward(uvw, lmn, sky, refs, occ)
    sky_d = torch.as_tensor(sky, dtype=torch.float32, device=cuda_device)
    for shape in range(4):
        plan.set_shapes(shape, 0)
        Vs = plan.forward(sky_d).cpu().numpy().astype(np.complex128)
        assert np.abs(Vs - Vo).max() < 1e-2, (shape, np.abs(Vs - Vo).max())
    Vd = plan.forward(sky_d, fp64=True).cpu().numpy().astype(np.complex128)
    assert np.abs(Vd - Vo).max() < 1e-3
    ev, mixed, tot = plan.last_stats()
    assert 0 < mixed <= ev < tot        # the grazing tiles took the exact test; some were culled


def test_grazing_rows_adjoint(case, oracle, cuda_device):
    lmn, uvw, sky, refs, occ, plan = case
    rng = np.random.default_rng(9)
    a = (rng.standard_normal(len(uvw)) + 1j * rng.standard_normal(len(uvw))).astype(np.complex64)
    Co = oracle.adjoint(uvw, a.astype(np.complex128), lmn, refs, occ)
    a_d = torch.as_tensor(a, device=cuda_device)
    for shape in range(4):
        plan.set_shapes(0, shape)
        Cs = plan.adjoint(a_d).cpu().numpy().astype(np.float64)
        assert np.abs(Cs - Co).max() < 1e-2, (shape, np.abs(Cs - Co).max())
    Cd = plan.adjoint(a_d, fp64=True).cpu().numpy().astype(np.float64)
    assert np.abs(Cd - Co).max() < 1e-3


def test_refs_outside_the_table_are_rejected(viss, cuda_device):
    """A ref past the occulter table (or below -1) is an argument error, not an
    out-of-bounds read; the plan holds no samples afterwards."""
    from viss_optimize_3d_b200._capi import VissError
    lmn = api.pix2lmn(4, "ring", device=cuda_device)
    uvw = torch.zeros((8, 3), dtype=torch.float64, device=cuda_device)
    occ = torch.tensor([[0.0, 0.0, 1.0, 0.5]] * 3, dtype=torch.float64, device=cuda_device)
    for bad in (3, -2):
        refs = torch.full((8, 3), -1, dtype=torch.int32, device=cuda_device)
        refs[5, 1] = bad
        plan = api.Plan(lmn)
        with pytest.raises(VissError, match="outside"):
            plan.set_samples(uvw, None, refs, occ)
        with pytest.raises(VissError):
            plan.forward(torch.ones(lmn.shape[0], device=cuda_device))
    refs = torch.full((8, 3), 2, dtype=torch.int32, device=cuda_device)
    plan = api.Plan(lmn, uvw, None, refs, occ)     # the last row is in range
    assert plan.forward(torch.ones(lmn.shape[0], device=cuda_device)).shape == (8,)


@pytest.mark.parametrize("which", ["forward", "adjoint"])
def test_bounded_wait_reports_a_lost_copy(case, cuda_device, which):
    """Failure path without a GPU fault: the first thread block never receives
    one staging copy (viss_plan_debug_drop_copy), its bounded waits give up
    after about a second, the kernel ends and the call reports
    VISS_ERR_TIMEOUT; the same plan then computes the right result again."""
    from viss_optimize_3d_b200._capi import VissError, check, lib
    lmn, uvw, sky, refs, occ, plan = case
    plan.set_shapes(0, 0)
    sky_d = torch.as_tensor(sky, dtype=torch.float32, device=cuda_device)
    a = torch.ones(len(uvw), dtype=torch.complex64, device=cuda_device)
    run = (lambda: plan.forward(sky_d)) if which == "forward" else (lambda: plan.adjoint(a))
    good = run().cpu()
    plan.last_stats()
    check(lib.viss_plan_debug_drop_copy(plan._h, 1), "viss_plan_debug_drop_copy")
    run()
    with pytest.raises(VissError, match="bounded device wait"):
        plan.last_stats()
    again = run().cpu()
    plan.last_stats()                                  # no error: the flag was per call
    assert torch.equal(again, good)
