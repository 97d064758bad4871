"""Multi-rank path on CPU: two gloo ranks take the reference's round-robin days
(vissgen3d_blockage.cu:279), compute per-day images (here with the CPU oracle,
on a tiny observation) and all-reduce them into the notebooks' summed image
(healpix3d_blockage.ipynb:103-116); the result equals the single-process sum.
Also the max-over-ranks timing reduction bench.py uses."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _day_image(day):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    from oracle import oracle as O
    from viss_optimize_3d_b200 import synth

    cfg = synth.scaled(synth.CONFIGS["c2"], nside=2, n_snap=3, n_sat=3)
    import dataclasses
    obs = synth.make_observation(dataclasses.replace(cfg, day=float(day)))
    _, _, xyz = O.pix2ang(cfg.nside)
    lmn = O.lmn_from_xyz(xyz)
    occ = O.occulters(obs.occ_sat_positions, synth.R_MOON, 0)
    uvw = obs.uvw(1e7)
    V = O.forward(uvw, lmn, obs.sky, obs.refs, occ, nthreads=1)
    img = O.adjoint(uvw, V, lmn, obs.refs, occ, nthreads=1)
    if day == 3:
        img[0] = np.nan          # the notebooks' nan_to_num path
    return torch.as_tensor(img)


def _worker(rank, world, port, n_days, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from viss_optimize_3d_b200 import replicas
        days = replicas.days_for_rank(n_days, rank, world)
        assert days == list(range(1 + rank, n_days + 1, world))
        total = replicas.accumulate_days(n_days, 48, _day_image)
        mx = replicas.max_over_ranks([float(rank), 10.0 - rank])
        out[rank] = (total.numpy().tolist(), mx)
    finally:
        dist.destroy_process_group()


def test_two_rank_day_sum_matches_single_process():
    world, n_days = 2, 5
    port = _free_port()
    manager = mp.get_context("spawn").Manager()
    out = manager.dict()
    mp.start_processes(_worker, args=(world, port, n_days, out), nprocs=world, start_method="spawn")
    ref = sum(torch.nan_to_num(_day_image(d), nan=0.0) for d in range(1, n_days + 1)).numpy()
    for rank in range(world):
        total, mx = out[rank]
        np.testing.assert_allclose(total, ref, rtol=1e-12, atol=1e-12)
        assert mx == [1.0, 10.0]


def _bench_worker(rank, world, port, steps, out):
    """The day-sum path of bench.py --gpus N: every step adds this rank's day
    image into an FP64 sum (replicas.add_day_image, non-finite pixels as 0),
    and the last step all-reduces the sums (replicas.sum_images).  CPU
    tensors stand in for the device images."""
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from viss_optimize_3d_b200 import replicas
        day = replicas.days_for_rank(world, rank, world)[0]
        total = torch.zeros(48, dtype=torch.float64)
        for i in range(steps):
            img = _day_image(day).to(torch.float32)
            replicas.add_day_image(total, img)
            if i == steps - 1:
                replicas.sum_images(total)
        out[rank] = total.numpy().tolist()
    finally:
        dist.destroy_process_group()


def test_two_rank_bench_day_sum():
    world, steps = 2, 3
    port = _free_port()
    manager = mp.get_context("spawn").Manager()
    out = manager.dict()
    mp.start_processes(_bench_worker, args=(world, port, steps, out), nprocs=world, start_method="spawn")
    ref = np.zeros(48)
    for day in (1, 2):
        img = torch.nan_to_num(_day_image(day).to(torch.float32).double(), nan=0.0).numpy()
        ref += steps * img
    for rank in range(world):
        np.testing.assert_allclose(out[rank], ref, rtol=1e-12, atol=1e-12)


def test_days_for_rank_validates():
    from viss_optimize_3d_b200 import replicas
    assert replicas.days_for_rank(450, 3, 8)[:3] == [4, 12, 20]
    assert sum(len(replicas.days_for_rank(450, r, 8)) for r in range(8)) == 450
    with pytest.raises(ValueError):
        replicas.days_for_rank(10, 2, 2)
