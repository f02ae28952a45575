"""Sample-split rendering across ranks (the multi-GPU path of bench.py), on CPU.

Two gloo ranks each render their own sample range ([rank*spp, (rank+1)*spp)) of the
same image with the oracle, sum the per-rank frames with all_reduce (the frame
combine bench.py does with NCCL), and rank 0 compares the result with one render of
all samples: the RNG is keyed by (pixel, sample), so only the order of the float
additions differs.
"""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, spp, out_path):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import torch
    import torch.distributed as dist

    import pyoracle
    from offlinerenderer_b200 import scenes

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sd = scenes.cornell(24, 20, spp, seed=3)
        rgb, _, _, _ = pyoracle.Oracle().scene(sd).render(sample_begin=rank * spp, threads=2)
        frame = torch.from_numpy((rgb.astype(np.float32) * np.float32(spp)).copy())
        dist.all_reduce(frame)  # sum of the ranks' sample ranges
        if rank == 0:
            np.save(out_path, (frame / (world * spp)).numpy())
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_sample_split_over_two_gloo_ranks(tmp_path, oracle):
    import torch.multiprocessing as mp

    spp, world = 4, 2
    out = str(tmp_path / "frame.npy")
    mp.start_processes(_worker, args=(world, _free_port(), spp, out), nprocs=world, join=True, start_method="spawn")
    combined = np.load(out)
    from offlinerenderer_b200 import scenes

    full = oracle.scene(scenes.cornell(24, 20, world * spp, seed=3)).render()[0]
    np.testing.assert_allclose(combined, full, rtol=1e-5, atol=1e-6)
    # and the split really covers different samples than rank 0 alone
    half = oracle.scene(scenes.cornell(24, 20, spp, seed=3)).render()[0]
    assert np.abs(half - full).max() > 1e-3
