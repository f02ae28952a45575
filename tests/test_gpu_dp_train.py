"""Data-parallel denoiser training (one gradient all-reduce per step), two ranks as
processes with the gloo backend.  Both ranks use one GPU: their kernels never wait on
each other (the all-reduce goes through the host).  Checks: the averaged gradient of
two half batches equals the full-batch gradient (relative L2 < 1e-4: the same per-pixel
arithmetic, only the order of the f32 sums differs), and after a step the ranks hold
bit-identical weights."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _batch(k, B, H, W):
    rng = np.random.default_rng(100 + k)
    rgb = rng.gamma(0.6, 0.5, (B, H, W, 3)).astype(np.float32)
    return (rgb, rng.uniform(0, 1, (B, H, W, 3)).astype(np.float32),
            rng.uniform(-1, 1, (B, H, W, 3)).astype(np.float32),
            (rgb * rng.uniform(0.5, 1.5, (B, H, W, 3))).astype(np.float32))


def _rank(rank, world, port, q):
    import datetime
    import sys

    import torch
    import torch.distributed as dist

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    from offlinerenderer_b200 import denoise_train, wrk

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        B, H, W = 2, 64, 128
        dn = wrk.Denoiser(seed=4)
        arrs = [wrk.DeviceArray.from_numpy(a) for a in _batch(rank, B, H, W)]
        g = torch.empty(dn.num_params, dtype=torch.float32, device="cuda:0")
        denoise_train.dp_step(dn, dist, g, *arrs, B, H, W, 1e-3)
        mean_grad = g.cpu().numpy()
        params = torch.tensor(dn.get_params())
        allp = [torch.empty_like(params) for _ in range(world)]
        dist.all_gather(allp, params)
        same = all(torch.equal(allp[0], p) for p in allp)
        err = None
        if rank == 0:
            full = [np.concatenate([a, b]) for a, b in zip(_batch(0, B, H, W), _batch(1, B, H, W))]
            ref = wrk.Denoiser(seed=4)
            _, gfull = ref.gradients(*[wrk.DeviceArray.from_numpy(a) for a in full], 2 * B, H, W)
            err = float(np.linalg.norm(mean_grad - gfull) / np.linalg.norm(gfull))
        q.put((rank, same, err))
    finally:
        dist.destroy_process_group()


def test_data_parallel_step_matches_full_batch(gpu):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=300)
    codes = [p.exitcode for p in ps]
    assert codes == [0, 0], codes
    res = {r: (same, err) for r, same, err in (q.get(timeout=5) for _ in range(2))}
    assert res[0][0] and res[1][0], "ranks hold different weights after the step"
    assert res[0][1] < 1e-4, res[0][1]
