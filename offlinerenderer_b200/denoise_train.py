"""Training of the learned denoiser, on the GPU end to end.

    python -m offlinerenderer_b200.denoise_train [--scenes 16] [--views 24] [--steps 12000] [--out PATH]
    python -m offlinerenderer_b200.denoise_train --evaluate label=weights.wrkw [label=...]
    python -m torch.distributed.run --nproc-per-node N -m offlinerenderer_b200.denoise_train ...   (data parallel)

The renderer itself generates the training pairs: seeded variants of the
scale-test scene (heightfield + 250 icospheres of the five BSDFs + 64 emissive
triangles; scene seeds 101.. -- the benchmark scene, seed 1, is held out),
seen from the scale-test camera and from random orbit cameras (radius U(1,3)
around the scene centre, the serving workload's poses).  For every view it
renders a high-spp target and noisy inputs at 1..32 spp from disjoint sample
indices (radiance + first-hit albedo + normal, the 9 channels libWR gives its
denoiser, libWR/src/internal/denoiser.cpp:98-116).  Training takes random crops
with random flips and runs the network's forward, backward and Adam step through
wrk_denoiser_train_step (tcgen05 convolutions).  torch only holds the data in
device memory and gathers the crops.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time

import numpy as np

from . import scenes, wrk

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_WEIGHTS = os.path.join(HERE, "weights", "unet_scale.wrkw")
INPUT_SPPS = (1, 2, 4, 8, 16, 32)


def relmse(x: np.ndarray, ref: np.ndarray) -> float:
    """mean over pixels and channels of (x - r)^2 / (r^2 + 1e-2)."""
    x = np.asarray(x, np.float64)
    r = np.asarray(ref, np.float64)
    return float(np.mean((x - r) ** 2 / (r * r + 1e-2)))


def orbit_camera(rng, width: int, height: int, center=(0.5, 0.05, 0.5)) -> scenes.Camera:
    """Camera on an orbit of radius U(1,3) around the scene centre, looking at it."""
    r = float(rng.uniform(1.0, 3.0))
    th = float(rng.uniform(0.0, 2.0 * math.pi))
    el = float(rng.uniform(math.radians(20.0), math.radians(55.0)))
    c = np.asarray(center, np.float64)
    pos = c + r * np.array([math.cos(el) * math.cos(th), math.sin(el), math.cos(el) * math.sin(th)])
    fov = float(np.clip(2.0 * math.atan(0.8 / r), math.radians(15.0), math.radians(60.0)))
    return scenes.Camera(position=tuple(float(v) for v in pos), target=tuple(float(v) for v in c), up=(0.0, 1.0, 0.0),
                         fovY=fov, aspect=float(np.float32(width) / np.float32(height)))


_Ptr = wrk.TensorPtr


def render_views(scene, renderer, cams, size, spp, sample_offset, torch, device, out=None):
    """Renders every camera at `spp` into (V, size, size, 3) rgb / albedo / normal tensors
    (new ones, or the given `out` triple of views)."""
    V = len(cams)
    if out is None:
        rgb = torch.empty((V, size, size, 3), dtype=torch.float32, device=f"cuda:{device}")
        alb = torch.empty_like(rgb)
        nrm = torch.empty_like(rgb)
    else:
        rgb, alb, nrm = out
    st = scene._data.settings
    st = scenes.RenderSettings(size, size, spp, maxBounces=st.maxBounces, russianRouletteDepth=st.russianRouletteDepth,
                               seed=st.seed, useNEE=st.useNEE)
    for v, cam in enumerate(cams):
        renderer.render_device(scene, None, camera=cam, settings=st, d_rgb_ptr=_Ptr(rgb[v]).ptr,
                               d_albedo=_Ptr(alb[v]), d_normal=_Ptr(nrm[v]), sample_offset=sample_offset)
    return rgb, alb, nrm


def generate(scene_seeds, views, size, target_spp, device=0, log=print):
    """Renders the training set straight into preallocated device tensors (views of
    all scenes stacked); returns a dict: "target" -> (V, size, size, 3) and, per input
    spp, (rgb, albedo, normal)."""
    import torch

    rng = np.random.default_rng(12345)
    renderer = wrk.Renderer(device=device)
    V = len(scene_seeds) * views
    shape = (V, size, size, 3)
    dev = f"cuda:{device}"
    data = {"target": torch.empty(shape, dtype=torch.float32, device=dev)}
    scratch = (torch.empty((views, size, size, 3), dtype=torch.float32, device=dev),
               torch.empty((views, size, size, 3), dtype=torch.float32, device=dev))
    for k in INPUT_SPPS:
        data[k] = tuple(torch.empty(shape, dtype=torch.float32, device=dev) for _ in range(3))
    t0 = time.time()
    for j, s in enumerate(scene_seeds):
        sd = scenes.scale_test(size, size, 4, seed=s)
        scene = wrk.Scene.from_data(sd, device)
        cams = [scenes.Camera(position=sd.camera.position, target=sd.camera.target, up=sd.camera.up,
                              fovY=sd.camera.fovY, aspect=1.0)]
        cams += [orbit_camera(rng, size, size) for _ in range(views - 1)]
        sl = slice(j * views, (j + 1) * views)
        render_views(scene, renderer, cams, size, target_spp, 0, torch, device,
                     out=(data["target"][sl], scratch[0], scratch[1]))
        off = target_spp
        for k in INPUT_SPPS:
            render_views(scene, renderer, cams, size, k, off, torch, device, out=tuple(t[sl] for t in data[k]))
            off += k
        del scene
        log(f"scene seed {s}: {len(cams)} views rendered ({time.time() - t0:.1f} s)")
    torch.cuda.synchronize()
    return data


def dp_step(dn, dist, gbuf, d_rgb, d_alb, d_nrm, d_tgt, B, H, W, lr) -> float:
    """One data-parallel step: local forward / backward, gradients averaged across
    ranks with one all-reduce, then the same Adam step on every rank (the weights
    stay identical because every rank starts from the same seed)."""
    loss = dn.gradients_device(d_rgb, d_alb, d_nrm, d_tgt, B, H, W)
    dn.grads_copy(_Ptr(gbuf).ptr)
    dist.all_reduce(gbuf)
    gbuf /= dist.get_world_size()
    dn.grads_set(_Ptr(gbuf).ptr)  # waits for the all-reduce and the division on torch's stream
    dn.apply(lr)
    return loss


def train(data, steps, batch=16, crop=128, lr=1e-3, seed=1, device=0, log=print, dn=None, dist=None):
    import torch

    rank = dist.get_rank() if dist is not None else 0
    world = dist.get_world_size() if dist is not None else 1
    g = torch.Generator(device=f"cuda:{device}")
    g.manual_seed(seed + 7919 * rank)  # every rank draws its own crops
    dn = dn or wrk.Denoiser(device=device, seed=seed)
    gbuf = torch.empty(dn.num_params, dtype=torch.float32, device=f"cuda:{device}") if world > 1 else None
    V, S = data["target"].shape[0], data["target"].shape[1]
    losses = []
    t0 = time.time()
    for it in range(steps):
        k = INPUT_SPPS[int(torch.randint(len(INPUT_SPPS), (1,), generator=g, device=f"cuda:{device}").item())]
        vi = torch.randint(V, (batch,), generator=g, device=f"cuda:{device}")
        oy = torch.randint(S - crop + 1, (batch,), generator=g, device=f"cuda:{device}")
        ox = torch.randint(S - crop + 1, (batch,), generator=g, device=f"cuda:{device}")
        ar = torch.arange(crop, device=f"cuda:{device}")
        yy = (oy[:, None] + ar[None, :])[:, :, None]
        xx = (ox[:, None] + ar[None, :])[:, None, :]
        b = vi[:, None, None]

        def take(t):
            return t[b, yy, xx].contiguous()

        rgb, alb, nrm = (take(t) for t in data[k])
        tgt = take(data["target"])
        if it % 2:
            rgb, alb, nrm, tgt = (t.flip(2).contiguous() for t in (rgb, alb, nrm, tgt))
            nrm[..., 0] = -nrm[..., 0]
        cur = lr * (0.1 + 0.9 * 0.5 * (1.0 + math.cos(math.pi * it / max(1, steps))))
        if world > 1:
            loss = dp_step(dn, dist, gbuf, _Ptr(rgb), _Ptr(alb), _Ptr(nrm), _Ptr(tgt), batch, crop, crop, cur)
        else:
            loss = dn.train_step(_Ptr(rgb), _Ptr(alb), _Ptr(nrm), _Ptr(tgt), batch, crop, crop, cur)
        losses.append(loss)
        if it % 250 == 0 or it == steps - 1:
            log(f"step {it}: loss {np.mean(losses[-50:]):.4f} lr {cur:.2e} ({time.time() - t0:.1f} s)")
    torch.cuda.synchronize()
    return dn, losses, time.time() - t0


def evaluate(weights, size=256, spps=(1, 4, 16), ref_spp=4096, device=0, log=print) -> dict:
    """Held-out quality of denoiser weights: the benchmark scene (scale test, seed 1,
    never trained on) from its own camera and 3 orbit views, at `spps`; relMSE of the
    denoised and of the noisy image against an FP64-accumulated ref_spp reference.
    `weights` maps a label to a WRKUNET1 file; every file is scored on the same
    renders."""
    import torch

    from . import quality

    renderer = wrk.Renderer(device=device)
    sd = scenes.scale_test(size, size, 4, seed=1)
    scene = wrk.Scene.from_data(sd, device)
    rng = np.random.default_rng(777)
    cams = [scenes.Camera(position=sd.camera.position, target=sd.camera.target, up=sd.camera.up,
                          fovY=sd.camera.fovY, aspect=1.0)] + [orbit_camera(rng, size, size) for _ in range(3)]
    st0 = scenes.RenderSettings(size, size, 1, maxBounces=sd.settings.maxBounces,
                                russianRouletteDepth=sd.settings.russianRouletteDepth, seed=sd.settings.seed)
    dns = {}
    for label, path in weights.items():
        dns[label] = wrk.Denoiser(device=device)
        load_weights(dns[label], path)
    rows = []
    for v, cam in enumerate(cams):
        ref = quality.reference(renderer, scene, cam, st0, total_spp=ref_spp, chunk=512, device=device)
        for s in spps:
            rgb, alb, nrm, _ = quality.render(renderer, scene, cam, st0, s, 0, torch, device, True)
            row = {"view": v, "spp": s, "noisy": quality.relmse(rgb, ref)}
            for label, dn in dns.items():
                out = torch.empty_like(rgb)
                dn.infer_device(_Ptr(rgb), _Ptr(alb), _Ptr(nrm), 1, size, size, _Ptr(out))
                row[label] = quality.relmse(out, ref)
            rows.append(row)
            log(json.dumps(row))
    summary = {k: float(np.mean([r[k] for r in rows])) for k in ["noisy"] + list(weights)}
    return {"views": len(cams), "size": size, "spps": list(spps), "reference_spp": ref_spp, "rows": rows,
            "mean_relmse": summary}


def write_weights(path: str, params: np.ndarray, meta: dict) -> None:
    """WRKUNET1 file: magic, u64 count, u64 metadata bytes, count bf16 bit patterns
    (the precision inference uses), JSON metadata.  wrk_denoiser_load reads it."""
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    bits = wrk.to_bf16_bits(np.asarray(params, np.float32))
    m = json.dumps(meta).encode()
    with open(path, "wb") as f:
        f.write(b"WRKUNET1")
        f.write(np.asarray([bits.size, len(m)], np.uint64).tobytes())
        f.write(bits.tobytes())
        f.write(m)


def read_meta(path: str) -> dict:
    with open(path, "rb") as f:
        if f.read(8) != b"WRKUNET1":
            raise ValueError(f"{path} is not a WRKUNET1 weights file")
        count, mlen = np.frombuffer(f.read(16), np.uint64)
        f.seek(24 + 2 * int(count))
        return json.loads(f.read(int(mlen)).decode())


def save_weights(dn: "wrk.Denoiser", path: str, meta: dict) -> None:
    write_weights(path, dn.get_params(), meta)


def load_weights(dn: "wrk.Denoiser", path: str = DEFAULT_WEIGHTS) -> dict:
    dn.load(path)
    return read_meta(path)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scenes", type=int, default=16)
    ap.add_argument("--views", type=int, default=24)
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--target-spp", type=int, default=1024)
    ap.add_argument("--steps", type=int, default=12000)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    ap.add_argument("--log", default=None)
    ap.add_argument("--evaluate", nargs="*", default=None, metavar="LABEL=PATH",
                    help="only score the given weights on the held-out benchmark scene and print JSON")
    args = ap.parse_args()
    if args.evaluate is not None:
        res = evaluate(dict(a.split("=", 1) for a in args.evaluate))
        print(json.dumps(res["mean_relmse"]))
        print(json.dumps(res))
        return
    logf = open(args.log, "w") if args.log else None

    def log(msg):
        print(msg, flush=True)
        if logf:
            logf.write(msg + "\n")
            logf.flush()

    import torch

    # one process per GPU under torch.distributed.run: every rank renders its own
    # share of the scene variants and the gradients are averaged each step
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    t0 = time.time()
    seeds = list(range(101, 101 + args.scenes))[rank::world]
    data = generate(seeds, args.views, args.size, args.target_spp, device=local, log=log)
    gen_s = time.time() - t0
    dn, losses, train_s = train(data, args.steps, batch=args.batch, lr=args.lr, device=local, log=log, dist=dist)
    meta = {"scenes": list(range(101, 101 + args.scenes)), "views": args.views, "size": args.size,
            "target_spp": args.target_spp, "input_spps": list(INPUT_SPPS), "steps": args.steps, "batch": args.batch,
            "crop": 128, "lr": args.lr, "gen_s": gen_s, "train_s": train_s,
            "final_loss": float(np.mean(losses[-100:]))}
    meta["ranks"] = world
    if rank == 0:
        save_weights(dn, args.out, meta)
        log(json.dumps(meta))
    del data
    torch.cuda.empty_cache()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
