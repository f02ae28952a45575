"""Open-loop load generator for the render server (the serving workload).

Requests arrive as a Poisson process at `rate` per second against one resident
scene; each has an orbit camera (radius U(1,3) around the scene centre) drawn
from a fixed set of poses, a resolution drawn from `resolutions` and spp from
`spps`, and asks for the learned denoiser.  The driver submits a request as soon as its arrival time has
passed, steps the server while anything is in flight, and takes every ready
result into device memory.  Latency = result ready - arrival (queueing included).
"""
from __future__ import annotations

import time

import numpy as np

from . import scenes, wrk
from .denoise_train import orbit_camera


def _group_summary(rows) -> dict:
    out = {}
    for key in sorted({(r["size"], r["spp"]) for r in rows}):
        g = [r for r in rows if (r["size"], r["spp"]) == key]
        served = np.asarray([r["relmse_served"] for r in g])
        out[f"{key[0]}^2@{key[1]}spp"] = {"requests": len(g), "relmse_served_mean": float(served.mean()),
                                         "relmse_served_max": float(served.max()),
                                         "relmse_plain_same_spp": float(np.mean([r["relmse_plain"] for r in g]))}
    return out


def run(server: "wrk.Server", scene: "wrk.Scene", n_requests: int = 1000, rate: float = 50.0, seed: int = 7,
        resolutions=(256, 512, 1024), spps=(1, 4, 16), denoise: bool = True, device: int = 0,
        quality_renderer=None, poses: int = 6, ref_spp: int = 1024) -> dict:
    """Serves n_requests Poisson arrivals; with quality_renderer, every served image
    is then scored: relMSE against an FP64-accumulated ref_spp reference of its
    camera pose and size (one reference per (pose, size): the cameras are drawn from
    a fixed set of `poses` orbit cameras so references can be shared), next to the
    relMSE of the plain render at the same spp (the fallback without the denoiser)."""
    import torch

    from . import quality

    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n_requests))
    pose_cams = [orbit_camera(np.random.default_rng(seed * 1000 + k), 1, 1) for k in range(poses)]
    jobs = []
    base = scene._data.settings
    for _ in range(n_requests):
        res = int(rng.choice(resolutions))
        spp = int(rng.choice(spps))
        pose = int(rng.integers(poses))
        st = scenes.RenderSettings(res, res, spp, maxBounces=base.maxBounces,
                                   russianRouletteDepth=base.russianRouletteDepth, seed=base.seed)
        jobs.append((pose, st))
    keep = quality_renderer is not None
    results = [None] * n_requests
    out = torch.empty((max(resolutions) ** 2 * 3,), dtype=torch.float32, device=f"cuda:{device}")
    if keep:  # every result is kept on the device and scored after the timed run
        results = [torch.empty((st.height, st.width, 3), dtype=torch.float32, device=f"cuda:{device}")
                   for _, st in jobs]
    lat, wait, service, samples = [], [], [], 0
    pending = {}
    i = 0
    steps = 0
    busy_ms = 0.0
    t0 = time.perf_counter()
    while i < n_requests or pending:
        now = time.perf_counter() - t0
        while i < n_requests and arrivals[i] <= now:
            pose, st = jobs[i]
            t_sub = time.perf_counter() - t0
            tk = server.submit(scene, camera=pose_cams[pose], settings=st, denoise=denoise)
            pending[tk] = (i, arrivals[i], t_sub, st.width * st.height * st.spp)
            i += 1
        if not pending:
            time.sleep(min(2e-4, max(0.0, arrivals[i] - (time.perf_counter() - t0))) if i < n_requests else 0)
            continue
        s = server.step()
        steps += 1
        busy_ms += s["lastChunkMs"]
        for tk in [t for t in pending if server.ready(t)]:
            k, arr, t_sub, nsamp = pending.pop(tk)
            dst = results[k] if keep else out
            info = server.result_device(tk, wrk.TensorPtr(dst).ptr)
            ready = t_sub + (info["readyMs"] - info["submitMs"]) / 1e3
            lat.append(ready - arr)
            wait.append((t_sub - arr) + (info["admitMs"] - info["submitMs"]) / 1e3)
            service.append((info["readyMs"] - info["admitMs"]) / 1e3)
            samples += nsamp
    wall = time.perf_counter() - t0
    lat_ms = np.asarray(lat) * 1e3
    res = {"requests": n_requests, "rate_per_s": rate, "resolutions": list(resolutions), "spps": list(spps),
           "denoised": denoise, "p50_ms": float(np.percentile(lat_ms, 50)), "p99_ms": float(np.percentile(lat_ms, 99)),
           "mean_ms": float(lat_ms.mean()), "max_ms": float(lat_ms.max()),
           "mean_wait_ms": float(np.mean(wait) * 1e3), "mean_service_ms": float(np.mean(service) * 1e3),
           "wall_s": wall, "steps": steps, "gpu_busy_frac": busy_ms / 1e3 / wall,
           "served_msamples_per_s": samples / wall / 1e6, "camera_poses": poses}
    if keep:
        refs, plains, rows = {}, {}, []
        for k, (pose, st) in enumerate(jobs):
            if (pose, st.width) not in refs:
                refs[(pose, st.width)] = quality.reference(quality_renderer, scene, pose_cams[pose], st,
                                                           total_spp=ref_spp, chunk=256, device=device).float()
            ref = refs[(pose, st.width)]
            if (pose, st.width, st.spp) not in plains:
                plain, _, _, _ = quality.render(quality_renderer, scene, pose_cams[pose], st, st.spp, 0, torch,
                                                device, guides=False)
                plains[(pose, st.width, st.spp)] = quality.relmse(plain, ref)
            rows.append({"size": st.width, "spp": st.spp, "relmse_served": quality.relmse(results[k], ref),
                         "relmse_plain": plains[(pose, st.width, st.spp)]})
        served = np.asarray([r["relmse_served"] for r in rows])
        res["quality"] = {
            "reference": f"FP64-accumulated {ref_spp} spp per (pose, size): {len(refs)} references",
            "relmse_served_mean": float(served.mean()), "relmse_served_p50": float(np.median(served)),
            "relmse_served_max": float(served.max()),
            "relmse_plain_same_spp_mean": float(np.mean([r["relmse_plain"] for r in rows])),
            "by_size_spp": _group_summary(rows),
            "relmse_per_request": [float(f"{v:.4g}") for v in served]}
    return res
