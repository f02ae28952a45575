"""Open-loop load generator for the render server (the serving workload).

Requests arrive as a Poisson process at `rate` per second against one resident
scene; each has a random orbit camera (radius U(1,3) around the scene centre),
a resolution drawn from `resolutions` and spp from `spps`, and asks for the
learned denoiser.  The driver submits a request as soon as its arrival time has
passed, steps the server while anything is in flight, and takes every ready
result into device memory.  Latency = result ready - arrival (queueing included).
"""
from __future__ import annotations

import time

import numpy as np

from . import scenes, wrk
from .denoise_train import orbit_camera


def audit(server: "wrk.Server", renderer: "wrk.Renderer", scene: "wrk.Scene", jobs, ref_spp: int = 512,
          device: int = 0) -> list:
    """relMSE of served images against FP64-accumulated references: each audited
    request is served again (same camera, size, spp and seed, so the same samples),
    its denoised result and the plain render are compared with a ref_spp reference."""
    import torch

    from . import quality

    out = []
    for cam, st in jobs:
        H, W = st.height, st.width
        ref = quality.reference(renderer, scene, cam, st, total_spp=ref_spp, chunk=128, device=device)
        served = torch.empty((H, W, 3), dtype=torch.float32, device=f"cuda:{device}")
        tk = server.submit(scene, camera=cam, settings=st, denoise=True)
        server.wait(tk)
        server.result_device(tk, wrk.TensorPtr(served).ptr)
        plain, _, _, _ = quality.render(renderer, scene, cam, st, st.spp, 0, torch, device, guides=False)
        out.append({"size": W, "spp": st.spp, "relmse_served": quality.relmse(served, ref),
                    "relmse_plain": quality.relmse(plain, ref), "reference_spp": ref_spp})
    return out


def run(server: "wrk.Server", scene: "wrk.Scene", n_requests: int = 400, rate: float = 50.0, seed: int = 7,
        resolutions=(256, 512, 1024), spps=(1, 4, 16), denoise: bool = True, device: int = 0,
        audit_renderer=None, audit_requests: int = 4) -> dict:
    import torch

    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n_requests))
    jobs = []
    base = scene._data.settings
    for _ in range(n_requests):
        res = int(rng.choice(resolutions))
        spp = int(rng.choice(spps))
        cam = orbit_camera(rng, res, res)
        st = scenes.RenderSettings(res, res, spp, maxBounces=base.maxBounces,
                                   russianRouletteDepth=base.russianRouletteDepth, seed=base.seed)
        jobs.append((cam, st))
    out = torch.empty((max(resolutions) ** 2 * 3,), dtype=torch.float32, device=f"cuda:{device}")
    lat, wait, service, samples = [], [], [], 0
    pending = {}
    i = 0
    steps = 0
    busy_ms = 0.0
    t0 = time.perf_counter()
    while i < n_requests or pending:
        now = time.perf_counter() - t0
        while i < n_requests and arrivals[i] <= now:
            cam, st = jobs[i]
            t_sub = time.perf_counter() - t0
            tk = server.submit(scene, camera=cam, settings=st, denoise=denoise)
            pending[tk] = (arrivals[i], t_sub, st.width * st.height * st.spp)
            i += 1
        if not pending:
            time.sleep(min(2e-4, max(0.0, arrivals[i] - (time.perf_counter() - t0))) if i < n_requests else 0)
            continue
        s = server.step()
        steps += 1
        busy_ms += s["lastChunkMs"]
        for tk in [t for t in pending if server.ready(t)]:
            arr, t_sub, nsamp = pending.pop(tk)
            info = server.result_device(tk, wrk.TensorPtr(out).ptr)
            ready = t_sub + (info["readyMs"] - info["submitMs"]) / 1e3
            lat.append(ready - arr)
            wait.append((t_sub - arr) + (info["admitMs"] - info["submitMs"]) / 1e3)
            service.append((info["readyMs"] - info["admitMs"]) / 1e3)
            samples += nsamp
    wall = time.perf_counter() - t0
    lat_ms = np.asarray(lat) * 1e3
    checked = []
    if audit_renderer is not None and audit_requests:
        pick = np.random.default_rng(seed + 1).choice(n_requests, audit_requests, replace=False)
        small = [jobs[int(k)] for k in pick]
        # keep the audit bounded: references of the 1024^2 requests at 256^2 of the same view
        small = [(c, st) if st.width <= 512 else
                 (c, scenes.RenderSettings(256, 256, st.spp, maxBounces=st.maxBounces,
                                           russianRouletteDepth=st.russianRouletteDepth, seed=st.seed))
                 for c, st in small]
        checked = audit(server, audit_renderer, scene, small, device=device)
    return {"audit": checked, "requests": n_requests, "rate_per_s": rate, "resolutions": list(resolutions), "spps": list(spps),
            "denoised": denoise, "p50_ms": float(np.percentile(lat_ms, 50)), "p99_ms": float(np.percentile(lat_ms, 99)),
            "mean_ms": float(lat_ms.mean()), "max_ms": float(lat_ms.max()),
            "mean_wait_ms": float(np.mean(wait) * 1e3), "mean_service_ms": float(np.mean(service) * 1e3),
            "wall_s": wall, "steps": steps, "gpu_busy_frac": busy_ms / 1e3 / wall,
            "served_msamples_per_s": samples / wall / 1e6}
