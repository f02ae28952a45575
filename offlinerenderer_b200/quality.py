"""Image-quality measurement: FP64-accumulated references, relMSE, time-to-relMSE.

relMSE(x, r) = mean over pixels and channels of (x - r)^2 / (r^2 + 1e-2), with r
the FP64-accumulated high-spp reference of the same scene, camera and settings.

time_to_relmse: the plain renderer at `plain_spp` (256 for the scale test) sets
the quality bar; the denoised renderer searches the smallest spp whose denoised
image reaches that bar, and the ratio of GPU times (render + denoise vs plain
render) is the headline of the serving path.
"""
from __future__ import annotations

import numpy as np

from . import scenes, wrk


_Ptr = wrk.TensorPtr


def relmse(x, ref) -> float:
    """relMSE over the entries where the image is finite (non-finite entries are
    counted by `nonfinite`; a path that produced NaN is not a quality figure)."""
    import torch

    if isinstance(x, torch.Tensor):
        x64 = x.double()
        r64 = ref.double()
        e = (x64 - r64) ** 2 / (r64 * r64 + 1e-2)
        return float(e[torch.isfinite(e)].mean().item())
    x = np.asarray(x, np.float64)
    r = np.asarray(ref, np.float64)
    e = (x - r) ** 2 / (r * r + 1e-2)
    return float(np.mean(e[np.isfinite(e)]))


def nonfinite(x) -> int:
    import torch

    if isinstance(x, torch.Tensor):
        return int((~torch.isfinite(x)).sum().item())
    return int((~np.isfinite(np.asarray(x))).sum())


def _settings(st, spp):
    return scenes.RenderSettings(st.width, st.height, spp, maxBounces=st.maxBounces,
                                 russianRouletteDepth=st.russianRouletteDepth, useNEE=st.useNEE,
                                 fireflyClamp=st.fireflyClamp, seed=st.seed)


def render(renderer, scene, cam, st, spp, sample_offset, torch, device=0, guides=True):
    """(rgb, albedo, normal) device tensors (H, W, 3) of one render; gpu ms."""
    H, W = st.height, st.width
    rgb = torch.empty((H, W, 3), dtype=torch.float32, device=f"cuda:{device}")
    alb = torch.empty_like(rgb) if guides else None
    nrm = torch.empty_like(rgb) if guides else None
    s = renderer.render_device(scene, None, camera=cam, settings=_settings(st, spp), d_rgb_ptr=_Ptr(rgb).ptr,
                               d_albedo=_Ptr(alb) if guides else None, d_normal=_Ptr(nrm) if guides else None,
                               sample_offset=sample_offset)
    return rgb, alb, nrm, s["gpuMs"]


def reference(renderer, scene, cam, st, total_spp=4096, chunk=256, sample_offset=1 << 20, device=0, stats=None):
    """FP64-accumulated reference: chunks of `chunk` spp (f32 per-pixel sums inside a
    chunk) summed in float64 over disjoint sample ranges.  A chunk whose pixel sum
    is not finite (a path produced NaN or inf) is left out of that pixel's average;
    `stats["dropped"]` counts such pixel-chunks."""
    import torch

    acc = torch.zeros((st.height, st.width, 3), dtype=torch.float64, device=f"cuda:{device}")
    cnt = torch.zeros_like(acc)
    n = 0
    dropped = 0
    while n < total_spp:
        k = min(chunk, total_spp - n)
        rgb, _, _, _ = render(renderer, scene, cam, st, k, sample_offset + n, torch, device, guides=False)
        ok = torch.isfinite(rgb)
        dropped += int((~ok).sum().item())
        acc += torch.where(ok, rgb.double() * k, torch.zeros_like(acc))
        cnt += ok.double() * k
        n += k
    if stats is not None:
        stats["dropped"] = dropped
    return acc / cnt.clamp(min=1)


def relmse_trimmed(x, ref, drop: float = 1e-3) -> float:
    """relMSE with the largest `drop` fraction of per-pixel errors (mean over the
    three channels) left out: the figure without the firefly tail."""
    import torch

    x64 = torch.as_tensor(x).double()
    r64 = torch.as_tensor(ref).double().to(x64.device)
    e = ((x64 - r64) ** 2 / (r64 * r64 + 1e-2)).mean(-1).flatten()
    e = e[torch.isfinite(e)]
    keep = max(1, int(e.numel() * (1.0 - drop)))
    return float(torch.sort(e).values[:keep].mean().item())


def time_to_relmse(renderer, denoiser, scene, cam, st, ref, plain_spp=256, search=(1, 2, 4, 8, 16, 32, 64, 128),
                   device=0, repeats=2, level=1e-3, plain_search=(256, 512, 1024, 2048),
                   denoised_search=(1, 4, 16, 64, 256)):
    """Plain render at plain_spp vs render+denoise at increasing spp until the
    denoised relMSE reaches the plain one.  Times are device times (CUDA events).

    Also reports, for the fixed relMSE `level` (1e-3), the smallest spp of
    plain_search and of denoised_search at which each arm reaches it -- raw and
    with the top 0.1 % of per-pixel errors left out (the firefly tail) -- or None
    when neither spp of the search does."""
    import torch

    def timed(fn, reps=repeats):
        best = None
        out = None
        for _ in range(reps):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            out = fn()
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
        return out, best

    H, W = st.height, st.width

    def denoised_run(s):
        rgb, alb, nrm, _ = render(renderer, scene, cam, st, s, 0, torch, device, True)
        out = torch.empty_like(rgb)
        denoiser.infer_device(_Ptr(rgb), _Ptr(alb), _Ptr(nrm), 1, H, W, _Ptr(out))
        return rgb, out

    (plain, _, _, _), plain_ms = timed(lambda: render(renderer, scene, cam, st, plain_spp, 0, torch, device, False))
    bar = relmse(plain, ref)
    bar_trimmed = relmse_trimmed(plain, ref)
    plain_nonfinite = nonfinite(plain)
    rows = []
    found = None
    for s in search:
        (noisy, den), ms = timed(lambda: denoised_run(s))
        r = {"spp": s, "ms": ms, "relmse_noisy": relmse(noisy, ref), "relmse_denoised": relmse(den, ref),
             "relmse_denoised_trimmed": relmse_trimmed(den, ref), "nonfinite_denoised": nonfinite(den)}
        rows.append(r)
        if found is None and r["relmse_denoised"] <= bar:
            found = r
            break

    # the fixed level: both arms, raw and trimmed
    plain_rows = []
    for s in plain_search:
        (img, _, _, _), ms = timed(lambda: render(renderer, scene, cam, st, s, 0, torch, device, False), 1)
        plain_rows.append({"spp": s, "ms": ms, "relmse": relmse(img, ref), "relmse_trimmed": relmse_trimmed(img, ref)})
        del img
    den_rows = []
    for s in denoised_search:
        (_, den), ms = timed(lambda: denoised_run(s), 1)
        den_rows.append({"spp": s, "ms": ms, "relmse": relmse(den, ref), "relmse_trimmed": relmse_trimmed(den, ref)})
        del den

    def first(rows_, key):
        hit = [r for r in rows_ if r[key] <= level]
        return {"spp": hit[0]["spp"], "ms": hit[0]["ms"]} if hit else None

    at_level = {"level": level, "plain_search": plain_rows, "denoised_search": den_rows,
                "plain": first(plain_rows, "relmse"), "denoised": first(den_rows, "relmse"),
                "plain_trimmed": first(plain_rows, "relmse_trimmed"),
                "denoised_trimmed": first(den_rows, "relmse_trimmed"),
                "trimmed": "top 0.1 % of per-pixel errors left out"}
    return {"plain_spp": plain_spp, "plain_ms": plain_ms, "plain_relmse": bar, "plain_relmse_trimmed": bar_trimmed,
            "plain_nonfinite": plain_nonfinite, "search": rows,
            "denoised_spp": found["spp"] if found else None, "denoised_ms": found["ms"] if found else None,
            "time_ratio": (found["ms"] / plain_ms) if found else None, "at_level": at_level}
