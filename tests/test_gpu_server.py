"""Serving loop on the GPU: continuous batching of requests with different sizes,
spp, cameras and scenes in one set of wavefront queues.

Tolerance for "the same alone and in the mix": the RNG is keyed by (seed,
pixel, sample), so every path is identical; only the order of the f32 atomic
sums into a pixel changes, bounding the difference by a few ulps of the sum:
|a - b| <= 1e-5 * |b| + 1e-6 per channel.
"""
import numpy as np
import pytest

from offlinerenderer_b200 import scenes

pytestmark = pytest.mark.gpu


def _close(a, b):
    return np.all(np.abs(a - b) <= 1e-5 * np.abs(b) + 1e-6)


def _cam(pos, target=(0.5, 0.5, 0.0), aspect=1.0, fov=40.0):
    return scenes.Camera(position=pos, target=target, up=(0.0, 1.0, 0.0), fovY=float(scenes._radians(fov)),
                         aspect=aspect)


def _settings(w, h, spp, base):
    return scenes.RenderSettings(w, h, spp, maxBounces=base.maxBounces, russianRouletteDepth=base.russianRouletteDepth,
                                 seed=base.seed)


@pytest.fixture(scope="module")
def world(gpu):
    cb = gpu.Scene.from_data(scenes.cornell(64, 64, 4, seed=1))
    sc = gpu.Scene.from_data(scenes.material_showcase(64, 64, 4, seed=2, tex_size=256))
    return cb, sc


def _solo(gpu, scene, cam, st):
    r = gpu.Renderer(capacity=1 << 16)
    return r.render(scene, camera=cam, settings=st)


def test_requests_same_alone_and_in_the_mix(gpu, world):
    cb, sc = world
    base = cb._data.settings
    jobs = [(cb, _cam((0.5, 0.5, -1.4)), _settings(64, 64, 8, base)),
            (cb, _cam((0.3, 0.6, -1.2), aspect=2.0), _settings(96, 48, 4, base)),
            (sc, sc._data.camera, _settings(64, 64, 6, sc._data.settings)),
            (cb, _cam((0.7, 0.4, -1.6)), _settings(40, 24, 16, base))]  # not a multiple of the 8x4 tile
    srv = gpu.Server(capacity=1 << 15)
    tickets = [srv.submit(s, camera=c, settings=st) for s, c, st in jobs]
    for t in tickets:
        srv.wait(t)
    for t, (s, c, st) in zip(tickets, jobs):
        rgb, alb, nrm, info = srv.result(t)
        solo = _solo(gpu, s, c, st)
        assert _close(rgb, solo.rgb) and _close(alb, solo.albedo) and _close(nrm, solo.normal)
        assert info["width"] == st.width and info["spp"] == st.spp


def test_continuous_admission_and_limits(gpu, world):
    cb, _ = world
    base = cb._data.settings
    srv = gpu.Server(capacity=1 << 14, max_requests=2, pool_bytes=64 * 64 * 96 * 2)
    first = srv.submit(cb, settings=_settings(64, 64, 32, base))
    st = srv.step()
    assert st["running"] == 1
    # a request arriving while the first is in flight joins the running wavefront
    second = srv.submit(cb, camera=_cam((0.4, 0.5, -1.3)), settings=_settings(64, 64, 4, base))
    extra = [srv.submit(cb, camera=_cam((0.5, 0.45, -1.5 - 0.1 * k)), settings=_settings(64, 64, 2, base))
             for k in range(3)]
    # a ready request holds its pool region until its result is taken: take results
    # as they come so the queued ones can be admitted
    max_running = 0
    results = {}
    pending = [first, second] + extra
    for _ in range(100000):
        if not pending:
            break
        st = srv.step()
        max_running = max(max_running, st["running"])
        for t in [t for t in pending if srv.ready(t)]:
            results[t] = srv.result(t)
            pending.remove(t)
    assert not pending, "requests did not finish"
    assert max_running <= 2
    r1, r2 = results[first][3], results[second][3]
    assert r2["admitMs"] < r1["readyMs"], "second request was not admitted while the first was in flight"
    for k, t in enumerate(extra):
        solo = _solo(gpu, cb, _cam((0.5, 0.45, -1.5 - 0.1 * k)), _settings(64, 64, 2, base))
        assert _close(results[t][0], solo.rgb)


def test_wait_reports_a_request_that_cannot_be_admitted(gpu, world):
    cb, _ = world
    base = cb._data.settings
    srv = gpu.Server(capacity=1 << 14, pool_bytes=32 * 32 * 96)  # room for one 32x32 request
    a = srv.submit(cb, settings=_settings(32, 32, 2, base))
    b = srv.submit(cb, settings=_settings(32, 32, 2, base))
    srv.wait(a)  # ready, but its pool region stays held until the result is taken
    with pytest.raises(gpu.WrkError):
        srv.wait(b)
    srv.result(a)
    srv.wait(b)
    assert srv.result(b)[3]["spp"] == 2


def test_request_larger_than_pool_rejected(gpu, world):
    cb, _ = world
    srv = gpu.Server(capacity=1 << 14, pool_bytes=1 << 20)
    with pytest.raises(gpu.WrkError):
        srv.submit(cb, settings=_settings(512, 512, 1, cb._data.settings))


def test_denoised_requests(gpu, world):
    cb, _ = world
    base = cb._data.settings
    dn = gpu.Denoiser(seed=3)
    srv = gpu.Server(capacity=1 << 15)
    srv.set_denoiser(dn)
    st = _settings(64, 64, 4, base)
    t = srv.submit(cb, settings=st, denoise=True)
    srv.wait(t)
    rgb, alb, nrm, info = srv.result(t)
    assert info["denoised"] == 1
    solo = _solo(gpu, cb, cb._data.camera, st)
    ref = dn.infer(solo.rgb, solo.albedo, solo.normal)
    assert np.abs(np.log1p(rgb) - np.log1p(ref)).max() < 1e-2


def test_launch_shape_does_not_change_the_image(gpu, world):
    _, sc = world
    st = _settings(64, 64, 8, sc._data.settings)
    base = gpu.Renderer(capacity=1 << 16).render(sc, settings=st)
    for chunk, block in ((1, 128), (4, 256), (16, 128)):
        r = gpu.Renderer(capacity=1 << 13)
        r.set_launch(chunk, block)
        out = r.render(sc, settings=st)
        assert _close(out.rgb, base.rgb), (chunk, block)
        assert out.stats["extensionRays"] == base.stats["extensionRays"]


def test_autotune_picks_a_listed_shape(gpu, world):
    cb, _ = world
    res = gpu.autotune(cb, settings=_settings(64, 64, 4, cb._data.settings))
    # 6 shapes per capacity; capacities 1M .. 64M while their queues fit in free memory
    assert len(res["trials"]) in (6, 12, 18, 24, 30)
    for t in res["trials"]:
        assert t["capacity"] in (1 << 20, 1 << 22, 1 << 24, 1 << 25, 1 << 26)
        assert t["chunk"] in (4, 8, 16) and t["shadeBlock"] in (128, 256)
    best = min(res["trials"], key=lambda t: t["ms"])
    assert (res["capacity"], res["chunk"], res["shadeBlock"]) == (best["capacity"], best["chunk"], best["shadeBlock"])


def test_batched_variant_scenes_each_as_alone(gpu):
    """Batched scenes in one launch: Cornell variants, each its own scene (own BVH,
    materials, lights), rendered together; each image equals its solo render."""
    sds = [scenes.cornell_variant(k) for k in range(6)]
    scs = [gpu.Scene.from_data(sd) for sd in sds]
    sts = [_settings(48, 32, 4, sd.settings) for sd in sds]
    srv = gpu.Server(capacity=1 << 14)
    tickets = [srv.submit(sc, settings=st) for sc, st in zip(scs, sts)]
    for t in tickets:
        srv.wait(t)
    for t, sc, st in zip(tickets, scs, sts):
        rgb, alb, nrm, _ = srv.result(t)
        solo = _solo(gpu, sc, sc._data.camera, st)
        assert _close(rgb, solo.rgb) and _close(nrm, solo.normal)


def test_server_rejects_bad_requests(gpu, world):
    cb, _ = world
    srv = gpu.Server(capacity=1 << 13)
    with pytest.raises(gpu.WrkError):
        srv.submit(cb, settings=_settings(32, 32, 0, cb._data.settings))  # spp 0
    with pytest.raises(gpu.WrkError):
        srv.ready(12345)  # unknown ticket
    with pytest.raises(gpu.WrkError):
        srv.submit(cb, settings=_settings(32, 32, 1, cb._data.settings), denoise=True)  # no denoiser attached
    st = srv.step()  # nothing queued: a no-op
    assert st["running"] == 0 and st["queued"] == 0


def test_sample_split_across_requests(gpu, world):
    """Two requests over disjoint sample ranges [0, 4) and [4, 8) average to the
    request over [0, 8): the RNG is keyed by sample index, so they draw the same
    samples (up to f32 rounding of the sums)."""
    _, sc = world
    st4 = _settings(64, 64, 4, sc._data.settings)
    st8 = _settings(64, 64, 8, sc._data.settings)
    srv = gpu.Server(capacity=1 << 15)
    a = srv.submit(sc, settings=st4, sample_offset=0)
    b = srv.submit(sc, settings=st4, sample_offset=4)
    c = srv.submit(sc, settings=st8)
    for t in (a, b, c):
        srv.wait(t)
    ra, rb, rc = srv.result(a)[0], srv.result(b)[0], srv.result(c)[0]
    np.testing.assert_allclose(0.5 * (ra + rb), rc, rtol=2e-5, atol=2e-6)
