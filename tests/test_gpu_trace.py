"""Closest-hit and visibility parity of the GPU BVH traversal.

Against the oracle's FP32 Moller-Trumbore (same arithmetic): primitive ids and t
agree exactly.  Against the FP64 exact intersector over all triangles: primitive
ids agree on >= 99.99% of rays and t within 1e-5 relative (north-star level 2).
"""
import numpy as np
import pytest

from offlinerenderer_b200 import scenes

pytestmark = pytest.mark.gpu


def random_rays(sd, n, seed, origin_box=None):
    rng = np.random.default_rng(seed)
    lo, hi = sd.vertices.min(0), sd.vertices.max(0)
    if origin_box is not None:
        lo, hi = origin_box
    o = rng.uniform(lo, hi, (n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3], r[:, 3], r[:, 4:7], r[:, 7] = o, 0.0, d, 1e20
    return r


def camera_like_rays(oracle, sd, n, seed):
    st = sd.settings
    rng = np.random.default_rng(seed)
    px = rng.integers(0, st.width * st.height, n).astype(np.uint32)
    sm = rng.integers(0, 64, n).astype(np.uint32)
    return oracle.camera_rays(sd.camera, st.width, st.height, px, sm, 0)


@pytest.mark.parametrize("make", [lambda: scenes.cornell(64, 64, 1),
                                  lambda: scenes.material_showcase(64, 64, 1, tex_size=8),
                                  lambda: scenes.scale_test(64, 36, 1, grid=128, spheres=40, lights=16)])
def test_closest_hit_matches_fp32_oracle(gpu, oracle, make):
    sd = make()
    s = gpu.Scene.from_data(sd)
    osc = oracle.scene(sd)
    rays = np.concatenate([random_rays(sd, 100000, 1), camera_like_rays(oracle, sd, 50000, 2)])
    t, p = s.trace_closest(rays)
    to, po = osc.closest(rays, mode=0)
    assert np.array_equal(p, po)
    assert np.array_equal(t, to)


def test_closest_hit_vs_fp64_exact(gpu, oracle):
    sd = scenes.material_showcase(64, 64, 1, tex_size=8)
    s = gpu.Scene.from_data(sd)
    rays = np.concatenate([random_rays(sd, 40000, 3), camera_like_rays(oracle, sd, 20000, 4)])
    t, p = s.trace_closest(rays)
    t64, p64 = oracle.scene(sd).closest(rays, mode=1)
    agree = (p == p64).mean()
    assert agree >= 0.9999, agree
    hit = (p == p64) & (p != 0xFFFFFFFF)
    rel = np.abs(t[hit].astype(np.float64) - t64[hit]) / np.abs(t64[hit])
    assert rel.max() < 1e-5


def test_occlusion_matches_oracle(gpu, oracle):
    sd = scenes.material_showcase(32, 32, 1, tex_size=8)
    s = gpu.Scene.from_data(sd)
    rays = random_rays(sd, 100000, 5)
    rays[:, 3] = 1e-5
    rays[:, 7] = np.random.default_rng(6).uniform(0.0, 1.5, 100000).astype(np.float32)
    a = s.trace_occluded(rays)
    b = oracle.scene(sd).occluded(rays)
    assert np.array_equal(a, b)
    # occluded(any hit in [tmin,tmax]) agrees with the closest hit distance
    t, p = s.trace_closest(rays)
    assert np.array_equal(a.astype(bool), p != 0xFFFFFFFF)


def test_bvh_structure(gpu):
    for sd in (scenes.cornell(8, 8, 1), scenes.material_showcase(8, 8, 1, tex_size=8)):
        s = gpu.Scene.from_data(sd)
        info = s.bvh_info()
        assert info["numTriangles"] == sd.num_triangles
        assert 1 <= info["numNodes"] <= info["numBinaryNodes"]
        assert info["depth"] < 32


def test_tiny_and_degenerate_scenes(gpu, oracle):
    # one triangle; coplanar duplicates; a zero-area triangle
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 0], [1, 0, 0], [0, 1, 0], [2, 2, 2], [2, 2, 2], [2, 2, 2]],
                 np.float32)
    for nt in (1, 2, 3):
        b = scenes._Builder()
        m = b.lambertian((0.5, 0.5, 0.5))
        b.mesh(v[: 3 * nt], np.arange(3 * nt, dtype=np.uint32), m)
        sd = b.build(camera=scenes.Camera(), settings=scenes.RenderSettings(4, 4, 1))
        s = gpu.Scene.from_data(sd)
        rays = random_rays(sd, 20000, 7, origin_box=(np.array([-1, -1, -1.0]), np.array([2, 2, 1.0])))
        t, p = s.trace_closest(rays)
        to, po = oracle.scene(sd).closest(rays)
        assert np.array_equal(p, po) and np.array_equal(t, to)


def test_many_identical_triangles(gpu, oracle):
    """Centroids that coincide force the object-median split path of the builder."""
    b = scenes._Builder()
    m = b.lambertian((0.5, 0.5, 0.5))
    tri = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    for _ in range(3000):
        b.mesh(tri, [0, 1, 2], m)
    sd = b.build(camera=scenes.Camera(), settings=scenes.RenderSettings(4, 4, 1))
    s = gpu.Scene.from_data(sd)
    rays = random_rays(sd, 5000, 8, origin_box=(np.array([-0.5, -0.5, -1.0]), np.array([1, 1, 1.0])))
    t, p = s.trace_closest(rays)
    to, po = oracle.scene(sd).closest(rays)
    assert np.array_equal(p, po) and np.array_equal(t, to)


def test_large_scene_against_fp64_sample(gpu, oracle):
    """About 2.4M triangles (the scale-test scene): the BVH builds and a sample of
    rays agrees with the exact FP64 intersector."""
    sd = scenes.scale_test(64, 36, 1)
    s = gpu.Scene.from_data(sd)
    info = s.bvh_info()
    assert info["numTriangles"] == sd.num_triangles > 2_000_000
    rays = camera_like_rays(oracle, sd, 2000, 9)
    t, p = s.trace_closest(rays)
    osc = oracle.scene(sd)
    to, po = osc.closest(rays, mode=0)
    assert np.array_equal(p, po) and np.array_equal(t, to)
    t64, p64 = osc.closest(rays[:300], mode=1)
    assert (p[:300] == p64).mean() >= 0.99
