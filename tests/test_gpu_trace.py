"""Closest-hit and visibility parity of the GPU BVH traversal.

Against the oracle's FP32 Moller-Trumbore (same arithmetic): primitive ids and t
agree exactly.  Against the FP64 exact intersector: primitive ids agree on
>= 99.99% of rays and t within 1e-5 relative wherever both hit (parity level
2).  The exact intersector tests every triangle in FP64 (oracle mode 1); on the
2.41M-triangle scale scene it reaches the triangles by walking the oracle's CPU
BVH with conservatively widened FP64 boxes (mode 2, checked equal to mode 1).
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
    osc = oracle.scene(sd)
    t64, p64 = osc.closest(rays, mode=1)
    _check_level2(t, p, t64, p64)
    t2, p2 = osc.closest(rays, mode=2)
    assert np.array_equal(p2, p64) and np.array_equal(t2, t64)


def _check_level2(t, p, t64, p64):
    miss = np.uint32(0xFFFFFFFF)
    agree = (p == p64).mean()
    assert agree >= 0.9999, agree
    assert ((p != miss) == (p64 != miss)).mean() >= 0.9999
    # t of every ray whose primitive agrees (a ray that grazes a silhouette may hit
    # another surface in FP32 than in FP64: that is a primitive disagreement)
    hit = (p == p64) & (p != miss)
    # t relative to 1e-5 for hits at least 1e-3 away.  Closer than that (random rays
    # may start within 1e-5 of a surface; the renderer offsets every ray origin 1e-4)
    # the FP32 rounding of the origin coordinates alone, ~6e-8 absolute at unit
    # scale, exceeds 1e-5 of t: there t is held to 1e-8 absolute.
    far = hit & (t64 >= 1e-3)
    near = hit & (t64 < 1e-3)
    with np.errstate(invalid="ignore"):  # inf - inf on rays that miss
        dt = np.abs(t.astype(np.float64) - t64.astype(np.float64))
    assert (dt[far] / t64[far]).max() < 1e-5, (dt[far] / t64[far]).max()
    assert not near.any() or dt[near].max() < 1e-8, dt[near].max()
    return agree


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


def test_large_scene_against_fp64(gpu, oracle):
    """The full scale-test scene (1920x1080 camera, 1024^2 fBm heightfield + 250
    icospheres, ~2.41M triangles): 100k camera rays of the benchmark camera and
    100k random rays.  Bit-exact against the FP32 oracle; against the FP64 exact
    intersector (BVH walk, mode 2) >= 99.99% primitive-id agreement and t within
    1e-5 relative; mode 2 equals the all-triangle FP64 test on a sample."""
    sd = scenes.scale_test(1920, 1080, 1, seed=1)
    s = gpu.Scene.from_data(sd)
    info = s.bvh_info()
    assert info["numTriangles"] == sd.num_triangles > 2_000_000
    rays = np.concatenate([camera_like_rays(oracle, sd, 100000, 9), random_rays(sd, 100000, 10)])
    t, p = s.trace_closest(rays)
    osc = oracle.scene(sd)
    to, po = osc.closest(rays, mode=0)
    assert np.array_equal(p, po) and np.array_equal(t, to)
    t64, p64 = osc.closest(rays, mode=2)
    agree = _check_level2(t, p, t64, p64)
    assert (p[:100000] != 0xFFFFFFFF).mean() > 0.3  # the terrain fills ~44% of the benchmark view
    sample = np.r_[0:32, 100000:100032]
    t1, p1 = osc.closest(rays[sample], mode=1)
    assert np.array_equal(p1, p64[sample]) and np.array_equal(t1, t64[sample])
    print(f"level 2 on the scale scene: {agree:.6f} primitive-id agreement over {len(rays)} rays")
