"""The oracle pinned against the reference.

The reference publishes no golden vectors, so the fixtures in tests/golden come
from the reference's own shading headers and PNG writer compiled on the host
(tests/golden/make_golden.py).  The oracle's restatement must reproduce them bit
for bit; where the reference build is present it is also compared live.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from offlinerenderer_b200 import scenes


def _eq_nan(a, b):
    return (a == b) | (np.isnan(a) & np.isnan(b))


def test_bsdf_bitexact_vs_reference_fixture(oracle):
    d = np.load(os.path.join(GOLDEN, "bsdf_ref.npz"))
    out = oracle.bsdf(d["inputs"], prec=0)
    assert _eq_nan(out, d["outputs"]).all()


def test_rng_bitexact_vs_reference_fixture(oracle):
    d = np.load(os.path.join(GOLDEN, "rng_ref.npz"))
    h, u = oracle.rng(d["seeds"], d["dims"])
    assert np.array_equal(h, d["hash"]) and np.array_equal(u, d["u"])


def test_cdf_lower_bound_vs_reference_fixture(oracle):
    d = np.load(os.path.join(GOLDEN, "cdf_ref.npz"))
    for k, n in enumerate(d["n"]):
        got = oracle.cdf_sample(d["cdf"][k][:n], d["u"][k])
        assert np.array_equal(got, d["index"][k])


def test_aces_bytes_vs_reference_png_writer(oracle):
    d = np.load(os.path.join(GOLDEN, "aces_ref.npz"))
    assert np.array_equal(oracle.tonemap(d["rgb"]), d["bytes"])


def test_camera_rays_use_reference_camera_basis(oracle):
    """Rays from the oracle's camera basis match the basis GLM gives the reference."""
    d = np.load(os.path.join(GOLDEN, "camera_ref.npz"))
    for cam_v, basis in zip(d["cameras"], d["basis"]):
        cam = scenes.Camera(position=tuple(cam_v[0:3]), target=tuple(cam_v[3:6]), up=tuple(cam_v[6:9]),
                            fovY=float(cam_v[9]), aspect=1.0)
        # centre pixel of a 1x1 image with jitter: direction = normalize(fwd + right*ndcX*t + up*ndcY*t)
        rays = oracle.camera_rays(cam, 1, 1, [0], [0], 0)
        js = np.uint32(0x9e3779b9)
        seq = []
        for _ in range(2):
            js = np.uint32((int(js) * 1664525 + 1013904223) & 0xffffffff)
            seq.append(np.float32(int(js) >> 8) / np.float32(16777216.0))
        f, r, u, t = basis[0:3], basis[3:6], basis[6:9], np.float32(basis[9])
        nx = (np.float32(2.0) * (np.float32(0.0) + seq[0]) / np.float32(1.0) - np.float32(1.0)) * np.float32(1.0)
        ny = np.float32(1.0) - np.float32(2.0) * (np.float32(0.0) + seq[1]) / np.float32(1.0)
        v = (f + (r * nx) * t) + (u * ny) * t
        v = v.astype(np.float32)
        dd = np.float32(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])
        inv = np.float32(1.0 / np.sqrt(np.float64(dd)))
        np.testing.assert_array_equal(rays[0, 4:7], (v * inv).astype(np.float32))
        np.testing.assert_array_equal(rays[0, 0:3], np.asarray(cam.position, np.float32))


def test_cornell_image_bitexact_vs_reference_fixture(oracle):
    """Whole render path: the oracle with the host compiler's argument order
    reproduces the image the reference's shading code renders, bit for bit."""
    d = np.load(os.path.join(GOLDEN, "cornell_ref.npz"))
    sd = scenes.cornell(32, 32, 8, seed=0)
    rgb, alb, nrm, st = oracle.scene(sd).render(draw_order=1)
    assert np.array_equal(rgb, d["rgb"])
    assert np.array_equal(alb, d["albedo"]) and np.array_equal(nrm, d["normal"])
    assert st["extension_rays"] == int(d["extension_rays"]) and st["shadow_rays"] == int(d["shadow_rays"])


@pytest.mark.parametrize("make", [lambda: scenes.cornell(24, 16, 4, seed=3),
                                  lambda: scenes.material_showcase(24, 24, 2, seed=2, tex_size=64)])
def test_render_bitexact_vs_live_reference(oracle, reference, make):
    sd = make()
    a = oracle.scene(sd).render(draw_order=1)
    b = reference.scene(sd).render()
    for x, y in zip(a[:3], b[:3]):
        assert np.array_equal(x, y)
    assert a[3] == b[3]


def test_bsdf_live_reference_random(oracle, reference):
    import pyoracle

    inp = pyoracle.random_bsdf_inputs(3000, seed=99)
    assert _eq_nan(oracle.bsdf(inp), reference.bsdf(inp)).all()


def test_fp64_transcription_close_to_fp32(oracle):
    """The FP64 transcription (the per-kernel 1e-5 yardstick) agrees with FP32 on
    well-conditioned records."""
    import pyoracle

    inp = pyoracle.random_bsdf_inputs(2000, seed=5)
    a, b = oracle.bsdf(inp, 0), oracle.bsdf(inp, 1)
    ok = np.isfinite(a) & np.isfinite(b) & (np.abs(b) > 1e-3)
    rel = np.abs(a[ok] - b[ok]) / np.abs(b[ok])
    assert np.median(rel) < 1e-6


def test_light_cdf_restatement(oracle):
    sd = scenes.cornell(8, 8, 1)
    tris, cdf = oracle.scene(sd).light_cdf()
    assert list(tris) == [10, 11]  # the light quad follows the 10 room triangles
    assert cdf.dtype == np.float32 and cdf[-1] == np.float32(1.0)
    # two equal-area, equal-emission triangles: the first CDF entry is exactly 1/2
    assert cdf[0] == np.float32(0.5)


def _light_cdf_numpy(sd):
    """scene.cpp:423-491 restated in numpy float32, independently of the oracle: per
    emissive triangle in index order, power = (ex + ey + ez) * area with area =
    0.5 * |cross(v1 - v0, v2 - v0)| (correctly rounded float32 steps, left to right),
    a serial float32 prefix sum, then each entry divided by the total."""
    f = np.float32
    tris, cdf, total = [], [], f(0.0)
    for t in range(sd.num_triangles):
        m = sd.materials[sd.tri_material[t]]
        if m["type"] != scenes.EMISSIVE:
            continue
        a, b, c = (sd.vertices[sd.indices[t][k]].astype(np.float32) for k in range(3))
        e1, e2 = b - a, c - a
        cr = np.array([e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                       e1[0] * e2[1] - e1[1] * e2[0]], np.float32)
        area = f(0.5) * np.sqrt(f(f(cr[0] * cr[0] + cr[1] * cr[1]) + cr[2] * cr[2]))
        em = m["emission"]
        power = f(f(em[0] + em[1]) + em[2]) * area
        total = f(total + power)
        tris.append(t)
        cdf.append(total)
    return np.array(tris, np.uint32), (np.array(cdf, np.float32) / total).astype(np.float32)


def test_light_cdf_scale_scene_matches_numpy_restatement(oracle):
    """The 64 lights of unequal power of the scale scene: the oracle's light list and
    CDF equal the numpy restatement bit for bit (the GPU tests then compare the
    product's CDF with the oracle's)."""
    sd = scenes.scale_test(48, 32, 1, seed=1)
    tris, cdf = oracle.scene(sd).light_cdf()
    want_t, want_c = _light_cdf_numpy(sd)
    assert len(tris) == 64
    assert np.array_equal(tris, want_t)
    assert np.array_equal(cdf.view(np.uint32), want_c.view(np.uint32))


@pytest.mark.parametrize("full", [False, True])
def test_fp64_bvh_walk_equals_all_triangle_test(oracle, full):
    """Oracle mode 2 (the FP64 test on the triangles a widened FP64 BVH walk reaches)
    returns exactly what mode 1 (FP64 over every triangle) returns: on a small scale
    scene for 4000 rays, and on the full 2.41M-triangle scale scene for a sample."""
    from test_gpu_trace import camera_like_rays, random_rays

    sd = scenes.scale_test(1920, 1080, 1, seed=1) if full else \
        scenes.scale_test(64, 36, 1, grid=96, spheres=30, lights=16, seed=2)
    n = 24 if full else 2000
    rays = np.concatenate([camera_like_rays(oracle, sd, n, 21), random_rays(sd, n, 22)])
    osc = oracle.scene(sd)
    t1, p1 = osc.closest(rays, mode=1)
    t2, p2 = osc.closest(rays, mode=2)
    assert np.array_equal(p1, p2) and np.array_equal(t1, t2)
    assert (p1 != 0xFFFFFFFF).sum() > n // 4


def test_level1_caps_hold_for_the_reference_build(oracle):
    """The level-1 criterion and its exclusion caps, applied to the reference's own
    FP32 outputs (the golden fixture from the reference build): every
    well-conditioned output of the reference is within 1e-5 of the FP64
    transcription (so the GPU test's bound is met by the reference itself)."""
    from level1 import check_against_fp64

    d = np.load(os.path.join(GOLDEN, "bsdf_ref.npz"))
    check_against_fp64(d["outputs"], d["outputs"], d["inputs"], oracle, "reference")


def test_iteration_cap_drops_paths(oracle):
    """maxIterations bounds the wavefront iterations; fewer iterations can only
    drop energy (paths still alive at the cap are not accumulated)."""
    sd = scenes.cornell(16, 16, 4, seed=1)
    sc = oracle.scene(sd)
    lo = sc.render(max_iterations=2)[0].sum()
    hi = sc.render(max_iterations=8)[0].sum()
    inf = sc.render(max_iterations=64)[0].sum()
    assert lo < hi <= inf


def test_compact_oracle():
    import pyoracle

    o = pyoracle.Oracle()
    stage = np.array([0, 3, 1, 3, 2], np.uint32)
    assert list(o.compact(stage, np.array([4, 3, 2, 1, 0], np.uint32))) == [4, 2, 0]
    assert len(o.compact(stage, np.zeros(0, np.uint32))) == 0
