"""Procedural benchmark scenes: sizes and the properties the render path relies on."""
import numpy as np

from offlinerenderer_b200 import scenes


def _normals(sd, tris):
    v = sd.vertices[sd.indices[tris]]
    n = np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0])
    return n / np.linalg.norm(n, axis=1, keepdims=True)


def test_cornell_layout():
    sd = scenes.cornell()
    assert sd.num_triangles == 36
    assert sd.settings.width == 256 and sd.settings.spp == 64 and sd.settings.maxBounces == 8
    em = np.where(sd.materials["type"][sd.tri_material] == scenes.EMISSIVE)[0]
    assert len(em) == 2
    np.testing.assert_allclose(_normals(sd, em), [[0, -1, 0], [0, -1, 0]], atol=1e-6)  # light faces down
    np.testing.assert_allclose(sd.materials["emission"][sd.tri_material[em[0]]][:3], [17, 12, 4])
    assert sd.vertices.min() >= 0.0 and sd.vertices.max() <= 1.0 + 1e-6


def test_showcase_layout():
    sd = scenes.material_showcase()
    assert sd.num_triangles == 12 + 3 * 5120
    assert sd.settings.width == 512 and sd.settings.spp == 256 and sd.settings.maxBounces == 16
    assert len(sd.textures) == 2 and sd.textures[0].shape == (1024, 1024, 4)
    types = set(sd.materials["type"].tolist())
    assert {scenes.GLASS, scenes.GGX_REFLECTION, scenes.GGX_TRANSMISSION, scenes.LAMBERTIAN} <= types
    assert sd.uvs is not None and sd.normals is not None


def test_scale_test_layout():
    sd = scenes.scale_test(grid=64, spheres=10, lights=64)
    assert sd.num_triangles == 2 * 63 * 63 + 10 * 1280 + 64
    em = np.where(sd.materials["type"][sd.tri_material] == scenes.EMISSIVE)[0]
    assert len(em) == 64
    assert (_normals(sd, em)[:, 1] < -0.99).all()


def test_scenes_are_deterministic():
    a, b = scenes.material_showcase(tex_size=64), scenes.material_showcase(tex_size=64)
    assert np.array_equal(a.vertices, b.vertices) and np.array_equal(a.textures[1], b.textures[1])
    c = scenes.scale_test(grid=32, spheres=4, lights=4, seed=2)
    d = scenes.scale_test(grid=32, spheres=4, lights=4, seed=2)
    assert np.array_equal(c.vertices, d.vertices)


def test_icosphere_counts():
    for k in range(4):
        v, f = scenes.icosphere(k)
        assert f.shape[0] == 20 * 4 ** k
        np.testing.assert_allclose(np.linalg.norm(v, axis=1), 1.0, atol=1e-12)
