"""The GPU-built 8-wide BVH, read back and checked on the CPU by an independent
decoder of its node format (oracle/port/orc_render.cpp, orc_bvh8_*): every
triangle appears exactly once, every triangle lies inside its quantized child
box, and a CPU traversal of the exported tree finds the same closest hits as the
GPU kernel and as the oracle's own BVH."""
import numpy as np
import pytest

from offlinerenderer_b200 import scenes
from test_gpu_trace import camera_like_rays, random_rays

pytestmark = pytest.mark.gpu

CASES = {
    "cornell": lambda: scenes.cornell(64, 64, 1),
    "showcase": lambda: scenes.material_showcase(64, 64, 1, tex_size=8),
    "scale_small": lambda: scenes.scale_test(64, 36, 1, grid=256, spheres=60, lights=16),
}


@pytest.mark.parametrize("name", list(CASES))
def test_exported_bvh_is_valid_and_traces_identically(gpu, oracle, name):
    sd = CASES[name]()
    s = gpu.Scene.from_data(sd)
    nodes, tris = s.bvh_export()
    rc, depth, internal, leaf = oracle.bvh8_validate(nodes, tris)
    assert rc == 0, rc
    assert depth == s.bvh_info()["depth"]
    assert internal == nodes.shape[0] - 1  # every node but the root is some node's child
    rays = np.concatenate([camera_like_rays(oracle, sd, 20000, 1), random_rays(sd, 20000, 2)])
    t, p, visits, tests = oracle.bvh8_trace(nodes, tris, rays)
    tg, pg = s.trace_closest(rays)
    assert np.array_equal(p, pg) and np.array_equal(t, tg)
    print(f"{name}: {sd.num_triangles} tris, {nodes.shape[0]} nodes, depth {depth}, "
          f"visits/ray {visits.mean():.1f}, tests/ray {tests.mean():.1f}")
