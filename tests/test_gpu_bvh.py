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


def _sah_numpy(nodes):
    """SAH cost of an exported 8-wide tree, decoded in numpy (float64): 1 for the
    root plus, per child box, area / root area x (1 node test or the leaf's count)."""
    n = nodes.astype(np.uint64)
    p = nodes[:, 0:3].copy().view(np.float32).astype(np.float64)
    e = np.stack([(n[:, 3] >> np.uint64(8 * a)) & np.uint64(0xff) for a in range(3)], 1).astype(np.int64) - 127
    sc = np.ldexp(1.0, e)
    imask = (n[:, 3] >> np.uint64(24)).astype(np.int64)
    meta = np.concatenate([nodes[:, 6:8].copy().view(np.uint8)], 1).reshape(-1, 8).astype(np.int64)
    b = nodes[:, 8:20].copy().view(np.uint8).reshape(-1, 6, 8).astype(np.float64)  # qlo x,y,z ; qhi x,y,z
    lo = p[:, :, None] + b[:, 0:3] * sc[:, :, None]
    hi = p[:, :, None] + b[:, 3:6] * sc[:, :, None]
    valid = (b[:, 0:3] <= b[:, 3:6]).all(1)
    d = np.maximum(hi - lo, 0.0)
    area = d[:, 0] * d[:, 1] + d[:, 1] * d[:, 2] + d[:, 2] * d[:, 0]
    internal = ((imask[:, None] >> np.arange(8)) & 1) == 1
    work = np.where(internal, 1.0, (meta >> 5) + 1.0)
    total = (area * work * valid).sum()
    rl = np.where(valid[0][None], lo[0], np.inf).min(1)
    rh = np.where(valid[0][None], hi[0], -np.inf).max(1)
    rd = rh - rl
    root = rd[0] * rd[1] + rd[1] * rd[2] + rd[2] * rd[0]
    return 1.0 + total / root


@pytest.mark.parametrize("name", list(CASES))
def test_reported_sah_cost_matches_the_exported_tree(gpu, name):
    s = gpu.Scene.from_data(CASES[name]())
    nodes, _ = s.bvh_export()
    sah = s.bvh_info()["sahCost"]
    assert sah > 1.0
    assert abs(sah - _sah_numpy(nodes)) <= 1e-4 * sah
