"""BVH build throughput on the scale scene (1920x1080 config: 1024^2 fBm heightfield
plus 250 icospheres, about 2.41M triangles).

    python -m offlinerenderer_b200.bvh_bench [--repeat 3]

Uploads the scene `repeat` times (each upload builds the 8-wide BVH on the GPU) and
prints the device time of each build, the triangle rate, the node count and the
tree's SAH cost (wrk_scene_bvh_info).
"""
from __future__ import annotations

import argparse
import json

from . import scenes, wrk


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--repeat", type=int, default=3)
    args = ap.parse_args()
    sd = scenes.scale_test(1920, 1080, 64, seed=1)
    builds = []
    for _ in range(args.repeat):
        s = wrk.Scene.from_data(sd)
        builds.append(s.bvh_info())
        del s
    ms = [b["buildMs"] for b in builds]
    b = builds[-1]
    print(json.dumps({"triangles": b["numTriangles"], "nodes8": b["numNodes"], "binary_nodes": b["numBinaryNodes"],
                      "depth": b["depth"], "sah_cost": b["sahCost"], "build_ms": ms,
                      "mtris_per_s_best": b["numTriangles"] / (min(ms) / 1e3) / 1e6}))


if __name__ == "__main__":
    main()
