"""Regenerate the golden fixtures in tests/golden from the reference itself.

Runs the reference renderer's own BVH template and ray/triangle test
(oracle/_ref/libref_bvh.so, built by `make -C oracle` from the reference
sources) on small seeded inputs and stores inputs and outputs:

  bvh_soup_2k.npz  2,000-triangle soup (the ray-cast microbenchmark's
                   distribution), 4,096 closest-hit rays and 4,096 shadow
                   rays: the reference BVH2/BVH4 node arrays, leaf order, hit
                   ids, double-precision hit distances and occlusion flags.
  ray_triangle.json  the reference's Moller-Trumbore known answers
                   (tests/RayTriangleIntersectionTest.cpp cases) evaluated by
                   the reference code.

Usage: python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from rise_b200 import scenes  # noqa: E402

# Cases of tests/RayTriangleIntersectionTest.cpp:16-129 (origin, direction,
# v0, edgeA, edgeB) plus two of our own near-edge and grazing cases.
RT_CASES = [
    ("interior", (0.25, 0.25, 1.0), (0, 0, -1), (0, 0, 0), (1, 0, 0), (0, 1, 0)),
    ("edge_mid", (0.5, 0.5, 2.0), (0, 0, -2), (0, 0, 0), (1, 0, 0), (0, 1, 0)),
    ("vertex", (1.0, 0.0, 3.0), (0, 0, -3), (0, 0, 0), (1, 0, 0), (0, 1, 0)),
    ("miss_outside", (0.75, 0.75, 1.0), (0, 0, -1), (0, 0, 0), (1, 0, 0), (0, 1, 0)),
    ("miss_behind", (0.25, 0.25, -1.0), (0, 0, -1), (0, 0, 0), (1, 0, 0), (0, 1, 0)),
    ("miss_parallel", (0.25, 0.25, 1.0), (1, 0, 0), (0, 0, 0), (1, 0, 0), (0, 1, 0)),
    ("winding_fwd", (0.2, 0.3, 1.0), (0, 0, -1), (0, 0, 0), (1, 0, 0), (0, 1, 0)),
    ("winding_rev", (0.2, 0.3, 1.0), (0, 0, -1), (0, 0, 0), (0, 1, 0), (1, 0, 0)),
    ("oblique", (0.1, 0.2, 0.9), (0.3, -0.2, -1.0), (0, 0, 0), (1, 0, 0), (0, 1, 0)),
    ("outside_by_1e-13", (0.5 + 5e-14, 0.5 + 5e-14, 1.0), (0, 0, -1), (0, 0, 0), (1, 0, 0), (0, 1, 0)),
]


def main():
    if oracle.ref() is None:
        raise SystemExit("build the reference harness first: make -C oracle")
    tri = scenes.soup_triangles(2000, seed=11)
    rays = scenes.sphere_rays(4096, seed=11)
    srays = scenes.sphere_rays(4096, seed=11, shadow=True)
    R = oracle.BVH(tri, "ref")
    nodes2, prims, nodes4 = R.nodes()
    ids, t = R.closest(rays)
    occ = R.any(srays)
    np.savez_compressed(os.path.join(HERE, "bvh_soup_2k.npz"), tri9=tri, rays=rays, shadow_rays=srays,
                        nodes2=nodes2.view(np.uint8), prims=prims, nodes4=nodes4.view(np.uint8),
                        ids=ids, t=t, occluded=occ)
    out = []
    for name, o, d, v0, ea, eb in RT_CASES:
        hit, tt, a, b = oracle.ray_triangle(o, d, v0, ea, eb, kind="ref")
        out.append({"name": name, "o": o, "d": d, "v0": v0, "ea": ea, "eb": eb, "hit": hit,
                    "t": tt if hit else None, "alpha": a if hit else None, "beta": b if hit else None})
    with open(os.path.join(HERE, "ray_triangle.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", len(ids), "rays,", len(nodes2), "BVH2 nodes,", len(out), "triangle cases")


if __name__ == "__main__":
    main()
