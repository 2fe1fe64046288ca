"""The oracle itself, pinned against the reference (CPU only).

* the port (oracle/bvh_oracle.cpp) against the committed golden fixtures the
  reference produced (tests/golden/make_golden.py);
* the port against the reference harness oracle/_ref (when built here);
* both against the reference's own Moller-Trumbore known answers
  (tests/RayTriangleIntersectionTest.cpp of the reference).
"""
import json
import os

import numpy as np
import pytest

import oracle
from rise_b200 import scenes

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _golden():
    return np.load(os.path.join(GOLDEN, "bvh_soup_2k.npz"))


def test_port_matches_golden_tree():
    g = _golden()
    b = oracle.BVH(g["tri9"], "port")
    n2, prims, n4 = b.nodes()
    assert n2.view(np.uint8).tobytes() == g["nodes2"].tobytes()
    assert (prims == g["prims"]).all()
    r4 = g["nodes4"].view(oracle.NODE4_DTYPE)
    for f in oracle.NODE4_FIELDS:
        assert (n4[f] == r4[f]).all(), f


def test_port_matches_golden_hits():
    g = _golden()
    b = oracle.BVH(g["tri9"], "port")
    ids, t = b.closest(g["rays"])
    assert (ids == g["ids"]).all()
    assert (t == g["t"]).all()
    assert (b.any(g["shadow_rays"]) == g["occluded"]).all()


def test_golden_has_hits_and_misses():
    g = _golden()
    assert 0.05 < (g["ids"] >= 0).mean() < 0.99
    assert 0.02 < g["occluded"].mean() < 0.99


@pytest.mark.parametrize("case", json.load(open(os.path.join(GOLDEN, "ray_triangle.json"))),
                         ids=lambda c: c["name"])
def test_ray_triangle_known_answers(case):
    hit, t, a, b = oracle.ray_triangle(case["o"], case["d"], case["v0"], case["ea"], case["eb"])
    assert hit == case["hit"]
    if hit:
        assert t == case["t"] and a == case["alpha"] and b == case["beta"]


def test_reference_known_answers_from_reference_test_file():
    # tests/RayTriangleIntersectionTest.cpp:16-129 of the reference, restated.
    v0, ea, eb = (0, 0, 0), (1, 0, 0), (0, 1, 0)
    hit, t, a, b = oracle.ray_triangle((0.25, 0.25, 1.0), (0, 0, -1), v0, ea, eb)
    assert hit and abs(t - 1) < 1e-6 and abs(a - .25) < 1e-6 and abs(b - .25) < 1e-6
    hit, t, a, b = oracle.ray_triangle((0.5, 0.5, 2.0), (0, 0, -2), v0, ea, eb)
    assert hit and abs(t - 1) < 1e-6 and abs(a - .5) < 1e-6 and abs(b - .5) < 1e-6
    hit, t, a, b = oracle.ray_triangle((1.0, 0.0, 3.0), (0, 0, -3), v0, ea, eb)
    assert hit and abs(t - 1) < 1e-6 and abs(a - 1) < 1e-6 and abs(b) < 1e-6
    assert not oracle.ray_triangle((0.75, 0.75, 1.0), (0, 0, -1), v0, ea, eb)[0]
    assert not oracle.ray_triangle((0.25, 0.25, -1.0), (0, 0, -1), v0, ea, eb)[0]
    assert not oracle.ray_triangle((0.25, 0.25, 1.0), (1, 0, 0), v0, ea, eb)[0]
    f = oracle.ray_triangle((0.2, 0.3, 1.0), (0, 0, -1), v0, (1, 0, 0), (0, 1, 0))
    r = oracle.ray_triangle((0.2, 0.3, 1.0), (0, 0, -1), v0, (0, 1, 0), (1, 0, 0))
    assert f[0] and r[0] and abs(f[1] - r[1]) < 1e-6


def test_port_bvh_matches_brute_force():
    tri = scenes.soup_triangles(3000, seed=3)
    rays = scenes.sphere_rays(3000, seed=3)
    ids, t = oracle.BVH(tri, "port").closest(rays)
    bi, bt = oracle.closest_brute(tri, rays)
    assert (ids == bi).all()
    assert np.allclose(t[ids >= 0], bt[ids >= 0], rtol=0, atol=0)


needs_ref = pytest.mark.skipif(oracle.ref() is None, reason="reference harness oracle/_ref not built here")


@needs_ref
@pytest.mark.parametrize("n_tri", [1, 4, 5, 17, 1000, 100000])
def test_port_matches_reference_harness(n_tri):
    tri = scenes.soup_triangles(n_tri, seed=n_tri)
    rays = scenes.sphere_rays(20000, seed=n_tri)
    srays = scenes.sphere_rays(20000, seed=n_tri, shadow=True)
    P, R = oracle.BVH(tri, "port"), oracle.BVH(tri, "ref")
    p2, pp, p4 = P.nodes()
    r2, rp, r4 = R.nodes()
    assert p2.tobytes() == r2.tobytes() and (pp == rp).all()
    for f in oracle.NODE4_FIELDS:
        assert (p4[f] == r4[f]).all()
    pi, pt = P.closest(rays)
    ri, rt = R.closest(rays)
    assert (pi == ri).all() and (pt == rt).all()
    assert (P.any(srays) == R.any(srays)).all()


@needs_ref
def test_reference_harness_known_answers():
    for case in json.load(open(os.path.join(GOLDEN, "ray_triangle.json"))):
        hit, t, a, b = oracle.ray_triangle(case["o"], case["d"], case["v0"], case["ea"], case["eb"], kind="ref")
        assert hit == case["hit"]
