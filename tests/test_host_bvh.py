"""The product's host BVH builder (librtb200.so) reproduces the reference tree.

Checked byte for byte against the reference's golden node arrays and, at
larger sizes, against the oracle port (itself pinned to the reference).  No
device is needed: rtb200_bvh_host_* run on the host only.
"""
import os

import numpy as np
import pytest

import oracle
from rise_b200 import raycaster, scenes

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_host_builder_matches_golden():
    g = np.load(os.path.join(GOLDEN, "bvh_soup_2k.npz"))
    n2, prims, n4 = raycaster.build_host_bvh(g["tri9"])
    assert n2.view(np.uint8).tobytes() == g["nodes2"].tobytes()
    assert (prims == g["prims"]).all()
    r4 = g["nodes4"].view(raycaster.NODE4_DTYPE)
    for f in oracle.NODE4_FIELDS:
        assert (n4[f] == r4[f]).all(), f


@pytest.mark.parametrize("n_tri,threads", [(1, 0), (4, 0), (5, 2), (300, 3), (70000, 0), (300000, 8)])
def test_host_builder_matches_port(n_tri, threads):
    tri = scenes.soup_triangles(n_tri, seed=100 + n_tri)
    n2, prims, n4 = raycaster.build_host_bvh(tri, threads=threads)
    p2, pp, p4 = oracle.BVH(tri, "port").nodes()
    assert n2.tobytes() == p2.tobytes()
    assert (prims == pp).all()
    for f in oracle.NODE4_FIELDS:
        assert (n4[f] == p4[f]).all(), f


def test_host_builder_degenerate_inputs():
    # All triangles share one centroid: the reference makes one big leaf.
    tri = np.tile(np.array([[0, 0, 0, 1, 0, 0, 0, 1, 0]], np.float32), (40, 1))
    n2, prims, n4 = raycaster.build_host_bvh(tri)
    p2, pp, p4 = oracle.BVH(tri, "port").nodes()
    assert n2.tobytes() == p2.tobytes() and len(n2) == 1 and n2[0]["count"] == 40
    # Collinear centroids along one axis with duplicates.
    x = np.repeat(np.arange(10, dtype=np.float32), 7)
    tri = np.zeros((len(x), 9), np.float32)
    tri[:, 0] = x
    tri[:, 3] = x + 0.5
    tri[:, 7] = 1.0
    n2, prims, n4 = raycaster.build_host_bvh(tri)
    p2, pp, p4 = oracle.BVH(tri, "port").nodes()
    assert n2.tobytes() == p2.tobytes() and (prims == pp).all()


def test_host_builder_empty():
    n2, prims, n4 = raycaster.build_host_bvh(np.zeros((0, 9), np.float32))
    assert len(n2) == 0 and len(prims) == 0 and len(n4) == 0


def stack_bound(nodes4):
    """Largest sum of (children - 1) over the internal nodes of one
    root-to-node path: the deferred entries a depth-first BVH4 walk can hold."""
    best, todo = 0, [(0, 0)]
    while todo:
        ni, above = todo.pop()
        n = nodes4[ni]
        here = above + max(int(n["nchild"]) - 1, 0)
        best = max(best, here)
        todo.extend((int(n["child"][i]), here) for i in range(int(n["nchild"])) if n["count"][i] == 0)
    return best


def test_traversal_stack_bounds():
    # The shared-memory stack holds 40 entries; these scenes stay within it
    # (the path-tracer scenes up to 3.4M triangles included) ...
    assert stack_bound(raycaster.build_host_bvh(scenes.soup_triangles(100_000, 7))[2]) <= 40
    assert stack_bound(raycaster.build_host_bvh(scenes.cornell_box(8, 8).tri9)[2]) <= 40
    # ... and the nested-cluster scene needs the local-memory continuation.
    b = stack_bound(raycaster.build_host_bvh(scenes.nested_clusters())[2])
    assert 40 < b <= 128


# ---- the eight-wide layout (rise_b200/csrc/bvh_wide.cpp) --------------------

def _w8_checker(tmp_path_factory):
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = os.path.join(root, "rise_b200", "csrc")
    exe = str(tmp_path_factory.mktemp("w8") / "w8_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", src, os.path.join(root, "tests", "cpp", "w8_check.cpp"),
                    os.path.join(src, "bvh_build.cpp"), os.path.join(src, "bvh_wide.cpp"), "-o", exe, "-lpthread"],
                   check=True)
    return exe


@pytest.fixture(scope="module")
def w8_check(tmp_path_factory):
    return _w8_checker(tmp_path_factory)


@pytest.mark.parametrize("case", ["soup", "tiny1", "tiny5", "deep"])
def test_wide_nodes_are_conservative_and_find_every_closest_hit(w8_check, tmp_path, case):
    """The eight-wide encoding: each triangle once, links and runs in range,
    every 8-bit child box containing its triangles, and the device's
    traversal rules (octant order, groups, one stack entry per level) finding
    the brute-force closest hit of every ray."""
    import subprocess
    from rise_b200 import scenes
    if case == "soup":
        tri, rays = scenes.soup_triangles(20000, seed=4), scenes.sphere_rays(1500, seed=4)
    elif case == "deep":
        tri = scenes.nested_clusters()
        rays = scenes.cluster_rays(tri, 1500, seed=5)
    else:
        n = 1 if case == "tiny1" else 5
        tri, rays = scenes.soup_triangles(n, seed=n), scenes.sphere_rays(500, seed=n)
    tp, rp = tmp_path / "tri.bin", tmp_path / "rays.bin"
    np.ascontiguousarray(tri, np.float32).tofile(tp)
    np.ascontiguousarray(rays, np.float32).tofile(rp)
    out = subprocess.run([w8_check, str(tp), str(rp)], capture_output=True, text=True)
    assert out.returncode == 0 and out.stdout.startswith("ok"), out.stdout + out.stderr


# ---- the half-precision layout (EncodeHalfNodes in rise_b200/csrc/bvh_build.cpp) ----

@pytest.fixture(scope="module")
def f16_check(tmp_path_factory):
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = os.path.join(root, "rise_b200", "csrc")
    exe = str(tmp_path_factory.mktemp("f16") / "f16_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", src, os.path.join(root, "tests", "cpp", "f16_check.cpp"),
                    os.path.join(src, "bvh_build.cpp"), "-o", exe, "-lpthread"], check=True)
    return exe


def test_half_values_are_ieee_binary16(f16_check, tmp_path):
    import subprocess
    out = tmp_path / "h.bin"
    subprocess.run([f16_check, "halves", str(out)], check=True)
    got = np.fromfile(out, np.float32)
    want = np.arange(65536, dtype=np.uint16).view(np.float16).astype(np.float32)
    nan = np.isnan(want)
    assert (np.isnan(got) == nan).all() and (got[~nan] == want[~nan]).all()


def test_directed_rounding_to_half_brackets_every_float(f16_check, tmp_path):
    """Down and up roundings: down <= x <= up, equal when x is a half, else
    neighbours; beyond the half range the outward side is infinite."""
    import subprocess
    rng = np.random.default_rng(3)
    x = np.concatenate([rng.uniform(-2, 2, 20000), rng.normal(0, 1e-5, 2000), rng.uniform(-7e4, 7e4, 2000),
                        np.arange(-2048, 2048, dtype=np.float16).astype(np.float64) / 256.0,
                        [0.0, -0.0, 65504.0, -65504.0, 65520.0, 1e6, -1e6, 6e-8, -6e-8, 1e-9]]).astype(np.float32)
    inp, out = tmp_path / "x.bin", tmp_path / "r.bin"
    x.tofile(inp)
    subprocess.run([f16_check, "round", str(inp), str(out)], check=True)
    r = np.fromfile(out, np.uint16).reshape(-1, 2)
    dn, up = r[:, 0].view(np.float16).astype(np.float64), r[:, 1].view(np.float16).astype(np.float64)
    xd = x.astype(np.float64)
    assert (dn <= xd).all() and (up >= xd).all()
    with np.errstate(over="ignore"):
        exact = x.astype(np.float16).astype(np.float64) == xd
    assert (dn[exact] == xd[exact]).all() and (up[exact] == xd[exact]).all()
    fin = ~exact & np.isfinite(dn) & np.isfinite(up)
    assert (np.nextafter(dn[fin].astype(np.float16), np.float16(np.inf)).astype(np.float64) == up[fin]).all()
    assert np.isinf(up[xd > 65504]).all() and np.isinf(dn[xd < -65504]).all()


@pytest.mark.parametrize("case", ["soup", "tiny1", "deep"])
def test_half_nodes_contain_the_fp32_boxes(f16_check, tmp_path, case):
    import subprocess
    from rise_b200 import scenes
    tri = {"soup": lambda: scenes.soup_triangles(20000, seed=4), "tiny1": lambda: scenes.soup_triangles(1, seed=1),
           "deep": scenes.nested_clusters}[case]()
    tp = tmp_path / "tri.bin"
    np.ascontiguousarray(tri, np.float32).tofile(tp)
    out = subprocess.run([f16_check, "nodes", str(tp)], capture_output=True, text=True)
    assert out.returncode == 0 and out.stdout.startswith("ok"), out.stdout + out.stderr
