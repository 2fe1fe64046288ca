""".risemesh reading (host side, no GPU): the reference's mesh format with its
BVH2 cache.  The cache fixture is the reference's own BVH over the 2,000
triangle golden soup (tests/golden/bvh_soup_2k.npz, made by the reference's
BVH template): read back from a .risemesh, its collapse to four-wide nodes
must equal the reference's, byte for byte."""
import os
import struct

import numpy as np
import pytest

from rise_b200 import raycaster
from rise_b200._native import RTB200Error

from risemesh_io import risemesh_bytes, soup_mesh

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def soup():
    g = np.load(os.path.join(GOLDEN, "bvh_soup_2k.npz"))
    return g


def parse(data):
    return raycaster.RiseMesh(data)


@pytest.mark.parametrize("version", [3, 4, 5])
def test_cached_bvh_collapses_to_the_reference_nodes(soup, version):
    pts, tris = soup_mesh(soup["tri9"])
    m = parse(risemesh_bytes(pts, tris, version=version, nodes2=soup["nodes2"], prims=soup["prims"],
                             normals=np.ones((7, 3)), coords=np.zeros((5, 2)), colors=np.ones((3, 3))))
    try:
        info = m.info()
        assert info == {"version": version, "n_points": 6000, "n_tri": 2000, "double_sided": True,
                        "n_bvh_nodes": len(soup["nodes2"]) // 32}
        n2, prims, n4 = m.host_bvh(True)
        assert n2.tobytes() == soup["nodes2"].tobytes()
        assert np.array_equal(prims, soup["prims"])
        assert n4.tobytes() == soup["nodes4"].tobytes()
    finally:
        m.close()


@pytest.mark.parametrize("version", [1, 2, 4, 5])
def test_without_cache_builds_the_reference_bvh(soup, version):
    pts, tris = soup_mesh(soup["tri9"])
    m = parse(risemesh_bytes(pts, tris, version=version, double_sided=False))
    try:
        assert m.info()["n_bvh_nodes"] == 0 and not m.info()["double_sided"]
        n2, prims, n4 = m.host_bvh(True)
        assert n2.tobytes() == soup["nodes2"].tobytes() and n4.tobytes() == soup["nodes4"].tobytes()
    finally:
        m.close()


def test_cache_with_a_different_layout_is_kept(soup):
    """A valid cache that is not what a fresh build gives (the reference's
    tree with every box grown by 0.01) is used as read, not rebuilt."""
    tri9 = soup["tri9"]
    n2 = soup["nodes2"].view(raycaster.NODE2_DTYPE).copy()
    n2["bmin"] -= 0.01
    n2["bmax"] += 0.01
    prims = soup["prims"]
    pts, tris = soup_mesh(tri9)
    m = parse(risemesh_bytes(pts, tris, nodes2=n2, prims=prims))
    try:
        c2, cp, _ = m.host_bvh(True)
        assert c2.tobytes() == n2.tobytes() and np.array_equal(cp, prims)
        assert c2.tobytes() != soup["nodes2"].tobytes()
        b2, _, _ = m.host_bvh(False)
        assert b2.tobytes() == soup["nodes2"].tobytes()
    finally:
        m.close()


def test_malformed_files_are_refused(soup):
    pts, tris = soup_mesh(soup["tri9"][:50])
    n2, prims, _ = raycaster.build_host_bvh(soup["tri9"][:50])
    good = risemesh_bytes(pts, tris, nodes2=n2, prims=prims)
    parse(good).close()
    bad = [
        b"RISETMGX" + good[8:],                                            # signature
        good[:8] + struct.pack("<I", 6) + good[12:],                       # version
        risemesh_bytes(pts, np.where(tris == 7, 10 ** 6, tris)),           # point index
        risemesh_bytes(pts, tris, nodes2=n2, prims=np.where(prims == 3, 50, prims)),   # leaf index
        risemesh_bytes(pts, tris, nodes2=n2, prims=prims[:-1]),           # leaf order too short
        risemesh_bytes(pts, tris, version=3, legacy_tree=True),          # legacy tree block
    ]
    # every truncation of the good file
    bad += [good[:k] for k in range(0, len(good), max(1, len(good) // 97))]
    for data in bad:
        with pytest.raises(RTB200Error):
            parse(data)


def test_malformed_cache_is_refused_when_used(soup):
    tri9 = soup["tri9"][:200]
    n2, prims, _ = raycaster.build_host_bvh(tri9)
    pts, tris = soup_mesh(tri9)
    loop = n2.copy()
    inner = np.nonzero(n2["count"] == 0)[0][1]
    loop["first"][inner] = inner          # an internal node whose children would be itself
    inverted = n2.copy()
    inverted["bmin"][0, 0] = inverted["bmax"][0, 0] + 1.0
    deep_leaf = n2.copy()
    leaf = np.nonzero(n2["count"] >= 2)[0][0]
    deep_leaf["first"][leaf] = 199        # leaf range past the end of the leaf order
    for nodes in (loop, inverted, deep_leaf):
        m = parse(risemesh_bytes(pts, tris, nodes2=nodes, prims=prims))
        try:
            with pytest.raises(RTB200Error):
                m.host_bvh(True)
            m.host_bvh(False)             # without the cache the mesh still builds
        finally:
            m.close()
