"""GPU ray casting against the reference BVH (through the C ABI).

Closest-hit ids must equal the reference's, hit distances must be within 4
FP32 ulps of the reference's double distance, and shadow-ray occlusion must
agree, except for the rays tests/parity.py explains (edge band 1e-6, equal
distance ties, blockers at the shadow ray's end).  Both BVH layouts (FP32
and 8-bit quantised child boxes) are held to the same bar.
"""
import os

import numpy as np
import pytest

import oracle
from rise_b200 import raycaster, scenes

from parity import any_report, closest_report

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
LAYOUTS = ["f32", "q8", "w8", "f16"]


@pytest.fixture(scope="module")
def ctx():
    c = raycaster.Context(0)
    yield c
    c.close()


def make_caster(ctx, tri9, layout):
    s = raycaster.Scene(ctx)
    s.add_triangles(tri9)
    s.commit(layout)
    return s, raycaster.RayCaster(s)


@pytest.mark.parametrize("layout", LAYOUTS)
def test_golden_closest_and_any(ctx, layout):
    g = np.load(os.path.join(GOLDEN, "bvh_soup_2k.npz"))
    s, rc = make_caster(ctx, g["tri9"], layout)
    hits = rc.cast_rays(g["rays"])
    rep = closest_report(g["tri9"], g["rays"], hits, g["ids"], g["t"])
    assert rep["bad"] == [] and rep["t_over"] == 0, rep
    occ = rc.cast_shadow_rays(g["shadow_rays"])
    arep = any_report(g["tri9"], g["shadow_rays"], occ, g["occluded"])
    assert arep["bad"] == [], arep
    s.close()


@pytest.mark.parametrize("layout", LAYOUTS)
@pytest.mark.parametrize("n_tri,n_rays", [(1, 1000), (5, 1000), (50000, 100000), (300000, 100000)])
def test_random_soup_parity(ctx, layout, n_tri, n_rays):
    tri = scenes.soup_triangles(n_tri, seed=n_tri + 1)
    rays = scenes.sphere_rays(n_rays, seed=n_tri + 1)
    srays = scenes.sphere_rays(n_rays, seed=n_tri + 2, shadow=True)
    s, rc = make_caster(ctx, tri, layout)
    ob = oracle.BVH(tri, "port")
    ids, t = ob.closest(rays)
    hits = rc.cast_rays(rays)
    rep = closest_report(tri, rays, hits, ids, t)
    assert rep["bad"] == [] and rep["t_over"] == 0, {k: rep[k] for k in ("bad", "t_over", "max_ulp")}
    assert len(rep["excluded"]) <= max(2, n_rays // 1000)
    occ = rc.cast_shadow_rays(srays)
    arep = any_report(tri, srays, occ, ob.any(srays))
    assert arep["bad"] == [], arep
    s.close()


@pytest.mark.parametrize("layout", LAYOUTS)
def test_edge_cases(ctx, layout):
    # One unit triangle in z = 0 plus a far one; axis-aligned rays with zero
    # direction components, rays clipped by tmax / tmin, rays from behind.
    tri = np.array([[0, 0, 0, 1, 0, 0, 0, 1, 0],
                    [0, 0, 5, 1, 0, 5, 0, 1, 5]], np.float32)
    s, rc = make_caster(ctx, tri, layout)
    inf = np.inf
    rays = np.array([
        [0.25, 0.25, 1, 0, 0, 0, -1, inf],      # straight down: hit tri 0 at t=1
        [0.25, 0.25, 1, 0, 0, 0, -1, 0.5],      # clipped by tmax
        [0.25, 0.25, 1, 1.5, 0, 0, -1, inf],    # tmin past tri 0 -> nothing below
        [0.25, 0.25, 10, 0, 0, 0, -1, inf],     # hits tri 1 (z=5) first at t=5
        [0.75, 0.75, 1, 0, 0, 0, -1, inf],      # outside the hypotenuse: miss
        [0.25, 0.25, -1, 0, 0, 0, 1, inf],      # from below: back face, t=1
        [0.25, 0.25, 1, 0, 1, 0, 0, inf],       # parallel to the plane: miss
        [-5, 0.25, 0.0, 0, 1, 0, 0, inf],       # in the plane: degenerate, miss
    ], np.float32)
    hits = rc.cast_rays(rays)
    assert list(hits["prim"]) == [0, -1, -1, 1, -1, 0, -1, -1]
    assert hits["t"][0] == 1.0 and hits["t"][3] == 5.0 and hits["t"][5] == 1.0
    assert abs(hits["a"][0] - 0.25) < 1e-6 and abs(hits["b"][0] - 0.25) < 1e-6
    sr = rays.copy()
    sr[:, 7] = [2, 0.5, inf, 4.9, 2, 2, 2, 2]
    occ = rc.cast_shadow_rays(sr)
    assert list(occ) == [1, 0, 0, 0, 0, 1, 0, 0]
    assert len(rc.cast_rays(np.zeros((0, 8), np.float32))) == 0
    s.close()


@pytest.mark.parametrize("layout", LAYOUTS)
def test_deep_bvh_local_stack_parity(ctx, layout):
    # A BVH whose traversal stack bound (46) exceeds the shared-memory part
    # (40) runs the kernels that continue the stack in local memory.
    tri = scenes.nested_clusters()
    rays = scenes.cluster_rays(tri, 20000, seed=3)
    srays = scenes.cluster_rays(tri, 20000, seed=4, shadow=True)
    s, rc = make_caster(ctx, tri, layout)
    ob = oracle.BVH(tri, "port")
    ids, t = ob.closest(rays)
    hits = rc.cast_rays(rays)
    rep = closest_report(tri, rays, hits, ids, t)
    assert rep["bad"] == [] and rep["t_over"] == 0, {k: rep[k] for k in ("bad", "t_over", "max_ulp")}
    assert (ids >= 0).mean() > 0.3   # rays at triangles below the 1e-12 determinant miss
    occ = rc.cast_shadow_rays(srays)
    arep = any_report(tri, srays, occ, ob.any(srays))
    assert arep["bad"] == [], arep
    s.close()


def test_layouts_agree_and_are_deterministic(ctx):
    tri = scenes.soup_triangles(200000, seed=5)
    rays = scenes.sphere_rays(500000, seed=5)
    sf, rf = make_caster(ctx, tri, "f32")
    sq, rq = make_caster(ctx, tri, "q8")
    sw, rw = make_caster(ctx, tri, "w8")
    sh, rh = make_caster(ctx, tri, "f16")
    a = rf.cast_rays(rays)
    b = rq.cast_rays(rays)
    c = rf.cast_rays(rays)
    w = rw.cast_rays(rays)
    w2 = rw.cast_rays(rays)
    assert (a["prim"] == c["prim"]).all() and (a["t"] == c["t"]).all()
    assert (w["prim"] == w2["prim"]).all() and (w["t"] == w2["t"]).all()
    assert (a["prim"] == b["prim"]).mean() > 0.99999
    assert (a["prim"] == w["prim"]).mean() > 0.99999
    h = rh.cast_rays(rays)
    assert (a["prim"] == h["prim"]).mean() > 0.99999
    sh.close()
    sf.close()
    sq.close()
    sw.close()


def test_device_api_matches_host_api(ctx):
    torch = pytest.importorskip("torch")
    tri = scenes.soup_triangles(20000, seed=9)
    rays = scenes.sphere_rays(65536, seed=9)
    s, rc = make_caster(ctx, tri, "f32")
    host = rc.cast_rays(rays)
    d_rays = torch.from_numpy(rays).cuda()
    d_hits = torch.empty((len(rays), 4), dtype=torch.float32, device="cuda")
    rc.cast_rays_device(d_rays.data_ptr(), d_hits.data_ptr(), len(rays), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    dev = d_hits.cpu().numpy().view(raycaster.HIT_DTYPE).reshape(-1)
    assert (dev["prim"] == host["prim"]).all() and (dev["t"] == host["t"]).all()
    s.close()


@pytest.mark.parametrize("layout", LAYOUTS)
def test_full_size_microbench_sample(ctx, layout):
    """1,000,000 triangles, 4,194,304 rays (the microbenchmark's full size):
    every ray is cast; a seeded sample of 20,000 is checked against the
    oracle, and the whole batch for hit rate and determinism."""
    tri = scenes.soup_triangles(1_000_000, seed=7)
    rays = scenes.sphere_rays(4_194_304, seed=7)
    s, rc = make_caster(ctx, tri, layout)
    hits = rc.cast_rays(rays)
    again = rc.cast_rays(rays)
    assert (hits["prim"] == again["prim"]).all()
    assert (hits["prim"] >= 0).mean() > 0.999
    idx = np.random.default_rng(0).choice(len(rays), 20000, replace=False)
    ids, t = oracle.BVH(tri, "port").closest(rays[idx])
    rep = closest_report(tri, rays[idx], hits[idx], ids, t)
    assert rep["bad"] == [] and rep["t_over"] == 0, {k: rep[k] for k in ("bad", "t_over", "max_ulp")}
    s.close()


@pytest.mark.parametrize("layout", LAYOUTS)
def test_risemesh_cache_traversal_matches_reference(ctx, layout):
    """A scene of one .risemesh whose BVH2 cache is the reference's own tree
    over the golden soup traverses that tree: the reference's hits."""
    from risemesh_io import risemesh_bytes, soup_mesh
    g = np.load(os.path.join(GOLDEN, "bvh_soup_2k.npz"))
    pts, tris = soup_mesh(g["tri9"])
    m = raycaster.RiseMesh(risemesh_bytes(pts, tris, nodes2=g["nodes2"], prims=g["prims"]))
    s = raycaster.Scene(ctx)
    try:
        s.add_risemesh(m)
        s.commit(layout)
        rc = raycaster.RayCaster(s)
        hits = rc.cast_rays(g["rays"])
        rep = closest_report(g["tri9"], g["rays"], hits, g["ids"], g["t"])
        assert rep["bad"] == [] and rep["t_over"] == 0, rep
        occ = rc.cast_shadow_rays(g["shadow_rays"])
        assert any_report(g["tri9"], g["shadow_rays"], occ, g["occluded"])["bad"] == []
    finally:
        s.close()
        m.close()


@pytest.mark.parametrize("layout", LAYOUTS)
def test_two_level_scene_with_cached_and_built_meshes(ctx, layout):
    """Cached meshes beside plain ones: the scene is a top level over per-mesh
    trees; hits equal the oracle's over all triangles."""
    from risemesh_io import risemesh_bytes, soup_mesh
    parts = [scenes.soup_triangles(3000, seed=41), scenes.soup_triangles(2000, seed=42) + np.float32(0.4),
             scenes.soup_triangles(1000, seed=43) - np.float32(0.3)]
    s = raycaster.Scene(ctx)
    meshes = []
    try:
        for k, tri in enumerate(parts):
            if k == 1:
                s.add_triangles(tri)           # built with the reference SAH at commit
                continue
            n2, prims, _ = raycaster.build_host_bvh(tri)
            pts, tris = soup_mesh(tri)
            m = raycaster.RiseMesh(risemesh_bytes(pts, tris, nodes2=n2, prims=prims))
            meshes.append(m)
            s.add_risemesh(m)
        s.commit(layout)
        allt = np.concatenate(parts)
        rays = scenes.sphere_rays(50000, seed=44)
        srays = scenes.sphere_rays(50000, seed=45, shadow=True)
        rc = raycaster.RayCaster(s)
        ob = oracle.BVH(allt, "port")
        ids, t = ob.closest(rays)
        rep = closest_report(allt, rays, rc.cast_rays(rays), ids, t)
        assert rep["bad"] == [] and rep["t_over"] == 0, {k: rep[k] for k in ("bad", "t_over", "max_ulp")}
        assert len(rep["excluded"]) <= 50
        assert any_report(allt, srays, rc.cast_shadow_rays(srays), ob.any(srays))["bad"] == []
    finally:
        s.close()
        for m in meshes:
            m.close()
