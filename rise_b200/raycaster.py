"""Host-side mirror of the reference's ray-caster surface, over the C ABI.

The reference casts one ray per virtual call (IRayCaster::CastRay /
CastShadowRay, src/Library/Interfaces/IRayCaster.h:87-199, implemented by
RayCaster.cpp:1958-1966 and ObjectManager::IntersectRay /
IntersectShadowRay, src/Library/Managers/ObjectManager.cpp:270-374).  Here
the same queries are batched: `RayCaster.cast_rays` is the closest-hit query
and `RayCaster.cast_shadow_rays` the any-hit (occlusion) query, each over an
array of rays, on the GPU.
"""
import ctypes

import numpy as np

from . import _native
from ._native import check, lib

RAY_DTYPE = np.dtype([("ox", "<f4"), ("oy", "<f4"), ("oz", "<f4"), ("tmin", "<f4"),
                      ("dx", "<f4"), ("dy", "<f4"), ("dz", "<f4"), ("tmax", "<f4")])
HIT_DTYPE = np.dtype([("t", "<f4"), ("prim", "<i4"), ("a", "<f4"), ("b", "<f4")])
NODE2_DTYPE = np.dtype([("bmin", "<f4", 3), ("bmax", "<f4", 3), ("first", "<u4"),
                        ("count", "<u2"), ("axis", "u1"), ("pad", "u1")])
NODE4_DTYPE = np.dtype([("minx", "<f4", 4), ("miny", "<f4", 4), ("minz", "<f4", 4),
                        ("maxx", "<f4", 4), ("maxy", "<f4", 4), ("maxz", "<f4", 4),
                        ("child", "<i4", 4), ("count", "<u2", 4), ("nchild", "u1"),
                        ("axis", "u1"), ("pad", "u1", 6)])

LAYOUTS = {"f32": _native.BVH_F32, "q8": _native.BVH_Q8, "w8": _native.BVH_W8, "f16": _native.BVH_F16}


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


class Context:
    """Owns a CUDA stream and all device memory of its scenes and jobs."""

    def __init__(self, device=0, budget_bytes=0):
        h = ctypes.c_void_p()
        check(lib().rtb200_ctx_create(device, budget_bytes, ctypes.byref(h)))
        self.h = h
        self.device = device

    def bytes_in_use(self):
        return lib().rtb200_ctx_bytes_in_use(self.h)

    def close(self):
        if self.h:
            lib().rtb200_ctx_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class Scene:
    """Triangle geometry plus its BVH, resident on the device once committed."""

    def __init__(self, ctx):
        self.ctx = ctx
        h = ctypes.c_void_p()
        check(lib().rtb200_scene_create(ctx.h, ctypes.byref(h)), ctx.h)
        self.h = h
        self.n_tri = 0

    def add_mesh(self, xyz, tri, material=0, double_sided=True):
        xyz = np.ascontiguousarray(xyz, np.float32).reshape(-1, 3)
        tri = np.ascontiguousarray(tri, np.uint32).reshape(-1, 3)
        check(lib().rtb200_scene_add_mesh(self.h, _ptr(xyz), len(xyz), _ptr(tri), len(tri),
                                          int(material), int(bool(double_sided))), self.ctx.h)
        self.n_tri += len(tri)

    def add_triangles(self, tri9, material=0, double_sided=True, normals9=None):
        """Add a triangle soup given as (n, 9) floats: v0, v1, v2 per row;
        normals9, the same shape, gives vertex normals per corner for smooth
        shading."""
        tri9 = np.ascontiguousarray(tri9, np.float32).reshape(-1, 9)
        idx = np.arange(3 * len(tri9), dtype=np.uint32).reshape(-1, 3)
        if normals9 is None:
            self.add_mesh(tri9.reshape(-1, 3), idx, material, double_sided)
            return
        nrm = np.ascontiguousarray(normals9, np.float32).reshape(-1, 3)
        xyz = tri9.reshape(-1, 3)
        check(lib().rtb200_scene_add_mesh_normals(self.h, _ptr(xyz), len(xyz), _ptr(idx), len(idx), _ptr(nrm),
                                                  len(nrm), _ptr(idx), int(material), int(bool(double_sided))),
              self.ctx.h)
        self.n_tri += len(idx)

    def add_risemesh(self, mesh, material=0, use_cached_bvh=True):
        """Add a parsed RiseMesh; its BVH2 cache (if any) replaces the SAH
        build of this mesh when use_cached_bvh."""
        check(lib().rtb200_scene_add_risemesh(self.h, mesh.h, int(material), int(bool(use_cached_bvh))), self.ctx.h)
        self.n_tri += mesh.info()["n_tri"]

    def commit(self, layout="f32"):
        check(lib().rtb200_scene_commit(self.h, LAYOUTS[layout]), self.ctx.h)
        self.layout = layout

    def info(self):
        n_tri, n_nodes, nbytes = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        secs = ctypes.c_double()
        check(lib().rtb200_scene_info(self.h, ctypes.byref(n_tri), ctypes.byref(n_nodes),
                                      ctypes.byref(nbytes), ctypes.byref(secs)), self.ctx.h)
        return {"n_tri": n_tri.value, "n_nodes": n_nodes.value, "device_bytes": nbytes.value,
                "build_seconds": secs.value}

    def close(self):
        if self.h:
            lib().rtb200_scene_destroy(self.h)
            self.h = None


class RayCaster:
    """Batched closest-hit and shadow queries against one committed scene."""

    def __init__(self, scene):
        self.scene = scene

    def cast_rays(self, rays):
        """Closest hit per ray (host arrays).  rays: (n, 8) float32 or RAY_DTYPE."""
        rays = np.ascontiguousarray(rays).view(np.float32).reshape(-1, 8)
        hits = np.empty(len(rays), HIT_DTYPE)
        check(lib().rtb200_cast_closest(self.scene.h, _ptr(rays), len(rays), _ptr(hits)), self.scene.ctx.h)
        return hits

    def cast_shadow_rays(self, rays):
        """Occlusion per ray within (tmin, tmax) (host arrays) -> uint8 array."""
        rays = np.ascontiguousarray(rays).view(np.float32).reshape(-1, 8)
        occ = np.empty(len(rays), np.uint8)
        check(lib().rtb200_cast_any(self.scene.h, _ptr(rays), len(rays), _ptr(occ)), self.scene.ctx.h)
        return occ

    def cast_rays_device(self, d_rays, d_hits, n, stream=None):
        """Closest hit on device pointers (ints), asynchronous on `stream`."""
        check(lib().rtb200_cast_closest_device(self.scene.h, ctypes.c_void_p(d_rays), n,
                                               ctypes.c_void_p(d_hits), ctypes.c_void_p(stream)),
              self.scene.ctx.h)

    def cast_shadow_rays_device(self, d_rays, d_occ, n, stream=None):
        check(lib().rtb200_cast_any_device(self.scene.h, ctypes.c_void_p(d_rays), n,
                                           ctypes.c_void_p(d_occ), ctypes.c_void_p(stream)),
              self.scene.ctx.h)


class RiseMesh:
    """A parsed .risemesh file (the reference's mesh format, v1..v5, with its
    optional BVH2 cache)."""

    def __init__(self, data):
        data = bytes(data)
        buf = ctypes.create_string_buffer(data, len(data))
        h = ctypes.c_void_p()
        check(lib().rtb200_risemesh_parse(buf, len(data), ctypes.byref(h)))
        self.h = h

    @classmethod
    def from_file(cls, path):
        with open(path, "rb") as f:
            return cls(f.read())

    def info(self):
        v, ds = ctypes.c_int32(), ctypes.c_int32()
        npt, ntri, nn = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        check(lib().rtb200_risemesh_info(self.h, ctypes.byref(v), ctypes.byref(npt), ctypes.byref(ntri),
                                         ctypes.byref(ds), ctypes.byref(nn)))
        return {"version": v.value, "n_points": npt.value, "n_tri": ntri.value, "double_sided": bool(ds.value),
                "n_bvh_nodes": nn.value}

    def triangles(self):
        """(n, 9) float32 triangles (v0, v1, v2)."""
        out = np.zeros((self.info()["n_tri"], 9), np.float32)
        check(lib().rtb200_risemesh_triangles(self.h, _ptr(out)))
        return out

    def normals(self):
        """(n, 9) float32 vertex normals per triangle corner, or None when the
        mesh shades with face normals."""
        out = np.zeros((self.info()["n_tri"], 9), np.float32)
        if lib().rtb200_risemesh_normals(self.h, _ptr(out)) != 0:
            return None
        return out

    def host_bvh(self, use_cached_bvh=True):
        """(nodes2, prims, nodes4) as a scene commit would use them."""
        h = ctypes.c_void_p()
        check(lib().rtb200_bvh_host_from_risemesh(self.h, int(bool(use_cached_bvh)), ctypes.byref(h)))
        return _export_host_bvh(h, self.info()["n_tri"])

    def close(self):
        if self.h:
            lib().rtb200_risemesh_destroy(self.h)
            self.h = None


def _export_host_bvh(h, n_tri):
    try:
        n2, n4 = ctypes.c_int64(), ctypes.c_int64()
        check(lib().rtb200_bvh_host_info(h, ctypes.byref(n2), ctypes.byref(n4)))
        nodes2 = np.zeros(n2.value, NODE2_DTYPE)
        prims = np.zeros(n_tri, np.uint32)
        nodes4 = np.zeros(n4.value, NODE4_DTYPE)
        check(lib().rtb200_bvh_host_export(h, _ptr(nodes2), _ptr(prims), _ptr(nodes4)))
        return nodes2, prims, nodes4
    finally:
        lib().rtb200_bvh_host_destroy(h)


def build_host_bvh(tri9, threads=0):
    """Build the reference BVH on the host: (nodes2, prims, nodes4) arrays."""
    tri9 = np.ascontiguousarray(tri9, np.float32).reshape(-1, 9)
    h = ctypes.c_void_p()
    check(lib().rtb200_bvh_host_build(_ptr(tri9), len(tri9), threads, ctypes.byref(h)))
    return _export_host_bvh(h, len(tri9))
