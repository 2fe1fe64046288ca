"""Writer of .risemesh byte streams for the tests, following the layout of the
reference's TriangleMeshGeometryIndexed::Serialize
(Geometry/TriangleMeshGeometryIndexed.cpp:615-745) and BVH::Serialize
(Acceleration/BVH.h:353-373): little-endian, signature "RISETMGI", version,
geometry lists, indexed triangles, double-sided flag, optional BVH2 cache.
"""
import struct

import numpy as np


def risemesh_bytes(points, tris, double_sided=True, version=5, nodes2=None, prims=None, normals=None,
                   coords=None, colors=None, face_normals=False, legacy_tree=False):
    points = np.asarray(points, np.float64).reshape(-1, 3)
    tris = np.asarray(tris, np.uint32).reshape(-1, 3)
    normals = np.zeros((0, 3)) if normals is None else np.asarray(normals, np.float64).reshape(-1, 3)
    coords = np.zeros((0, 2)) if coords is None else np.asarray(coords, np.float64).reshape(-1, 2)
    colors = np.zeros((0, 3)) if colors is None else np.asarray(colors, np.float64).reshape(-1, 3)
    out = [b"RISETMGI", struct.pack("<I", version)]
    if version < 4:
        out.append(struct.pack("<Ib", 8, 24))         # legacy octree settings
    out.append(struct.pack("<b", 1 if face_normals else 0))
    for arr in (points, normals, coords):
        out.append(struct.pack("<I", len(arr)))
        out.append(np.ascontiguousarray(arr, "<f8").tobytes())
    if version >= 5:
        out.append(struct.pack("<I", len(colors)))
        out.append(np.ascontiguousarray(colors, "<f8").tobytes())
    out.append(struct.pack("<I", len(tris)))
    idx = np.zeros((len(tris), 3, 3), np.uint32)
    idx[:, :, 0] = tris
    if len(normals):
        idx[:, :, 1] = tris % len(normals)
    if len(coords):
        idx[:, :, 2] = tris % len(coords)
    out.append(np.ascontiguousarray(idx, "<u4").tobytes())
    out.append(struct.pack("<b", 1 if double_sided else 0))
    if version < 4:
        out.append(struct.pack("<bb", 0, 1 if legacy_tree else 0))
    if version >= 3 and len(tris):
        if nodes2 is None:
            out.append(struct.pack("<b", 0))
        else:
            nodes2 = np.ascontiguousarray(nodes2).view(np.uint8)
            out.append(struct.pack("<b", 1))
            out.append(b"BVH2" + struct.pack("<II", 1, len(nodes2) // 32))
            out.append(nodes2.tobytes())
            prims = np.asarray(prims, np.uint32)
            out.append(struct.pack("<I", len(prims)) + np.ascontiguousarray(prims, "<u4").tobytes())
            lo, hi = points.min(axis=0), points.max(axis=0)
            out.append(struct.pack("<6d", *lo, *hi))
    return b"".join(out)


def soup_mesh(tri9):
    """Points and indexed triangles of a triangle soup (3 points per triangle)."""
    tri9 = np.asarray(tri9, np.float32).reshape(-1, 9)
    return tri9.reshape(-1, 3).astype(np.float64), np.arange(3 * len(tri9), dtype=np.uint32).reshape(-1, 3)
