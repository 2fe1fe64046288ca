"""Parity rules for hit ids and distances against the reference BVH.

The reference intersects in double precision with a 1e-12 barycentric slack
(src/Library/Intersection/RayTriangleIntersection.cpp:21-68); the device
path intersects in FP32 with a watertight test.  They can legitimately
disagree only where a ray is within 1e-6 of a triangle edge, where two
triangles are hit at the same distance to within 4 FP32 ulps (ties are
resolved by traversal order in both), or, for shadow rays, where the only
blocker sits within 1e-6 (relative) of the ray's end.  Every other ray must
agree exactly: same triangle id, same hit/miss, distance within 4 ulps of
the reference's distance rounded to FP32.
"""
import numpy as np

EDGE_BAND = 1e-6
T_ULPS = 4


def _mt_all(tri9, o, d):
    """Double Moller-Trumbore of one ray against all triangles (numpy)."""
    v0 = tri9[:, 0:3].astype(np.float64)
    ea = tri9[:, 3:6].astype(np.float64) - v0
    eb = tri9[:, 6:9].astype(np.float64) - v0
    d = np.asarray(d, np.float64)
    o = np.asarray(o, np.float64)
    pv = np.cross(d[None, :], eb)
    det = np.einsum("ij,ij->i", ea, pv)
    ok = np.abs(det) >= 1e-12
    inv = np.where(ok, 1.0 / np.where(ok, det, 1.0), 0.0)
    tv = o[None, :] - v0
    a = np.einsum("ij,ij->i", tv, pv) * inv
    qv = np.cross(tv, ea)
    b = (qv @ d) * inv
    t = np.einsum("ij,ij->i", eb, qv) * inv
    hit = ok & (a >= -1e-12) & (a <= 1 + 1e-12) & (b >= -1e-12) & (a + b <= 1 + 1e-12) & (t >= 1e-12)
    return hit, t, a, b


def _edge_dist(tri, p):
    def seg(a, c):
        ab = c - a
        l2 = ab @ ab
        s = 0.0 if l2 <= 0 else np.clip((p - a) @ ab / l2, 0.0, 1.0)
        return np.linalg.norm(a + s * ab - p)
    t = tri.reshape(3, 3).astype(np.float64)
    return min(seg(t[0], t[1]), seg(t[1], t[2]), seg(t[2], t[0]))


def ulp_diff(t_gpu, t_ref):
    tr = np.float32(t_ref)
    return abs(np.float64(t_gpu) - np.float64(tr)) / np.float64(np.spacing(np.abs(tr)))


def closest_report(tri9, rays, hits, ref_ids, ref_t):
    """Classify GPU closest hits against the reference.  Returns a dict with
    'bad' (unexplained mismatches), 'excluded' (edge-band or tie rays),
    'max_ulp' over agreeing rays."""
    tri9 = np.asarray(tri9).reshape(-1, 9)
    rays = np.asarray(rays, np.float32).reshape(-1, 8)
    gid = hits["prim"].astype(np.int64)
    gt = hits["t"].astype(np.float64)
    same = gid == ref_ids
    excluded, bad = [], []
    for i in np.nonzero(~same)[0]:
        o, d = rays[i, 0:3].astype(np.float64), rays[i, 4:7].astype(np.float64)
        hit, t, _, _ = _mt_all(tri9, o, d)
        near_edge = False
        for tid, tt in ((ref_ids[i], ref_t[i]), (gid[i], None)):
            if tid >= 0:
                tt = t[tid] if tt is None else tt
                if np.isfinite(tt) and _edge_dist(tri9[tid], o + tt * d) < EDGE_BAND:
                    near_edge = True
        tie = False
        if ref_ids[i] >= 0 and gid[i] >= 0 and hit[gid[i]]:
            tie = ulp_diff(t[gid[i]], ref_t[i]) <= T_ULPS
        (excluded if (near_edge or tie) else bad).append(int(i))
    agree = same & (ref_ids >= 0)
    ulps = np.array([ulp_diff(gt[i], ref_t[i]) for i in np.nonzero(agree)[0]]) if agree.any() else np.zeros(0)
    return {"n": len(rays), "bad": bad, "excluded": excluded,
            "max_ulp": float(ulps.max()) if len(ulps) else 0.0,
            "t_over": int((ulps > T_ULPS).sum())}


def any_report(tri9, rays, occ, ref_occ):
    """Classify GPU occlusion flags against the reference."""
    tri9 = np.asarray(tri9).reshape(-1, 9)
    rays = np.asarray(rays, np.float32).reshape(-1, 8)
    excluded, bad = [], []
    for i in np.nonzero(occ.astype(bool) != ref_occ.astype(bool))[0]:
        o, d = rays[i, 0:3].astype(np.float64), rays[i, 4:7].astype(np.float64)
        tmax = float(rays[i, 7])
        hit, t, _, _ = _mt_all(tri9, o, d)
        cand = np.nonzero(hit & (t < tmax * (1 + EDGE_BAND)))[0]
        marginal = len(cand) > 0 and all(
            abs(t[c] - tmax) <= EDGE_BAND * max(1.0, tmax) or _edge_dist(tri9[c], o + t[c] * d) < EDGE_BAND
            for c in cand)
        (excluded if marginal else bad).append(int(i))
    return {"n": len(rays), "bad": bad, "excluded": excluded}


# ---- image statistics ---------------------------------------------------------
# Per-pixel z-test of two renderers at equal samples per pixel: each side gives
# K independent batches; z = (mean_a - mean_b) / sqrt(var_a / K + var_b / K)
# per pixel and channel (var with ddof 1).  With Gaussian batch means, |z| > 3
# has probability 0.27 %; the test allows three times that, which covers the
# heavier tails of a statistic whose variances are themselves estimated from
# 16 batches (about 0.5 % expected).
Z_LIMIT = 3.0
Z_GAUSS_RATE = 0.0027
Z_ALLOWED_RATE = 3 * Z_GAUSS_RATE


def z_scores(mean_a, var_a, k_a, mean_b, var_b, k_b):
    """z per pixel and channel where either side has any variance."""
    den = np.sqrt(var_a / k_a + var_b / k_b)
    ok = den > 0
    return (mean_a - mean_b)[ok] / den[ok], ok


def rel_mse(x, ref):
    """Mean over pixels and channels of (x - r)^2 / (r^2 + 1e-2)."""
    return float(np.mean((x - ref) ** 2 / (ref ** 2 + 1e-2)))
