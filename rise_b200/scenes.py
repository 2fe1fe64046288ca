"""Seeded synthetic workloads for the ray caster and the path tracer.

Ray-cast microbenchmark (`soup_triangles`, `sphere_rays`): N random
triangles whose centroids are uniform in the unit cube and whose three
vertices are offset from the centroid by N(0, 0.01^2) per coordinate; rays
start uniformly on a sphere of radius 2 around the cube centre (0.5, 0.5,
0.5) and point at uniform targets inside the cube.  Closest-hit rays have an
unbounded range; any-hit (shadow) rays end at their target.

All arrays are float32.  Rays are packed 8 floats each:
(ox, oy, oz, tmin, dx, dy, dz, tmax) with a unit direction.
"""
import numpy as np

CUBE_CENTRE = np.array([0.5, 0.5, 0.5], np.float64)
SPHERE_RADIUS = 2.0
VERTEX_SIGMA = 0.01


def soup_triangles(n_tri, seed=7):
    """Triangle soup, (n_tri, 9) float32: v0, v1, v2 per row."""
    rng = np.random.default_rng(seed)
    c = rng.random((n_tri, 1, 3))
    v = c + rng.normal(0.0, VERTEX_SIGMA, (n_tri, 3, 3))
    return v.reshape(n_tri, 9).astype(np.float32)


def sphere_rays(n_rays, seed=7, shadow=False):
    """Rays from a radius-2 sphere towards uniform targets in the unit cube.

    Closest-hit rays get tmax = +inf; shadow rays (`shadow=True`) get
    tmax = |target - origin| so they test visibility of the target point.
    Uses its own stream (seed + 1) so the triangles and rays of one seed are
    independent.
    """
    rng = np.random.default_rng(seed + 1)
    z = rng.normal(size=(n_rays, 3))
    z /= np.linalg.norm(z, axis=1, keepdims=True)
    o = CUBE_CENTRE + SPHERE_RADIUS * z
    tgt = rng.random((n_rays, 3))
    d = tgt - o
    dist = np.linalg.norm(d, axis=1)
    d /= dist[:, None]
    rays = np.empty((n_rays, 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 3] = 0.0
    rays[:, 4:7] = d
    rays[:, 7] = dist if shadow else np.inf
    return rays
