"""Seeded synthetic workloads for the ray caster and the path tracer.

Ray-cast microbenchmark (`soup_triangles`, `sphere_rays`): N random
triangles whose centroids are uniform in the unit cube and whose three
vertices are offset from the centroid by N(0, 0.01^2) per coordinate; rays
start uniformly on a sphere of radius 2 around the cube centre (0.5, 0.5,
0.5) and point at uniform targets inside the cube.  Closest-hit rays have an
unbounded range; any-hit (shadow) rays end at their target.

Path-tracing scenes are described by `SceneDesc` (triangle meshes with one
material each, spectra tabulated at 81 samples over 380..780 nm in 5 nm
steps, materials, optional uniform sky, pinhole camera and render
settings); `cornell_box` builds the 32-triangle spectral Cornell box.

All geometry is float32.  Rays are packed 8 floats each:
(ox, oy, oz, tmin, dx, dy, dz, tmax) with a unit direction.
"""
from dataclasses import dataclass, field

import math

import numpy as np

CUBE_CENTRE = np.array([0.5, 0.5, 0.5], np.float64)
SPHERE_RADIUS = 2.0
VERTEX_SIGMA = 0.01

WAVELENGTHS = np.arange(380.0, 781.0, 5.0)  # 81 spectrum samples
MAT_LAMBERTIAN, MAT_GGX, MAT_DIELECTRIC = 0, 1, 2


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


def nested_clusters(levels=30, ratio=0.3, per=5, scale=1e3, seed=1):
    """Self-similar clusters whose BVH is deep: level k holds three clusters of
    `per` small triangles near the corners (0.9,0.1,0.1), (0.1,0.9,0.1),
    (0.1,0.1,0.9) of a cube of side scale * ratio**k at the origin, and the
    next level nests inside it.  Every BVH4 node on the path down the levels
    has siblings to defer, so the traversal stack grows with the level count
    (46 deferred entries for the defaults)."""
    rng = np.random.default_rng(seed)
    corners = np.array([(0.9, 0.1, 0.1), (0.1, 0.9, 0.1), (0.1, 0.1, 0.9)])
    rows = []
    for k in range(levels):
        s = scale * ratio ** k
        for cc in corners:
            c = (cc + rng.uniform(-0.05, 0.05, (per, 3))) * s
            e = 0.03 * s
            rows.append(np.concatenate([c + [e, 0, 0], c + [0, e, 0], c + [0, 0, e]], axis=1))
    return np.concatenate(rows).astype(np.float32)


def cluster_rays(tri9, n_rays, seed=7, shadow=False):
    """Rays aimed at random triangles of `tri9` from 20 triangle sizes away,
    so rays reach every scale of a `nested_clusters` scene.  Shadow rays stop
    0.1 % short of the aim point, as a renderer's shadow ray stops short of the
    surface point it connects to (ending exactly on the aimed triangle would
    leave its occlusion to FP32 rounding)."""
    rng = np.random.default_rng(seed)
    t = tri9.reshape(-1, 3, 3).astype(np.float64)
    pick = rng.integers(0, len(t), n_rays)
    w = rng.dirichlet((1.0, 1.0, 1.0), n_rays)
    tgt = np.einsum("nk,nkj->nj", w, t[pick])
    size = np.linalg.norm(t[pick, 1] - t[pick, 0], axis=1)
    z = rng.normal(size=(n_rays, 3))
    z /= np.linalg.norm(z, axis=1, keepdims=True)
    o = tgt + 20.0 * size[:, None] * z
    d = tgt - o
    dist = np.linalg.norm(d, axis=1)
    d /= dist[:, None]
    rays = np.empty((n_rays, 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 3] = 0.0
    rays[:, 4:7] = d
    rays[:, 7] = dist * 0.999 if shadow else np.inf
    return rays


# ---- spectra -----------------------------------------------------------------

def flat_spectrum(value, lo=380.0, hi=780.0, outside=0.0):
    """`value` on [lo, hi] nm (inclusive grid points), `outside` elsewhere."""
    s = np.full(81, outside, np.float32)
    s[(WAVELENGTHS >= lo) & (WAVELENGTHS <= hi)] = value
    return s


# ---- path-tracing scene description ------------------------------------------

@dataclass
class Material:
    type: int = MAT_LAMBERTIAN
    reflectance: int = -1   # spectrum id
    emission: int = -1      # spectrum id (radiance)
    eta: int = -1
    kappa: int = -1
    alpha: float = 0.0
    ior: float = 1.5


@dataclass
class SpectralPacket:
    """A binned spectrum (the reference's SpectralPacket): len(amps) bins over
    [begin, end]; the value at nm is the amplitude of the bin holding it, 0
    outside the range."""
    begin: float
    end: float
    amps: np.ndarray

    def value_at(self, nm):
        nm = np.asarray(nm, np.float64)
        n = len(self.amps)
        delta = (float(self.end) - float(self.begin)) / n
        idx = np.minimum(((nm - self.begin) / delta).astype(np.int64), n - 1)
        inside = (nm >= self.begin) & (nm <= self.end)
        return np.where(inside, np.asarray(self.amps, np.float64)[np.clip(idx, 0, n - 1)], 0.0)


@dataclass
class SigmoidSpectrum:
    """An RGB colour's spectrum: scale * s(c0 t^2 + c1 t + c2), t = (nm -
    380) / 400 on 380..780 nm, s(x) = 1/2 + x / (2 sqrt(1 + x^2))."""
    c0: float
    c1: float
    c2: float
    scale: float = 1.0

    def value_at(self, nm):
        nm = np.asarray(nm, np.float64)
        t = (nm - 380.0) / 400.0
        x = self.c0 * t * t + self.c1 * t + self.c2
        v = self.scale * (0.5 + x / (2.0 * np.sqrt(1.0 + x * x)))
        return np.where((nm >= 380.0) & (nm <= 780.0), v, 0.0)


@dataclass
class BlackbodySpectrum:
    """A black body: scale * Planck's function (wavelength in metres), the
    scale divided by the function's value at 0.0029 / T m when normalize
    (BlackBodyPainter)."""
    temperature: float
    scale: float = 1.0
    normalize: bool = True

    @staticmethod
    def planck(t, lam):
        c, h, k = 2.99792458e8, 6.6260755e-34, 1.380658e-23
        c1, c2 = 2.0 * math.pi * h * (c * c), (h * c) / k
        return c1 / np.power(lam, 5.0) * (1.0 / (np.exp(c2 / (lam * t)) - 1.0))

    def effective_scale(self):
        s = float(self.scale)
        if self.normalize:
            s /= float(self.planck(float(self.temperature), 0.0029 / float(self.temperature)))
        return s

    def value_at(self, nm):
        t = float(np.float32(self.temperature))
        k = float(np.float32(self.effective_scale()))
        return k * self.planck(t, np.asarray(nm, np.float64) * 1e-9)


RGB_ALBEDO, RGB_UNBOUNDED = 0, 1


def rgb_spectrum(rgb, kind=RGB_ALBEDO):
    """The spectrum the reference's RGB painters give a linear Rec.709
    colour (Jakob-Hanika uplift, computed by the library's table): ALBEDO
    clamps to [0, 1], UNBOUNDED keeps the largest channel as a scale."""
    import ctypes
    from ._native import check, lib
    c = np.ascontiguousarray(rgb, np.float64).reshape(3)
    out = np.zeros(4)
    check(lib().rtb200_rgb_uplift(c.ctypes.data_as(ctypes.c_void_p), int(kind), out.ctypes.data_as(ctypes.c_void_p)))
    return SigmoidSpectrum(*out.tolist())


def spectral_painter(nm, amplitudes, nmbegin=400.0, nmend=700.0):
    """The spectrum of the reference's spectral_painter chunk
    (Job::AddSpectralColorPainter, Job.cpp:1557-1582): the control points
    (nm, amplitude) define a piecewise-linear function, constant beyond the
    first and last points (PiecewiseLinearFunction1D,
    Utilities/PiecewiseLinearFunction.h:60-90); it is sampled at
    nmbegin + i * (nmend - nmbegin) / n for the n = len(nm) bins of a
    SpectralPacket (SpectralPacket.h:80-100).  The chunk's `scale` scales
    only the painter's RGB colour, not its spectrum, so it has no argument
    here."""
    x = np.asarray(nm, np.float64)
    y = np.asarray(amplitudes, np.float64)
    order = np.argsort(x, kind="stable")
    x, y = x[order], y[order]
    n = len(x)
    delta = (float(nmend) - float(nmbegin)) / n
    amps = np.empty(n)
    for i in range(n):
        s = nmbegin + i * delta
        if n < 2:
            amps[i] = 1.0
        elif s <= x[0]:
            amps[i] = y[0]
        elif s >= x[-1]:
            amps[i] = y[-1]
        else:
            k = int(np.searchsorted(x, s, side="left"))
            if x[k] == s:
                amps[i] = y[k]
            elif x[k - 1] == s:
                amps[i] = y[k - 1]
            else:
                d = (s - x[k - 1]) / (x[k] - x[k - 1])
                amps[i] = d * (y[k] - y[k - 1]) + y[k - 1]
    return SpectralPacket(float(nmbegin), float(nmend), amps.astype(np.float32))


SAMPLER_HASH = 0    # counter-based hash of (seed, pixel, sample, dimension)
SAMPLER_SOBOL = 1   # the reference's Owen-scrambled padded Sobol
SAMPLER_SOBOL_SHUFFLED = 2   # the same with the index shuffled per dimension pair (converges per pixel)
SPECTRAL_HWSS = 0    # hero wavelength + 3 companions per path (the reference's hwss true)
SPECTRAL_SINGLE = 1  # one wavelength per path (the reference's default, hwss false)


@dataclass
class RenderSettings:
    width: int = 256
    height: int = 256
    cam_pos: tuple = (0.5, 0.5, -1.4)
    cam_look: tuple = (0.5, 0.5, 0.0)
    cam_up: tuple = (0.0, 1.0, 0.0)
    fov_deg: float = 39.3
    lambda_min: float = 400.0
    lambda_max: float = 700.0
    max_depth: int = 8
    rr_min_depth: int = 3
    rr_threshold: float = 0.05
    nee_per_lambda: int = 1
    seed: int = 1
    max_paths: int = 0
    filter: int = 0           # 0 box; 1 Gaussian (GaussianPixelFilter; splatted when size / 2 > 0.501)
    filter_size: float = 2.0  # Gaussian kernel width in pixels
    filter_sigma: float = 0.5 # Gaussian standard deviation in pixels
    adaptive_max_spp: int = 0       # adaptive sampling: maximum samples per pixel (0 = off)
    adaptive_threshold: float = 0.01  # adaptive sampling: relative standard error to converge
    light_selection: int = 0  # 0 light BVH (more than one luminary), 1 by emitted power
    sampler: int = 0          # 0 counter-based hash, 1 the reference's Owen-scrambled Sobol, 2 shuffled Sobol
    max_diffuse_bounce: int = None       # per-type bounce limits (None = unlimited)
    max_glossy_bounce: int = None
    max_transmission_bounce: int = None
    spectral_mode: int = 0    # 0 hero + 3 companions (hwss true), 1 one wavelength per path (hwss false)
    num_wavelengths: int = 0  # single-wavelength mode: wavelength bins (0 = continuous)
    spectral_samples: int = 1 # paths per pixel sample


@dataclass
class EnvMap:
    """An image environment: the rasterizer's radiance_map bound to an HDR
    texture painter (light-probe mapping, bilinear, per-lookup RGB uplift)."""
    rgb: np.ndarray                       # (height, width, 3) linear Rec.709, rows top to bottom
    scale: float = 1.0                    # radiance_scale
    orient_deg: tuple = (0.0, 0.0, 0.0)   # radiance_orient (x, y, z Euler angles)


@dataclass
class SceneDesc:
    tri9: np.ndarray = None
    meshes: list = field(default_factory=list)     # (first, count, material, double_sided)
    spectra: list = field(default_factory=list)    # 81 floats each, or a SpectralPacket
    materials: list = field(default_factory=list)  # Material
    env: int = -1
    env_visible: int = 1
    env_map: object = None     # EnvMap: an image environment (replaces env)
    point_lights: list = field(default_factory=list)  # (position, colour, power)
    settings: RenderSettings = field(default_factory=RenderSettings)
    _tris: list = field(default_factory=list)
    _nrms: list = field(default_factory=list)

    def add_spectrum(self, s):
        self.spectra.append(s if isinstance(s, (SpectralPacket, SigmoidSpectrum, BlackbodySpectrum))
                            else np.asarray(s, np.float32).reshape(81))
        return len(self.spectra) - 1

    def add_point_light(self, position, color, power=1.0):
        """An omni_light (Lights/PointLight.h): radiant intensity colour x power."""
        self.point_lights.append((tuple(float(v) for v in position), tuple(float(v) for v in color), float(power)))

    def add_material(self, m):
        self.materials.append(m)
        return len(self.materials) - 1

    def add_mesh(self, tri9, material, double_sided=True, normals9=None):
        """normals9: vertex normals per triangle corner, (n, 9), for smooth
        shading (None: face normals)."""
        tri9 = np.asarray(tri9, np.float32).reshape(-1, 9)
        first = sum(len(t) for t in self._tris)
        self._tris.append(tri9)
        self._nrms.append(None if normals9 is None else np.asarray(normals9, np.float32).reshape(-1, 9))
        self.meshes.append((first, len(tri9), material, int(bool(double_sided))))
        self.tri9 = np.concatenate(self._tris).astype(np.float32)

    @property
    def nrm9(self):
        """Vertex normals of every triangle corner, zeros for flat meshes; None
        when no mesh has normals."""
        if not any(n is not None for n in self._nrms):
            return None
        return np.concatenate([n if n is not None else np.zeros((len(t), 9), np.float32)
                               for n, t in zip(self._nrms, self._tris)]).astype(np.float32)

    @property
    def n_tri(self):
        return 0 if self.tri9 is None else len(self.tri9)


def _quad(p0, p1, p2, p3):
    """Two triangles (p0, p1, p2), (p0, p2, p3); normal = (p1-p0) x (p2-p0)."""
    return np.array([p0 + p1 + p2, p0 + p2 + p3], np.float32)


def _box(cx, cz, sx, sy, sz, angle_deg):
    """Five faces (no bottom) of a box on the floor, rotated about y."""
    a = np.radians(angle_deg)
    c, s = np.cos(a), np.sin(a)

    def P(x, y, z):
        x -= sx / 2
        z -= sz / 2
        return [cx + c * x + s * z, y, cz - s * x + c * z]
    v = {k: P(*k) for k in [(0, 0, 0), (sx, 0, 0), (sx, 0, sz), (0, 0, sz),
                            (0, sy, 0), (sx, sy, 0), (sx, sy, sz), (0, sy, sz)]}
    q = [
        ((0, sy, 0), (0, sy, sz), (sx, sy, sz), (sx, sy, 0)),   # top
        ((0, 0, 0), (0, sy, 0), (sx, sy, 0), (sx, 0, 0)),       # front (z = 0 side)
        ((sx, 0, sz), (sx, sy, sz), (0, sy, sz), (0, 0, sz)),   # back
        ((0, 0, sz), (0, sy, sz), (0, sy, 0), (0, 0, 0)),       # left
        ((sx, 0, 0), (sx, sy, 0), (sx, sy, sz), (sx, 0, sz)),   # right
    ]
    return np.concatenate([_quad(*(v[k] for k in f)) for f in q])


def fbm_heights(n, seed, octaves=6, amplitude=0.1):
    """(n, n) heights: seeded value-noise fBm (lacunarity 2, gain 0.5), scaled
    so the sum of octave amplitudes is `amplitude`."""
    rng = np.random.default_rng(seed)
    u = np.linspace(0.0, 1.0, n)
    h = np.zeros((n, n))
    amp, total = 1.0, 0.0
    for o in range(octaves):
        f = 4 * (2 ** o)
        g = rng.random((f + 2, f + 2)) * 2.0 - 1.0
        x = u * f
        i = np.floor(x).astype(int)
        t = x - i
        t = t * t * (3 - 2 * t)
        gx0, gx1 = i, i + 1
        a = g[np.ix_(gx0, gx0)] * (1 - t)[None, :] + g[np.ix_(gx0, gx1)] * t[None, :]
        b = g[np.ix_(gx1, gx0)] * (1 - t)[None, :] + g[np.ix_(gx1, gx1)] * t[None, :]
        h += amp * (a * (1 - t)[:, None] + b * t[:, None])
        total += amp
        amp *= 0.5
    return h * (amplitude / total)


def heightfield(n, seed, amplitude=0.1, y0=0.0):
    """(2 (n-1)^2, 9) triangles of an n x n vertex grid over x, z in [0, 1]."""
    hgt = fbm_heights(n, seed, amplitude=amplitude) + y0
    u = np.linspace(0.0, 1.0, n)
    X, Z = np.meshgrid(u, u)
    P = np.stack([X, hgt.T, Z], axis=-1).astype(np.float32)   # P[z, x]
    a = P[:-1, :-1].reshape(-1, 3)
    b = P[:-1, 1:].reshape(-1, 3)
    c = P[1:, 1:].reshape(-1, 3)
    d = P[1:, :-1].reshape(-1, 3)
    t1 = np.concatenate([a, d, c], axis=1)   # normals up (+y)
    t2 = np.concatenate([a, c, b], axis=1)
    return np.concatenate([t1, t2]).astype(np.float32), hgt


def uv_sphere(center, radius, n_tri):
    """Closed UV sphere with about n_tri triangles, outward-facing winding."""
    # nu segments around, nv rings: 2 nu (nv - 2) triangles (one per segment
    # at each pole row).
    nu = max(8, int(round(np.sqrt(n_tri / 2.0))))
    nv = max(4, int(round(n_tri / (2.0 * nu))) + 2)
    th = np.linspace(0.0, np.pi, nv)
    ph = np.linspace(0.0, 2 * np.pi, nu + 1)
    st, ct = np.sin(th), np.cos(th)
    V = np.stack([st[:, None] * np.cos(ph)[None, :], np.broadcast_to(ct[:, None], (nv, nu + 1)),
                  st[:, None] * np.sin(ph)[None, :]], axis=-1) * radius + np.asarray(center)
    tris = []
    for i in range(nv - 1):
        a, b = V[i, :-1], V[i, 1:]
        c, d = V[i + 1, :-1], V[i + 1, 1:]
        if i > 0:
            tris.append(np.concatenate([a, b, c], axis=1))
        if i < nv - 2:
            tris.append(np.concatenate([b, d, c], axis=1))
    return np.concatenate(tris).astype(np.float32)


def sphere_normals(tri9, center):
    """Vertex normals of a sphere's triangle corners: the unit direction from
    the centre to each vertex, (n, 9) float32."""
    v = np.asarray(tri9, np.float64).reshape(-1, 3) - np.asarray(center, np.float64)
    return (v / np.linalg.norm(v, axis=1, keepdims=True)).reshape(-1, 9).astype(np.float32)


def gold_like_spectra():
    """Smooth conductor optical constants, eta and k over 380-780 nm."""
    t = (WAVELENGTHS - 380.0) / 400.0
    eta = (1.4 - 1.25 * t).astype(np.float32)
    k = (1.8 + 2.6 * t).astype(np.float32)
    return eta, k


def spheres_scene(grid=1024, n_spheres=64, sphere_tris=20000, width=1024, height=1024, seed=3,
                  max_depth=16, nee_per_lambda=1):
    """Displaced heightfield plus tessellated spheres, one area light and a sky.

    A grid x grid heightfield over the unit square with 6-octave fBm of
    amplitude 0.1 (2 (grid-1)^2 triangles, Lambertian 0.5); n_spheres spheres
    of sphere_tris triangles with radii U(0.02, 0.08) resting on it, half GGX
    conductors with roughness U(0.05, 0.5), half dielectrics of index 1.5; a
    0.3 x 0.3 area light of radiance 30 at height 1.2 and a uniform sky of
    radiance 0.3 (both on 400-700 nm).  With the defaults this is the
    large-scene configuration: 2,093,058 + 64 x 20,000 triangles, 1024 x 1024
    pixels, max depth 16.

    Max depth N is set as the reference's path-tracing rasterizer takes it
    from a scene file: per-type bounce limits of N - 1 diffuse, glossy and
    transmission scatters (max_diffuse_bounce etc., StabilityConfig) under
    its fixed cap of 128 path vertices (PathTracingIntegrator.h:187), so
    that a path through glass may have more than N vertices.
    """
    rng = np.random.default_rng(seed)
    d = SceneDesc()
    ground = d.add_spectrum(flat_spectrum(0.5))
    sky = d.add_spectrum(flat_spectrum(0.3, 400, 700))
    lightS = d.add_spectrum(flat_spectrum(30.0, 400, 700))
    eta, k = gold_like_spectra()
    s_eta, s_k = d.add_spectrum(eta), d.add_spectrum(k)
    m_ground = d.add_material(Material(MAT_LAMBERTIAN, ground))
    m_light = d.add_material(Material(MAT_LAMBERTIAN, -1, lightS))
    hf, hgt = heightfield(grid, seed, 0.1)
    d.add_mesh(hf, m_ground)
    for i in range(n_spheres):
        r = rng.uniform(0.02, 0.08)
        x, z = rng.uniform(0.1, 0.9, 2)
        gi, gj = int(round(x * (grid - 1))), int(round(z * (grid - 1)))
        y = hgt[gi, gj] + r
        if i % 2 == 0:
            m = d.add_material(Material(MAT_GGX, -1, -1, s_eta, s_k, float(rng.uniform(0.05, 0.5)), 1.5))
            d.add_mesh(uv_sphere((x, y, z), r, sphere_tris), m, double_sided=True)
        else:
            m = d.add_material(Material(MAT_DIELECTRIC, -1, -1, -1, -1, 0.0, 1.5))
            d.add_mesh(uv_sphere((x, y, z), r, sphere_tris), m, double_sided=False)
    lo, hi, ly = 0.35, 0.65, 1.2
    d.add_mesh(_quad([lo, ly, lo], [hi, ly, lo], [hi, ly, hi], [lo, ly, hi]), m_light, double_sided=False)
    d.env = sky
    d.env_visible = 1
    d.settings = RenderSettings(width=width, height=height, cam_pos=(0.5, 0.55, -0.45), cam_look=(0.5, 0.0, 0.55),
                                cam_up=(0.0, 1.0, 0.0), fov_deg=45.0, max_depth=128,
                                max_diffuse_bounce=max_depth - 1, max_glossy_bounce=max_depth - 1,
                                max_transmission_bounce=max_depth - 1, nee_per_lambda=nee_per_lambda, seed=1)
    return d


RESOLUTIONS = (128, 256, 512, 1024)


def batch_scene_params(n=48, seed=11, min_tri=10_000, max_tri=1_000_000, min_spp=4, max_spp=256,
                       resolutions=RESOLUTIONS):
    """Per-scene parameters of the batched-scenes distribution: triangle count
    and spp log-uniform, resolution drawn from `resolutions` (square), max
    depth 8-16."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        out.append({
            "n_tri": int(np.exp(rng.uniform(np.log(min_tri), np.log(max_tri)))),
            "res": int(rng.choice(resolutions)),
            "spp": int(round(np.exp(rng.uniform(np.log(min_spp), np.log(max_spp))))),
            "max_depth": int(rng.integers(8, 17)),
            "seed": int(rng.integers(1, 1 << 30)),
        })
    return out


def batch_scene(p):
    """A heightfield-plus-spheres scene of about p['n_tri'] triangles (60% in
    the heightfield, 40% in 16 spheres) at p['res'] x p['res'] pixels."""
    n_sph = 16
    grid = max(8, int(np.sqrt(0.6 * p["n_tri"] / 2.0)) + 1)
    sph = max(80, int(0.4 * p["n_tri"] / n_sph))
    return spheres_scene(grid=grid, n_spheres=n_sph, sphere_tris=sph, width=p["res"], height=p["res"],
                         seed=p["seed"] % 100000, max_depth=p["max_depth"])


def cornell_box(width=256, height=256, spp_seed=1, nee_per_lambda=1, max_depth=8):
    """The 32-triangle spectral Cornell box.

    Five unit-square walls (floor y=0, ceiling y=1, back z=1, red x=1, green
    x=0; 10 triangles), two boxes of five faces rotated about the vertical
    axis (20 triangles), and a 0.25 x 0.25 quad light just below the ceiling
    facing down (2 triangles).  Lambertian reflectances: white 0.75 flat; red
    0.6 on 600-700 nm, 0.05 elsewhere; green 0.6 on 500-570 nm, 0.05
    elsewhere.  The light emits radiance 15 on 400-700 nm.  Pinhole camera,
    max depth 8, Russian roulette from depth 3.
    """
    d = SceneDesc()
    white = d.add_spectrum(flat_spectrum(0.75))
    red = d.add_spectrum(flat_spectrum(0.6, 600, 700, 0.05))
    green = d.add_spectrum(flat_spectrum(0.6, 500, 570, 0.05))
    light = d.add_spectrum(flat_spectrum(15.0, 400, 700, 0.0))
    m_white = d.add_material(Material(MAT_LAMBERTIAN, white))
    m_red = d.add_material(Material(MAT_LAMBERTIAN, red))
    m_green = d.add_material(Material(MAT_LAMBERTIAN, green))
    m_light = d.add_material(Material(MAT_LAMBERTIAN, -1, light))
    floor = _quad([0, 0, 0], [0, 0, 1], [1, 0, 1], [1, 0, 0])
    ceil = _quad([0, 1, 0], [1, 1, 0], [1, 1, 1], [0, 1, 1])
    back = _quad([0, 0, 1], [0, 1, 1], [1, 1, 1], [1, 0, 1])
    d.add_mesh(np.concatenate([floor, ceil, back]), m_white)
    d.add_mesh(_quad([1, 0, 0], [1, 0, 1], [1, 1, 1], [1, 1, 0]), m_red)
    d.add_mesh(_quad([0, 0, 0], [0, 1, 0], [0, 1, 1], [0, 0, 1]), m_green)
    d.add_mesh(np.concatenate([_box(0.67, 0.35, 0.3, 0.3, 0.3, -17.0),
                               _box(0.33, 0.65, 0.3, 0.6, 0.3, 17.0)]), m_white)
    y = 0.999
    lo, hi = 0.375, 0.625
    # Winding chosen so the face normal points down (-y): one-sided emitter.
    d.add_mesh(_quad([lo, y, lo], [hi, y, lo], [hi, y, hi], [lo, y, hi]), m_light, double_sided=False)
    d.settings = RenderSettings(width=width, height=height, seed=spp_seed, nee_per_lambda=nee_per_lambda,
                                max_depth=max_depth)
    assert d.n_tri == 32
    return d
