"""Oracle loaders -- TEST INFRASTRUCTURE ONLY.

`port()` loads liboracle.so, the CPU restatement of the reference's BVH and
path-tracing algorithms (bvh_oracle.cpp, pt_oracle.cpp).  `ref()` loads
_ref/libref_bvh.so, the reference renderer's own BVH template and
ray/triangle test compiled from its sources (recipe: oracle/Makefile), or
returns None where it was not built.

Only tests/, `__graft_entry__.smoke()` and bench.py's CPU-baseline leg may
import this package.  The product (rise_b200) never does.
"""
import ctypes
import math
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_port = None
_ref = None

_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)
_i32p = ctypes.POINTER(ctypes.c_int32)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_vp = ctypes.c_void_p
_i64 = ctypes.c_int64

NODE2_DTYPE = np.dtype([("bmin", "<f4", 3), ("bmax", "<f4", 3), ("first", "<u4"),
                        ("count", "<u2"), ("axis", "u1"), ("pad", "u1")])
NODE4_DTYPE = np.dtype([("minx", "<f4", 4), ("miny", "<f4", 4), ("minz", "<f4", 4),
                        ("maxx", "<f4", 4), ("maxy", "<f4", 4), ("maxz", "<f4", 4),
                        ("child", "<i4", 4), ("count", "<u2", 4), ("nchild", "u1"),
                        ("axis", "u1"), ("pad", "u1", 6)])
NODE4_FIELDS = [f for f in NODE4_DTYPE.names if f != "pad"]
assert NODE2_DTYPE.itemsize == 32 and NODE4_DTYPE.itemsize == 128


def build():
    """Compile liboracle.so (and _ref when the reference tree is present)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _p(a, t):
    return a.ctypes.data_as(t)


def _setup(lib, prefix):
    b = getattr(lib, prefix + "bvh_build")
    b.restype = _vp
    b.argtypes = [_f32p, _i64]
    getattr(lib, prefix + "bvh_destroy").argtypes = [_vp]
    for nm in ("bvh_num_nodes2", "bvh_num_nodes4"):
        f = getattr(lib, prefix + nm)
        f.restype = _i64
        f.argtypes = [_vp]
    c = getattr(lib, prefix + "closest")
    c.restype = None
    a = getattr(lib, prefix + "any")
    a.restype = None
    a.argtypes = [_vp, _f32p, _i64, _u8p, ctypes.c_int]
    rt = getattr(lib, prefix + "ray_triangle")
    rt.restype = ctypes.c_int
    rt.argtypes = [_f64p] * 5 + [_f64p, _f64p, _f64p]


def port():
    global _port
    if _port is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        lib = ctypes.CDLL(path)
        _setup(lib, "orc_")
        lib.orc_closest.argtypes = [_vp, _f32p, _i64, _i32p, _f64p, _f64p, ctypes.c_int]
        lib.orc_bvh_export.argtypes = [_vp, _vp, _u32p, _vp]
        lib.orc_closest_brute.argtypes = [_f32p, _i64, _f32p, _i64, _i32p, _f64p]
        _port = lib
    return _port


def ref():
    global _ref
    if _ref is None:
        path = os.path.join(_HERE, "_ref", "libref_bvh.so")
        if not os.path.exists(path):
            return None
        lib = ctypes.CDLL(path)
        _setup(lib, "ref_")
        lib.ref_closest.argtypes = [_vp, _f32p, _i64, _i32p, _f64p, ctypes.c_int]
        lib.ref_bvh_export.argtypes = [_vp, _vp, _u32p]
        lib.ref_bvh_export4.argtypes = [_vp, _vp]
        _ref = lib
    return _ref


class BVH:
    """A BVH built by either the port (`kind='port'`) or the reference ('ref')."""

    def __init__(self, tri9, kind="port"):
        self.kind = kind
        self.lib = port() if kind == "port" else ref()
        if self.lib is None:
            raise RuntimeError("reference harness oracle/_ref/libref_bvh.so is not built")
        self.pre = "orc_" if kind == "port" else "ref_"
        self.tri9 = np.ascontiguousarray(tri9, dtype=np.float32).reshape(-1, 9)
        self.h = getattr(self.lib, self.pre + "bvh_build")(_p(self.tri9, _f32p), len(self.tri9))

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            getattr(self.lib, self.pre + "bvh_destroy")(h)
            self.h = None

    def nodes(self):
        n2 = getattr(self.lib, self.pre + "bvh_num_nodes2")(self.h)
        n4 = getattr(self.lib, self.pre + "bvh_num_nodes4")(self.h)
        nodes2 = np.zeros(n2, NODE2_DTYPE)
        prims = np.zeros(len(self.tri9), np.uint32)
        nodes4 = np.zeros(n4, NODE4_DTYPE)
        if self.kind == "port":
            self.lib.orc_bvh_export(self.h, nodes2.ctypes.data, _p(prims, _u32p), nodes4.ctypes.data)
        else:
            self.lib.ref_bvh_export(self.h, nodes2.ctypes.data, _p(prims, _u32p))
            self.lib.ref_bvh_export4(self.h, nodes4.ctypes.data)
        return nodes2, prims, nodes4

    def closest(self, rays, threads=os.cpu_count(), edge=False):
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        n = len(rays)
        ids = np.empty(n, np.int32)
        t = np.empty(n, np.float64)
        if self.kind == "port":
            e = np.empty(n, np.float64) if edge else None
            self.lib.orc_closest(self.h, _p(rays, _f32p), n, _p(ids, _i32p), _p(t, _f64p),
                                 _p(e, _f64p) if edge else None, threads)
            return (ids, t, e) if edge else (ids, t)
        self.lib.ref_closest(self.h, _p(rays, _f32p), n, _p(ids, _i32p), _p(t, _f64p), threads)
        return ids, t

    def any(self, rays, threads=os.cpu_count()):
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        occ = np.empty(len(rays), np.uint8)
        getattr(self.lib, self.pre + "any")(self.h, _p(rays, _f32p), len(rays), _p(occ, _u8p), threads)
        return occ


def closest_brute(tri9, rays):
    lib = port()
    tri9 = np.ascontiguousarray(tri9, dtype=np.float32).reshape(-1, 9)
    rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
    ids = np.empty(len(rays), np.int32)
    t = np.empty(len(rays), np.float64)
    lib.orc_closest_brute(_p(tri9, _f32p), len(tri9), _p(rays, _f32p), len(rays), _p(ids, _i32p), _p(t, _f64p))
    return ids, t


class _OrcEnvImage(ctypes.Structure):
    _fields_ = [("rgb", _f32p), ("width", ctypes.c_int32), ("height", ctypes.c_int32), ("scale", ctypes.c_double),
                ("orient_rad", ctypes.c_double * 3), ("uplift", _f32p)]


_UPLIFT = None


def uplift_table():
    """The Jakob-Hanika RGB -> sigmoid-coefficient table (3 x 64^3 x 3
    floats) as rise_b200 generates it (held to the reference generator's
    output by tests/test_oracle_pt.py): data for the oracle's image
    environment, which restates the lookup itself."""
    global _UPLIFT
    if _UPLIFT is None:
        from rise_b200 import _native
        t = np.empty(3 * 64 ** 3 * 3, np.float32)
        _native.check(_native.lib().rtb200_rgb_uplift_table(t.ctypes.data_as(ctypes.c_void_p)))
        _UPLIFT = t
    return _UPLIFT


def cie_table():
    """The reference's CIE 1931 table (tests/golden/cie1931_5nm.json), 3 x 81."""
    import json
    path = os.path.join(os.path.dirname(_HERE), "tests", "golden", "cie1931_5nm.json")
    d = json.load(open(path))
    return np.array([d["x"], d["y"], d["z"]], np.float64)


def spectrum_table(spectra):
    """The spectrum table the oracle reads (the device's layout): a header of
    4 floats per id -- {0, 380, 780, offset} for 81 grid samples, {n, begin,
    end, offset} for a binned packet (an object with .begin, .end, .amps) --
    then the samples; offset is the samples' float index stored as int32
    bits."""
    head = np.zeros((len(spectra), 4), np.float32)
    data = []
    off = 4 * len(spectra)
    for i, sp in enumerate(spectra):
        if hasattr(sp, "temperature"):
            vals = np.array([sp.temperature, sp.effective_scale()], np.float32)
            head[i, :3] = (-2.0, 0.0, 1e30)
        elif hasattr(sp, "c0"):
            vals = np.array([sp.c0, sp.c1, sp.c2, sp.scale], np.float32)
            head[i, :3] = (-1.0, 380.0, 780.0)
        elif hasattr(sp, "amps"):
            vals = np.asarray(sp.amps, np.float32)
            head[i, :3] = (len(vals), sp.begin, sp.end)
        else:
            vals = np.asarray(sp, np.float32).reshape(81)
            head[i, :3] = (0.0, 380.0, 780.0)
        head[i, 3] = np.array([off], np.int32).view(np.float32)[0]
        data.append(vals)
        off += len(vals)
    return np.ascontiguousarray(np.concatenate([head.ravel()] + data).astype(np.float32))


def _bounce_limits(st):
    lim = [getattr(st, "max_diffuse_bounce", None), getattr(st, "max_glossy_bounce", None),
           getattr(st, "max_transmission_bounce", None)]
    return (int(any(v is not None for v in lim)),) + tuple(int(v) if v is not None else 255 for v in lim)


def pt_render(desc, spp, sample_begin=0, crop=None, threads=None, settings=None, return_counts=False):
    """Render a scenes.SceneDesc with the path-tracing oracle.

    Returns the mean XYZ of samples sample_begin .. sample_begin+spp-1 per
    pixel as float64 (h, w, 3) over `crop` = (x0, y0, x1, y1) (default: the
    whole image); with the Gaussian filter, the resolved splat film.  With
    adaptive sampling (settings.adaptive_max_spp > 0) every pixel takes
    batches of `spp` samples until it converges or reaches the maximum;
    return_counts adds the (h, w) int32 samples per pixel."""
    lib = port()
    st = settings or desc.settings
    x0, y0, x1, y1 = crop or (0, 0, st.width, st.height)
    tri9 = np.ascontiguousarray(desc.tri9, np.float32)
    meshes = np.array(desc.meshes, np.int64).reshape(-1, 4)
    spectra = spectrum_table(desc.spectra)
    mats_i = np.array([[m.type, m.reflectance, m.emission, m.eta, m.kappa] for m in desc.materials], np.int32)
    mats_f = np.array([[m.alpha, m.ior] for m in desc.materials], np.float32)
    envi = np.array([desc.env, desc.env_visible], np.int32)
    cam = np.array(list(st.cam_pos) + list(st.cam_look) + list(st.cam_up) + [st.fov_deg], np.float64)
    setd = np.array([st.lambda_min, st.lambda_max, st.rr_threshold, getattr(st, "filter_size", 2.0),
                     getattr(st, "filter_sigma", 0.5), getattr(st, "adaptive_threshold", 0.01)], np.float64)
    seti = np.array([st.width, st.height, st.max_depth, st.rr_min_depth, st.nee_per_lambda, st.seed,
                     getattr(st, "filter", 0), getattr(st, "adaptive_max_spp", 0),
                     getattr(st, "light_selection", 0), getattr(st, "sampler", 0)] + list(_bounce_limits(st)) +
                    [getattr(st, "spectral_mode", 0), getattr(st, "num_wavelengths", 0),
                     getattr(st, "spectral_samples", 1)], np.int32)
    out = np.zeros((y1 - y0, x1 - x0, 3), np.float64)
    counts = np.zeros((y1 - y0, x1 - x0), np.int32)
    cie = np.ascontiguousarray(cie_table())
    f = lib.orc_pt_render
    f.restype = ctypes.c_int
    i32 = ctypes.c_int32
    f.argtypes = [_f32p, _i64, _vp, i32, _f32p, i32, _vp, _f32p, i32, _vp, _f64p, _f64p, _vp, i32, i32,
                  i32, i32, i32, i32, i32, _f64p, _f64p, _vp, i32, _f64p, _f32p, _vp]
    points = np.array([list(p) + list(c) + [w] for p, c, w in getattr(desc, "point_lights", [])],
                      np.float64).reshape(-1, 7)
    nrm9 = getattr(desc, "nrm9", None)
    if nrm9 is not None:
        nrm9 = np.ascontiguousarray(nrm9, np.float32)
    env_arg, keep = None, None
    em = getattr(desc, "env_map", None)
    if em is not None:
        rgb = np.ascontiguousarray(em.rgb, np.float32)
        table = uplift_table()
        ei = _OrcEnvImage(rgb.ctypes.data_as(_f32p), rgb.shape[1], rgb.shape[0], float(em.scale),
                          (ctypes.c_double * 3)(*[math.radians(a) for a in em.orient_deg]),
                          table.ctypes.data_as(_f32p))
        env_arg, keep = ctypes.byref(ei), (rgb, table, ei)
    rc = f(_p(tri9, _f32p), len(tri9), meshes.ctypes.data, len(meshes), _p(spectra, _f32p), len(desc.spectra),
           mats_i.ctypes.data, _p(mats_f, _f32p), len(mats_i), envi.ctypes.data, _p(cam, _f64p), _p(setd, _f64p),
           seti.ctypes.data, int(spp), int(sample_begin), x0, y0, x1, y1, threads or os.cpu_count(),
           _p(out, _f64p), _p(cie, _f64p), counts.ctypes.data, len(points), _p(points, _f64p),
           _p(nrm9, _f32p) if nrm9 is not None else None, env_arg)
    if rc != 0:
        raise RuntimeError("oracle path tracer rejected the scene")
    return (out, counts) if return_counts else out


def ray_triangle(o, d, v0, ea, eb, kind="port"):
    """The reference's double Moller-Trumbore on one triangle: (hit, t, alpha, beta)."""
    lib = port() if kind == "port" else ref()
    fn = lib.orc_ray_triangle if kind == "port" else lib.ref_ray_triangle
    arrs = [np.ascontiguousarray(x, dtype=np.float64) for x in (o, d, v0, ea, eb)]
    t, a, b = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    hit = fn(*[_p(x, _f64p) for x in arrs], ctypes.byref(t), ctypes.byref(a), ctypes.byref(b))
    return bool(hit), t.value, a.value, b.value


# ---- path-tracer building blocks: port vs the reference's own code -------------

_D = ctypes.c_double
_BLOCK_SIGS = {
    # name: (restype, argtypes) -- identical in both libraries unless noted
    "sample_wavelengths": (None, [_D, _D, _D, _f64p]),
    "ggx_d": (_D, [_D, _D]),
    "ggx_lambda": (_D, [_D, _D]),
    "ggx_g2": (_D, [_D, _D, _D]),
    "vndf_pdf": (_D, [_f64p, _f64p, _f64p, _D]),
    "lookup_ess": (_D, [_D, _D]),
    "lookup_eavg": (_D, [_D]),
    "ms_z": (_D, [_D]),
    "ms_pdf": (_D, [_D, _D, _D]),
    "ms_sample_cos": (_D, [_D, _D]),
    "fresnel_avg": (_D, [_D, _D, _D]),
    "fms": (_D, [_D, _D]),
    "power_heuristic": (_D, [_D, _D]),
    "gaussian_weight": (_D, [_D, _D, _D, _D]),
}
_ref_pt = None


def _bind_blocks(lib, prefix):
    for name, (res, args) in _BLOCK_SIGS.items():
        f = getattr(lib, prefix + name)
        f.restype = res
        f.argtypes = args


def _bind_colour(lib, prefix):
    f = getattr(lib, prefix + "xyz_to_rec709")
    f.restype, f.argtypes = None, [_f64p, _f64p]
    f = getattr(lib, prefix + "display")
    f.restype, f.argtypes = None, [_f64p, _D, ctypes.c_int, _vp]
    if prefix == "ref_pt_":
        f = lib.ref_pt_spectral_packet
        f.restype, f.argtypes = None, [_f64p, _f64p, ctypes.c_int, _D, _D, _f64p, ctypes.c_int, _f64p]


def light_bvh(lib, prefix, pos, power, pts, xi):
    """The light BVH over point lights of the port ('orc_pt_') or the
    reference ('ref_pt_'): (picked light, its probability) per query and the
    (m, n) probabilities of every light from every query point."""
    pos = np.ascontiguousarray(pos, np.float64).reshape(-1, 3)
    power = np.ascontiguousarray(power, np.float64)
    pts = np.ascontiguousarray(pts, np.float64).reshape(-1, 3)
    xi = np.ascontiguousarray(xi, np.float64)
    n, m = len(pos), len(pts)
    picked = np.zeros(m, np.int32)
    pdf = np.zeros(m)
    pdf_all = np.zeros((m, n))
    f = getattr(lib, prefix + "light_bvh")
    f.restype = None
    f.argtypes = [ctypes.c_int, _f64p, _f64p, ctypes.c_int, _f64p, _f64p, _vp, _f64p, _f64p]
    f(n, _p(pos, _f64p), _p(power, _f64p), m, _p(pts, _f64p), _p(xi, _f64p), picked.ctypes.data,
      _p(pdf, _f64p), _p(pdf_all, _f64p))
    return picked, pdf, pdf_all


def xyz_to_rec709(lib, prefix, xyz):
    """Per-pixel XYZ -> linear Rec.709 of the port ('orc_pt_') or the
    reference ('ref_pt_') over an (..., 3) array."""
    x = np.ascontiguousarray(xyz, np.float64).reshape(-1, 3)
    out = np.empty_like(x)
    f = getattr(lib, prefix + "xyz_to_rec709")
    for i in range(len(x)):
        f(_p(x[i], _f64p), _p(out[i], _f64p))
    return out.reshape(np.shape(xyz))


def display8(lib, prefix, rgb, exposure_ev=0.0, tone=0):
    """8-bit sRGB output of linear Rec.709 pixels, (..., 3) uint8."""
    x = np.ascontiguousarray(rgb, np.float64).reshape(-1, 3)
    out = np.empty(x.shape, np.uint8)
    f = getattr(lib, prefix + "display")
    for i in range(len(x)):
        f(_p(x[i], _f64p), float(exposure_ev), int(tone), out[i].ctypes.data)
    return out.reshape(np.shape(rgb))


def port_blocks():
    """liboracle.so with the path-tracer building blocks bound (orc_pt_*)."""
    lib = port()
    if not getattr(lib, "_blocks_bound", False):
        _bind_blocks(lib, "orc_pt_")
        lib.orc_pt_xyz_from_nm.restype = ctypes.c_int
        lib.orc_pt_xyz_from_nm.argtypes = [_D, _f64p, _f64p]
        lib.orc_pt_vndf_sample.restype = None
        lib.orc_pt_vndf_sample.argtypes = [_f64p, _f64p, _f64p, _f64p, _D, _D, _D, _f64p]
        lib.orc_pt_conductor_f.restype = _D
        lib.orc_pt_conductor_f.argtypes = [_D, _D, _D, _D]
        lib.orc_pt_dielectric_r.restype = _D
        lib.orc_pt_dielectric_r.argtypes = [_D, _D, _D, _D]
        lib.orc_pt_russian_roulette.restype = ctypes.c_int
        lib.orc_pt_russian_roulette.argtypes = [ctypes.c_int, ctypes.c_int, _D, _D, _D, _D, _f64p]
        lib.orc_pt_tables.restype = None
        lib.orc_pt_tables.argtypes = [_f64p, _f64p]
        lib.orc_pt_set_tables.restype = None
        lib.orc_pt_set_tables.argtypes = [_f64p, _f64p]
        _bind_colour(lib, "orc_pt_")
        lib._blocks_bound = True
    return lib


def ref_blocks():
    """_ref/libref_pt.so (the reference's own helpers, ref_pt_*) or None."""
    global _ref_pt
    if _ref_pt is None:
        path = os.path.join(_HERE, "_ref", "libref_pt.so")
        if not os.path.exists(path):
            return None
        lib = ctypes.CDLL(path)
        _bind_blocks(lib, "ref_pt_")
        lib.ref_pt_xyz_from_nm.restype = ctypes.c_int
        lib.ref_pt_xyz_from_nm.argtypes = [_D, _f64p]
        lib.ref_pt_cie_y_integral.restype = _D
        lib.ref_pt_cie_y_integral.argtypes = [_D, _D]
        lib.ref_pt_vndf_sample.restype = None
        lib.ref_pt_vndf_sample.argtypes = [_f64p, _f64p, _D, _D, _D, _f64p, _f64p]
        lib.ref_pt_conductor_f.restype = _D
        lib.ref_pt_conductor_f.argtypes = [_f64p, _f64p, _D, _D, _D]
        lib.ref_pt_dielectric_r.restype = _D
        lib.ref_pt_dielectric_r.argtypes = [_f64p, _f64p, _f64p, _D, _D]
        lib.ref_pt_russian_roulette.restype = ctypes.c_int
        lib.ref_pt_russian_roulette.argtypes = [ctypes.c_uint, ctypes.c_uint, _D, _D, _D, _D, _f64p]
        lib.ref_pt_tables.restype = None
        lib.ref_pt_tables.argtypes = [_f64p, _f64p]
        _bind_colour(lib, "ref_pt_")
        _ref_pt = lib
    return _ref_pt


def energy_tables(lib, prefix):
    """(E_ss 32 x 32, E_avg 32) of the port (prefix 'orc_pt_') or reference ('ref_pt_')."""
    ess = np.zeros(1024)
    eavg = np.zeros(32)
    getattr(lib, prefix + "tables")(_p(ess, _f64p), _p(eavg, _f64p))
    return ess.reshape(32, 32), eavg


# ---- the reference renderer (oracle/_ref/librise_ref.so) ----------------------

_rise = None


RISE_THREADS = os.cpu_count() or 1


def rise_ref():
    """The reference renderer's library with our harness
    (oracle/ref_render_harness.cpp, recipe oracle/rise_ref.mk), or None where
    it was not built.  Its render thread pool is set to every host core
    (RISE_THREADS) through an options file (RISE_OPTIONS_FILE,
    force_number_of_threads, render_thread_reserve_count 0: the reference's
    benchmark mode), written before the library first reads its options."""
    global _rise
    if _rise is None:
        path = os.path.join(_HERE, "_ref", "librise_ref.so")
        if not os.path.exists(path):
            return None
        import tempfile
        fd, opts = tempfile.mkstemp(prefix="rise_options_", suffix=".options")
        with os.fdopen(fd, "w") as f:
            f.write(f"force_number_of_threads {RISE_THREADS}\nrender_thread_reserve_count 0\n")
        os.environ["RISE_OPTIONS_FILE"] = opts
        lib = ctypes.CDLL(path)
        lib.rr_load.restype = _vp
        lib.rr_load.argtypes = [ctypes.c_char_p]
        lib.rr_free.argtypes = [_vp]
        lib.rr_size.restype = ctypes.c_int
        lib.rr_size.argtypes = [_vp, _u32p, _u32p]
        lib.rr_render.restype = ctypes.c_int
        lib.rr_render.argtypes = [_vp, _f64p, ctypes.c_uint, ctypes.c_uint]
        lib.rr_integrate.restype = ctypes.c_int
        lib.rr_integrate.argtypes = [_vp] + [ctypes.c_uint] * 6 + [ctypes.c_int, ctypes.c_int, _f64p]
        _rise = lib
    return _rise


_RISE_CWD = None


class _StdoutToStderr:
    """The reference library logs on the process's standard output and into a
    log file in the working directory; while it runs, route the output to
    standard error and work in a scratch directory, so a caller's output and
    folders stay its own."""

    def __enter__(self):
        import sys
        import tempfile
        global _RISE_CWD
        if _RISE_CWD is None:
            _RISE_CWD = tempfile.mkdtemp(prefix="rise_ref_")
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)
        self.cwd = os.getcwd()
        os.chdir(_RISE_CWD)
        return self

    def __exit__(self, *a):
        import ctypes.util
        libc = ctypes.CDLL(ctypes.util.find_library("c"))
        libc.fflush(None)
        os.chdir(self.cwd)
        os.dup2(self.saved, 1)
        os.close(self.saved)


class RefRenderer:
    """A .RISEscene loaded into the reference renderer.

    render(): the reference's whole pipeline (Job::Rasterize); returns the
    resolved linear Rec.709 image (height, width, 3) in float64.
    integrate(spp, batch, rect): the reference's per-sample function over a
    box-filter pixel loop with the batch number mixed into the Sobol seed
    (batch 0 = the reference's own seed); returns mean XYZ per pixel.
    Referenced files resolve against the scene's folder."""

    def __init__(self, scene_path):
        lib = rise_ref()
        if lib is None:
            raise OSError("oracle/_ref/librise_ref.so is not built (make -C oracle rise)")
        self.lib = lib
        path = os.path.abspath(scene_path)
        with _StdoutToStderr():
            self.h = lib.rr_load(path.encode())
        if not self.h:
            raise RuntimeError(f"the reference could not load {scene_path}")
        w, h = ctypes.c_uint(), ctypes.c_uint()
        if not lib.rr_size(self.h, ctypes.byref(w), ctypes.byref(h)):
            raise RuntimeError("scene has no film")
        self.width, self.height = w.value, h.value

    def render(self):
        out = np.zeros((self.height, self.width, 3), np.float64)
        with _StdoutToStderr():
            ok = self.lib.rr_render(self.h, _p(out, _f64p), self.width, self.height)
        if not ok:
            raise RuntimeError("reference render failed")
        return out

    def integrate(self, spp, batch=0, rect=None, threads=None, independent=False):
        x0, y0, x1, y1 = rect if rect is not None else (0, 0, self.width, self.height)
        out = np.zeros((y1 - y0, x1 - x0, 3), np.float64)
        n = threads or os.cpu_count() or 1
        with _StdoutToStderr():
            ok = self.lib.rr_integrate(self.h, x0, y0, x1, y1, spp, batch, n, int(bool(independent)),
                                       _p(out, _f64p))
        if not ok:
            raise RuntimeError("reference integrate failed")
        return out

    def close(self):
        if self.h:
            self.lib.rr_free(self.h)
            self.h = None


def sobol(index, dim, seed, kind="port"):
    """Scrambled Sobol values: the port's 32-bit integers, or the reference's
    SobolSequence::Sample doubles (value / 2^32)."""
    index = np.ascontiguousarray(index, np.uint32)
    dim = np.ascontiguousarray(np.broadcast_to(dim, index.shape), np.uint32)
    seed = np.ascontiguousarray(np.broadcast_to(seed, index.shape), np.uint32)
    n = index.size
    if kind == "port":
        lib = port()
        out = np.zeros(n, np.uint32)
        lib.orc_pt_sobol.restype = None
        lib.orc_pt_sobol.argtypes = [_u32p, _u32p, _u32p, _i64, _u32p]
        lib.orc_pt_sobol(_p(index, _u32p), _p(dim, _u32p), _p(seed, _u32p), n, _p(out, _u32p))
        return out
    lib = ref_blocks()
    out = np.zeros(n, np.float64)
    lib.ref_pt_sobol.restype = None
    lib.ref_pt_sobol.argtypes = [_u32p, _u32p, _u32p, _i64, _f64p]
    lib.ref_pt_sobol(_p(index, _u32p), _p(dim, _u32p), _p(seed, _u32p), n, _p(out, _f64p))
    return out


def hash_combine(a, b, kind="port"):
    a = np.ascontiguousarray(a, np.uint32)
    b = np.ascontiguousarray(np.broadcast_to(b, a.shape), np.uint32)
    lib, name = (port(), "orc_pt_hash_combine") if kind == "port" else (ref_blocks(), "ref_pt_hash_combine")
    f = getattr(lib, name)
    f.restype = None
    f.argtypes = [_u32p, _u32p, _i64, _u32p]
    out = np.zeros(a.size, np.uint32)
    f(_p(a, _u32p), _p(b, _u32p), a.size, _p(out, _u32p))
    return out
