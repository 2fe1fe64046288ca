"""Host-side mirror of the reference's spectral path-tracing rasterizer.

`SpectralRasterizer` plays the part of PathTracingSpectralRasterizer on top
of PixelBasedRasterizerHelper (src/Library/Rendering/
PathTracingSpectralRasterizer.cpp, PixelBasedRasterizerHelper.cpp): it owns
a scene on the device and a render job, `rasterize_scene(spp)` adds spp
samples per pixel (a progressive pass), and `film()` returns the mean XYZ
per pixel.  Everything runs through the C ABI (include/rtb200.h).
"""
import ctypes

import numpy as np

from . import _native
from ._native import check, lib
from .raycaster import Scene


class Material(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int32), ("reflectance", ctypes.c_int32), ("emission", ctypes.c_int32),
                ("eta", ctypes.c_int32), ("kappa", ctypes.c_int32), ("alpha", ctypes.c_float),
                ("ior", ctypes.c_float)]


class RenderSettings(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int32), ("height", ctypes.c_int32),
                ("cam_pos", ctypes.c_float * 3), ("cam_look", ctypes.c_float * 3), ("cam_up", ctypes.c_float * 3),
                ("fov_deg", ctypes.c_float), ("lambda_min", ctypes.c_float), ("lambda_max", ctypes.c_float),
                ("max_depth", ctypes.c_int32), ("rr_min_depth", ctypes.c_int32), ("rr_threshold", ctypes.c_float),
                ("nee_per_lambda", ctypes.c_int32), ("seed", ctypes.c_uint32), ("max_paths", ctypes.c_int32),
                ("filter", ctypes.c_int32), ("filter_size", ctypes.c_float), ("filter_sigma", ctypes.c_float),
                ("adaptive_max_spp", ctypes.c_int32), ("adaptive_threshold", ctypes.c_float),
                ("light_selection", ctypes.c_int32), ("sampler", ctypes.c_int32), ("bounce_limits", ctypes.c_int32),
                ("max_diffuse_bounce", ctypes.c_int32), ("max_glossy_bounce", ctypes.c_int32),
                ("max_transmission_bounce", ctypes.c_int32), ("spectral_mode", ctypes.c_int32),
                ("num_wavelengths", ctypes.c_int32), ("spectral_samples", ctypes.c_int32)]


class Stats(ctypes.Structure):
    _fields_ = [("spp", ctypes.c_int64), ("samples", ctypes.c_int64), ("segments", ctypes.c_int64),
                ("shadow_rays", ctypes.c_int64), ("seconds", ctypes.c_double), ("active_pixels", ctypes.c_int64)]


def upload_scene(ctx, desc, layout="f32"):
    """Create and commit a device scene from a scenes.SceneDesc."""
    s = Scene(ctx)
    L = lib()
    for sp in desc.spectra:
        out = ctypes.c_int32()
        if hasattr(sp, "temperature"):
            check(L.rtb200_scene_add_blackbody(s.h, float(sp.temperature), float(sp.scale), int(bool(sp.normalize)),
                                               ctypes.byref(out)), ctx.h)
        elif hasattr(sp, "c0"):
            cs = np.array([sp.c0, sp.c1, sp.c2, sp.scale], np.float64)
            check(L.rtb200_scene_add_rgb_spectrum(s.h, ctypes.c_void_p(cs.ctypes.data), ctypes.byref(out)), ctx.h)
        elif hasattr(sp, "amps"):
            a = np.ascontiguousarray(sp.amps, np.float32)
            check(L.rtb200_scene_add_spectral_packet(s.h, float(sp.begin), float(sp.end), len(a),
                                                     ctypes.c_void_p(a.ctypes.data), ctypes.byref(out)), ctx.h)
        else:
            sp = np.ascontiguousarray(sp, np.float32)
            check(L.rtb200_scene_add_spectrum(s.h, ctypes.c_void_p(sp.ctypes.data), ctypes.byref(out)), ctx.h)
    for m in desc.materials:
        cm = Material(m.type, m.reflectance, m.emission, m.eta, m.kappa, m.alpha, m.ior)
        out = ctypes.c_int32()
        check(L.rtb200_scene_add_material(s.h, ctypes.byref(cm), ctypes.byref(out)), ctx.h)
    check(L.rtb200_scene_set_environment(s.h, desc.env, desc.env_visible), ctx.h)
    em = getattr(desc, "env_map", None)
    if em is not None:
        rgb = np.ascontiguousarray(em.rgb, np.float32)
        o3 = (ctypes.c_float * 3)(*em.orient_deg)
        check(L.rtb200_scene_set_environment_map(s.h, ctypes.c_void_p(rgb.ctypes.data), rgb.shape[1], rgb.shape[0],
                                                 float(em.scale), o3, desc.env_visible), ctx.h)
    nrm9 = desc.nrm9 if hasattr(desc, "nrm9") else None
    for k, (first, count, mat, ds) in enumerate(desc.meshes):
        smooth = nrm9 is not None and desc._nrms[k] is not None
        s.add_triangles(desc.tri9[first:first + count], material=mat, double_sided=ds,
                        normals9=nrm9[first:first + count] if smooth else None)
    for pos, color, power in getattr(desc, "point_lights", []):
        p3 = (ctypes.c_float * 3)(*pos)
        c3 = (ctypes.c_float * 3)(*color)
        check(L.rtb200_scene_add_point_light(s.h, p3, c3, float(power)), ctx.h)
    s.commit(layout)
    return s


# Tone curves of rtb200_job_read_display (RTB200_TONE_*).
TONE_NONE, TONE_REINHARD, TONE_ACES, TONE_AGX, TONE_HABLE = range(5)


def write_ppm(path, rgb8):
    """Write an (height, width, 3) uint8 image as binary PPM (P6), rows top
    to bottom, as the reference's PPM writer lays it out."""
    rgb8 = np.ascontiguousarray(rgb8, np.uint8)
    h, w = rgb8.shape[:2]
    with open(path, "wb") as f:
        f.write(b"P6\n%d %d\n255\n" % (w, h))
        f.write(rgb8.tobytes())


def settings_struct(st):
    return RenderSettings(st.width, st.height, (ctypes.c_float * 3)(*st.cam_pos), (ctypes.c_float * 3)(*st.cam_look),
                          (ctypes.c_float * 3)(*st.cam_up), st.fov_deg, st.lambda_min, st.lambda_max, st.max_depth,
                          st.rr_min_depth, st.rr_threshold, st.nee_per_lambda, st.seed, st.max_paths,
                          getattr(st, "filter", 0), getattr(st, "filter_size", 2.0), getattr(st, "filter_sigma", 0.5),
                          getattr(st, "adaptive_max_spp", 0), getattr(st, "adaptive_threshold", 0.01),
                          getattr(st, "light_selection", 0), getattr(st, "sampler", 0),
                          *bounce_limits(st), getattr(st, "spectral_mode", 0), getattr(st, "num_wavelengths", 0),
                          getattr(st, "spectral_samples", 1))


def bounce_limits(st):
    """(bounce_limits, max diffuse, max glossy, max transmission) of a
    scenes.RenderSettings: limits are on when any of them is set."""
    lim = [getattr(st, "max_diffuse_bounce", None), getattr(st, "max_glossy_bounce", None),
           getattr(st, "max_transmission_bounce", None)]
    on = any(v is not None for v in lim)
    return (int(on),) + tuple(int(v) if v is not None else 255 for v in lim)


PROGRESS_FN = ctypes.CFUNCTYPE(ctypes.c_int32, ctypes.c_void_p, ctypes.c_double, ctypes.c_double)


class SpectralRasterizer:
    """One progressive spectral path-traced image of one scene."""

    def __init__(self, ctx, desc, layout="f32", scene=None, settings=None):
        self.ctx = ctx
        self.desc = desc
        self.owns_scene = scene is None
        self.scene = scene if scene is not None else upload_scene(ctx, desc, layout)
        self.settings = settings if settings is not None else desc.settings
        h = ctypes.c_void_p()
        cs = settings_struct(self.settings)
        check(lib().rtb200_job_create(self.scene.h, ctypes.byref(cs), ctypes.byref(h)), ctx.h)
        self.h = h

    def rasterize_scene(self, spp):
        """Add `spp` samples per pixel (blocking).  Returns False when the
        progress callback stopped the pass (the film then holds the whole
        pixel samples finished), else True."""
        rc = lib().rtb200_job_render(self.h, int(spp))
        if rc == _native.E_CANCELLED:
            return False
        check(rc, self.ctx.h)
        return True

    def set_progress(self, fn):
        """fn(progress, total) -> bool, called after every engine step of a
        render (IProgressCallback::Progress); False stops the render.  None
        removes it."""
        if fn is None:
            self._progress = None
            check(lib().rtb200_job_set_progress(self.h, None, None), self.ctx.h)
            return
        self._progress = PROGRESS_FN(lambda user, done, total: 1 if fn(done, total) else 0)
        check(lib().rtb200_job_set_progress(self.h, ctypes.cast(self._progress, ctypes.c_void_p), None), self.ctx.h)

    def relmse(self, ref_xyz):
        """relMSE of the film against `ref_xyz` ((height, width, 3) XYZ),
        reduced on the device in FP64."""
        ref = np.ascontiguousarray(ref_xyz, np.float32)
        st = self.settings
        if ref.shape != (st.height, st.width, 3):
            raise ValueError("reference image has the wrong shape")
        out = ctypes.c_double()
        check(lib().rtb200_job_relmse(self.h, ctypes.c_void_p(ref.ctypes.data), ctypes.byref(out)), self.ctx.h)
        return out.value

    def film(self):
        """Mean XYZ per pixel, (height, width, 3) float32."""
        st = self.settings
        out = np.empty((st.height, st.width, 3), np.float32)
        check(lib().rtb200_job_read_film(self.h, ctypes.c_void_p(out.ctypes.data)), self.ctx.h)
        return out

    def stats(self):
        s = Stats()
        check(lib().rtb200_job_stats(self.h, ctypes.byref(s)), self.ctx.h)
        return {"spp": s.spp, "samples": s.samples, "segments": s.segments, "shadow_rays": s.shadow_rays,
                "seconds": s.seconds, "active_pixels": s.active_pixels}

    def rgb(self):
        """Linear Rec.709 RGB per pixel (the rasterizer's resolve of each
        pixel's XYZ), (height, width, 3) float32."""
        st = self.settings
        out = np.empty((st.height, st.width, 3), np.float32)
        check(lib().rtb200_job_read_rgb(self.h, ctypes.c_void_p(out.ctypes.data)), self.ctx.h)
        return out

    def display(self, exposure_ev=0.0, tone=TONE_NONE):
        """8-bit sRGB image for LDR files: exposure 2^ev, tone curve, sRGB
        encode, clamp, truncate; (height, width, 3) uint8."""
        st = self.settings
        out = np.empty((st.height, st.width, 3), np.uint8)
        check(lib().rtb200_job_read_display(self.h, float(exposure_ev), int(tone),
                                            ctypes.c_void_p(out.ctypes.data)), self.ctx.h)
        return out

    def sample_counts(self):
        """Samples each pixel took, (height, width) uint32 (adaptive sampling
        stops converged pixels early)."""
        st = self.settings
        out = np.empty((st.height, st.width), np.uint32)
        check(lib().rtb200_job_read_sample_counts(self.h, ctypes.c_void_p(out.ctypes.data)), self.ctx.h)
        return out

    def close(self):
        if self.h:
            lib().rtb200_job_destroy(self.h)
            self.h = None
        if self.owns_scene and self.scene is not None:
            self.scene.close()
            self.scene = None


class Engine:
    """A shared wavefront (path pool + queues) for many jobs at once.

    `render` batches whole requests; `submit` / `step` / `progress` /
    `retire` drive continuous batching, where jobs join while others are in
    flight (see rtb200_engine_* in include/rtb200.h).
    """

    def __init__(self, ctx, capacity=0):
        self.ctx = ctx
        h = ctypes.c_void_p()
        check(lib().rtb200_engine_create(ctx.h, int(capacity), ctypes.byref(h)), ctx.h)
        self.h = h

    def render(self, rasterizers, spp, use_graph=True):
        n = len(rasterizers)
        jobs = (ctypes.c_void_p * n)(*[r.h.value for r in rasterizers])
        counts = (ctypes.c_int32 * n)(*[int(s) for s in spp])
        rc = lib().rtb200_engine_render(self.h, jobs, counts, n, int(bool(use_graph)))
        if rc == _native.E_CANCELLED:
            return False
        check(rc, self.ctx.h)
        return True

    def set_poll(self, iterations):
        """Wavefront iterations between host progress polls in `render`."""
        check(lib().rtb200_engine_set_poll(self.h, int(iterations)), self.ctx.h)

    def submit(self, rasterizer, spp):
        check(lib().rtb200_engine_submit(self.h, rasterizer.h, int(spp)), self.ctx.h)

    def step(self, iterations=4, use_graph=True):
        check(lib().rtb200_engine_step(self.h, int(iterations), int(bool(use_graph))), self.ctx.h)

    def progress(self, rasterizer):
        done, total = ctypes.c_int64(), ctypes.c_int64()
        check(lib().rtb200_engine_progress(self.h, rasterizer.h, ctypes.byref(done), ctypes.byref(total)),
              self.ctx.h)
        return done.value, total.value

    def retire(self, rasterizer):
        check(lib().rtb200_engine_retire(self.h, rasterizer.h), self.ctx.h)

    def cancel(self, rasterizer):
        """Start no more pixel samples of the job's request; retire it once
        progress reports done == total."""
        check(lib().rtb200_engine_cancel(self.h, rasterizer.h), self.ctx.h)

    def close(self):
        if self.h:
            lib().rtb200_engine_destroy(self.h)
            self.h = None

