"""Scene ingest: the reference's ASCII scene files (.RISEscene, "RISE ASCII
SCENE 5..7") for the chunks this renderer draws, into a scenes.SceneDesc.

The file is a list of chunks -- a keyword on its own line, "{" and "}" on
their own lines around "parameter value..." lines -- with '#' line comments
and /* */ block comments (src/Library/Parsers/README.md, Cst/Cst.cpp:80-115).
Each supported chunk is restated from its parser in
src/Library/Parsers/ChunkParserRegistry.cpp (defaults included):

  spectral_painter            -> scenes.spectral_painter (binned SpectralPacket)
  blackbody_painter           -> scenes.BlackbodySpectrum (Planck, optionally unit peak)
  scene_options               -> accepted (scene_unit does not affect a pinhole camera)
  omni_light                  -> point light: position, linear RGB colour x power
                                 (ChunkParserRegistry.cpp:6855-6865, Lights/PointLight.h)
  hdr_painter                 -> a Radiance HDR image (scale, shift; bilinear, clamp),
                                 drawn as the rasterizer's radiance_map (scenes.EnvMap)
  uniformcolor_painter        -> scenes.rgb_spectrum (Jakob-Hanika albedo uplift of the
                                 colour in linear Rec.709; sRGB colours linearised)
  lambertian_material         -> Lambertian, reflectance painter
  lambertian_luminaire_material -> emitter: radiance = exitance * scale / pi
                                 (LambertianEmitter.cpp:72-87), reflective part
                                 from a lambertian `material` or none
  ggx_material                -> GGX conductor (rd none, isotropic alpha)
  scalar_painter              -> a scalar per wavelength: value, values r g b,
                                 file of (nm, value) lines, sellmeier
  dielectric_material         -> smooth dielectric: IOR constant or per wavelength
                                 (scalar painter, inline r g b, number), transmitted
                                 Phong lobe (scattering), clear interior (tau 1)
  rawmesh2_geometry           -> vertices with normals (smooth shading)
  clippedplane_geometry       -> two triangles (a, b, c), (a, c, d)
  rawmesh_geometry            -> "tri" / "quad" lines (TriangleMeshLoaderRAW.cpp:33-110)
  risemesh_geometry           -> the .risemesh reader of the C ABI
  box_geometry                -> 12 triangles, centred on the origin
  standard_object             -> position + Euler orientation (degrees, Z
                                 then Y then X) + scale (Transformable.cpp:339-343,436-441)
  film, pinhole_camera        -> image size, camera (vertical field of view)
  pathtracing_spectral_rasterizer, pixelintegratingspectral_rasterizer
                              -> samples, wavelength range, pixel filter
                                 (default Gaussian 2.0 / 0.35), adaptive sampling,
                                 Russian roulette, maximum depth (128), per-type
                                 bounce limits, light BVH or power selection,
                                 hero bundles (hwss true) or one wavelength per
                                 path in num_wavelengths bins (the default),
                                 spectral_samples
  pathtracing_shaderop, standard_shader, file_rasterizeroutput -> accepted

A parameter or chunk that would change the image in a way this renderer
cannot draw (other painters, materials, geometry, cameras, lights, modifiers,
volumes, non-unit pixel aspect, hidden luminaires, ...) raises
SceneFileError naming it.  Options that do not change the estimator's
expectation (the pixel sampler, OIDN denoising of the output) are recorded
in LoadedScene.notes.
"""
import math
import os
import re
from dataclasses import dataclass, field

import numpy as np

from . import scenes


class SceneFileError(ValueError):
    pass


@dataclass
class Chunk:
    keyword: str
    line: int
    params: list = field(default_factory=list)   # (key, value string, line)

    def get(self, key, default=None):
        vals = [v for k, v, _ in self.params if k == key]
        return vals[-1] if vals else default

    def all(self, key):
        return [v for k, v, _ in self.params if k == key]

    def has(self, key):
        return any(k == key for k, _, _ in self.params)


@dataclass
class LoadedScene:
    desc: scenes.SceneDesc
    spp: int
    outputs: list = field(default_factory=list)
    notes: list = field(default_factory=list)


def _strip_comments(text):
    text = re.sub(r"/\*.*?\*/", lambda m: "\n" * m.group(0).count("\n"), text, flags=re.S)
    return [re.sub(r"#.*", "", ln).strip() for ln in text.split("\n")]


def parse_chunks(text):
    """The chunks of a scene file, in order."""
    lines = _strip_comments(text)
    i = 0
    while i < len(lines) and not lines[i]:
        i += 1
    m = re.match(r"RISE ASCII SCENE (\d+)$", lines[i] if i < len(lines) else "")
    if not m or not 5 <= int(m.group(1)) <= 7:
        raise SceneFileError("not a RISE ASCII SCENE (versions 5 to 7) file")
    i += 1
    chunks = []
    while i < len(lines):
        ln = lines[i]
        if not ln:
            i += 1
            continue
        if len(ln.split()) != 1 or ln in ("{", "}"):
            raise SceneFileError(f"line {i + 1}: expected a chunk name, got {ln!r}")
        c = Chunk(ln, i + 1)
        i += 1
        while i < len(lines) and not lines[i]:
            i += 1
        if i >= len(lines) or lines[i] != "{":
            raise SceneFileError(f"line {c.line}: chunk {ln} without '{{'")
        i += 1
        while i < len(lines) and lines[i] != "}":
            if lines[i]:
                parts = lines[i].split(None, 1)
                c.params.append((parts[0], parts[1].strip() if len(parts) > 1 else "", i + 1))
            i += 1
        if i >= len(lines):
            raise SceneFileError(f"line {c.line}: chunk {ln} without '}}'")
        i += 1
        chunks.append(c)
    return chunks


def _floats(s, n, what):
    try:
        v = [float(x) for x in s.split()]
    except ValueError:
        raise SceneFileError(f"{what}: expected {n} numbers, got {s!r}") from None
    if len(v) != n:
        raise SceneFileError(f"{what}: expected {n} numbers, got {s!r}")
    return v


def _bool(s):
    return str(s).strip().lower() in ("true", "1", "yes", "on")


_GRID = np.arange(81, dtype=np.float64) * 5.0 + 380.0   # the device's spectral grid (nm)


def _uniform_scalar(v):
    return lambda nm: np.full(np.shape(nm), float(v))


def _rgb_scalar(r, g, b):
    # RGBScalarPainter::GetValueAtNM: b up to 450 nm, g at 550, r from 650,
    # linear between.
    def fn(nm):
        nm = np.asarray(nm, np.float64)
        lo = b + (nm - 450.0) / 100.0 * (g - b)
        hi = g + (nm - 550.0) / 100.0 * (r - g)
        return np.where(nm <= 450.0, b, np.where(nm >= 650.0, r, np.where(nm <= 550.0, lo, hi)))
    return fn


def _piecewise_scalar(pts):
    # PiecewiseLinearScalarPainter::EvalAtNM: clamped to the end values.
    pts = sorted(pts)
    xs = np.array([p[0] for p in pts]), np.array([p[1] for p in pts])
    return lambda nm: np.interp(np.asarray(nm, np.float64), xs[0], xs[1])


def _sellmeier_scalar(b1, b2, b3, c1, c2, c3):
    # SellmeierScalarPainter::EvalAtNM: n^2 = 1 + sum B l^2 / (l^2 - C), l in um.
    def fn(nm):
        l2 = (np.asarray(nm, np.float64) * 1e-3) ** 2
        n2 = 1.0
        for b, cc in ((b1, c1), (b2, c2), (b3, c3)):
            den = l2 - cc
            n2 = n2 + np.where(np.abs(den) < 1e-9, 0.0, b * l2 / np.where(den == 0, 1.0, den))
        return np.where(n2 > 0, np.sqrt(np.maximum(n2, 0.0)), 1.0)
    return fn


def read_hdr(path):
    """A Radiance HDR (RGBE) file as (height, width, 3) float32 linear RGB,
    rows top to bottom (the reference's HDRReader, through rtb200_hdr_decode)."""
    import ctypes
    from . import _native
    with open(path, "rb") as f:
        data = f.read()
    buf = np.frombuffer(data, np.uint8)
    w, h = ctypes.c_int32(), ctypes.c_int32()
    L = _native.lib()
    if L.rtb200_hdr_decode(ctypes.c_void_p(buf.ctypes.data), len(buf), ctypes.byref(w), ctypes.byref(h), None):
        raise SceneFileError(f"{path}: not a readable Radiance HDR file")
    out = np.empty((h.value, w.value, 3), np.float32)
    if L.rtb200_hdr_decode(ctypes.c_void_p(buf.ctypes.data), len(buf), ctypes.byref(w), ctypes.byref(h),
                           ctypes.c_void_p(out.ctypes.data)):
        raise SceneFileError(f"{path}: not a readable Radiance HDR file")
    return out


def _number(s):
    try:
        return float(s)
    except (TypeError, ValueError):
        return None


def _rot(ax, ay, az):
    """Rx(ax) Ry(ay) Rz(az) for column vectors: Z applied first, then Y, then X."""
    cx, sx, cy, sy, cz, sz = math.cos(ax), math.sin(ax), math.cos(ay), math.sin(ay), math.cos(az), math.sin(az)
    rx = np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]])
    ry = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
    rz = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]])
    return rx @ ry @ rz


def _box(w, h, d):
    hw, hh, hd = 0.5 * w, 0.5 * h, 0.5 * d
    c = np.array([[x, y, z] for x in (-hw, hw) for y in (-hh, hh) for z in (-hd, hd)])
    # faces as corner indices (x, y, z bits: 4, 2, 1), wound for outward normals
    quads = [(0, 1, 3, 2), (4, 6, 7, 5), (0, 4, 5, 1), (2, 3, 7, 6), (0, 2, 6, 4), (1, 5, 7, 3)]
    tris = []
    for a, b, cc, dd in quads:
        tris.append(np.concatenate([c[a], c[b], c[cc]]))
        tris.append(np.concatenate([c[a], c[cc], c[dd]]))
    return np.array(tris)


class _Loader:
    def __init__(self, search):
        self.search = search
        self.desc = scenes.SceneDesc()
        self.painters = {}       # name -> spectrum id
        self.scalars = {}        # name -> function of wavelength (nm, array) -> value
        self.images = {}         # name -> (height, width, 3) float32 linear RGB (hdr_painter)
        self.materials = {}      # name -> (material id, kind, reflectance id)
        self.geometry = {}       # name -> ((n, 9) float64 triangles, double_sided)
        self.spp = None
        self.outputs = []
        self.notes = []
        self.st = {}

    def path(self, name, what):
        for d in self.search:
            p = os.path.join(d, name)
            if os.path.exists(p):
                return p
        raise SceneFileError(f"{what}: file {name!r} not found (searched {self.search})")

    def refuse(self, c, why):
        raise SceneFileError(f"line {c.line}: {c.keyword}: {why}")

    def only(self, c, allowed):
        for k, _, ln in c.params:
            if k not in allowed:
                raise SceneFileError(f"line {ln}: {c.keyword}: parameter {k!r} is not supported")

    # ---- painters ----------------------------------------------------------
    def spectral_painter(self, c):
        self.only(c, {"name", "nmbegin", "nmend", "scale", "cp", "file"})
        nm, amp = [], []
        for cp in c.all("cp"):
            a, b = _floats(cp, 2, "spectral_painter cp")
            nm.append(a)
            amp.append(b)
        if c.has("file"):
            with open(self.path(c.get("file"), "spectral_painter"), "r") as f:
                for ln in f:
                    parts = ln.split()
                    try:
                        a, b = float(parts[0]), float(parts[1])
                    except (IndexError, ValueError):
                        continue
                    nm.append(a)
                    amp.append(b)
        if not nm:
            self.refuse(c, "no samples")
        sp = scenes.spectral_painter(nm, amp, float(c.get("nmbegin", 400.0)), float(c.get("nmend", 700.0)))
        self.painters[c.get("name", "noname")] = self.desc.add_spectrum(sp)
        if c.has("scale"):
            self.notes.append(f"spectral_painter {c.get('name')}: scale applies to the RGB colour only")

    def uniformcolor_painter(self, c):
        # Job::AddUniformColorPainter (Job.cpp:2452-2484): the colour in its
        # colour space, converted to linear Rec.709; the painter's spectrum
        # is the albedo uplift (UniformColorPainter's default role).
        self.only(c, {"name", "color", "colorspace"})
        rgb = np.array(_floats(c.get("color", "0 0 0"), 3, "color"))
        space = c.get("colorspace", "Rec709RGB_Linear")
        if space == "sRGB":
            # ColorUtils::SRGBTransferFunctionInverse (ColorUtils.cpp:34-45).
            rgb = np.array([0.0 if v == 0 else (v / 12.92 if v <= 0.03928 else ((v + 0.055) / 1.055) ** 2.4)
                            for v in rgb])
        elif space not in ("Rec709RGB_Linear", "RISERGB"):
            self.refuse(c, f"colour space {space!r} is not supported (Rec709RGB_Linear, RISERGB, sRGB)")
        self.painters[c.get("name", "noname")] = self.desc.add_spectrum(scenes.rgb_spectrum(rgb, scenes.RGB_ALBEDO))

    def blackbody_painter(self, c):
        # Job::AddBlackBodyPainter: only temperature, scale and normalize
        # reach the spectrum (nmbegin / nmend / numfreq shape the RGB colour).
        self.only(c, {"name", "temperature", "nmbegin", "nmend", "numfreq", "scale", "normalize"})
        sp = scenes.BlackbodySpectrum(float(c.get("temperature", 5600.0)), float(c.get("scale", 1.0)),
                                      _bool(c.get("normalize", "true")))
        self.painters[c.get("name", "noname")] = self.desc.add_spectrum(sp)

    def hdr_painter(self, c):
        # Job::AddHDRTexturePainter (Job.cpp:2216-2265): the Radiance HDR
        # image, times `scale` then plus `shift` per channel, read with the
        # bilinear filter (the default filter_type) and clamp-to-edge wrap.
        self.only(c, {"name", "file", "scale", "shift", "lowmemory", "filter_type", "wrap_s", "wrap_t"})
        if c.get("filter_type", "bilinear") not in ("bilinear", "Bilinear"):
            self.refuse(c, "only the bilinear texture filter is supported")
        for k in ("wrap_s", "wrap_t"):
            if c.get(k, "clamp") != "clamp":
                self.refuse(c, f"{k} other than clamp is not supported")
        rgb = read_hdr(self.path(c.get("file", "none"), "hdr_painter"))
        scale = np.array(_floats(c.get("scale", "1 1 1"), 3, "hdr_painter scale"), np.float32)
        shift = np.array(_floats(c.get("shift", "0 0 0"), 3, "hdr_painter shift"), np.float32)
        if np.any(scale != 1):
            rgb = rgb * scale
        if np.any(shift != 0):
            rgb = rgb + shift
        self.images[c.get("name", "noname")] = np.ascontiguousarray(rgb, np.float32)

    def scalar_painter(self, c):
        # Physical scalars per wavelength (ScalarPainterAsciiChunkParser,
        # Parsers/ChunkParserRegistry.cpp:1216-1330): `value` (uniform),
        # `values r g b` (RGBScalarPainter), `file` of "nm value" lines
        # (PiecewiseLinearScalarPainter, clamped at its ends), `sellmeier B1 B2
        # B3 C1 C2 C3` (SellmeierScalarPainter, lambda in micrometres).
        forms = ("value", "values", "file", "sellmeier")
        self.only(c, {"name"} | set(forms))
        present = [k for k in forms if c.has(k)]
        if len(present) != 1:
            self.refuse(c, "exactly one of value, values, file or sellmeier is supported")
        form = present[0]
        if form == "value":
            v = _floats(c.get("value"), 1, "scalar_painter value")[0]
            fn = _uniform_scalar(v)
        elif form == "values":
            fn = _rgb_scalar(*_floats(c.get("values"), 3, "scalar_painter values"))
        elif form == "file":
            pts = []
            with open(self.path(c.get("file"), "scalar_painter"), "r") as f:
                for ln in f:
                    parts = ln.split()
                    if not parts or parts[0].startswith("#"):
                        continue
                    try:
                        pts.append((float(parts[0]), float(parts[1])))
                    except (IndexError, ValueError):
                        continue
            if not pts:
                self.refuse(c, "file produced no samples")
            fn = _piecewise_scalar(pts)
        else:
            fn = _sellmeier_scalar(*_floats(c.get("sellmeier"), 6, "scalar_painter sellmeier"))
        self.scalars[c.get("name", "noname")] = fn

    def _scalar(self, c, value, default):
        """A material's scalar slot (Job.cpp ResolveScalarPainterArg): a
        scalar_painter name, an inline `r g b` triple or a single number."""
        value = c.get(value, default)
        if value in self.scalars:
            return self.scalars[value]
        parts = value.split()
        if len(parts) == 3:
            return _rgb_scalar(*_floats(value, 3, "scalar"))
        v = _number(value)
        if v is None:
            self.refuse(c, f"unknown scalar painter {value!r}")
        return _uniform_scalar(v)

    def _scalar_spectrum(self, c, key, default):
        """A physical-scalar slot as a spectrum id on the device's 5 nm grid
        (a painter name is read as its spectrum)."""
        value = c.get(key, default)
        if value in self.painters:
            return self.painters[value]
        return self.desc.add_spectrum(self._scalar(c, key, default)(_GRID).astype(np.float32))

    def omni_light(self, c):
        # Job::AddPointOmniLight; shootphotons only matters to photon mapping.
        self.only(c, {"name", "power", "position", "color", "shootphotons"})
        pos = _floats(c.get("position", "0 0 0"), 3, "omni_light position")
        col = _floats(c.get("color", "0 0 0"), 3, "omni_light color")
        self.desc.add_point_light(pos, col, _floats(c.get("power", "1.0"), 1, "omni_light power")[0])

    def scene_options(self, c):
        # scene_unit sets the lens units of physical cameras; a pinhole has none.
        self.only(c, {"scene_unit"})

    def spectrum(self, c, name, allow_number=False):
        """Spectrum id of a painter reference, or a flat spectrum for a number."""
        if name in (None, "none"):
            return -1
        if name in self.painters:
            return self.painters[name]
        v = _number(name)
        if allow_number and v is not None:
            return self.desc.add_spectrum(np.full(81, v, np.float32))
        self.refuse(c, f"unknown painter {name!r}")

    def scaled(self, sid, k):
        sp = self.desc.spectra[sid]
        if isinstance(sp, scenes.SigmoidSpectrum):
            return self.desc.add_spectrum(scenes.SigmoidSpectrum(sp.c0, sp.c1, sp.c2, sp.scale * k))
        if isinstance(sp, scenes.BlackbodySpectrum):
            return self.desc.add_spectrum(scenes.BlackbodySpectrum(sp.temperature, sp.scale * k, sp.normalize))
        if isinstance(sp, scenes.SpectralPacket):
            return self.desc.add_spectrum(scenes.SpectralPacket(sp.begin, sp.end,
                                                                (np.asarray(sp.amps, np.float64) * k).astype(np.float32)))
        return self.desc.add_spectrum((np.asarray(sp, np.float64) * k).astype(np.float32))

    # ---- materials ---------------------------------------------------------
    def add_material(self, c, m, kind, refl=-1):
        self.materials[c.get("name", "noname")] = (self.desc.add_material(m), kind, refl)

    def lambertian_material(self, c):
        self.only(c, {"name", "reflectance"})
        r = self.spectrum(c, c.get("reflectance", "none"))
        self.add_material(c, scenes.Material(scenes.MAT_LAMBERTIAN, r), "lambertian", r)

    def lambertian_luminaire_material(self, c):
        self.only(c, {"name", "material", "exitance", "scale"})
        ex = self.spectrum(c, c.get("exitance", "none"))
        scale = float(c.get("scale", 1.0))
        emit = self.scaled(ex, scale / math.pi) if ex >= 0 else -1
        inner = c.get("material", "none")
        refl = -1
        if inner != "none":
            if inner not in self.materials or self.materials[inner][1] != "lambertian":
                self.refuse(c, f"reflective part {inner!r} must be a lambertian_material")
            refl = self.materials[inner][2]
        self.add_material(c, scenes.Material(scenes.MAT_LAMBERTIAN, refl, emit), "luminaire", refl)

    def ggx_material(self, c):
        self.only(c, {"name", "rd", "rs", "alphax", "alphay", "ior", "extinction", "fresnel_mode"})
        if c.get("rd", "none") != "none":
            self.refuse(c, "a diffuse layer (rd) is not supported")
        if c.get("fresnel_mode", "conductor") != "conductor":
            self.refuse(c, "only fresnel_mode conductor is supported")
        ax, ay = _number(c.get("alphax", "0.15")), _number(c.get("alphay", "0.15"))
        if ax is None or ay is None or ax != ay:
            self.refuse(c, "alphax and alphay must be equal numbers (isotropic)")
        # rs "none" is the job's built-in black painter (Job.cpp:536-540):
        # no specular layer at all.
        rs = c.get("rs", "none")
        spec = self.desc.add_spectrum(np.zeros(81, np.float32)) if rs == "none" else self.spectrum(c, rs)
        eta = self._scalar_spectrum(c, "ior", "2.45")
        kap = self._scalar_spectrum(c, "extinction", "3.45")
        self.add_material(c, scenes.Material(scenes.MAT_GGX, spec, -1, eta, kap, float(ax), 1.5), "ggx")

    def dielectric_material(self, c):
        # Job::AddDielectricMaterial: tau (interior transmittance per unit
        # length), ior, scattering (the Phong exponent of the transmitted
        # lobe, default 10000; 1e6 and above is a smooth interface).
        # The index of refraction is a scalar painter evaluated per
        # wavelength (DielectricSPF::GetSpecularInfoNM): constant, or
        # tabulated on the 5 nm grid (exact for piecewise-linear painters
        # whose knots lie on it, as the RGB triple's 450/550/650 do).
        self.only(c, {"name", "tau", "ior", "scattering"})
        if c.get("tau", "none") != "none" and np.any(self._scalar(c, "tau", "none")(_GRID) != 1.0):
            self.refuse(c, "an absorbing interior (tau other than 1) is not supported")
        ior = self._scalar(c, "ior", "1.33")(_GRID)
        scat = self._scalar(c, "scattering", "10000")(_GRID)
        if np.any(scat != scat[0]):
            self.refuse(c, "a scattering exponent that varies with wavelength is not supported")
        if np.all(ior == ior[0]):
            eta, n = -1, float(ior[0])
        else:
            eta, n = self.desc.add_spectrum(ior.astype(np.float32)), float(ior[34])
        self.add_material(c, scenes.Material(scenes.MAT_DIELECTRIC, -1, -1, eta, -1, float(min(scat[0], 1e6)), n),
                          "dielectric")

    # ---- geometry ----------------------------------------------------------
    def clippedplane_geometry(self, c):
        self.only(c, {"name", "pta", "ptb", "ptc", "ptd", "doublesided"})
        p = [np.array(_floats(c.get(k, "0 0 0"), 3, k)) for k in ("pta", "ptb", "ptc", "ptd")]
        tris = np.array([np.concatenate([p[0], p[1], p[2]]), np.concatenate([p[0], p[2], p[3]])])
        self.geometry[c.get("name", "noname")] = (tris, _bool(c.get("doublesided", "true")), None)

    def rawmesh_geometry(self, c):
        self.only(c, {"name", "file", "double_sided", "maxpolygons", "maxdepth"})
        tris = []
        with open(self.path(c.get("file", "none"), "rawmesh_geometry"), "r") as f:
            for ln in f:
                parts = ln.split()
                if not parts:
                    continue
                if parts[0] == "tri":
                    v = [float(x) for x in parts[1:10]]
                    tris.append(v)
                elif parts[0] == "quad":
                    v = [float(x) for x in parts[1:13]]
                    a, b, cc, d = v[0:3], v[3:6], v[6:9], v[9:12]
                    tris.append(a + b + cc)
                    tris.append(a + cc + d)
        self.geometry[c.get("name", "noname")] = (np.array(tris, np.float64).reshape(-1, 9),
                                                  _bool(c.get("double_sided", "false")), None)

    def risemesh_geometry(self, c):
        from .raycaster import RiseMesh
        self.only(c, {"name", "file", "loadintomemory", "face_normals"})
        m = RiseMesh.from_file(self.path(c.get("file", "none"), "risemesh_geometry"))
        try:
            # The file's own face-normals flag decides between its vertex
            # normals and face normals (TriangleMeshGeometryIndexed.cpp:444-490).
            nrm = m.normals()
            self.geometry[c.get("name", "noname")] = (m.triangles().astype(np.float64), m.info()["double_sided"],
                                                      None if nrm is None else nrm.astype(np.float64))
        finally:
            m.close()

    def rawmesh2_geometry(self, c):
        # TriangleMeshLoaderRAW2 (Geometry/TriangleMeshLoaderRAW2.cpp): a
        # "vertices triangles" header, "v x y z nx ny nz u v [r g b]" lines,
        # then "t a b c" lines indexing vertices, normals and coordinates alike;
        # face_normals shades with face normals instead.
        self.only(c, {"name", "file", "double_sided", "face_normals", "maxpolygons", "maxdepth"})
        with open(self.path(c.get("file", "none"), "rawmesh2_geometry"), "r") as f:
            lines = [ln.split() for ln in f if ln.strip()]
        try:
            nv, nt = int(lines[0][0]), int(lines[0][1])
            verts = np.array([[float(x) for x in ln[1:7]] for ln in lines[1:1 + nv]], np.float64).reshape(-1, 6)
            idx = np.array([[int(x) for x in ln[1:4]] for ln in lines[1 + nv:1 + nv + nt]], np.int64).reshape(-1, 3)
        except (IndexError, ValueError):
            self.refuse(c, "malformed RAW2 file")
        if len(verts) != nv or len(idx) != nt or (nt and (idx.min() < 0 or idx.max() >= nv)):
            self.refuse(c, "malformed RAW2 file")
        tris = verts[idx, 0:3].reshape(-1, 9)
        nrm = None if _bool(c.get("face_normals", "false")) else verts[idx, 3:6].reshape(-1, 9)
        self.geometry[c.get("name", "noname")] = (tris, _bool(c.get("double_sided", "false")), nrm)

    def box_geometry(self, c):
        self.only(c, {"name", "width", "height", "depth"})
        self.geometry[c.get("name", "noname")] = (
            _box(float(c.get("width", 1.0)), float(c.get("height", 1.0)), float(c.get("depth", 1.0))), False, None)

    # ---- objects -----------------------------------------------------------
    def standard_object(self, c):
        self.only(c, {"name", "geometry", "material", "position", "orientation", "scale", "casts_shadows",
                      "receives_shadows"})
        g = c.get("geometry", "none")
        if g not in self.geometry:
            self.refuse(c, f"unknown geometry {g!r}")
        mname = c.get("material", "none")
        if mname not in self.materials:
            self.refuse(c, f"unknown or missing material {mname!r}")
        if not _bool(c.get("casts_shadows", "true")) or not _bool(c.get("receives_shadows", "true")):
            self.refuse(c, "objects that cast or receive no shadows are not supported")
        tris, ds, nrm = self.geometry[g]
        pos = np.array(_floats(c.get("position", "0 0 0"), 3, "position"))
        ori = np.radians(_floats(c.get("orientation", "0 0 0"), 3, "orientation"))
        sc = np.array(_floats(c.get("scale", "1 1 1"), 3, "scale"))
        r = _rot(*ori)
        v = tris.reshape(-1, 3) * sc
        world = (v @ r.T + pos).reshape(-1, 9)
        # Normals go through the inverse transpose of rotation x scale
        # (Object.cpp:543): R S^-1 n; the device normalises after interpolating.
        wn = None if nrm is None else ((nrm.reshape(-1, 3) / sc) @ r.T).reshape(-1, 9).astype(np.float32)
        self.desc.add_mesh(world.astype(np.float32), self.materials[mname][0], bool(ds), normals9=wn)

    # ---- camera, film, rasterizer -----------------------------------------
    def film(self, c):
        self.only(c, {"width", "height", "pixelAR"})
        if float(c.get("pixelAR", 1.0)) != 1.0:
            self.refuse(c, "pixel aspect ratios other than 1 are not supported")
        self.st["width"] = int(c.get("width", 256))
        self.st["height"] = int(c.get("height", 256))

    def pinhole_camera(self, c):
        self.only(c, {"name", "location", "lookat", "up", "fov", "orientation", "pitch", "roll", "yaw",
                      "target_orientation", "theta", "phi", "exposure", "scanning_rate", "pixel_rate"})
        for k in ("orientation", "target_orientation"):
            if c.has(k) and any(x != 0.0 for x in map(float, c.get(k).split())):
                self.refuse(c, f"{k} is not supported")
        for k in ("pitch", "roll", "yaw", "theta", "phi"):
            if c.has(k) and float(c.get(k)) != 0.0:
                self.refuse(c, f"{k} is not supported")
        self.st["cam_pos"] = tuple(_floats(c.get("location", "0 0 0"), 3, "location"))
        self.st["cam_look"] = tuple(_floats(c.get("lookat", "0 0 -1"), 3, "lookat"))
        self.st["cam_up"] = tuple(_floats(c.get("up", "0 1 0"), 3, "up"))
        self.st["fov_deg"] = float(c.get("fov", 39.0))

    def _raster_common(self, c, extra):
        base = {"samples", "nmbegin", "nmend", "num_wavelengths", "hwss", "use_hwss", "spectral_samples",
                "pixel_filter", "pixel_filter_width", "pixel_filter_height", "pixel_filter_paramA",
                "pixel_filter_paramB", "pixel_sampler", "pixel_sampler_param", "blue_noise_sampler",
                "adaptive_max_samples", "adaptive_threshold", "rr_min_depth", "rr_threshold", "show_luminaires",
                "oidn_denoise", "oidn_quality", "oidn_device", "oidn_prefilter", "light_bvh", "defaultshader",
                "progressive_rendering", "progressive_samples_per_pass", "max_diffuse_bounce", "max_glossy_bounce",
                "max_transmission_bounce", "max_translucent_bounce", "max_volume_bounce", "radiance_map",
                "radiance_scale", "radiance_background", "radiance_orient"}
        self.only(c, base | extra)
        self.spp = int(c.get("samples", 32))
        lo, hi = float(c.get("nmbegin", 380.0)), float(c.get("nmend", 780.0))
        if lo < 380.0 or hi > 780.0 or not hi > lo:
            self.refuse(c, "wavelength range must lie within 380..780 nm")
        self.st["lambda_min"], self.st["lambda_max"] = lo, hi
        filt = c.get("pixel_filter", "gaussian").strip('"').lower()
        if filt == "gaussian":
            self.st["filter"] = 1
            self.st["filter_size"] = float(c.get("pixel_filter_paramA", 2.0))
            self.st["filter_sigma"] = float(c.get("pixel_filter_paramB", 0.35))
        elif filt == "box" and float(c.get("pixel_filter_width", 1.0)) == 1.0 \
                and float(c.get("pixel_filter_height", 1.0)) == 1.0:
            self.st["filter"] = 0
        else:
            self.refuse(c, f"pixel filter {filt!r} is not supported (gaussian, or box of width 1)")
        if c.has("adaptive_max_samples"):
            self.st["adaptive_max_spp"] = int(c.get("adaptive_max_samples"))
            self.st["adaptive_threshold"] = float(c.get("adaptive_threshold", 0.01))
        if c.has("rr_min_depth"):
            self.st["rr_min_depth"] = int(c.get("rr_min_depth"))
        if c.has("rr_threshold"):
            self.st["rr_threshold"] = float(c.get("rr_threshold"))
        # Per-type bounce limits (StabilityConfig); translucent and volume
        # bounces cannot occur with the materials read here.
        for k in ("max_diffuse_bounce", "max_glossy_bounce", "max_transmission_bounce"):
            if c.has(k):
                self.st[k] = int(c.get(k))
        # The reference's integrator always draws its path decisions from its
        # Owen-scrambled Sobol sampler (PathTracingSpectralRasterizer.cpp:206-479);
        # rendered here with the sample index shuffled per dimension pair, which
        # converges per pixel where the reference's padding does not
        # (scenes.SAMPLER_SOBOL is the reference's sequence as it is).
        self.st["sampler"] = scenes.SAMPLER_SOBOL_SHUFFLED
        if not _bool(c.get("show_luminaires", "true")):
            self.refuse(c, "hidden luminaires (show_luminaires false) are not supported")
        if c.has("pixel_sampler"):
            self.notes.append(f"{c.keyword}: camera jitter is drawn from the path's Sobol dimensions 0 and 1, "
                              "whatever pixel sampler is named")
        # The reference denoises with OIDN unless told not to (RasterizerDefaults::oidnDenoise).
        if _bool(c.get("oidn_denoise", "true")):
            self.notes.append(f"{c.keyword}: the film is not denoised")
        # Environment (RadianceMapConfig): a painter seen by escaping rays
        # through the light-probe mapping (Rendering/RadianceMap.h), times
        # radiance_scale; drawn here when the painter is uniform (a spectral
        # or uniform-colour painter: the same radiance in every direction,
        # so the orientation does not matter), visible to camera rays when
        # radiance_background (default true).
        env = c.get("radiance_map", "none")
        if env in self.images:
            self.desc.env = -1
            self.desc.env_map = scenes.EnvMap(self.images[env], float(c.get("radiance_scale", 1.0)),
                                              tuple(_floats(c.get("radiance_orient", "0 0 0"), 3, "radiance_orient")))
            self.desc.env_visible = int(_bool(c.get("radiance_background", "true")))
        elif env != "none":
            if env not in self.painters:
                self.refuse(c, f"radiance_map {env!r}: only uniform painters (spectral_painter, "
                               "uniformcolor_painter, blackbody_painter) are supported")
            scale = float(c.get("radiance_scale", 1.0))
            sid = self.painters[env]
            if scale != 1.0:
                import dataclasses
                sp = self.desc.spectra[sid]
                if isinstance(sp, np.ndarray):
                    sp = (sp * scale).astype(np.float32)
                elif hasattr(sp, "amps"):
                    sp = dataclasses.replace(sp, amps=np.asarray(sp.amps) * scale)
                else:
                    sp = dataclasses.replace(sp, scale=sp.scale * scale)
                sid = self.desc.add_spectrum(sp)
            self.desc.env = sid
            self.desc.env_visible = int(_bool(c.get("radiance_background", "true")))
            if c.get("radiance_orient", "0 0 0").split() != ["0", "0", "0"]:
                self.notes.append(f"{c.keyword}: radiance_orient does not change a uniform painter's sky")
        # StabilityConfig::useLightBVH (default true): the light BVH, else
        # the alias table over emitted power.
        self.st["light_selection"] = 0 if _bool(c.get("light_bvh", "true")) else 1
        # SpectralConfig (Utilities/SpectralConfig.h): hero-wavelength bundles
        # with `hwss true`, else one wavelength per path in num_wavelengths
        # bins (default 10); spectral_samples paths per pixel sample.
        hwss = _bool(c.get("hwss", c.get("use_hwss", "false")))
        self.st["spectral_mode"] = scenes.SPECTRAL_HWSS if hwss else scenes.SPECTRAL_SINGLE
        self.st["num_wavelengths"] = int(c.get("num_wavelengths", 10))
        self.st["spectral_samples"] = int(c.get("spectral_samples", 1))
        if self.st["num_wavelengths"] < 1 or not 1 <= self.st["spectral_samples"] <= 256:
            self.refuse(c, "num_wavelengths must be positive and spectral_samples within 1..256")

    def pathtracing_spectral_rasterizer(self, c):
        self._raster_common(c, set())
        self.st["max_depth"] = 128

    def pixelintegratingspectral_rasterizer(self, c):
        self._raster_common(c, {"lum_samples", "max_recursion"})
        self.st["max_depth"] = int(c.get("max_recursion", 10))

    def file_rasterizeroutput(self, c):
        self.outputs.append({k: v for k, v, _ in c.params})

    def accept(self, c):
        pass

    pathtracing_shaderop = accept
    standard_shader = accept


def load_scene(path=None, text=None, search=()):
    """Read a .RISEscene (or its text) into a LoadedScene.  Referenced files
    are looked up in `search` (e.g. the reference's media root), then next to
    the scene file, then in the working directory."""
    if text is None:
        with open(path, "r") as f:
            text = f.read()
    dirs = list(search) + ([os.path.dirname(os.path.abspath(path))] if path else []) + [os.getcwd()]
    ld = _Loader(dirs)
    for c in parse_chunks(text):
        fn = getattr(ld, c.keyword, None)
        if fn is None or c.keyword.startswith("_"):
            raise SceneFileError(f"line {c.line}: chunk {c.keyword} is not supported")
        fn(c)
    if ld.spp is None:
        raise SceneFileError("no spectral rasterizer chunk")
    if not ld.desc.meshes:
        raise SceneFileError("no objects")
    st = scenes.RenderSettings(**{**scenes.RenderSettings().__dict__, "max_depth": 128, **ld.st})
    ld.desc.settings = st
    return LoadedScene(ld.desc, ld.spp, ld.outputs, ld.notes)
