"""Write a scenes.SceneDesc in the reference's scene language, so the
reference renderer (oracle.RefRenderer) can render a synthetic scene of this
package: test and benchmark infrastructure, used where the reference
renderer is timed on the same scenes as the device (the serving arm of
bench.py).

The description's pieces map to the reference's chunks as the scene ingest
(rise_b200/scenefile.py) reads them back: a 81-sample spectrum becomes a
spectral_painter of 81 control points on 380..780 nm; Lambertian, emitting
(lambertian_luminaire_material, exitance = radiance with scale pi), GGX
conductor (ggx_material: ior / extinction scalar painters, isotropic alpha, rs
the reflectance painter or, for none, a unit one -- the reference's "none"
is black) and smooth dielectric (dielectric_material, tau 1, scattering 1e6)
materials; one RAW triangle file per mesh (rawmesh_geometry); the uniform
sky as the rasterizer's radiance_map of its spectrum; a pinhole camera and
the path-tracing spectral rasterizer with hero-wavelength bundles, the box
filter of width 1 and the settings' per-type bounce limits (else max depth - 1 of
each type).
"""
import math
import os

import numpy as np


def _spectrum_chunk(name, values):
    nm = np.arange(81) * 5.0 + 380.0
    out = ["spectral_painter", "{", f"\tname\t\t{name}", "\tnmbegin\t\t380", "\tnmend\t\t780"]
    out += [f"\tcp\t\t\t{a:g} {float(b):.9g}" for a, b in zip(nm, values)]
    return out + ["}", ""]


def write_risescene(desc, folder, name, spp=16, settings=None):
    """Write `desc` as folder/name.RISEscene (+ one RAW file per mesh);
    returns the scene file's path."""
    st = settings or desc.settings
    os.makedirs(folder, exist_ok=True)
    # Per-type bounce limits: the settings' own, else max depth - 1 of each
    # (the reference caps the path itself at 128 vertices).
    bounces = [getattr(st, k, None) for k in ("max_diffuse_bounce", "max_glossy_bounce", "max_transmission_bounce")]
    bounces = [max(1, st.max_depth - 1) if b is None else b for b in bounces]
    out = ["RISE ASCII SCENE 7", "", "pathtracing_shaderop", "{", "\tname\t\tpt", "}", "",
           "standard_shader", "{", "\tname\t\tglobal", "\tshaderop\tpt", "}", ""]
    raster = ["pathtracing_spectral_rasterizer", "{", f"\tsamples\t\t\t\t{spp}",
              f"\tnmbegin\t\t\t\t{st.lambda_min:g}", f"\tnmend\t\t\t\t{st.lambda_max:g}", "\thwss\t\t\t\ttrue",
              "\tspectral_samples\t1", "\tpixel_filter\t\tbox", "\tpixel_filter_width\t1", "\tpixel_filter_height\t1",
              f"\trr_min_depth\t\t{st.rr_min_depth}", f"\tmax_diffuse_bounce\t{bounces[0]}",
              f"\tmax_glossy_bounce\t{bounces[1]}", f"\tmax_transmission_bounce\t{bounces[2]}", "\toidn_denoise\t\tfalse"]
    if desc.env >= 0:
        raster += ["\tradiance_map\t\tpnt_%d" % desc.env, f"\tradiance_background\t{'true' if desc.env_visible else 'false'}"]
    out += ["film", "{", f"\twidth\t\t{st.width}", f"\theight\t\t{st.height}", "}", ""]
    out += ["pinhole_camera", "{", "\tlocation\t%g %g %g" % tuple(st.cam_pos), "\tlookat\t\t%g %g %g" % tuple(st.cam_look),
            "\tup\t\t\t%g %g %g" % tuple(st.cam_up), f"\tfov\t\t\t{st.fov_deg:g}", "}", ""]
    nm = np.arange(81) * 5.0 + 380.0
    out += _spectrum_chunk("pnt_one", np.ones(81))
    for i, sp in enumerate(desc.spectra):
        out += _spectrum_chunk(f"pnt_{i}", np.asarray(sp, np.float64))
        # The same values as a physical scalar (GGX ior / extinction slots).
        fn = f"{name}_scalar{i}.spectra"
        with open(os.path.join(folder, fn), "w") as f:
            f.writelines(f"{a:g} {float(b):.9g}\n" for a, b in zip(nm, np.asarray(sp, np.float64)))
        out += ["scalar_painter", "{", f"\tname\t\tscl_{i}", f"\tfile\t\t{fn}", "}", ""]
    out += raster + ["}", ""]
    for i, m in enumerate(desc.materials):
        if m.emission >= 0:
            out += ["lambertian_luminaire_material", "{", f"\tname\t\tmat_{i}", f"\texitance\tpnt_{m.emission}",
                    f"\tscale\t\t{math.pi:.17g}", "\tmaterial\tnone", "}", ""]
        elif m.type == 0:
            out += ["lambertian_material", "{", f"\tname\t\tmat_{i}", f"\treflectance\tpnt_{m.reflectance}", "}", ""]
        elif m.type == 1:
            rs = f"pnt_{m.reflectance}" if m.reflectance >= 0 else "pnt_one"
            out += ["ggx_material", "{", f"\tname\t\tmat_{i}", f"\trs\t\t\t{rs}", f"\tior\t\t\tscl_{m.eta}",
                    f"\textinction\tscl_{m.kappa}", f"\talphax\t\t{m.alpha:.9g}", f"\talphay\t\t{m.alpha:.9g}", "}", ""]
        else:
            out += ["dielectric_material", "{", f"\tname\t\tmat_{i}", "\ttau\t\t\t1.0", f"\tior\t\t\t{m.ior:.9g}",
                    "\tscattering\t1000000", "}", ""]
    for k, (first, count, mat, ds) in enumerate(desc.meshes):
        fn = f"{name}_mesh{k}.raw"
        tri = np.asarray(desc.tri9[first:first + count], np.float64)
        with open(os.path.join(folder, fn), "w") as f:
            f.writelines("tri " + " ".join(f"{v:.9g}" for v in t) + "\n" for t in tri)
        out += ["rawmesh_geometry", "{", f"\tname\t\tg_{k}", f"\tfile\t\t{fn}",
                f"\tdouble_sided\t{'true' if ds else 'false'}", "}", ""]
        out += ["standard_object", "{", f"\tname\t\to_{k}", f"\tgeometry\tg_{k}", f"\tmaterial\tmat_{mat}", "}", ""]
    path = os.path.join(folder, name + ".RISEscene")
    with open(path, "w") as f:
        f.write("\n".join(out))
    return path
