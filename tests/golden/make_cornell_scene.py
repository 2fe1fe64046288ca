"""Write the C1 spectral Cornell box as a scene in the reference's own scene
language: tests/golden/cornell_c1.RISEscene plus one RAW triangle file per
object (tests/golden/cornell_c1_*.raw).

The same files are loaded by the reference renderer (its .RISEscene parser,
through oracle/_ref/librise_ref.so) and by this package's scene ingest
(rise_b200.scenefile), so both render one scene description.

Geometry is scenes.cornell_box()'s 32 triangles: five unit-square walls as
triangle meshes (not clipped planes, which the reference intersects as
bilinear patches), two boxes rotated about the vertical axis, and a
0.25 x 0.25 light quad just below the ceiling facing down (one-sided).
Spectra are spectral_painter chunks with 30 control points every 10 nm on
400..700 nm, so the reference's painter (control points sampled into 30
bins, step lookup) gives exactly: white 0.75; red 0.6 on [600, 700], 0.05
below; green 0.6 on [500, 570), 0.05 elsewhere; light exitance 15 with
scale pi, i.e. radiance 15 (LambertianEmitter divides by pi).  HWSS with 4
wavelengths on 400..700 nm, box pixel filter of width 1, Russian roulette
from depth 3, at most 7 diffuse bounces (8 path vertices, the config's max
depth 8), 256 x 256, 16 samples per pixel.

    python tests/golden/make_cornell_scene.py           (the C1 scene)
    python tests/golden/make_cornell_scene.py smooth    (the smooth-shaded variant)
    python tests/golden/make_cornell_scene.py variants  (single-wavelength and dispersive variants)
    python tests/golden/make_cornell_scene.py overlap   (overlapping glass and metal spheres)
    python tests/golden/make_cornell_scene.py dsglass   (a double-sided glass sphere)
"""
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from rise_b200 import scenes  # noqa: E402

NAME = "cornell_c1"


def band(lo, hi, inside, outside):
    """Control points every 10 nm: `inside` for lo <= nm < hi, else `outside`."""
    nm = np.arange(400, 700, 10)
    return [(float(n), inside if lo <= n < hi else outside) for n in nm]


SPECTRA = {
    "pnt_white": band(400, 710, 0.75, 0.75),
    "pnt_red": band(600, 710, 0.6, 0.05),
    "pnt_green": band(500, 570, 0.6, 0.05),
    "pnt_light": band(400, 710, 15.0, 15.0),
}


def scene_text(width=256, height=256, spp=16):
    d = scenes.cornell_box(width, height)
    st = d.settings
    groups = [("walls_white", 0, "white", True), ("wall_red", 1, "red", True),
              ("wall_green", 2, "green", True), ("boxes", 3, "white", True), ("light", 4, "light", False)]
    raw = {}
    for name, mesh, _, _ in groups:
        first, count, _, _ = d.meshes[mesh]
        raw[name] = d.tri9[first:first + count]
    out = ["RISE ASCII SCENE 7", "",
           "# The C1 spectral Cornell box (written by tests/golden/make_cornell_scene.py).", ""]
    # The rasterizer's default shader must exist, even though the spectral
    # path tracer integrates on its own.
    out += ["pathtracing_shaderop", "{", "\tname\t\tpt", "}", "",
            "standard_shader", "{", "\tname\t\tglobal", "\tshaderop\tpt", "}", ""]
    out += ["pathtracing_spectral_rasterizer", "{",
            f"\tsamples\t\t\t\t{spp}", f"\tnmbegin\t\t\t\t{st.lambda_min:g}", f"\tnmend\t\t\t\t{st.lambda_max:g}",
            "\thwss\t\t\t\ttrue", "\tspectral_samples\t1", "\tpixel_filter\t\tbox", "\tpixel_filter_width\t1",
            "\tpixel_filter_height\t1", f"\trr_min_depth\t\t{st.rr_min_depth}",
            f"\tmax_diffuse_bounce\t{st.max_depth - 1}", "}", ""]
    out += ["film", "{", f"\twidth\t\t{width}", f"\theight\t\t{height}", "}", ""]
    out += ["pinhole_camera", "{", "\tlocation\t%g %g %g" % st.cam_pos, "\tlookat\t\t%g %g %g" % st.cam_look,
            "\tup\t\t\t%g %g %g" % st.cam_up, f"\tfov\t\t\t{st.fov_deg:g}", "}", ""]
    for name, cps in SPECTRA.items():
        out += ["spectral_painter", "{", f"\tname\t\t{name}", "\tnmbegin\t\t400", "\tnmend\t\t700"]
        out += [f"\tcp\t\t\t{a:g} {b:g}" for a, b in cps]
        out += ["}", ""]
    for m in ("white", "red", "green"):
        out += ["lambertian_material", "{", f"\tname\t\t{m}", f"\treflectance\tpnt_{m}", "}", ""]
    out += ["lambertian_luminaire_material", "{", "\tname\t\tlight", "\texitance\tpnt_light",
            f"\tscale\t\t{math.pi:.17g}", "\tmaterial\tnone", "}", ""]
    for name, _, mat, ds in groups:
        out += ["rawmesh_geometry", "{", f"\tname\t\tg_{name}", f"\tfile\t\t{NAME}_{name}.raw",
                f"\tdouble_sided\t{'true' if ds else 'false'}", "}", ""]
        out += ["standard_object", "{", f"\tname\t\to_{name}", f"\tgeometry\tg_{name}", f"\tmaterial\t{mat}",
                "}", ""]
    return "\n".join(out), raw


def raw_text(tri9):
    return "".join("tri " + " ".join(f"{float(v):.9g}" for v in t) + "\n" for t in tri9)


def main():
    text, raw = scene_text()
    with open(os.path.join(HERE, NAME + ".RISEscene"), "w") as f:
        f.write(text)
    for name, tri9 in raw.items():
        with open(os.path.join(HERE, f"{NAME}_{name}.raw"), "w") as f:
            f.write(raw_text(tri9))


if __name__ == "__main__" and not sys.argv[1:]:
    main()


# ---- a smooth-shaded variant --------------------------------------------------
# The C1 box without its two boxes, holding two UV spheres of 960 triangles
# with vertex normals (RAW2 files, which carry a normal per vertex): a
# Lambertian white one and a smooth dielectric (IOR 1.5) one.  Written by
# `python tests/golden/make_cornell_scene.py smooth`.
SMOOTH = "cornell_smooth"
SPHERES = [("sphere_matte", (0.3, 0.18, 0.55), 0.18, "white"), ("sphere_glass", (0.7, 0.2, 0.35), 0.2, "glass")]


def raw2_text(center, radius, n_tri):
    tri9 = scenes.uv_sphere(center, radius, n_tri).astype(np.float64)
    nrm9 = scenes.sphere_normals(tri9, center).astype(np.float64)
    v = tri9.reshape(-1, 3)
    n = nrm9.reshape(-1, 3)
    lines = [f"{len(v)} {len(tri9)}"]
    lines += [f"v {a[0]:.9g} {a[1]:.9g} {a[2]:.9g} {b[0]:.9g} {b[1]:.9g} {b[2]:.9g} 0 0" for a, b in zip(v, n)]
    lines += [f"t {3 * i} {3 * i + 1} {3 * i + 2}" for i in range(len(tri9))]
    return "\n".join(lines) + "\n"


def smooth_scene_text():
    text, _ = scene_text()
    text = text.replace("# The C1 spectral Cornell box (written by tests/golden/make_cornell_scene.py).",
                        "# The C1 box with two smooth-shaded spheres (written by tests/golden/make_cornell_scene.py).")
    text = text.replace(f"\tfile\t\t{NAME}_", "\tfile\t\tcornell_c1_")
    # No boxes; the spheres instead.
    cut = text.index("rawmesh_geometry\n{\n\tname\t\tg_boxes")
    end = text.index("rawmesh_geometry\n{\n\tname\t\tg_light")
    text = text[:cut] + text[end:]
    text = text.replace("max_diffuse_bounce\t7", "max_diffuse_bounce\t7\n\tmax_glossy_bounce\t8\n"
                        "\tmax_transmission_bounce\t8")
    extra = ["dielectric_material", "{", "\tname\t\tglass", "\ttau\t\t\t1.0", "\tior\t\t\t1.5",
             "\tscattering\t1000000", "}", ""]
    for name, c, r, mat in SPHERES:
        extra += ["rawmesh2_geometry", "{", f"\tname\t\tg_{name}", f"\tfile\t\t{SMOOTH}_{name}.raw2",
                  "\tdouble_sided\tfalse", "}", ""]
        extra += ["standard_object", "{", f"\tname\t\to_{name}", f"\tgeometry\tg_{name}", f"\tmaterial\t{mat}",
                  "}", ""]
    return text + "\n".join(extra)


def main_smooth():
    with open(os.path.join(HERE, SMOOTH + ".RISEscene"), "w") as f:
        f.write(smooth_scene_text())
    for name, c, r, _ in SPHERES:
        with open(os.path.join(HERE, f"{SMOOTH}_{name}.raw2"), "w") as f:
            f.write(raw2_text(c, r, 960))


if __name__ == "__main__" and sys.argv[1:] == ["smooth"]:
    main_smooth()


# ---- wavelength-sampling variants ---------------------------------------------
# cornell_nm: the C1 scene with `hwss false`, the reference's default of one
# wavelength per path in num_wavelengths (default 10) bins.
# cornell_prism: the C1 walls and light around a closed triangular glass
# prism (single-sided, outward winding) whose index of refraction varies with
# wavelength, raised 0.02 off the floor (`ior 1.3 1.5 2`: the reference's RGBScalarPainter, 2.0 at 450 nm
# and below, 1.5 at 550, 1.3 from 650), rendered with hero-wavelength
# bundles; cornell_prism_nm the same with one wavelength per path in 30 bins
# and two spectral samples per pixel sample.
#     python tests/golden/make_cornell_scene.py variants
PRISM = [(0.32, 0.02, 0.30), (0.68, 0.02, 0.30), (0.50, 0.02, 0.58)]
PRISM_HEIGHT = 0.42


def prism_tri9():
    a, b, c = (np.array(p, np.float64) for p in PRISM)
    up = np.array([0.0, PRISM_HEIGHT, 0.0])
    A, B, C = a + up, b + up, c + up
    tris = [(a, b, c), (A, C, B)]                         # bottom (facing down), top (facing up)
    for p, q in ((a, b), (b, c), (c, a)):                 # sides, counter-clockwise seen from outside
        P, Q = p + up, q + up
        tris += [(p, Q, q), (p, P, Q)]
    t = np.array([np.concatenate(x) for x in tris])
    cen = np.mean([a, b, c], axis=0) + 0.5 * up
    tt = t.reshape(-1, 3, 3)
    n = np.cross(tt[:, 1] - tt[:, 0], tt[:, 2] - tt[:, 0])
    assert ((n * (tt.mean(axis=1) - cen)).sum(axis=1) > 0).all()
    return t


def nm_scene_text():
    text, _ = scene_text()
    text = text.replace("# The C1 spectral Cornell box (written by tests/golden/make_cornell_scene.py).",
                        "# The C1 box, one wavelength per path (written by tests/golden/make_cornell_scene.py).")
    return text.replace("\thwss\t\t\t\ttrue\n", "\thwss\t\t\t\tfalse\n")


def prism_scene_text(hwss=True):
    text, _ = scene_text()
    what = "hero-wavelength bundles" if hwss else "one wavelength per path"
    text = text.replace("# The C1 spectral Cornell box (written by tests/golden/make_cornell_scene.py).",
                        f"# The C1 box around a dispersive glass prism, {what} "
                        "(written by tests/golden/make_cornell_scene.py).")
    text = text.replace(f"\tfile\t\t{NAME}_", "\tfile\t\tcornell_c1_")
    cut = text.index("rawmesh_geometry\n{\n\tname\t\tg_boxes")
    end = text.index("rawmesh_geometry\n{\n\tname\t\tg_light")
    text = text[:cut] + text[end:]
    text = text.replace("max_diffuse_bounce\t7", "max_diffuse_bounce\t7\n\tmax_glossy_bounce\t8\n"
                        "\tmax_transmission_bounce\t8")
    if not hwss:
        text = text.replace("\thwss\t\t\t\ttrue\n\tspectral_samples\t1\n",
                            "\thwss\t\t\t\tfalse\n\tnum_wavelengths\t\t30\n\tspectral_samples\t2\n")
    extra = ["dielectric_material", "{", "\tname\t\tglass", "\ttau\t\t\t1.0", "\tior\t\t\t1.3 1.5 2",
             "\tscattering\t1000000", "}", "",
             "rawmesh_geometry", "{", "\tname\t\tg_prism", "\tfile\t\tcornell_prism_prism.raw",
             "\tdouble_sided\tfalse", "}", "",
             "standard_object", "{", "\tname\t\to_prism", "\tgeometry\tg_prism", "\tmaterial\tglass", "}", ""]
    return text + "\n".join(extra)


def main_variants():
    for name, text in (("cornell_nm", nm_scene_text()), ("cornell_prism", prism_scene_text(True)),
                       ("cornell_prism_nm", prism_scene_text(False))):
        with open(os.path.join(HERE, name + ".RISEscene"), "w") as f:
            f.write(text)
    with open(os.path.join(HERE, "cornell_prism_prism.raw"), "w") as f:
        f.write(raw_text(prism_tri9()))


if __name__ == "__main__" and sys.argv[1:] == ["variants"]:
    main_variants()


# ---- overlapping media ---------------------------------------------------------
# cornell_overlap: the C1 walls and light around two overlapping glass spheres
# of different indices (1.5 and 1.33; single-sided, outward winding) and a
# GGX conductor sphere (double-sided) that cuts into the first.  The
# reference's index-of-refraction stack (Utilities/IORStack.h) gives the
# indices on either side of each crossing (1.5 -> 1.33 from the first sphere
# into the second, not air -> 1.33) and the conductor's Fresnel seen from
# inside the glass (incident index 1.5).  Hero-wavelength bundles.
#     python tests/golden/make_cornell_scene.py overlap
OVERLAP = [("glass_a", (0.42, 0.25, 0.45), 0.2, "glass_a", False),
           ("glass_b", (0.62, 0.22, 0.38), 0.16, "glass_b", False),
           ("metal", (0.30, 0.14, 0.30), 0.12, "metal", True)]


def overlap_scene_text():
    text, _ = scene_text()
    text = text.replace("# The C1 spectral Cornell box (written by tests/golden/make_cornell_scene.py).",
                        "# The C1 box around overlapping glass and metal spheres "
                        "(written by tests/golden/make_cornell_scene.py).")
    text = text.replace(f"\tfile\t\t{NAME}_", "\tfile\t\tcornell_c1_")
    cut = text.index("rawmesh_geometry\n{\n\tname\t\tg_boxes")
    end = text.index("rawmesh_geometry\n{\n\tname\t\tg_light")
    text = text[:cut] + text[end:]
    text = text.replace("max_diffuse_bounce\t7", "max_diffuse_bounce\t7\n\tmax_glossy_bounce\t8\n"
                        "\tmax_transmission_bounce\t8")
    extra = ["dielectric_material", "{", "\tname\t\tglass_a", "\ttau\t\t\t1.0", "\tior\t\t\t1.5",
             "\tscattering\t1000000", "}", "",
             "dielectric_material", "{", "\tname\t\tglass_b", "\ttau\t\t\t1.0", "\tior\t\t\t1.33",
             "\tscattering\t1000000", "}", "",
             "ggx_material", "{", "\tname\t\tmetal", "\trs\t\t\tpnt_white", "\tior\t\t\t0.4",
             "\textinction\t2.5", "\talphax\t\t0.2", "\talphay\t\t0.2", "}", ""]
    for name, c, r, mat, ds in OVERLAP:
        extra += ["rawmesh_geometry", "{", f"\tname\t\tg_{name}", f"\tfile\t\tcornell_overlap_{name}.raw",
                  f"\tdouble_sided\t{'true' if ds else 'false'}", "}", ""]
        extra += ["standard_object", "{", f"\tname\t\to_{name}", f"\tgeometry\tg_{name}", f"\tmaterial\t{mat}",
                  "}", ""]
    return text + "\n".join(extra)


def main_overlap():
    with open(os.path.join(HERE, "cornell_overlap.RISEscene"), "w") as f:
        f.write(overlap_scene_text())
    for name, c, r, _, _ in OVERLAP:
        with open(os.path.join(HERE, f"cornell_overlap_{name}.raw"), "w") as f:
            f.write(raw_text(scenes.uv_sphere(c, r, 960)))


if __name__ == "__main__" and sys.argv[1:] == ["overlap"]:
    main_overlap()


# ---- double-sided glass ----------------------------------------------------------
# cornell_dsglass: the C1 walls and light around one glass sphere (IOR 1.5,
# flat-shaded RAW mesh) marked double-sided.  The reference turns a double-
# sided mesh's normals towards the ray (TriangleMeshGeometry.cpp:94-120) while
# its dielectric takes inside / outside from the index-of-refraction stack, so
# a ray leaving the sphere sees the normal on its own side and the refracted
# ray fails the crossing test (DielectricSPF.cpp:274-279): only total internal
# reflection leaves the inside.
#     python tests/golden/make_cornell_scene.py dsglass
DSGLASS = ("glass_ds", (0.5, 0.25, 0.45), 0.22)


def dsglass_scene_text():
    text = overlap_scene_text()
    text = text.replace("# The C1 box around overlapping glass and metal spheres",
                        "# The C1 box around a double-sided glass sphere")
    cut = text.index("dielectric_material\n{\n\tname\t\tglass_b")
    text = text[:cut]
    name, c, r = DSGLASS
    extra = ["rawmesh_geometry", "{", f"\tname\t\tg_{name}", f"\tfile\t\tcornell_dsglass_{name}.raw",
             "\tdouble_sided\ttrue", "}", "",
             "standard_object", "{", f"\tname\t\to_{name}", f"\tgeometry\tg_{name}", "\tmaterial\tglass_a", "}", ""]
    return text + "\n".join(extra)


def main_dsglass():
    with open(os.path.join(HERE, "cornell_dsglass.RISEscene"), "w") as f:
        f.write(dsglass_scene_text())
    name, c, r = DSGLASS
    with open(os.path.join(HERE, f"cornell_dsglass_{name}.raw"), "w") as f:
        f.write(raw_text(scenes.uv_sphere(c, r, 960)))


if __name__ == "__main__" and sys.argv[1:] == ["dsglass"]:
    main_dsglass()
