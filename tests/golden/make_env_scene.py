"""Write an image-environment test scene in the reference's scene language:
tests/golden/cornell_env.RISEscene and its light probe
tests/golden/cornell_env_probe.hdr (a Radiance HDR file).

The probe is a 64 x 64 angular map (the reference's light-probe mapping,
Rendering/RadianceMap.h): a sky from blue at the zenith to a warm horizon, a
darker ground, and a small bright warm sun, generated here in closed form.
The scene has no other light: a large Lambertian floor, the C1 scene's two
white boxes and a rough gold-like GGX prism (tests/golden/cornell_prism_prism.raw)
under the map turned 30 degrees about y (radiance_orient) and scaled by 1.5
(radiance_scale), visible behind the objects; hero-wavelength bundles on
400..700 nm, box filter, Russian roulette from depth 3, 128 x 128.

    python tests/golden/make_env_scene.py
"""
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SIZE = 64


def probe_rgb(size=SIZE):
    """The probe's texels (size, size, 3), rows top to bottom: map-space
    direction per texel centre through the inverse light-probe mapping."""
    img = np.zeros((size, size, 3), np.float64)
    sun = np.array([0.35, 0.8, -0.48])
    sun /= np.linalg.norm(sun)
    for y in range(size):
        for x in range(size):
            s, t = (x + 0.5) / size, (y + 0.5) / size
            dx, dy = s - 0.5, -(t - 0.5)
            r = math.hypot(dx, dy)
            if r > 0.5:
                continue
            th = 2 * math.pi * r
            d = np.array([dx * math.sin(th) / r, dy * math.sin(th) / r, -math.cos(th)]) if r > 0 else np.array([0, 0, -1.0])
            up = d[1]
            if up >= 0:
                c = np.array([0.25, 0.45, 0.9]) * (0.6 + 0.8 * up) + np.array([0.9, 0.6, 0.3]) * (1 - up) ** 4
            else:
                c = np.array([0.18, 0.15, 0.12]) * (1 + up * 0.5)
            if float(d @ sun) > math.cos(math.radians(9.0)):
                c = c + np.array([60.0, 50.0, 38.0])
            img[y, x] = c
    return img.astype(np.float32)


def hdr_bytes(img):
    """Radiance RGBE, new-style run-length scanlines of literal runs."""
    h, w, _ = img.shape
    out = bytearray(b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n" + f"-Y {h} +X {w}\n".encode())
    for y in range(h):
        rows = np.zeros((4, w), np.uint8)
        for x in range(w):
            r, g, b = (float(v) for v in img[y, x])
            m = max(r, g, b)
            if m < 1e-32:
                continue
            mant, e = math.frexp(m)   # m = mant * 2^e, mant in [0.5, 1)
            f = 256.0 / 2.0 ** e
            rows[:, x] = [min(255, int(r * f)), min(255, int(g * f)), min(255, int(b * f)), e + 128]
        out += bytes([2, 2, w >> 8, w & 255])
        for comp in range(4):
            x = 0
            while x < w:
                n = min(128, w - x)
                out.append(n)
                out += bytes(rows[comp, x:x + n])
                x += n
    return bytes(out)


def scene_text():
    out = ["RISE ASCII SCENE 7", "",
           "# Image-environment test scene (written by tests/golden/make_env_scene.py).", "",
           "pathtracing_shaderop", "{", "\tname\t\tpt", "}", "",
           "standard_shader", "{", "\tname\t\tglobal", "\tshaderop\tpt", "}", "",
           "hdr_painter", "{", "\tname\t\tpnt_env", "\tfile\t\tcornell_env_probe.hdr", "}", ""]
    flat = lambda name, v: ["spectral_painter", "{", f"\tname\t\t{name}", "\tnmbegin\t\t400", "\tnmend\t\t700"] + \
        [f"\tcp\t\t\t{n} {v}" for n in range(400, 710, 10)] + ["}", ""]
    out += flat("pnt_white", 0.75) + flat("pnt_one", 1.0)
    nm = np.arange(380, 785, 5)
    for name, vals in (("eta", 1.4 - 1.25 * (nm - 380) / 400), ("kappa", 1.8 + 2.6 * (nm - 380) / 400)):
        with open(os.path.join(HERE, f"cornell_env_{name}.spectra"), "w") as f:
            f.writelines(f"{a} {b:.6f}\n" for a, b in zip(nm, vals))
        out += ["scalar_painter", "{", f"\tname\t\tscl_{name}", f"\tfile\t\tcornell_env_{name}.spectra", "}", ""]
    out += ["pathtracing_spectral_rasterizer", "{", "\tsamples\t\t\t\t16", "\tnmbegin\t\t\t\t400",
            "\tnmend\t\t\t\t700", "\thwss\t\t\t\ttrue", "\tspectral_samples\t1", "\tpixel_filter\t\tbox",
            "\tpixel_filter_width\t1", "\tpixel_filter_height\t1", "\trr_min_depth\t\t3",
            "\tmax_diffuse_bounce\t7", "\tmax_glossy_bounce\t8", "\tmax_transmission_bounce\t8",
            "\toidn_denoise\t\tfalse", "\tradiance_map\t\tpnt_env", "\tradiance_scale\t\t1.5",
            "\tradiance_orient\t\t0 30 0", "\tradiance_background\ttrue", "}", ""]
    out += ["film", "{", "\twidth\t\t128", "\theight\t\t128", "}", ""]
    out += ["pinhole_camera", "{", "\tlocation\t0.5 0.75 -1.3", "\tlookat\t\t0.5 0.15 0.5", "\tup\t\t\t0 1 0",
            "\tfov\t\t\t45", "}", ""]
    out += ["lambertian_material", "{", "\tname\t\twhite", "\treflectance\tpnt_white", "}", "",
            "ggx_material", "{", "\tname\t\tgold", "\trs\t\t\tpnt_one", "\tior\t\t\tscl_eta",
            "\textinction\tscl_kappa", "\talphax\t\t0.2", "\talphay\t\t0.2", "}", ""]
    with open(os.path.join(HERE, "cornell_env_floor.raw"), "w") as f:
        f.write("tri -2 0 -1 -2 0 3 3 0 3\ntri -2 0 -1 3 0 3 3 0 -1\n")
    for name, fn, mat, ds in (("floor", "cornell_env_floor.raw", "white", "true"),
                              ("boxes", "cornell_c1_boxes.raw", "white", "true"),
                              ("prism", "cornell_prism_prism.raw", "gold", "false")):
        out += ["rawmesh_geometry", "{", f"\tname\t\tg_{name}", f"\tfile\t\t{fn}", f"\tdouble_sided\t{ds}", "}", "",
                "standard_object", "{", f"\tname\t\to_{name}", f"\tgeometry\tg_{name}", f"\tmaterial\t{mat}",
                "}", ""]
    return "\n".join(out)


def main():
    with open(os.path.join(HERE, "cornell_env_probe.hdr"), "wb") as f:
        f.write(hdr_bytes(probe_rgb()))
    with open(os.path.join(HERE, "cornell_env.RISEscene"), "w") as f:
        f.write(scene_text())


if __name__ == "__main__":
    main()
