"""A C++ host program on the C ABI (tests/cpp/capi_render.cpp) renders the
same image as the Python host layer.

The program is what a RISE-side rasterizer does with rtb200: build the scene
from meshes, spectra and materials, create one job, render progressive passes
and read the film.  It is compiled here with g++ against include/rtb200.h
and the in-tree librtb200.so; its film must equal the film of the same job
driven through rise_b200.pathtracer (relative 1e-5: only the order of FP32
film additions can differ), and its statistics must match.
"""
import ctypes
import os
import struct
import subprocess

import numpy as np
import pytest

from rise_b200 import pathtracer, raycaster, scenes

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def write_scene(path, desc, passes):
    with open(path, "wb") as f:
        f.write(b"RTBS" + struct.pack("<i", 1))
        f.write(struct.pack("<i", len(desc.spectra)))
        for sp in desc.spectra:
            f.write(np.asarray(sp, "<f4").tobytes())
        f.write(struct.pack("<i", len(desc.materials)))
        for m in desc.materials:
            f.write(bytes(pathtracer.Material(m.type, m.reflectance, m.emission, m.eta, m.kappa, m.alpha, m.ior)))
        f.write(struct.pack("<ii", desc.env, desc.env_visible))
        f.write(struct.pack("<i", len(desc.meshes)))
        for first, count, mat, ds in desc.meshes:
            f.write(struct.pack("<qii", count, mat, ds))
            f.write(np.ascontiguousarray(desc.tri9[first:first + count], "<f4").tobytes())
        f.write(bytes(pathtracer.settings_struct(desc.settings)))
        f.write(struct.pack("<i", len(passes)))
        f.write(struct.pack(f"<{len(passes)}i", *passes))


@pytest.fixture(scope="module")
def program(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("cpp") / "capi_render")
    lib = os.path.join(ROOT, "rise_b200", "_lib")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "capi_render.cpp"), "-L" + lib, "-lrtb200",
                    "-Wl,-rpath," + lib, "-o", exe], check=True)
    return exe


@pytest.mark.parametrize("which", ["cornell", "spheres"])
def test_cpp_host_matches_python_host(program, tmp_path, which):
    if which == "cornell":
        desc = scenes.cornell_box(64, 48)
    else:
        desc = scenes.spheres_scene(grid=64, n_spheres=6, sphere_tris=800, width=48, height=40, max_depth=10)
    passes = [4, 4, 8]
    scene_file, film_file = str(tmp_path / "scene.bin"), str(tmp_path / "film.bin")
    write_scene(scene_file, desc, passes)
    run = subprocess.run([program, scene_file, film_file], capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stderr
    st = dict(kv.split("=") for kv in run.stdout.split())
    w, h = desc.settings.width, desc.settings.height
    cpp = np.fromfile(film_file, "<f4").reshape(h, w, 3)

    ctx = raycaster.Context(0)
    try:
        r = pathtracer.SpectralRasterizer(ctx, desc)
        for s in passes:
            r.rasterize_scene(s)
        py = r.film()
        ps = r.stats()
        r.close()
    finally:
        ctx.close()
    assert np.isfinite(cpp).all() and cpp.max() > 0
    assert np.allclose(cpp, py, rtol=1e-5, atol=1e-7)
    assert int(st["spp"]) == ps["spp"] == sum(passes)
    assert int(st["samples"]) == ps["samples"] and int(st["segments"]) == ps["segments"]
