"""The RISE-side adapter (rise_b200/adapter/) against this package's scene
ingest, on the CPU.

The adapter reads a scene through the reference renderer's own interfaces
(the scene parsed by the reference's job, oracle/_ref/librise_ref.so;
IScene, IObjectManager, TessellateToMesh, the material and painter classes,
ICamera::GenerateRay, RadianceMap) into the description the C ABI takes; the
test driver tests/cpp/rise_adapter_check.cpp (built by oracle/rise_ref.mk,
target adapter) writes that description out.  Here it must equal what
rise_b200.scenefile reads from the same file: the same world-space
triangles, the same materials and spectra wavelength by wavelength, the same
camera, film and environment.  (The GPU test renders both and compares the
images.)
"""
import json
import math
import os
import subprocess

import numpy as np
import pytest

from rise_b200 import scenes, scenefile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
EXE = os.path.join(ROOT, "oracle", "_ref", "rise_adapter_check")
SCENES = ["cornell_c1", "cornell_smooth", "cornell_prism", "cornell_env", "cornell_overlap", "cornell_dsglass"]
NM = np.arange(380.0, 781.0, 1.0) + 0.25


def _adapter():
    if not os.path.exists(EXE):
        pytest.skip("the RISE adapter test driver is not built (needs the reference tree)")
    return EXE


def extract(name, tmp_path):
    out = subprocess.run([_adapter(), "extract", os.path.join(GOLDEN, name + ".RISEscene"), str(tmp_path / name)],
                         capture_output=True, text=True, cwd=tmp_path)
    assert out.returncode == 0 and "ok" in out.stdout, out.stdout + out.stderr
    d = json.load(open(tmp_path / (name + ".json")))
    d["xyz"] = np.fromfile(tmp_path / (name + ".xyz"), np.float32).reshape(-1, 9)
    if d["env_image"][0]:
        d["env"] = np.fromfile(tmp_path / (name + ".env"), np.float32).reshape(d["env_image"][1], d["env_image"][0], 3)
    return d


def eval_extracted(s, nm):
    """An extracted spectrum at wavelengths nm."""
    nm = np.asarray(nm, np.float64)
    if s["kind"] == 0:
        a = np.array(s["amps"], np.float64)
        b, e = s["begin"], s["end"]
        i = np.minimum(((nm - b) * len(a) / (e - b)).astype(int), len(a) - 1)
        return np.where((nm >= b) & (nm <= e), a[np.clip(i, 0, len(a) - 1)], 0.0)
    if s["kind"] == 1:
        c = s["coeffs"]
        t = (nm - 380.0) / 400.0
        x = c[0] * t * t + c[1] * t + c[2]
        return np.where((nm >= 380) & (nm <= 780), c[3] * (0.5 + x / (2 * np.sqrt(1 + x * x))), 0.0)
    return np.interp(nm, np.arange(81) * 5.0 + 380.0, np.array(s["amps"], np.float64))


def eval_ingest(sp, nm):
    """A scene-ingest spectrum (scenes.SceneDesc.spectra entry) at nm."""
    nm = np.asarray(nm, np.float64)
    if isinstance(sp, np.ndarray):
        return np.interp(nm, np.arange(81) * 5.0 + 380.0, sp.astype(np.float64))
    if hasattr(sp, "amps"):
        a = np.asarray(sp.amps, np.float64)
        i = np.minimum(((nm - sp.begin) * len(a) / (sp.end - sp.begin)).astype(int), len(a) - 1)
        return np.where((nm >= sp.begin) & (nm <= sp.end), a[np.clip(i, 0, len(a) - 1)], 0.0)
    if hasattr(sp, "c0"):
        t = (nm - 380.0) / 400.0
        x = sp.c0 * t * t + sp.c1 * t + sp.c2
        return np.where((nm >= 380) & (nm <= 780), sp.scale * (0.5 + x / (2 * np.sqrt(1 + x * x))), 0.0)
    raise AssertionError(f"spectrum kind {type(sp)} not compared here")


def tri_key(t):
    return tuple(np.round(t.astype(np.float64), 5))


@pytest.mark.parametrize("name", SCENES)
def test_adapter_reads_the_reference_scene_as_the_ingest_does(name, tmp_path):
    ex = extract(name, tmp_path)
    assert ex["refused"] == []
    ls = scenefile.load_scene(os.path.join(GOLDEN, name + ".RISEscene"))
    desc, st = ls.desc, ls.desc.settings
    # Film and camera.
    assert (ex["width"], ex["height"]) == (st.width, st.height)
    assert abs(ex["fov_deg"] - st.fov_deg) < 1e-4
    assert np.allclose(ex["cam_pos"], st.cam_pos, atol=1e-6)
    f_in = np.subtract(st.cam_look, st.cam_pos)
    f_ex = np.subtract(ex["cam_look"], ex["cam_pos"])
    assert np.allclose(f_in / np.linalg.norm(f_in), f_ex / np.linalg.norm(f_ex), atol=1e-6)
    up = np.array(st.cam_up, np.float64)
    up -= f_in * (up @ f_in) / (f_in @ f_in)
    assert np.allclose(up / np.linalg.norm(up), ex["cam_up"], atol=1e-6)
    # Geometry: the same world-space triangles, each with the same material.
    assert len(ex["xyz"]) == desc.n_tri
    mats_ex = np.repeat([m["material"] for m in ex["meshes"]], [m["triangles"] for m in ex["meshes"]])
    mats_in = np.concatenate([[mat] * cnt for (_, cnt, mat, _) in desc.meshes])
    ds_ex = np.repeat([m["double_sided"] for m in ex["meshes"]], [m["triangles"] for m in ex["meshes"]])
    ds_in = np.concatenate([[d] * cnt for (_, cnt, _, d) in desc.meshes])
    by_key = {tri_key(t): i for i, t in enumerate(desc.tri9)}
    matched = [by_key.get(tri_key(t), -1) for t in ex["xyz"]]
    assert min(matched) >= 0 and len(set(matched)) == desc.n_tri
    order = np.array(matched)
    assert np.allclose(ex["xyz"], desc.tri9[order], atol=2e-6)
    assert (ds_ex == ds_in[order]).all()
    # Materials, spectra wavelength by wavelength.
    for me, mi in set(zip(mats_ex.tolist(), mats_in[order].tolist())):
        e = ex["materials"][me]
        m = desc.materials[mi]
        assert e[0] == m.type
        assert abs(e[5] - m.alpha) <= 1e-6 * max(1.0, abs(m.alpha))
        for slot, ours in ((1, m.reflectance), (2, m.emission), (3, m.eta), (4, m.kappa)):
            if ours < 0 and e[slot] < 0:
                continue
            if m.type == scenes.MAT_GGX and slot == 1 and ours >= 0 and e[slot] >= 0:
                pass
            assert (ours >= 0) == (e[slot] >= 0), (slot, ours, e[slot])
            a = eval_extracted(ex["spectra"][e[slot]], NM)
            b = eval_ingest(desc.spectra[ours], NM)
            assert np.allclose(a, b, rtol=1e-5, atol=1e-6), (slot, np.abs(a - b).max())
        if m.type == scenes.MAT_DIELECTRIC and m.eta < 0:
            assert abs(e[6] - m.ior) < 1e-6
    # Environment.
    if desc.env_map is not None:
        assert np.array_equal(ex["env"], desc.env_map.rgb)
        assert abs(ex["env_image"][2] - desc.env_map.scale) < 1e-6
        ax, ay, az = (math.radians(a) for a in desc.env_map.orient_deg)
        rx = np.array([[1, 0, 0], [0, math.cos(ax), math.sin(ax)], [0, -math.sin(ax), math.cos(ax)]])
        ry = np.array([[math.cos(ay), 0, -math.sin(ay)], [0, 1, 0], [math.sin(ay), 0, math.cos(ay)]])
        rz = np.array([[math.cos(az), math.sin(az), 0], [-math.sin(az), math.cos(az), 0], [0, 0, 1]])
        # The reference's storage _rc of X * Y * Z, applied as out_c = sum_r m_rc v_r.
        m = (rx.T @ ry.T @ rz.T).T
        assert np.allclose(np.array(ex["env_rot"]).reshape(3, 3), m.T, atol=1e-6)
    else:
        assert ex["env_image"][0] == 0 and (ex["env_spectrum"] >= 0) == (desc.env >= 0)
