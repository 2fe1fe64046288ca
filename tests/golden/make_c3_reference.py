"""Generate tests/golden/spheres_fp64_crop.npz: a 128x128 crop of the large
spheres scene (1024x1024 fBm heightfield of 2,093,058 triangles + 64 spheres of
20,000 triangles, half GGX conductors, half glass, area light + uniform sky;
1024x1024 pixels, 4 wavelengths, max depth 16) rendered by the FP64 oracle
(oracle/pt_oracle.cpp) at 2048 samples per pixel with seed 424242, which no
GPU run uses.  Crop: pixels x 448..575, y 448..575 (the image centre, with
spheres of both materials over the heightfield).  Stored as float32 XYZ.

The full 1024x1024 image at the 16384 spp the configuration names would take
days of host time; the crop's oracle noise at 2048 spp is 1/32 of the GPU's
at 64 spp, so GPU relMSE against it measures the GPU's own noise plus bias.

    make -C oracle && python tests/golden/make_c3_reference.py
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from rise_b200 import scenes  # noqa: E402

SPP = 2048
SEED = 424242
CROP = (448, 448, 576, 576)
CHUNK = 256


def main():
    desc = scenes.spheres_scene()
    settings = scenes.RenderSettings(**{**desc.settings.__dict__, "seed": SEED})
    x0, y0, x1, y1 = CROP
    acc = np.zeros((y1 - y0, x1 - x0, 3), np.float64)
    t0 = time.time()
    for begin in range(0, SPP, CHUNK):
        acc += oracle.pt_render(desc, CHUNK, sample_begin=begin, crop=CROP, settings=settings) * CHUNK
        print(f"{begin + CHUNK}/{SPP} spp, {time.time() - t0:.0f} s", flush=True)
    img = (acc / SPP).astype(np.float32)
    path = os.path.join(HERE, "spheres_fp64_crop.npz")
    np.savez_compressed(path, xyz=img, spp=SPP, seed=SEED, crop=np.array(CROP))
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
