"""Generate tests/golden/cornell_fp64_16384spp.npz: the converged spectral
Cornell box (256x256, HWSS 4 wavelengths, max depth 8, Russian roulette from
depth 3, per-wavelength next-event estimation) rendered by the FP64 oracle
(oracle/pt_oracle.cpp) at 16384 samples per pixel with seed 424242, which no
GPU run uses.  Stored as float32 XYZ (256, 256, 3).

The oracle's noise at 16384 spp (relMSE ~2e-5) is far below the 1e-3 level the
relMSE figures are judged at, so GPU relMSE against this image measures the
GPU's own noise plus any bias.

    make -C oracle && python tests/golden/make_cornell_reference.py   # ~30 min on 8 cores
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from rise_b200 import scenes  # noqa: E402

SPP = 16384
SEED = 424242
CHUNK = 256


def main():
    desc = scenes.cornell_box(256, 256)
    settings = scenes.RenderSettings(**{**desc.settings.__dict__, "seed": SEED})
    acc = np.zeros((256, 256, 3), np.float64)
    t0 = time.time()
    for begin in range(0, SPP, CHUNK):
        acc += oracle.pt_render(desc, CHUNK, sample_begin=begin, settings=settings) * CHUNK
        print(f"{begin + CHUNK}/{SPP} spp, {time.time() - t0:.0f} s", flush=True)
    img = (acc / SPP).astype(np.float32)
    path = os.path.join(HERE, "cornell_fp64_16384spp.npz")
    np.savez_compressed(path, xyz=img, spp=SPP, seed=SEED)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
