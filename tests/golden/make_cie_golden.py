"""Extract the reference's CIE 1931 2-degree colour-matching table as a fixture.

Reads src/Library/Utilities/Color/ColorUtils.cpp of the reference tree as
text (namespace CIE_DATA: x_2, y_2, z_2 at 5 nm from 380 to 780 nm) and
writes tests/golden/cie1931_5nm.json.  The product embeds the same standard
CIE data in rise_b200/csrc/spectral.h; tests check the two agree and that
the interpolation (XYZFromNM, ColorUtils.cpp:270-325) and the Y integral
(CIE_Y_Integral, ColorUtils.cpp:327-348) match the reference's.

Usage: python tests/golden/make_cie_golden.py [reference_root]
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    src = open(os.path.join(root, "src/Library/Utilities/Color/ColorUtils.cpp")).read()
    block = src[src.index("namespace CIE_DATA"):]
    out = {"min_nm": 380, "max_nm": 780, "step_nm": 5}
    for name in ("x_2", "y_2", "z_2"):
        body = block[block.index("spd_table " + name):]
        body = body[body.index("{") + 1:body.index("}")]
        vals = [float(v) for v in re.findall(r"[-+]?\d*\.\d+(?:[eE][-+]?\d+)?|\d+", body)]
        # The reference lists fewer than 81 values for z_2; C++ aggregate
        # initialisation zero-fills the rest of the array.
        assert 0 < len(vals) <= 81, (name, len(vals))
        out[name[0]] = vals + [0.0] * (81 - len(vals))
    with open(os.path.join(HERE, "cie1931_5nm.json"), "w") as f:
        json.dump(out, f)
    print("wrote 3 x 81 CIE values")


if __name__ == "__main__":
    main()
