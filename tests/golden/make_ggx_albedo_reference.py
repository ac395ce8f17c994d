"""Extracts the reference's embedded GGX directional-albedo tables (GGX_E_LUT,
GGX_EAVG_LUT in pt-webgpu/src/wgsl/pathTrace/material.wgsl.ts:2852-2869) as
text into ggx_albedo_reference.json, the fixture the generated
vitrum_b200/csrc/ggx_albedo_lut.h is checked against.

    python tests/golden/make_ggx_albedo_reference.py <reference checkout root>
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_ggx_albedo_reference.py <reference checkout root>")
    root = sys.argv[1]
    src = open(os.path.join(root, "packages/pt-webgpu/src/wgsl/pathTrace/material.wgsl.ts")).read()

    def grab(name):
        m = re.search(name + r"\s*=\s*array<f32,\s*(\d+)>\(([^)]*)\)", src)
        vals = [float(v) for v in re.findall(r"[-+]?\d*\.?\d+(?:[eE][-+]?\d+)?", m.group(2))]
        assert len(vals) == int(m.group(1)), name
        return vals

    out = {"source": "pt-webgpu/src/wgsl/pathTrace/material.wgsl.ts:2852-2869",
           "e_ss": grab("GGX_E_LUT"), "e_avg": grab("GGX_EAVG_LUT")}
    with open(os.path.join(HERE, "ggx_albedo_reference.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
