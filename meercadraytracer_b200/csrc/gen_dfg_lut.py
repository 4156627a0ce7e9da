"""Writes dfg_lut.h: three.js r187's DFG lookup table as 16-bit half floats.

The table is data, not code: 16 x 16 texels of (scale, bias) that three.js
precomputed for its split-sum specular (src/renderers/shaders/DFGLUTData.js,
MIT licence, Copyright 2010-2025 three.js authors). The reference vendors the
same values (src/dfgData.ts:4-39); shading only matches three.js, and the
reference, if the numbers are identical, so they are read from there.

Usage: python gen_dfg_lut.py [path/to/dfgData.ts]
"""
import os
import re
import sys

DEFAULT = "/root/reference/src/dfgData.ts"


def main() -> None:
    source = sys.argv[1] if len(sys.argv) > 1 else DEFAULT
    text = open(source).read()
    body = text[text.index("Uint16Array(["):]
    values = [int(v, 16) for v in re.findall(r"0x([0-9a-fA-F]{4})", body)]
    if len(values) != 16 * 16 * 2:
        raise SystemExit(f"expected 512 halves, found {len(values)}")
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "dfg_lut.h")
    lines = [
        "/* Generated by gen_dfg_lut.py. three.js r187 DFG lookup table",
        " * (src/renderers/shaders/DFGLUTData.js), MIT licence, Copyright 2010-2025",
        " * three.js authors: 16 x 16 texels of (scale, bias) as IEEE half floats,",
        " * roughness along each row and dot(N, V) down the rows. */",
        "#ifndef MCRT_DFG_LUT_H",
        "#define MCRT_DFG_LUT_H",
        "#define MCRT_DFG_LUT_SIZE 16",
        "static const unsigned short MCRT_DFG_LUT_HALF[512] = {",
    ]
    for row in range(0, 512, 16):
        lines.append("  " + ", ".join(f"0x{v:04x}" for v in values[row:row + 16]) + ",")
    lines += ["};", "#endif", ""]
    with open(out, "w") as f:
        f.write("\n".join(lines))
    print(f"wrote {out}")


if __name__ == "__main__":
    main()
