"""Extracts the literal known answers of the reference's tests/color.test.ts into
reference_kats.json (run once, in a checkout that has the reference's sources):

    python tests/golden/extract_kats.py /path/to/MeerCADRaytracer

Each entry is one `expect(fn(args)).toBe(value)` or `.toBeCloseTo(value, digits)`
of a plain function call with numeric (or hex) arguments, for the functions the
oracle restates. The tests use the JSON only; they never read the reference.
"""
import json
import os
import re
import sys

FUNCS = {"halfToFloat": "half_to_float", "linearToSrgb": "linear_to_srgb", "fresnelWeight": "fresnel_weight",
         "smoothstep": "smoothstep", "distanceAttenuation": "distance_attenuation"}
NUM = r"-?(?:0x[0-9a-fA-F]+|\d+(?:\.\d+)?(?:e-?\d+)?)"
PATTERN = re.compile(r"expect\((\w+)\(((?:\s*" + NUM + r"\s*,?)+)\)\)\.(toBe|toBeCloseTo|toBeLessThan)\((" + NUM +
                     r")(?:,\s*(\d+))?\)")


def number(text: str) -> float:
    return float(int(text, 16)) if text.lower().startswith("0x") else float(text)


def main(root: str) -> None:
    path = os.path.join(root, "tests", "color.test.ts")
    with open(path) as f:
        source = f.read()
    out = []
    for m in PATTERN.finditer(source):
        fn, args, matcher, value, digits = m.groups()
        if fn not in FUNCS:
            continue
        line = source.count("\n", 0, m.start()) + 1
        out.append({"function": FUNCS[fn], "args": [number(a) for a in args.split(",") if a.strip()],
                    "matcher": matcher, "value": number(value), "digits": int(digits) if digits else None,
                    "source": f"tests/color.test.ts:{line}"})
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "reference_kats.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(f"{len(out)} known answers")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python extract_kats.py <reference checkout>")
    main(sys.argv[1])
