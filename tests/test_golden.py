"""The oracle against the reference's literal known answers (tests/golden/reference_kats.json,
extracted from the reference's tests/color.test.ts by tests/golden/extract_kats.py), with the
reference's own matchers: toBe is exact, toBeCloseTo(v, d) is |x - v| < 10^-d / 2, toBeLessThan
is x < v."""
import json
import os

import pytest

from oracle import cpu

HERE = os.path.dirname(os.path.abspath(__file__))
KATS = json.load(open(os.path.join(HERE, "golden", "reference_kats.json")))


def test_every_helper_of_the_reference_has_known_answers():
    assert {k["function"] for k in KATS} >= {"half_to_float", "linear_to_srgb", "fresnel_weight", "smoothstep",
                                             "distance_attenuation"}


@pytest.mark.parametrize("kat", KATS, ids=[f"{k['function']}{tuple(k['args'])}@{k['source']}" for k in KATS])
def test_oracle_meets_reference_known_answer(kat):
    fn = getattr(cpu, kat["function"])
    args = [int(a) if kat["function"] == "half_to_float" else a for a in kat["args"]]
    x = fn(*args)
    if kat["matcher"] == "toBe":
        assert x == kat["value"]
    elif kat["matcher"] == "toBeCloseTo":
        digits = kat["digits"] if kat["digits"] is not None else 2
        assert abs(x - kat["value"]) < 10 ** (-digits) / 2
    else:
        assert x < kat["value"]
