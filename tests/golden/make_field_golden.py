"""Writes tests/golden/field_fix_states.json: the engine field model's fixed states.

The reference publishes no field-model samples and cannot run here (no JavaScript runtime);
test_field.py checks the cycle against README.md:73-75 and :97 and the samples by properties.
This file records fix_states() for the three aircraft at two conditions with and without the
afterburner, so later changes to field.py or engine.py are caught.
Run: python tests/golden/make_field_golden.py
"""
import importlib
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
aero = importlib.import_module("3d_aero_lab_b200")
field = importlib.import_module("3d_aero_lab_b200.field")

CASES = [(t, h, M, a, thr, ab) for t in ("airliner", "interceptor", "fighter")
         for (h, M, a) in ((0.0, 0.6, 3.0), (11000.0, 0.78, 2.5)) for thr in (1.0, 0.8) for ab in (False, True)]


def states():
    out = []
    for t, h, M, a, thr, ab in CASES:
        ac = aero.build_aircraft(t)
        F, fx = field.fix_states(ac, h, M, a, thr, ab)
        out.append({"type": t, "h": h, "M": M, "alpha": a, "thr": thr, "ab": ab, "F": F, "fix": fx})
    return out


if __name__ == "__main__":
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "field_fix_states.json")
    json.dump({"source": "3d_aero_lab_b200/field.py fix_states (src/air_cfd.js:526-533)", "cases": states()},
              open(path, "w"), indent=1)
    print("wrote", path)
