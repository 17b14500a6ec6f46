"""Writes tests/golden/oracle_fighter30k.json: the oracle's force history on the README case.

The reference cannot run here (no JavaScript runtime); its only published numbers are the
README.md:98 C_L/C_D, which test_oracle.py checks directly.  This file records the oracle's
grid size, cell counts and force history so later changes to the oracle are caught.
Run: python tests/golden/make_golden.py
"""
import importlib
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]
aero = importlib.import_module("3d_aero_lab_b200")
import ref  # noqa: E402
from helpers import oracle_case  # noqa: E402

ac, sh, g, geo, s = oracle_case(aero, ref, "fighter", 30000, 3.0)
hist = []
for it in (50, 100, 150, 200):
    s.step(it - s.it)
    f = s.forces(3.0, 0.6, ac.ref["S"], ac.ref["xcg"], 0.0, ac.ref["c"])
    hist.append({"it": it, "CL": f["CL"], "CD": f["CD"], "Cm": f["Cm"]})
out = {"case": "fighter, 30000 cells, M0.6, alpha 3, delta 3, fixed = free stream (tools/test_cfd3.js:4-12)",
       "cells": 30000, "delta": 3.0, "dims": [g.NX, g.NY, g.NZ], "nSolid": geo.nSolid, "nCut": geo.nCut,
       "readme": {"CL": 0.1927, "CD": 0.04406, "source": "README.md:98"}, "history": hist}
json.dump(out, open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle_fighter30k.json"), "w"), indent=1)
print(json.dumps(out, indent=1))
