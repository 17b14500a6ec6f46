"""Host side of the batched and served workloads: the seeded case list (type, cells, M, alpha,
delta drawn uniformly over the three aircraft, 20k-2M cells, M 0.3-0.85, alpha -2..8,
delta -5..5), the geometry pool behind warm starts, the fixed states of a request and the
Poisson arrival times."""
import importlib
import math

import numpy as np

serve = importlib.import_module("3d_aero_lab_b200.serve")


def test_case_list_is_seeded_and_within_the_distribution():
    a, b = serve.requests(1, 64), serve.requests(1, 64)
    assert a == b and serve.requests(2, 64) != a
    assert {r["type"] for r in a} == {"airliner", "interceptor", "fighter"}
    for r in a:
        assert 20e3 <= r["cells"] <= 2.0e6
        assert 0.3 <= r["M"] <= 0.85 and -2.0 <= r["alpha"] <= 8.0 and -5.0 <= r["delta"] <= 5.0
        assert r["fix"] == "free"
    cells = np.array([r["cells"] for r in a])
    assert 0.7e6 < cells.mean() < 1.3e6  # uniform over 20k-2M: mean about 1M


def test_geometry_pool_limits_distinct_geometries():
    reqs = serve.requests(7, 32, geometries=10)
    geo = {(r["type"], r["cells"], r["delta"]) for r in reqs}
    assert 1 < len(geo) <= 10
    # conditions still vary per request
    assert len({(r["M"], r["alpha"]) for r in reqs}) == 32


def test_cycle_fix_draws_the_same_cases():
    free, cyc = serve.requests(3, 16), serve.requests(3, 16, fix="cycle")
    for f, c in zip(free, cyc):
        assert {k: v for k, v in f.items() if k != "fix"} == {k: v for k, v in c.items() if k != "fix"}
        assert c["fix"] == "cycle"


def test_request_fix_states():
    aero = importlib.import_module("3d_aero_lab_b200")
    ac = aero.build_aircraft("airliner")
    r = {"type": "airliner", "cells": 30000, "M": 0.78, "alpha": 2.5, "delta": 0.0, "fix": "free"}
    F = aero.cfd.freestream(r["M"], r["alpha"])
    assert serve.request_fix(r, ac, F) == [F, F, F]
    fx = serve.request_fix(dict(r, fix="cycle", h=11000.0), ac, F)
    assert len(fx) == 3 and all(len(U) == 5 and all(math.isfinite(v) for v in U) for U in fx)
    assert fx == list(aero.fix_states(ac, 11000.0, 0.78, 2.5)[1])
    assert all(list(U) != list(F) for U in fx)  # intake sink, bypass and core jet all sample a stream


def test_poisson_arrivals():
    t = serve.arrivals(7, 4000, 20.0)
    assert np.all(np.diff(t) > 0) and np.array_equal(t, serve.arrivals(7, 4000, 20.0))
    gaps = np.diff(np.concatenate([[0.0], t]))
    assert abs(gaps.mean() - 1 / 20.0) < 0.1 / 20.0   # mean gap 1/rate
    assert abs(gaps.std() / gaps.mean() - 1) < 0.1    # exponential: coefficient of variation 1
