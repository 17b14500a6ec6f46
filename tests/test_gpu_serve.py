"""Continuous-batching server: results in the mix equal results alone; warm starts; budget."""
import importlib

import pytest

pytestmark = pytest.mark.gpu

REQS = [{"type": "fighter", "cells": 30000, "M": 0.6, "alpha": 3.0, "delta": 3.0},
        {"type": "interceptor", "cells": 45000, "M": 0.8, "alpha": 1.0, "delta": -2.0},
        {"type": "airliner", "cells": 60000, "M": 0.78, "alpha": 2.5, "delta": 0.0},
        {"type": "fighter", "cells": 25000, "M": 0.45, "alpha": 6.0, "delta": 4.0}]
KW = {"residual_drop": 0.1, "chunk": 25, "max_iters": 400}


@pytest.mark.parametrize("fix", ["free", "cycle"])
def test_results_in_the_mix_equal_results_alone(aero, fix):
    """fix="cycle": engine cells hold the engine field model's states (sea level, full throttle)."""
    serve = importlib.import_module("3d_aero_lab_b200.serve")
    reqs = [dict(r, fix=fix) for r in REQS]
    sv = serve.Server(max_active=8, chunk=KW["chunk"], max_iters=KW["max_iters"], residual_drop=KW["residual_drop"],
                      warm_start=False)
    ids = [sv.submit(r) for r in reqs]           # all arrive together and overlap on the GPU
    mixed = [sv.wait(i, 600) for i in ids]
    st = sv.stats()
    sv.close()
    assert st["completed"] == len(reqs) and st["rounds"] < sum(m["iterations"] for m in mixed) / KW["chunk"]
    for r, m in zip(reqs, mixed):
        alone = serve.solve_plain(r, kernel=serve.SERVED_KERNEL, kz=16, chunks=1, **KW)  # the served configuration
        assert m["status"] == 0 and m["iterations"] == alone["iterations"]
        for k in ("CL", "CD", "Cm", "CDi"):
            assert abs(m[k] - alone[k]) <= 1e-12 * max(1.0, abs(alone[k])), (r, k, m[k], alone[k])


def test_warm_start_reuses_the_resident_case(aero):
    serve = importlib.import_module("3d_aero_lab_b200.serve")
    sv = serve.Server(max_active=4, chunk=KW["chunk"], max_iters=KW["max_iters"], residual_drop=KW["residual_drop"])
    a = sv.wait(sv.submit(REQS[0]), 600)
    b = sv.wait(sv.submit(REQS[0]), 600)  # same geometry and conditions: starts converged
    st = sv.stats()
    sv.close()
    assert a["warm"] == 0 and b["warm"] == 1 and st["warm_starts"] == 1
    assert b["res0"] == a["res0"] and b["iterations"] < a["iterations"]
    assert abs(b["CL"] - a["CL"]) < 1e-3


def test_request_beyond_the_budget_is_refused(aero):
    serve = importlib.import_module("3d_aero_lab_b200.serve")
    L = importlib.import_module("3d_aero_lab_b200._lib")
    sv = serve.Server(budget_gb=0.5, max_active=2)
    with pytest.raises(L.AeroError) as e:
        sv.submit(dict(REQS[0], cells=2.0e7))
    assert e.value.status == 6
    sv.close()


def test_grid_sequencing_matches_cold_solves(aero):
    """Sequenced requests (coarse case at cells/8 first, then interpState onto the requested grid)
    converge to the cold solution in fewer iterations on the requested grid, with the same res0."""
    serve = importlib.import_module("3d_aero_lab_b200.serve")
    kw = dict(max_active=8, chunk=50, max_iters=3000, residual_drop=1e-2, warm_start=False)
    runs = {}
    for seq in (0, 8):
        sv = serve.Server(sequence=seq, sequence_drop=0.05, sequence_max_iters=1500, **kw)
        runs[seq] = [sv.wait(sv.submit(r), 600) for r in REQS]
        sv.close()
    for cold, seq in zip(runs[0], runs[8]):
        assert cold["status"] == 0 and seq["status"] == 0
        assert cold["coarse_iterations"] == 0 and seq["coarse_iterations"] > 0
        assert seq["res0"] == cold["res0"]  # the requested case's own free-stream res0, bit for bit
        for k in ("CL", "CD"):
            assert abs(seq[k] - cold[k]) < 1e-3, (k, seq[k], cold[k])
    assert sum(s["iterations"] for s in runs[8]) < sum(c["iterations"] for c in runs[0])


def test_app_controller_loop(aero):
    """The app's loop (CFD3.tick/readback) on a small case: readbacks every 100 iterations until
    its convergence rule holds or 3000 iterations have run."""
    ctl = importlib.import_module("3d_aero_lab_b200.controller")
    case = aero.Case(aircraft_type="fighter", cells=30000, M=0.6, alpha=3.0, delta=3.0)
    c = ctl.Controller(case, check_every=100)
    rec = c.run(max_iters=3000)
    assert rec is not None and len(c.hist) == case.solver.it // 100
    assert c.res0 and c.res0 > 0 and all(h["res"] is None or h["res"] > 0 for h in c.hist)
    assert 0 < rec["Mmax"] < 3 and rec["CDi"] >= 0
    if c.conv:
        assert c.res / c.res0 < 2e-3
    f = case.forces()
    assert f["CL"] == rec["CL"]
    case.solver.dispose()
