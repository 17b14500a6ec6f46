"""Parity at the headline sizes: the GPU solve against the float32 oracle (the CfdCPU restatement,
float32 storage and float64 arithmetic, src/air_cfd.js:157-259) on the bench's own inputs.

C2 - the fighter at ~4M cells (311 x 108 x 123 = 4,131,324 cells), M0.6, alpha 3, delta 3, the
engine field model's fixed states at sea level, full dry throttle (the bench case).  The same
number of iterations on both sides, the oracle on all host threads.  Tolerances are the parity
bar of the reference's own GPU/CPU check:
  * max|gpu - cpu| / max|cpu| per variable (tools/gpucmp.mjs:19-21) <= 3e-6 for all five;
  * per-cell relative difference <= 3e-6 for rho and E (the variables that never cross zero);
  * C_L and C_D agree to 4 significant digits.
The default 60 iterations keep the oracle near 10 s; A3D_C2_PARITY_ITERS=2000 runs the bench's
full solve (about 15 minutes of oracle time) with the same assertions.

C5 - the twin-engine airliner at ~120M cells with its under-wing nacelle's intake-sink, bypass
and core-jet cells (src/air_cfd.js:117-131) holding the 11 km cycle states, M0.78, alpha 2.5:
two iterations against the oracle, then forces and Trefftz drag from one state on both sides.
"""
import math
import os

import numpy as np
import pytest

from helpers import freestream, rel_max_diff

pytestmark = pytest.mark.gpu

TOL = 3e-6


def sig4(x):
    return float(f"{x:.4g}")


def cases(aero, ref, typ, cells, M, alpha, delta, h):
    ac = aero.build_aircraft(typ)
    sh = aero.shape_of(ac)
    F = freestream(M, alpha)
    fix = aero.fix_states(ac, h, M, alpha)[1]
    g = ref.grid(sh, cells)
    o = ref.CfdCPU(g, ref.geom(sh, g, delta), threads=ref.max_threads())
    s = aero.CfdGPU(aero.cfd_grid(sh, cells), shape=sh, delta=delta)
    for x in (o, s):
        x.setFree(F)
        x.setFix(fix)
        x.reset()
    return ac, g, o, s


def compare(Qg, Qo):
    errs = [rel_max_diff(Qg[c], Qo[c]) for c in range(5)]
    cell = [float(np.max(np.abs(Qg[c] - Qo[c]) / np.abs(Qo[c]))) for c in (0, 4)]
    return errs, cell


def test_c2_fighter_4m_matches_oracle(aero, ref):
    its = int(os.environ.get("A3D_C2_PARITY_ITERS", "60"))
    ac, g, o, s = cases(aero, ref, "fighter", 4.0e6, 0.6, 3.0, 3.0, 0.0)
    assert (g.NX, g.NY, g.NZ) == (311, 108, 123)
    assert s.kernel()[0] == 4  # the default stage kernel, the one the bench times
    s.step(its)
    o.step(its)
    Qg, Qo = s.read_array(), o.read()
    errs, cell = compare(Qg, Qo)
    print(f"C2 {its} iterations: gpucmp {['%.2e' % e for e in errs]}, per cell rho/E {['%.2e' % c for c in cell]}")
    assert all(e <= TOL for e in errs), errs
    assert all(c <= TOL for c in cell), cell
    r = ac.ref
    fg = s.forces(3.0, 0.6, r["S"], r["xcg"], 0.0, r["c"])
    fo = o.forces(3.0, 0.6, r["S"], r["xcg"], 0.0, r["c"])
    assert sig4(fg["CL"]) == sig4(fo["CL"]) and sig4(fg["CD"]) == sig4(fo["CD"]), (fg, fo)
    s.dispose()


def test_c5_airliner_120m_spot_parity(aero, ref):
    ac, g, o, s = cases(aero, ref, "airliner", 1.2e8, 0.78, 2.5, 0.0, 11000.0)
    assert g.N > 1.1e8
    s.step(2)
    o.step(2)
    Qg, Qo = s.read_array(), o.read()
    errs, cell = compare(Qg, Qo)
    print(f"C5 2 iterations: gpucmp {['%.2e' % e for e in errs]}, per cell rho/E {['%.2e' % c for c in cell]}")
    assert all(e <= TOL for e in errs), errs
    assert all(c <= TOL for c in cell), cell
    # the nacelle's fixed-state cells (intake sink 3, bypass 4, core jet 5) hold their states
    geo = ref.geom(aero.shape_of(ac), g, 0.0)
    tt = np.asarray(geo.t)
    fix = aero.fix_states(ac, 11000.0, 0.78, 2.5)[1]
    for k in (3, 4, 5):
        m = tt == k
        assert m.sum() > 0, k
        for c in range(5):
            assert np.all(Qg[c][m] == np.float32(fix[k - 3][c])), (k, c)
    del tt, geo
    # forces and Trefftz drag from one state on both sides (FP64 reductions)
    s.write(Qo.astype(np.float32))
    del Qg
    r = ac.ref
    fg = s.forces(2.5, 0.78, r["S"], r["xcg"], 0.0, r["c"])
    fo = o.forces(2.5, 0.78, r["S"], r["xcg"], 0.0, r["c"])
    for k in ("CL", "CD", "Cm"):
        assert math.isclose(fg[k], fo[k], rel_tol=1e-9, abs_tol=1e-12), k
    xT = aero.trefftz_x(ac)
    assert math.isclose(s.trefftz(xT, 2.5, 0.78, r["S"]), o.trefftz(xT, 2.5, 0.78, r["S"]), rel_tol=1e-9)
    s.dispose()
