"""One case on z slabs (split.py) against the same case unsplit, on one GPU.

With the halo planes exchanged after each stage, a slab's own planes see the numbers of the
unsplit solve.  The per-cell kernel and the z-marching TMA tile with slab boundaries aligned
to its z runs give the same state bit for bit.  Unaligned, the TMA tile differs only where a
z run starts elsewhere, within the 4e-6 of its prologue rounding.  The FP64 reductions sum
the same terms in another order.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def full_case(aero, typ, cells, M, alpha, delta, kernel, fixed):
    c = aero.Case(aircraft_type=typ, cells=cells, M=M, alpha=alpha, delta=delta, kernel=kernel, fixed=fixed)
    c.solver.set_kernel(kernel, 16)
    return c


@pytest.mark.parametrize("kernel,slabs,align,exact", [(0, 2, 1, True), (0, 3, 1, True), (2, 3, 16, True),
                                                      (2, 2, 1, False)])
def test_slabs_reproduce_the_unsplit_solve(aero, kernel, slabs, align, exact):
    split = importlib_split()
    typ, cells, M, alpha, delta = "fighter", 400000, 0.6, 3.0, 3.0
    full = full_case(aero, typ, cells, M, alpha, delta, kernel, "cycle")
    sc = split.SplitCase(typ, cells, M, alpha, delta, slabs=slabs, kernel=kernel, kz=16, align=align, fixed="cycle")
    assert len(sc.slabs) == slabs and sc.g.N == full.g.N
    assert full.solver.residual(1) is None and sc.residual(1) is None
    full.solver.step(30)
    sc.step(30)
    A, B = full.solver.read_array(), sc.read_array()
    if exact:
        assert np.array_equal(A, B)
    else:
        for c in range(5):
            d = np.abs(A[c] - B[c]) / np.maximum(np.abs(A[c]), 1e-3)
            assert float(d.max()) < 4e-6, c
    ff, fs = full.forces(), sc.forces()
    for k in ("CL", "CD", "Cm"):
        assert math.isclose(fs[k], ff[k], rel_tol=1e-9 if exact else 1e-5, abs_tol=1e-12), k
    assert math.isclose(sc.trefftz(), full.trefftz(), rel_tol=1e-9 if exact else 1e-5)
    assert math.isclose(sc.residual(1), full.solver.residual(1), rel_tol=1e-9 if exact else 1e-4)
    assert math.isclose(sc.mach_max(1), full.solver.mach_max(1), rel_tol=1e-12 if exact else 1e-5)
    sc.dispose()


def importlib_split():
    import importlib
    return importlib.import_module("3d_aero_lab_b200.split")
