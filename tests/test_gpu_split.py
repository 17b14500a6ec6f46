"""One case on z slabs (split.py) against the same case unsplit, on one GPU.

With the halo planes exchanged after each stage, a slab's own planes see the numbers of the
unsplit solve.  The per-cell kernel and the z-marching TMA tiles (single-cell and paired) with
slab boundaries aligned to their z runs give the same state bit for bit.  Unaligned, a tile
differs only where a z run starts elsewhere, within the 4e-6 of its prologue rounding.  The FP64 reductions sum
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


@pytest.mark.parametrize("push", [True, False])
@pytest.mark.parametrize("kernel,slabs,align,exact", [(0, 2, 1, True), (0, 3, 1, True), (2, 3, 16, True),
                                                      (2, 2, 1, False), (4, 3, 16, True), (4, 2, 1, False)])
def test_slabs_reproduce_the_unsplit_solve(aero, kernel, slabs, align, exact, push):
    """push: stage kernels store the neighbours' halo planes into their buffers; otherwise the
    halos are copied between the stages."""
    split = importlib_split()
    typ, cells, M, alpha, delta = "fighter", 400000, 0.6, 3.0, 3.0
    full = full_case(aero, typ, cells, M, alpha, delta, kernel, "cycle")
    sc = split.SplitCase(typ, cells, M, alpha, delta, slabs=slabs, kernel=kernel, kz=16, align=align, fixed="cycle",
                         push=push)
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


def test_pushing_slabs_refuse_unordered_use(aero):
    split = importlib_split()
    sc = split.SplitCase("fighter", 60000, 0.6, 3.0, 0.0, slabs=2, kernel=2)
    s0, s1 = sc.slabs
    with pytest.raises(aero.AeroError):
        s0.step(1)                                  # a pushing slab advances by stages only
    s0.stage(1)
    with pytest.raises(aero.AeroError):
        s0.stage(1)                                 # stage 1 twice
    with pytest.raises(aero.AeroError):
        s1.stage(2)                                 # stage 2 before its stage 1
    s1.stage(1)
    s0.sync_neighbors()
    s1.sync_neighbors()
    s0.stage(2)
    s1.stage(2)
    with pytest.raises(aero.AeroError):
        aero.Batch([s0, s1])                        # slab solvers are not batched
    with pytest.raises(aero.AeroError):
        s0.set_kernel(1, 16)                        # retired stage kernel numbers are refused
    sc.dispose()


def importlib_split():
    import importlib
    return importlib.import_module("3d_aero_lab_b200.split")
