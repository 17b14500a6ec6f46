"""Batched persistent-kernel runs: every case bit-identical to the same case stepped alone."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [("fighter", 30000, 0.6, 3.0, 3.0), ("interceptor", 50000, 0.85, 2.0, -2.0),
         ("airliner", 80000, 0.78, 2.5, 0.0), ("fighter", 20000, 0.4, 6.0, 5.0)]


def make(aero, typ, cells, M, alpha, delta):
    c = aero.Case(aircraft_type=typ, cells=cells, M=M, alpha=alpha, delta=delta)
    c.solver.set_kernel(3, 32)
    return c


@pytest.mark.parametrize("n", [21, 8])
def test_batch_equals_individual_steps(aero, n):
    alone = [make(aero, *c) for c in CASES]
    batched = [make(aero, *c) for c in CASES]
    for k, c in enumerate(alone):  # alone with other tile depths: the result must not depend on tiling
        c.solver.set_kernel(3, (32, 64, 8, 16)[k])
        c.solver.step(n)
    b = aero.Batch([c.solver for c in batched])
    b.set_schedule(16, 2)
    b.step(n)
    b.sync()
    for a, c in zip(alone, batched):
        assert c.solver.it == a.solver.it == n
        assert np.array_equal(c.solver.read_array(), a.solver.read_array())
        fa, fc = a.forces(), c.forces()
        assert fa["CL"] == fc["CL"] and fa["CD"] == fc["CD"]
    # after the batch each solver still steps on its own (roles carried over)
    for a, c in zip(alone, batched):
        a.solver.step(3)
        c.solver.step(3)
        assert np.array_equal(c.solver.read_array(), a.solver.read_array())
    b.dispose()


def test_tuner_restores_state_and_picks_a_schedule(aero):
    cases = [make(aero, *c) for c in CASES]
    for c in cases:
        c.solver.step(5)
    before = [c.solver.read_array() for c in cases]
    b = aero.Batch([c.solver for c in cases])
    best = b.tune(4)
    assert best["kz"] in (8, 16, 32, 64) and best["ctas_per_sm"] in (1, 2) and best["ms_per_iteration"] > 0
    assert b.schedule()["kz"] == best["kz"]
    for c, q in zip(cases, before):
        assert c.solver.it == 5
        assert np.array_equal(c.solver.read_array(), q)
    b.step(2)
    b.sync()
    b.dispose()
