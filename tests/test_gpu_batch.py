"""Batched persistent-kernel runs: every case bit-identical to the same case stepped alone, for
both batch tiles (kernel 2: the TMA tile, kernel 4: the paired-cell tile).  The tiles form the
first z face of a run in their prologue, where the compiler may round one operation
differently, so a case is bit-identical at equal run length and agrees to float32 rounding
across run lengths."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [("fighter", 30000, 0.6, 3.0, 3.0), ("interceptor", 50000, 0.85, 2.0, -2.0),
         ("airliner", 80000, 0.78, 2.5, 0.0), ("fighter", 20000, 0.4, 6.0, 5.0)]


def make(aero, kernel, typ, cells, M, alpha, delta):
    c = aero.Case(aircraft_type=typ, cells=cells, M=M, alpha=alpha, delta=delta)
    c.solver.set_kernel(kernel, 16)
    return c


@pytest.mark.parametrize("kernel", [2, 4])
@pytest.mark.parametrize("n", [21, 8])
def test_batch_equals_individual_steps(aero, n, kernel):
    alone = [make(aero, kernel, *c) for c in CASES]
    batched = [make(aero, kernel, *c) for c in CASES]
    for c in alone:
        c.solver.step(n)
    b = aero.Batch([c.solver for c in batched])
    b.set_mode(0)  # the persistent kernel
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
    # and the batch again after the solvers moved on alone (it rebuilds its case table)
    b.step(2)
    b.sync()
    for a in alone:
        a.solver.step(2)
    for a, c in zip(alone, batched):
        assert np.array_equal(c.solver.read_array(), a.solver.read_array())
    b.dispose()


@pytest.mark.parametrize("n", [21, 8])
def test_stream_mode_equals_individual_steps(aero, n):
    """Mode 1 (each case's own launches, concurrent in one graph): bit-identical to each case
    stepped alone with the same stage kernel and z run, odd step counts included."""
    alone = [make(aero, 2, *c) for c in CASES]
    batched = [make(aero, 2, *c) for c in CASES]
    for k in range(len(CASES)):
        for c in (alone[k], batched[k]):
            c.solver.set_kernel(2, (32, 64, 8, 16)[k])
    for c in alone:
        c.solver.step(n)
    b = aero.Batch([c.solver for c in batched])
    b.set_mode(1)
    b.step(n)
    b.sync()
    for a, c in zip(alone, batched):
        assert c.solver.it == a.solver.it == n
        assert np.array_equal(c.solver.read_array(), a.solver.read_array())
    for a, c in zip(alone, batched):  # roles carried over: both go on alike
        a.solver.step(3)
        c.solver.step(3)
        assert np.array_equal(c.solver.read_array(), a.solver.read_array())
    b.step(2)  # the batch again after the solvers moved on alone
    b.sync()
    for a in alone:
        a.solver.step(2)
    for a, c in zip(alone, batched):
        assert np.array_equal(c.solver.read_array(), a.solver.read_array())
    b.dispose()


def test_tma_tile_z_run_changes_only_rounding(aero):
    """The TMA tile with z runs of 8 and 64 planes: the same solution to float32 rounding."""
    a, b = make(aero, 2, *CASES[1]), make(aero, 2, *CASES[1])
    a.solver.set_kernel(2, 8)
    b.solver.set_kernel(2, 64)
    a.solver.step(60)
    b.solver.step(60)
    qa, qb = a.solver.read_array().astype(np.float64), b.solver.read_array().astype(np.float64)
    for c in range(5):
        assert np.max(np.abs(qa[c] - qb[c])) <= 4e-6 * np.max(np.abs(qb[c])), c
    assert abs(a.forces()["CL"] - b.forces()["CL"]) < 1e-5


@pytest.mark.parametrize("kernel", [2, 4])
def test_tuner_restores_state_and_picks_a_schedule(aero, kernel):
    cases = [make(aero, kernel, *c) for c in CASES]
    for c in cases:
        c.solver.step(5)
    before = [c.solver.read_array() for c in cases]
    b = aero.Batch([c.solver for c in cases])
    best = b.tune(4)
    assert best["mode"] in (0, 1) and best["kz"] in (8, 16, 32, 64) and best["ctas_per_sm"] in ((1, 2, 3) if kernel == 2 else (1, 2)) and best["ms_per_iteration"] > 0
    assert b.schedule()["kz"] == best["kz"]
    for c, q in zip(cases, before):
        assert c.solver.it == 5
        assert np.array_equal(c.solver.read_array(), q)
    b.step(2)
    b.sync()
    b.dispose()


def test_stream_mode_captures_chunked_steps(aero):
    """Cases set to pipelined z chunks (their own streams and events): the batch graph runs
    their whole-case stage launches and the odd iteration runs as their own chunked step, and
    the result stays bit-identical to the cases stepped alone (chunked throughout)."""
    cases = [("fighter", 200000, 0.6, 3.0, 3.0), ("airliner", 150000, 0.78, 2.5, 0.0)]
    alone = [make(aero, 2, *c) for c in cases]
    batched = [make(aero, 2, *c) for c in cases]
    for k, c in enumerate(alone + batched):
        c.solver.set_kernel(2, 4)
        c.solver.set_chunks(3 + k % 2)
    assert all(c.solver.chunks() > 1 for c in alone + batched)
    for c in alone:
        c.solver.step(9)
    b = aero.Batch([c.solver for c in batched])
    b.set_mode(1)
    b.step(9)
    b.sync()
    for a, c in zip(alone, batched):
        assert np.array_equal(c.solver.read_array(), a.solver.read_array())
    b.dispose()
