"""a3d_forces_noalloc: the force integral for callers that cannot allocate device memory.

Such a caller (for example an addon inside a host application that owns a fixed device pool)
already holds the state and the force list on the device; the entry point must give the same
C_L, C_D, C_m as the solver's own a3d_solver_forces, call after call, while using only the
library's static scratch.  This file is collected last so that a failure here comes after every
other test has run; it also passes on its own in a fresh process.
"""
import ctypes as C
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_forces_match_solver_forces_twice(aero):
    import torch
    L = importlib.import_module("3d_aero_lab_b200._lib")
    lib = L.lib()
    case = aero.Case(aircraft_type="fighter", cells=30000, M=0.6, alpha=3.0, delta=3.0, device=0)
    s = case.solver
    r = case.ac.ref
    dev = torch.device("cuda", 0)
    fl = s.force_list()
    d_fl = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in fl.items()}
    for rep in range(2):
        s.step(25)
        want = s.forces(case.alpha, case.M, r["S"], r["xcg"], r["zcg"], r["c"])
        H = s.read()
        d_state = [torch.from_numpy(H[k].copy()).to(dev) for k in ("r", "ru", "rv", "rw", "E")]
        torch.cuda.synchronize()
        out = np.zeros(3)
        rc = lib.a3d_forces_noalloc(*(C.c_void_p(t.data_ptr()) for t in d_state), len(fl["q"]),
                                    *(C.c_void_p(d_fl[k].data_ptr()) for k in ("q", "cx", "cz", "x", "z")),
                                    case.alpha, case.M, r["S"], r["xcg"], r["zcg"], r["c"], None, out)
        L.check(rc)
        for i, k in enumerate(("CL", "CD", "Cm")):
            assert abs(out[i] - want[k]) <= 1e-9 * abs(want[k]) + 1e-12, (rep, k, out[i], want[k])
    s.dispose()


def test_noalloc_rejects_lists_beyond_the_scratch_limit(aero):
    L = importlib.import_module("3d_aero_lab_b200._lib")
    lib = L.lib()
    out = np.zeros(3)
    p = C.c_void_p(1)
    rc = lib.a3d_forces_noalloc(p, p, p, p, p, 1048577, p, p, p, p, p, 3.0, 0.6, 1.0, 0.0, 0.0, 1.0, None, out)
    assert rc == 1 and b"static scratch limit" in lib.a3d_last_error()
