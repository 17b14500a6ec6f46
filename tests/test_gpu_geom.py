"""GPU cut-cell geometry and force list vs the oracle, cell by cell (bit-exact)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [("fighter", 30000, 3.0), ("fighter", 250000, -4.0), ("interceptor", 60000, 5.0),
         ("airliner", 150000, 0.0), ("airliner", 500000, 2.5), ("fighter", 4.0e6, 3.0)]


@pytest.mark.parametrize("typ,cells,delta", CASES)
def test_geometry_matches_oracle(aero, ref, typ, cells, delta):
    sh = aero.shape_of(aero.build_aircraft(typ))
    g = aero.cfd_grid(sh, cells)
    geo = aero.cfd_geom(sh, g, delta)
    o = ref.geom(sh, ref.grid(sh, cells), delta)
    assert np.array_equal(geo.t, o.t), f"type mismatches: {np.count_nonzero(geo.t != o.t)}"
    assert np.array_equal(geo.phi, o.phi), f"phi mismatches: {np.count_nonzero(geo.phi != o.phi)}"
    for d in range(4):
        assert np.array_equal(geo.ap[d], o.ap[d]), f"ap{d} mismatches: {np.count_nonzero(geo.ap[d] != o.ap[d])}"
    assert (geo.nSolid, geo.nCut) == (o.nSolid, o.nCut)
    assert (geo.volW, geo.volH, geo.volV) == (o.volW, o.volH, o.volV)
    if typ == "airliner":
        assert {3, 4, 5} <= set(np.unique(geo.t).tolist())


@pytest.mark.parametrize("typ,cells,delta", CASES[:4])
def test_force_list_matches_oracle(aero, ref, typ, cells, delta):
    sh = aero.shape_of(aero.build_aircraft(typ))
    g = aero.cfd_grid(sh, cells)
    s = aero.CfdGPU(g, shape=sh, delta=delta)
    fl = s.force_list()
    og = ref.grid(sh, cells)
    ofl = ref.force_list(og, ref.geom(sh, og, delta))
    for k in ("q", "cx", "cz", "x", "z"):
        assert np.array_equal(fl[k], ofl[k]), k
    s.dispose()


def test_solver_from_host_arrays_equals_solver_from_shape(aero):
    sh = aero.shape_of(aero.build_aircraft("fighter"))
    g = aero.cfd_grid(sh, 20000)
    geo = aero.cfd_geom(sh, g, 3.0)
    a = aero.CfdGPU(g, geo)
    b = aero.CfdGPU(g, shape=sh, delta=3.0)
    F = aero.freestream(0.6, 3.0)
    for s in (a, b):
        s.setFree(F)
        s.setFix([F, F, F])
        s.reset()
        s.step(10)
    assert np.array_equal(a.read_array(), b.read_array())
