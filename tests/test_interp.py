"""Grid sequencing, interpState (src/app_cfd.js:322-357) in 3-D.

CPU: known answers of the oracle restatement - identity on the same grid, exact reproduction
of a field linear in the cell centres where every corner is fluid, the nearest-fluid and
free-stream fallbacks.  GPU: the device interpolation is bit-identical to the oracle's on the
same coarse state (FP64 weights and sums in the same order on both sides), for a random box
and for an aircraft case coarse -> fine.
"""
import numpy as np
import pytest

from helpers import BoxGrid, box_geometry, freestream, oracle_case


def _box(ref, bg, t, F):
    geo = ref.Geom()
    N = bg.N
    geo.t = t
    geo.phi = np.ones(N, np.float32)
    geo.ap = [np.ones(N, np.float32) for _ in range(3)] + [np.zeros(N, np.float32)]
    s = ref.CfdCPU(bg, geo, prec=64)
    s.setFree(F)
    s.reset()
    return s


class _Faces:
    def __init__(self, xf, yf, zf):
        self.xf, self.yf, self.zf = (np.asarray(v, np.float64) for v in (xf, yf, zf))
        self.dims = np.array([len(self.xf) - 1, len(self.yf) - 1, len(self.zf) - 1], np.int32)
        self.NX, self.NY, self.NZ = (int(v) for v in self.dims)
        self.N = self.NX * self.NY * self.NZ
        self.h = 1.0


def _centres(f):
    return (0.5 * (f[:-1] + f[1:])).astype(np.float32).astype(np.float64)


def _refine(f):
    m = 0.5 * (f[:-1] + f[1:])
    out = np.empty(2 * len(f) - 1)
    out[0::2], out[1::2] = f, m
    return out


F0 = freestream(0.6, 3.0)


def test_identity_on_same_grid(ref):
    rng = np.random.default_rng(0)
    bg = BoxGrid(rng, 9, 7, 6)
    t = np.where(rng.random(bg.N) < 0.1, 1, 0).astype(np.uint8)
    a, b = _box(ref, bg, t, F0), _box(ref, bg, t, F0)
    Q = rng.uniform(0.5, 2.0, (5, bg.N))
    a.write(Q)
    ref.interp_state(a, b)
    Qb = b.read()
    fl = t == 0
    assert np.array_equal(Qb[:, fl], Q[:, fl])
    assert np.array_equal(Qb[:, ~fl], np.repeat(np.array(F0)[:, None], (~fl).sum(), 1))
    assert b.it == 0


def test_linear_field_reproduced(ref):
    rng = np.random.default_rng(1)
    bg = BoxGrid(rng, 10, 8, 7)
    fine = _Faces(_refine(bg.xf), _refine(bg.yf), _refine(bg.zf))
    a = _box(ref, bg, np.zeros(bg.N, np.uint8), F0)
    b = _box(ref, fine, np.zeros(fine.N, np.uint8), F0)
    xc, yc, zc = _centres(bg.xf), _centres(bg.yf), _centres(bg.zf)
    Z, Y, X = np.meshgrid(zc, yc, xc, indexing="ij")
    coef = rng.uniform(-1, 1, (5, 4))
    lin = lambda X, Y, Z: np.stack([c[0] + c[1] * X + c[2] * Y + c[3] * Z for c in coef]).reshape(5, -1)
    a.write(lin(X, Y, Z))
    ref.interp_state(a, b)
    fx, fy, fz = _centres(fine.xf), _centres(fine.yf), _centres(fine.zf)
    Zf, Yf, Xf = np.meshgrid(fz, fy, fx, indexing="ij")
    inside = ((Xf >= xc[0]) & (Xf <= xc[-1]) & (Yf >= yc[0]) & (Yf <= yc[-1]) & (Zf >= zc[0]) & (Zf <= zc[-1])).reshape(-1)
    want = lin(Xf, Yf, Zf)
    got = b.read()
    assert inside.sum() > 0.5 * fine.N
    assert np.max(np.abs(got[:, inside] - want[:, inside])) < 1e-12 * (1 + np.max(np.abs(want)))


def test_fallbacks(ref):
    """All eight corners solid -> nearest fluid within +-3; none within reach -> free stream."""
    rng = np.random.default_rng(2)
    bg = BoxGrid(rng, 12, 4, 4)
    t = np.ones(bg.N, np.uint8)
    t[11] = 0  # one fluid cell at (11, 0, 0)
    a = _box(ref, bg, t, F0)
    Q = rng.uniform(0.5, 2.0, (5, bg.N))
    a.write(Q)
    b = _box(ref, bg, np.zeros(bg.N, np.uint8), F0)
    ref.interp_state(a, b)
    Qb = b.read()
    i = np.arange(bg.N) % 12
    near = i >= 8
    assert np.array_equal(Qb[:, near], np.repeat(Q[:, 11:12], near.sum(), 1))
    assert np.array_equal(Qb[:, ~near], np.repeat(np.array(F0)[:, None], (~near).sum(), 1))


@pytest.mark.gpu
def test_gpu_interp_random_box_bitwise(aero, ref):
    rng = np.random.default_rng(5)
    bgA = BoxGrid(rng, 13, 9, 11)
    fine = _Faces(_refine(bgA.xf)[1:-2], _refine(bgA.yf), np.concatenate([[-1.0], _refine(bgA.zf), [bgA.zf[-1] + 3]]))
    tA, phiA, apA = box_geometry(rng, 13, 9, 11)
    tB, phiB, apB = box_geometry(rng, fine.NX, fine.NY, fine.NZ)
    sides = []
    for g_, t_, phi_, ap_ in ((bgA, tA, phiA, apA), (fine, tB, phiB, apB)):
        geo = ref.Geom()
        geo.t, geo.phi, geo.ap = t_, phi_, ap_
        o = ref.CfdCPU(g_, geo)
        hg = aero.cfd.Geom(g_.N)
        hg.t, hg.phi, hg.ap = t_, phi_, ap_
        s = aero.CfdGPU(aero.cfd.Grid(g_.xf, g_.yf, g_.zf), hg)
        for x in (o, s):
            x.setFree(F0)
            x.reset()
        sides.append((o, s))
    (oA, sA), (oB, sB) = sides
    Q = rng.uniform(0.5, 2.0, (5, bgA.N)).astype(np.float32)
    oA.write(Q.astype(np.float64))
    sA.write(Q)
    ref.interp_state(oA, oB)
    aero.cfd.interp_state(sA, sB)
    assert sB.it == 0
    assert np.array_equal(sB.read_array(), oB.read().astype(np.float32))


@pytest.mark.gpu
def test_gpu_interp_aircraft_coarse_to_fine_bitwise(aero, ref):
    ac, sh, ogA, _, oA = oracle_case(aero, ref, "fighter", 8000, 3.0)
    ogB = ref.grid(sh, 60000)
    oB = ref.CfdCPU(ogB, ref.geom(sh, ogB, 3.0))
    oB.setFree(F0)
    oB.reset()
    sA = aero.CfdGPU(aero.cfd_grid(sh, 8000), shape=sh, delta=3.0)
    sB = aero.CfdGPU(aero.cfd_grid(sh, 60000), shape=sh, delta=3.0)
    for s in (sA, sB):
        s.setFree(F0)
        s.setFix([F0, F0, F0])
        s.reset()
    sA.step(60)
    QA = sA.read_array()
    oA.write(QA.astype(np.float64))
    ref.interp_state(oA, oB)
    sB.interp_from(sA)
    QB = sB.read_array()
    assert np.array_equal(QB, oB.read().astype(np.float32))
    # the interpolated start is a flow state on the fine grid: positive density, finite
    assert np.all(np.isfinite(QB)) and QB[0].min() > 0
