"""ctypes wrapper of the CPU oracle (oracle/liboracle.so) - test infrastructure only.

Loaded by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg, nowhere else.
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_u8 = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_i32 = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64 = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")


def build():
    """Compile the oracle with its Makefile (g++ -fopenmp)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = C.CDLL(_LIB)
        L.ref_grid_build.argtypes = [C.c_void_p, C.c_double, C.c_int32, _dp, _dp, _dp, _i32, C.POINTER(C.c_double), _dp]
        L.ref_grid_build.restype = C.c_int
        L.ref_geom_build.argtypes = [C.c_void_p, _i32, _dp, _dp, _dp, C.c_double, C.c_double,
                                     _u8, _fp, _fp, _fp, _fp, _fp, _i64, _i32]
        L.ref_geom_build.restype = C.c_int
        L.ref_force_list.argtypes = [_i32, _dp, _dp, _dp, _u8, _fp, _fp, C.c_int64, _i64, _dp, _dp, _dp, _dp]
        L.ref_force_list.restype = C.c_int64
        L.ref_solver_new.argtypes = [C.c_int, _i32, _dp, _dp, _dp, _u8, _fp, _fp, _fp, _fp, _fp]
        L.ref_solver_new.restype = C.c_void_p
        for name, args in (("ref_solver_free", []), ("ref_solver_threads", [C.c_int]),
                           ("ref_solver_opt", [C.c_double, C.c_int]), ("ref_solver_set_free", [_dp]),
                           ("ref_solver_set_fix", [_dp]), ("ref_solver_reset", []), ("ref_solver_step", [C.c_int]),
                           ("ref_solver_read", [_dp]), ("ref_solver_write", [_dp]),
                           ("ref_solver_forces", [C.c_double] * 6 + [_dp])):
            f = getattr(L, name)
            f.argtypes = [C.c_void_p] + args
            f.restype = None
        L.ref_solver_iterations.argtypes = [C.c_void_p]
        L.ref_solver_iterations.restype = C.c_long
        L.ref_solver_trefftz.argtypes = [C.c_void_p] + [C.c_double] * 4
        L.ref_solver_trefftz.restype = C.c_double
        L.ref_solver_residual.argtypes = [C.c_void_p, C.c_int]
        L.ref_solver_residual.restype = C.c_double
        L.ref_solver_mach_max.argtypes = [C.c_void_p, C.c_int]
        L.ref_solver_mach_max.restype = C.c_double
        L.ref_max_threads.restype = C.c_int
        _lib = L
    return _lib


class Grid:
    """cfdGrid output: face coordinates (f64) plus the float32 centres/sizes the reference keeps."""

    def __init__(self, xf, yf, zf, h=1.0, core=None):
        self.xf, self.yf, self.zf, self.h, self.core = xf, yf, zf, h, core
        self.dims = np.array([len(xf) - 1, len(yf) - 1, len(zf) - 1], dtype=np.int32)
        self.NX, self.NY, self.NZ = (int(v) for v in self.dims)
        self.N = self.NX * self.NY * self.NZ
        mk = lambda f: ((0.5 * (f[:-1] + f[1:])).astype(np.float32), (f[1:] - f[:-1]).astype(np.float32))
        (self.xc, self.xd), (self.yc, self.yd), (self.zc, self.zd) = mk(xf), mk(yf), mk(zf)


def grid(shape, target_cells, cap=8192):
    L = lib()
    xf, yf, zf = (np.zeros(cap) for _ in range(3))
    dims = np.zeros(3, np.int32)
    h = C.c_double()
    core = np.zeros(5)
    rc = L.ref_grid_build(C.byref(shape), float(target_cells), cap, xf, yf, zf, dims, C.byref(h), core)
    assert rc == 0, rc
    return Grid(xf[:dims[0] + 1].copy(), yf[:dims[1] + 1].copy(), zf[:dims[2] + 1].copy(), h.value, core)


class Geom:
    pass


def geom(shape, g, delta_deg):
    L = lib()
    N = g.N
    o = Geom()
    o.t = np.zeros(N, np.uint8)
    o.phi = np.zeros(N, np.float32)
    o.ap = [np.zeros(N, np.float32) for _ in range(4)]
    counts = np.zeros(2, np.int64)
    vol = np.zeros(3, np.int32)
    rc = L.ref_geom_build(C.byref(shape), g.dims, g.xf, g.yf, g.zf, g.h, float(delta_deg), o.t, o.phi,
                          o.ap[0], o.ap[1], o.ap[2], o.ap[3], counts, vol)
    assert rc == 0, rc
    o.nSolid, o.nCut = int(counts[0]), int(counts[1])
    o.volW, o.volH, o.volV = (bool(v) for v in vol)
    return o


def force_list(g, geo):
    L = lib()
    n = L.ref_force_list(g.dims, g.xf, g.yf, g.zf, geo.t, geo.ap[0], geo.ap[2], 0,
                         np.zeros(1, np.int64), np.zeros(1), np.zeros(1), np.zeros(1), np.zeros(1))
    q = np.zeros(max(n, 1), np.int64)
    cx, cz, x, z = (np.zeros(max(n, 1)) for _ in range(4))
    L.ref_force_list(g.dims, g.xf, g.yf, g.zf, geo.t, geo.ap[0], geo.ap[2], n, q, cx, cz, x, z)
    return {"q": q[:n], "cx": cx[:n], "cz": cz[:n], "x": x[:n], "z": z[:n]}


class CfdCPU:
    """The oracle solver with the reference's CfdCPU surface (src/air_cfd.js:157-259).

    prec=32 stores the state in float32 (the reference), prec=64 in float64.
    """

    def __init__(self, g, geo, prec=32, threads=1):
        L = lib()
        self.g, self.geo, self._L = g, geo, L
        self._h = L.ref_solver_new(prec, g.dims, g.xf, g.yf, g.zf, geo.t, geo.phi, *geo.ap)
        L.ref_solver_threads(self._h, threads)

    def __del__(self):
        if getattr(self, "_h", None):
            self._L.ref_solver_free(self._h)
            self._h = None

    def set_opt(self, cfl=0.7, order=2):
        self._L.ref_solver_opt(self._h, cfl, order)

    def setFree(self, F):
        self._L.ref_solver_set_free(self._h, np.asarray(F, np.float64))

    def setFix(self, fx):
        self._L.ref_solver_set_fix(self._h, np.asarray(fx, np.float64).reshape(15))

    def reset(self):
        self._L.ref_solver_reset(self._h)

    def step(self, n):
        self._L.ref_solver_step(self._h, int(n))

    @property
    def it(self):
        return self._L.ref_solver_iterations(self._h)

    def read(self):
        out = np.zeros(5 * self.g.N)
        self._L.ref_solver_read(self._h, out)
        return out.reshape(5, self.g.N)

    def write(self, Q):
        self._L.ref_solver_write(self._h, np.ascontiguousarray(Q, np.float64).reshape(-1))

    def forces(self, alpha, M, S, xcg, zcg, cref):
        out = np.zeros(3)
        self._L.ref_solver_forces(self._h, alpha, M, S, xcg, zcg, cref, out)
        return {"CL": out[0], "CD": out[1], "Cm": out[2]}

    def trefftz(self, xT, alpha, M, S):
        return self._L.ref_solver_trefftz(self._h, xT, alpha, M, S)

    def residual(self, stride=3):
        return self._L.ref_solver_residual(self._h, stride)

    def mach_max(self, stride=2):
        return self._L.ref_solver_mach_max(self._h, stride)


def max_threads():
    return lib().ref_max_threads()


def hllc(L, R, d):
    """HLLC flux of the oracle (cfdHLLC) for primitive states L, R along direction d."""
    lb = lib()
    lb.ref_hllc.argtypes = [_dp, _dp, C.c_int, _dp]
    lb.ref_hllc.restype = None
    out = np.zeros(5)
    lb.ref_hllc(np.asarray(L, np.float64), np.asarray(R, np.float64), int(d), out)
    return out


def prim(U):
    lb = lib()
    lb.ref_prim.argtypes = [_dp, _dp]
    lb.ref_prim.restype = None
    out = np.zeros(5)
    lb.ref_prim(np.asarray(U, np.float64), out)
    return out


def sample(solver, xyz):
    """cfdStencil + cfdSample of the oracle at points xyz (n x 3): (n x 5 primitives, ok flags)."""
    lb = lib()
    lb.ref_solver_sample.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _i32]
    lb.ref_solver_sample.restype = None
    xyz = np.ascontiguousarray(xyz, np.float64).reshape(-1, 3)
    out = np.zeros((len(xyz), 5))
    ok = np.zeros(len(xyz), np.int32)
    lb.ref_solver_sample(solver._h, len(xyz), xyz.reshape(-1), out.reshape(-1), ok)
    return out, ok.astype(bool)


def interp_state(coarse, fine):
    """Grid sequencing (interpState, src/app_cfd.js:322-357, restated in 3-D): fine's state from coarse's."""
    lb = lib()
    lb.ref_interp_state.argtypes = [C.c_void_p, C.c_void_p]
    lb.ref_interp_state.restype = C.c_int
    assert lb.ref_interp_state(fine._h, coarse._h) == 0
    return fine


def fallback_count(reset=False):
    """How often the oracle's first-order fallback (src/air_cfd.js:221) has fired."""
    lb = lib()
    lb.ref_fallback_count.argtypes = [C.c_int]
    lb.ref_fallback_count.restype = C.c_long
    return int(lb.ref_fallback_count(1 if reset else 0))
