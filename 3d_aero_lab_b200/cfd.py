"""Host mirror of the reference's 3D CFD entry points (src/air_cfd.js), over libaero3d.so.

Reference name             here
-------------------------  ----------------------------------------------
cfdGrid(ac, level)         cfd_grid(ac, cells)
cfdGeom(ac, G, g, delta)   cfd_geom(ac, g, delta)
cfdForceList(g, geo)       CfdGPU.force_list()  (built on the device with the solver)
new CfdGPU(g, geo)         CfdGPU(g, geo) or CfdGPU(g, shape=..., delta=...)
  .setFree/.setFix/.reset  same names
  .step(n)/.read()/.it     same names; read() returns solver-owned arrays reused across calls
  .dispose()               same name
cfdForces(g, list, H, ...) CfdGPU.forces(alpha, M, S, xcg, zcg, cref)   (FP64 on the device)
Trefftz block of readback  CfdGPU.trefftz(xT, alpha, M, S)
residual of readback       CfdGPU.residual(stride)

Errors are raised as `AeroError` (the reference's constructor throws `Error`; its step and
read do not report failures).  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib
from .aircraft import shape_of, trefftz_x
from .abi import a3d_shape

GAMMA = 1.4
MAX_FACES = 16384


class Axis:
    """One grid axis: faces f (float64), centres c and sizes d (float32), n cells."""

    def __init__(self, f):
        self.f = np.ascontiguousarray(f, dtype=np.float64)
        self.n = len(f) - 1
        self.c = (0.5 * (self.f[:-1] + self.f[1:])).astype(np.float32)
        self.d = (self.f[1:] - self.f[:-1]).astype(np.float32)


class Grid:
    """cfdGrid result (src/air_cfd.js:36-38)."""

    def __init__(self, xf, yf, zf, h=0.0, core=None):
        self.X, self.Y, self.Z = Axis(xf), Axis(yf), Axis(zf)
        self.NX, self.NY, self.NZ = self.X.n, self.Y.n, self.Z.n
        self.N = self.NX * self.NY * self.NZ
        self.h = h
        self.core = core
        self.dims = np.array([self.NX, self.NY, self.NZ], dtype=np.int32)

    def cidx(self, i, j, k):
        return (k * self.NY + j) * self.NX + i


class Geom:
    """cfdGeom result: t, phi, ap[0..3], counts (src/air_cfd.js:140)."""

    def __init__(self, N):
        self.t = np.zeros(N, np.uint8)
        self.phi = np.zeros(N, np.float32)
        self.ap = [np.zeros(N, np.float32) for _ in range(4)]
        self.nSolid = self.nCut = 0
        self.volW = self.volH = self.volV = False


def _shape(x):
    return x if isinstance(x, a3d_shape) else shape_of(x)


# the app's grid levels (CFD_GRIDS, src/air_cfd.js:10)
CFD_GRIDS = {"coarse": 150e3, "medium": 380e3, "fine": 820e3}


def cfd_grid(ac, cells):
    """Stretched half-domain grid with about `cells` cells, or a level name of CFD_GRIDS
    (cfdGrid, src/air_cfd.js:21-44)."""
    if isinstance(cells, str):
        cells = CFD_GRIDS[cells]
    sh = _shape(ac)
    L = _lib.lib()
    xf, yf, zf = (np.zeros(MAX_FACES) for _ in range(3))
    dims = np.zeros(3, np.int32)
    h = C.c_double()
    core = np.zeros(5)
    _lib.check(L.a3d_grid_build(C.byref(sh), float(cells), MAX_FACES, xf, yf, zf, dims, C.byref(h), core))
    return Grid(xf[:dims[0] + 1].copy(), yf[:dims[1] + 1].copy(), zf[:dims[2] + 1].copy(), h.value, core)


def cfd_geom(ac, g, delta_deg=0.0):
    """Cut-cell geometry on the GPU (cfdGeom, src/air_cfd.js:50-141)."""
    sh = _shape(ac)
    L = _lib.lib()
    o = Geom(g.N)
    counts = np.zeros(2, np.int64)
    vol = np.zeros(3, np.int32)
    _lib.check(L.a3d_geom_build(C.byref(sh), g.dims, g.X.f, g.Y.f, g.Z.f, float(g.h), float(delta_deg), o.t, o.phi,
                                o.ap[0], o.ap[1], o.ap[2], o.ap[3], counts, vol))
    o.nSolid, o.nCut = int(counts[0]), int(counts[1])
    o.volW, o.volH, o.volV = (bool(v) for v in vol)
    return o


def freestream(M, alpha_deg):
    """Nondimensional free-stream conservative state (src/air_cfd.js:523-524)."""
    a = alpha_deg * math.pi / 180
    return [1.0, M * math.cos(a), 0.0, M * math.sin(a), 1 / (GAMMA * (GAMMA - 1)) + 0.5 * M * M]


class CfdGPU:
    """The solver object (CfdGPU surface, src/air_cfd.js:367-438) on a B200."""

    kind = "gpu"

    def __init__(self, g, geo=None, shape=None, delta=0.0, device=0):
        L = _lib.lib()
        self.g = g
        self._h = C.c_void_p()
        if geo is not None:
            _lib.check(L.a3d_solver_create(g.dims, g.X.f, g.Y.f, g.Z.f, geo.t, geo.phi, geo.ap[0], geo.ap[1],
                                           geo.ap[2], geo.ap[3], int(device), C.byref(self._h)))
        else:
            if shape is None:
                raise ValueError("CfdGPU needs either geometry arrays or an aircraft shape")
            _lib.check(L.a3d_solver_create_shape(C.byref(_shape(shape)), g.dims, g.X.f, g.Y.f, g.Z.f, float(g.h),
                                                 float(delta), int(device), C.byref(self._h)))
        self.geo = geo
        self._opt = {"cfl": 0.7, "order": 2}
        self.F = [1.0, 0.0, 0.0, 0.0, 1 / (GAMMA * (GAMMA - 1))]
        self.fix = [list(self.F)] * 3
        self.host = None

    # -- lifecycle --
    def dispose(self):
        if self._h:
            _lib.lib().a3d_solver_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.dispose()
        except Exception:
            pass

    # -- options (opt.cfl, opt.order) --
    @property
    def opt(self):
        return dict(self._opt)

    def set_opt(self, cfl=None, order=None):
        if cfl is not None:
            self._opt["cfl"] = float(cfl)
        if order is not None:
            self._opt["order"] = int(order)
        _lib.check(_lib.lib().a3d_solver_set_opt(self._h, self._opt["cfl"], self._opt["order"]))

    def set_kernel(self, kernel, march_kz=0):
        """Stage kernel and z planes per CTA (0: picked from the grid size)."""
        _lib.check(_lib.lib().a3d_solver_set_kernel(self._h, int(kernel), int(march_kz)))

    def kernel(self):
        """(stage kernel, z planes per CTA) in use."""
        k, kz = C.c_int32(), C.c_int32()
        _lib.check(_lib.lib().a3d_solver_get_kernel(self._h, C.byref(k), C.byref(kz)))
        return k.value, kz.value

    WAIT_LIMIT_DEFAULT = 4194304

    def set_wait_limit(self, limit):
        """Try_waits a stage kernel spends on one TMA copy before it gives up (0: at once)."""
        _lib.check(_lib.lib().a3d_solver_set_wait_limit(self._h, int(limit)))

    def set_chunks(self, chunks):
        """Pipelined z chunks of step() (kernels 2 and 4): 0 automatic, 1 none, 2..4 chunks."""
        _lib.check(_lib.lib().a3d_solver_set_chunks(self._h, int(chunks)))

    def chunks(self):
        """Stage launches per RK stage that step() uses for this case."""
        v = C.c_int32()
        _lib.check(_lib.lib().a3d_solver_get_chunks(self._h, C.byref(v)))
        return v.value

    # -- reference surface --
    def setFree(self, F):
        self.F = [float(v) for v in F]
        _lib.check(_lib.lib().a3d_solver_set_free(self._h, np.asarray(self.F, np.float64)))

    def setFix(self, fx):
        self.fix = [[float(v) for v in a] for a in fx]
        _lib.check(_lib.lib().a3d_solver_set_fix(self._h, np.asarray(self.fix, np.float64).reshape(15)))

    def reset(self):
        _lib.check(_lib.lib().a3d_solver_reset(self._h))

    def step(self, n):
        _lib.check(_lib.lib().a3d_solver_step(self._h, int(n)))

    @property
    def it(self):
        v = C.c_int64()
        _lib.check(_lib.lib().a3d_solver_iterations(self._h, C.byref(v)))
        return v.value

    def read(self, out=None):
        """State as {r, ru, rv, rw, E} float32 arrays; the arrays are reused across calls."""
        if out is None:
            if self.host is None:
                self.host = {k: np.empty(self.g.N, np.float32) for k in ("r", "ru", "rv", "rw", "E")}
            out = self.host
        _lib.check(_lib.lib().a3d_solver_read(self._h, *(_lib.ptr(out[k]) for k in ("r", "ru", "rv", "rw", "E"))))
        return out

    def read_dt(self):
        """The `dt` field of CfdGPU.read(): each fluid cell's local time step in the last iteration."""
        out = np.empty(self.g.N, np.float32)
        _lib.check(_lib.lib().a3d_solver_read_dt(self._h, _lib.ptr(out)))
        return out

    def read_array(self):
        H = self.read()
        return np.stack([H[k] for k in ("r", "ru", "rv", "rw", "E")]).copy()

    def write(self, Q):
        Q = np.ascontiguousarray(Q, dtype=np.float32).reshape(5, self.g.N)
        _lib.check(_lib.lib().a3d_solver_write(self._h, *(_lib.ptr(Q[c]) for c in range(5))))

    @property
    def stream(self):
        """The solver's cudaStream_t as an integer handle."""
        v = C.c_void_p()
        _lib.check(_lib.lib().a3d_solver_stream(self._h, C.byref(v)))
        return v.value or 0

    def sync(self):
        _lib.check(_lib.lib().a3d_solver_sync(self._h))

    def force_list(self):
        L = _lib.lib()
        n = C.c_int64()
        _lib.check(L.a3d_solver_force_list(self._h, C.byref(n), 0, None, None, None, None, None))
        m = n.value
        q = np.zeros(max(m, 1), np.int64)
        cx, cz, x, z = (np.zeros(max(m, 1)) for _ in range(4))
        _lib.check(L.a3d_solver_force_list(self._h, C.byref(n), m, *(_lib.ptr(a) for a in (q, cx, cz, x, z))))
        return {"q": q[:m], "cx": cx[:m], "cz": cz[:m], "x": x[:m], "z": z[:m]}

    def forces(self, alpha_deg, M, S, xcg, zcg, cref):
        out = np.zeros(3)
        _lib.check(_lib.lib().a3d_solver_forces(self._h, alpha_deg, M, S, xcg, zcg, cref, out))
        return {"CL": out[0], "CD": out[1], "Cm": out[2]}

    def trefftz(self, xT, alpha_deg, M, S):
        v = C.c_double()
        _lib.check(_lib.lib().a3d_solver_trefftz(self._h, xT, alpha_deg, M, S, C.byref(v)))
        return v.value

    def residual(self, stride=3):
        """RMS density change per iteration since the previous call (None on the first)."""
        v = C.c_double()
        _lib.check(_lib.lib().a3d_solver_residual(self._h, int(stride), C.byref(v)))
        return None if v.value < 0 else v.value

    # -- z-slab decomposition (split.py) --
    @classmethod
    def slab(cls, g, shape, z_lo, z_hi, delta=0.0, device=0):
        """Solver of planes [z_lo, z_hi) of the case built on the full grid g (a3d_solver_create_shape_slab)."""
        self = cls.__new__(cls)
        self.g = Grid(g.X.f, g.Y.f, g.Z.f[z_lo:z_hi + 1].copy(), g.h, g.core)
        self._h = C.c_void_p()
        _lib.check(_lib.lib().a3d_solver_create_shape_slab(C.byref(_shape(shape)), g.dims, g.X.f, g.Y.f, g.Z.f,
                                                           float(g.h), float(delta), int(z_lo), int(z_hi),
                                                           int(device), C.byref(self._h)))
        self.geo = None
        self._opt = {"cfl": 0.7, "order": 2}
        self.F = [1.0, 0.0, 0.0, 0.0, 1 / (GAMMA * (GAMMA - 1))]
        self.fix = [list(self.F)] * 3
        self.host = None
        return self

    def set_owned(self, k0, k1):
        """Planes [k0, k1) that forces, Trefftz, residual and Mach maximum cover."""
        _lib.check(_lib.lib().a3d_solver_set_owned(self._h, int(k0), int(k1)))

    def stage(self, which):
        """One RK stage (1 or 2); stage 2 completes the iteration."""
        _lib.check(_lib.lib().a3d_solver_stage(self._h, int(which)))

    def copy_planes_from(self, src, dst_k0, src_k0, nk, which):
        """Planes of src's current (which=0) or stage-1 (which=1) state into this solver's."""
        _lib.check(_lib.lib().a3d_solver_copy_planes(self._h, int(dst_k0), src._h, int(src_k0), int(nk), int(which)))

    def plane_ptr(self, which, c, k):
        """(device address, floats per plane) of plane k of component c."""
        p, n = C.c_void_p(), C.c_int64()
        _lib.check(_lib.lib().a3d_solver_plane_ptr(self._h, int(which), int(c), int(k), C.byref(p), C.byref(n)))
        return p.value, n.value

    def set_neighbors(self, lo, hi):
        """Stage kernels push the planes lo / hi keep as halo planes into their buffers."""
        _lib.check(_lib.lib().a3d_solver_set_neighbors(self._h, lo._h if lo is not None else None,
                                                       hi._h if hi is not None else None))

    def sync_neighbors(self):
        """The next stage waits for the neighbours' last stages (and their pushes)."""
        _lib.check(_lib.lib().a3d_solver_sync_neighbors(self._h))

    def residual_parts(self):
        """(sum of squared density changes, cell count) behind the last residual()."""
        out = np.zeros(2)
        _lib.check(_lib.lib().a3d_solver_residual_parts(self._h, out))
        return float(out[0]), float(out[1])

    def sample(self, xyz):
        """Primitive states at points (n x 3): (n x 5 array, ok flags) - cfdStencil + cfdSample."""
        xyz = np.ascontiguousarray(xyz, np.float64).reshape(-1, 3)
        out = np.zeros((len(xyz), 5))
        ok = np.zeros(len(xyz), np.int32)
        _lib.check(_lib.lib().a3d_solver_sample(self._h, len(xyz), xyz.reshape(-1), out.reshape(-1), ok))
        return out, ok.astype(bool)

    def interp_from(self, coarse):
        """Start from `coarse`'s state interpolated onto this grid (interpState, grid sequencing)."""
        _lib.check(_lib.lib().a3d_solver_interp_state(self._h, coarse._h))

    def mach_max(self, stride=2):
        v = C.c_double()
        _lib.check(_lib.lib().a3d_solver_mach_max(self._h, int(stride), C.byref(v)))
        return v.value


def interp_state(coarse, fine):
    """interpState (src/app_cfd.js:331-357) in 3-D: `fine` takes `coarse`'s state on its cells."""
    fine.interp_from(coarse)
    return fine


class Case:
    """One solve: aircraft -> grid -> device geometry -> solver, set up like tools/test_cfd3.js:5-10.

    fixed: None or "free" - free-stream fixed states, as tools/test_cfd3.js:10 sets them;
    "cycle" - the engine field model's states at altitude h, throttle thr and afterburner ab,
    as the app's applyCond pushes them (src/air_cfd.js:521-533); or three explicit states.
    """

    def __init__(self, aircraft_type="fighter", cells=30000, M=0.6, alpha=3.0, delta=0.0, fixed=None, device=0,
                 ac=None, kernel=None, h=0.0, thr=1.0, ab=False):
        from .aircraft import build_aircraft
        self.ac = ac if ac is not None else build_aircraft(aircraft_type)
        self.shape = shape_of(self.ac)
        self.M, self.alpha, self.delta = M, alpha, delta
        self.g = cfd_grid(self.shape, cells)
        self.solver = CfdGPU(self.g, shape=self.shape, delta=delta, device=device)
        if kernel is not None:
            self.solver.set_kernel(kernel)
        self.F = freestream(M, alpha)
        self.solver.setFree(self.F)
        if isinstance(fixed, str) and fixed == "cycle":
            from .field import fix_states
            fixed = fix_states(self.ac, h, M, alpha, thr, ab)[1]
        elif fixed is None or (isinstance(fixed, str) and fixed == "free"):
            fixed = [self.F, self.F, self.F]
        self.fixed = [list(map(float, f)) for f in fixed]
        self.solver.setFix(self.fixed)
        self.solver.reset()
        self.xT = trefftz_x(self.ac)

    def forces(self):
        r = self.ac.ref
        return self.solver.forces(self.alpha, max(self.M, 0.05), r["S"], r["xcg"], r["zcg"], r["c"])

    def trefftz(self):
        return self.solver.trefftz(self.xT, self.alpha, self.M, self.ac.ref["S"])


class Batch:
    """Many solver cases advanced together (a3d_batch_*): concurrent per-case launches in one
    graph (mode 1, default) or one persistent launch per RK stage (mode 0)."""

    def __init__(self, solvers):
        self.solvers = list(solvers)
        arr = (C.c_void_p * len(self.solvers))(*[s._h.value for s in self.solvers])
        self._h = C.c_void_p()
        _lib.check(_lib.lib().a3d_batch_create(arr, len(self.solvers), C.byref(self._h)))

    def step(self, n):
        _lib.check(_lib.lib().a3d_batch_step(self._h, int(n)))

    def sync(self):
        _lib.check(_lib.lib().a3d_batch_sync(self._h))

    def tune(self, trial_iters=20):
        kz, ct, ms = C.c_int32(), C.c_int32(), C.c_float()
        _lib.check(_lib.lib().a3d_batch_tune(self._h, int(trial_iters), C.byref(kz), C.byref(ct), C.byref(ms)))
        return {"kz": kz.value, "ctas_per_sm": ct.value, "ms_per_iteration": ms.value, "mode": self.mode()}

    def set_mode(self, mode):
        """0: one persistent kernel per RK stage; 1: concurrent per-case launches in one graph."""
        _lib.check(_lib.lib().a3d_batch_set_mode(self._h, int(mode)))

    def mode(self):
        m = C.c_int32()
        _lib.check(_lib.lib().a3d_batch_get_mode(self._h, C.byref(m)))
        return m.value

    def set_schedule(self, kz, ctas_per_sm):
        _lib.check(_lib.lib().a3d_batch_set_schedule(self._h, int(kz), int(ctas_per_sm)))

    def schedule(self):
        kz, ct, tiles = C.c_int32(), C.c_int32(), C.c_int64()
        _lib.check(_lib.lib().a3d_batch_get_schedule(self._h, C.byref(kz), C.byref(ct), C.byref(tiles)))
        return {"kz": kz.value, "ctas_per_sm": ct.value, "tiles": tiles.value}

    def dispose(self):
        if self._h:
            _lib.lib().a3d_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.dispose()
        except Exception:
            pass
