"""One case split into z slabs: several devices of one process, or one slab per rank.

The reference solves one case in one WebGL context (src/air_cfd.js:367-438), so a case is
limited to what one device holds.  Here a case's planes are cut into near-equal z slabs.  Each
slab solver stores its own planes plus up to HALO = 2 halo planes on each side that it shares
with its neighbour.  Two planes are what the MUSCL stencil of a face reads on either side.
Per SSP-RK2 iteration:

    stage 1 on every slab      S1 = Q + dt R(Q)
    exchange S1 halo planes
    stage 2 on every slab      B = Q/2 + (S1 + dt R(S1))/2
    exchange B halo planes     (B is the new Q)

A slab's update of its own planes reads only its own and halo planes, so after each exchange
the own planes hold the same numbers as the unsplit solve.  The fluxes involved are the
cross-plane face fluxes, the local time step and the wall source.  Halo planes are computed
too and then overwritten.  Forces, the Trefftz integral and the residual sums are restricted
to own planes and add up across slabs; Mach maxima combine by max.

`SplitCase` drives the slabs from one process.  By default the stage kernels push: each
slab's stage kernel stores the planes its neighbours keep as halo planes straight into their
buffers, peer stores over NVLink when they live on other devices.  Stream waits on the
neighbours' events then order the next stage, and no copy runs between stages.  With
push=False the halos move by `a3d_solver_copy_planes` after each stage instead.  `DistSplit` runs one slab per rank of a
torch.distributed group.  It exchanges the halo planes with point-to-point send/recv on the
solver's stream (NCCL over NVLink for CUDA ranks) and all-reduces the force and residual sums.
"""
from __future__ import annotations

import math

import numpy as np

HALO = 2


def slab_bounds(NZ, n, halo=HALO, align=1):
    """Own ranges [a, b) and stored ranges [lo, hi) (own plus halos) of n z slabs.

    Interior boundaries sit near i NZ / n.  align > 1 rounds each to a multiple of align.
    The stage kernels run over a slab's own planes, so a z-marching tile of align planes then
    starts its runs where the unsplit solve starts them.
    """
    if n < 1:
        raise ValueError("need at least one slab")
    cuts = [0]
    for i in range(1, n):
        b = int(round(i * NZ / n))
        if align > 1:
            b = int(round(b / align)) * align
        cuts.append(b)
    cuts.append(NZ)
    for i in range(n):
        if cuts[i + 1] - cuts[i] < halo:
            raise ValueError(f"slab {i} would own {cuts[i + 1] - cuts[i]} planes; at least {halo} needed "
                             f"(NZ={NZ}, n={n}, align={align})")
    out = []
    for i in range(n):
        a, b = cuts[i], cuts[i + 1]
        out.append({"own": (a, b), "stored": (max(0, a - halo), min(NZ, b + halo))})
    return out


class SplitCase:
    """A case on z slabs driven from one process (the slabs may live on several devices)."""

    def __init__(self, aircraft_type="fighter", cells=30000, M=0.6, alpha=3.0, delta=0.0, slabs=2, devices=(0,),
                 fixed=None, h=0.0, thr=1.0, ab=False, kernel=None, kz=16, align=1, ac=None, push=True):
        from .aircraft import build_aircraft, trefftz_x
        from .cfd import CfdGPU, cfd_grid, freestream, shape_of
        self.ac = ac if ac is not None else build_aircraft(aircraft_type)
        self.shape = shape_of(self.ac)
        self.M, self.alpha, self.delta = M, alpha, delta
        self.g = cfd_grid(self.shape, cells)
        self.bounds = slab_bounds(self.g.NZ, slabs, HALO, align)
        self.F = freestream(M, alpha)
        if isinstance(fixed, str) and fixed == "cycle":
            from .field import fix_states
            fixed = fix_states(self.ac, h, M, alpha, thr, ab)[1]
        elif fixed is None or (isinstance(fixed, str) and fixed == "free"):
            fixed = [self.F, self.F, self.F]
        self.fixed = fixed
        self.slabs = []
        self.push = push
        try:
            for n, b in enumerate(self.bounds):
                lo, hi = b["stored"]
                s = CfdGPU.slab(self.g, self.shape, lo, hi, delta=delta, device=devices[n % len(devices)])
                self.slabs.append(s)
                if kernel is not None:
                    s.set_kernel(kernel, kz)
                s.setFree(self.F)
                s.setFix(fixed)
                s.set_owned(b["own"][0] - lo, b["own"][1] - lo)
                s.reset()
            if push:
                for n, s in enumerate(self.slabs):
                    s.set_neighbors(self.slabs[n - 1] if n > 0 else None,
                                    self.slabs[n + 1] if n + 1 < len(self.slabs) else None)
        except Exception:
            self.dispose()
            raise
        self.xT = trefftz_x(self.ac)
        self.it = 0
        self._res_it = None

    def _exchange(self, which):
        for n in range(len(self.slabs) - 1):
            L, U = self.slabs[n], self.slabs[n + 1]
            (aL, bL), (loL, hiL) = self.bounds[n]["own"], self.bounds[n]["stored"]
            (aU, bU), (loU, hiU) = self.bounds[n + 1]["own"], self.bounds[n + 1]["stored"]
            nlo, nhi = aU - loU, hiL - bL  # U's lower halo planes, L's upper halo planes
            U.copy_planes_from(L, 0, loU - loL, nlo, which)            # L's top own planes -> U's halo
            L.copy_planes_from(U, bL - loL, aU - loU, nhi, which)      # U's bottom own planes -> L's halo

    def step(self, n):
        for _ in range(int(n)):
            for which in (1, 2):
                for s in self.slabs:
                    s.stage(which)
                if self.push:
                    for s in self.slabs:
                        s.sync_neighbors()
                else:
                    self._exchange(1 if which == 1 else 0)
            self.it += 1

    def sync(self):
        for s in self.slabs:
            s.sync()

    def read_array(self):
        """State of the full grid, (5, N): each slab's own planes."""
        NXY = self.g.NX * self.g.NY
        out = np.empty((5, self.g.N), np.float32)
        for s, b in zip(self.slabs, self.bounds):
            (a, e), (lo, _) = b["own"], b["stored"]
            Q = s.read_array()
            out[:, a * NXY:e * NXY] = Q[:, (a - lo) * NXY:(e - lo) * NXY]
        return out

    def forces(self, alpha=None, M=None):
        alpha = self.alpha if alpha is None else alpha
        M = max(self.M, 0.05) if M is None else M
        r = self.ac.ref
        tot = {"CL": 0.0, "CD": 0.0, "Cm": 0.0}
        for s in self.slabs:
            f = s.forces(alpha, M, r["S"], r["xcg"], r["zcg"], r["c"])
            for k in tot:
                tot[k] += f[k]
        return tot

    def trefftz(self):
        return sum(s.trefftz(self.xT, self.alpha, self.M, self.ac.ref["S"]) for s in self.slabs)

    def residual(self, stride=3):
        """RMS density change per iteration over all slabs' own cells (None on the first call)."""
        vals = [s.residual(stride) for s in self.slabs]
        first = self._res_it is None
        n_it = self.it - (self._res_it or 0)
        self._res_it = self.it
        if first or any(v is None for v in vals) or n_it <= 0:
            return None
        parts = [s.residual_parts() for s in self.slabs]
        return math.sqrt(sum(p[0] for p in parts) / max(1.0, sum(p[1] for p in parts))) / n_it

    def mach_max(self, stride=2):
        return max(s.mach_max(stride) for s in self.slabs)

    def dispose(self):
        for s in self.slabs:
            s.dispose()
        self.slabs = []


class _CudaView:
    """A device address range seen by torch (CUDA array interface)."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": "<f4", "data": (int(ptr), False),
                                         "version": 3, "strides": None}


class GpuSlab:
    """The slab protocol `DistSplit` drives, over a slab solver (CfdGPU.slab) on one device."""

    def __init__(self, solver, device):
        import torch
        self.s, self.device = solver, torch.device("cuda", device)
        self._stream = torch.cuda.ExternalStream(solver.stream, device=self.device)
        self._res_it = None
        self.it = 0

    def stage(self, which):
        self.s.stage(which)
        self.it += which == 2

    def planes(self, which, c, k0, nk):
        """torch view of planes [k0, k0 + nk) of component c (no copy)."""
        import torch
        ptr, pf = self.s.plane_ptr(which, c, k0)
        return torch.as_tensor(_CudaView(ptr, nk * pf), device=self.device)

    def stream(self):
        import torch
        return torch.cuda.stream(self._stream)

    def force_sums(self, alpha, M, ref, xT):
        """C_L, C_D, C_m and Trefftz CD_i of the own planes (FP64 partial sums)."""
        f = self.s.forces(alpha, M, ref["S"], ref["xcg"], ref["zcg"], ref["c"])
        return [f["CL"], f["CD"], f["Cm"], self.s.trefftz(xT, alpha, M, ref["S"])]

    def residual_parts(self, stride):
        """[sum of squared density changes, cell count, iterations since the last call, valid]."""
        v = self.s.residual(stride)
        n_it = self.it - (self._res_it or 0)
        first = self._res_it is None
        self._res_it = self.it
        if first or v is None:
            return [0.0, 0.0, float(n_it), 0.0]
        sq, cnt = self.s.residual_parts()
        return [sq, cnt, float(n_it), 1.0]

    def mach_max(self, stride):
        return self.s.mach_max(stride)


class DistSplit:
    """One slab per rank of a torch.distributed group; halos by point-to-point send/recv.

    `slab` implements stage(which), planes(which, c, k0, nk) -> tensor view, stream() (a
    context manager selecting the stream the slab's work runs on), force_sums(...),
    residual_parts(stride) and mach_max(stride); `bounds` is this rank's entry of
    slab_bounds(NZ, world_size).  Every rank takes the same collective steps in the same
    order; `device` is where the reduction tensors live (None: CPU, for gloo).
    """

    def __init__(self, slab, bounds, group=None, device=None):
        import torch.distributed as dist
        self.dist, self.group, self.device = dist, group, device
        self.rank, self.size = dist.get_rank(group), dist.get_world_size(group)
        self.slab, self.b = slab, bounds
        self.it = 0

    def _peer(self, r):
        return self.dist.get_global_rank(self.group, r) if self.group is not None else r

    def _ops(self, which):
        dist = self.dist
        (a, e), (lo, hi) = self.b["own"], self.b["stored"]
        ops = []
        for c in range(5):
            if self.rank > 0 and a > lo:              # lower neighbour: own bottom planes out, lower halo in
                n = a - lo
                ops.append(dist.P2POp(dist.isend, self.slab.planes(which, c, a - lo, n), self._peer(self.rank - 1),
                                      self.group))
                ops.append(dist.P2POp(dist.irecv, self.slab.planes(which, c, 0, n), self._peer(self.rank - 1),
                                      self.group))
            if self.rank < self.size - 1 and hi > e:  # upper neighbour: own top planes out, upper halo in
                n = hi - e
                ops.append(dist.P2POp(dist.isend, self.slab.planes(which, c, e - lo - n, n),
                                      self._peer(self.rank + 1), self.group))
                ops.append(dist.P2POp(dist.irecv, self.slab.planes(which, c, e - lo, n), self._peer(self.rank + 1),
                                      self.group))
        return ops

    def _exchange(self, which):
        ops = self._ops(which)
        if ops:
            with self.slab.stream():
                for r in self.dist.batch_isend_irecv(ops):
                    r.wait()

    def step(self, n):
        for _ in range(int(n)):
            self.slab.stage(1)
            self._exchange(1)
            self.slab.stage(2)
            self._exchange(0)
            self.it += 1

    def _allreduce(self, values, op):
        # host values (the slab's reductions have synchronised): reduce on the stream that made
        # the tensor
        import torch
        t = torch.tensor(values, dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=op, group=self.group)
        return t.tolist()

    def forces(self, alpha, M, ref, xT):
        """{CL, CD, Cm, CDi} of the whole case."""
        v = self._allreduce(self.slab.force_sums(alpha, M, ref, xT), self.dist.ReduceOp.SUM)
        return dict(zip(("CL", "CD", "Cm", "CDi"), v))

    def residual(self, stride=3):
        """RMS density change per iteration over all ranks' own cells (None on the first call)."""
        sq, cnt, n_it, valid = self._allreduce(self.slab.residual_parts(stride), self.dist.ReduceOp.SUM)
        n_it /= self.size
        if valid < self.size or n_it <= 0:
            return None
        return math.sqrt(sq / max(1.0, cnt)) / n_it

    def mach_max(self, stride=2):
        return self._allreduce([self.slab.mach_max(stride)], self.dist.ReduceOp.MAX)[0]
