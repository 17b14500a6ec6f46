"""z-slab decomposition on CPU: the slab bounds and the rank-to-rank halo exchange of
DistSplit over gloo (world sizes 2 and 3).

The ranks drive a stand-in slab with the solver's slab protocol: a five-component state on
planes, two RK stages whose update reads two planes on either side, far-field planes beyond
the stored range.  Exchanging the right halo planes at the right time is what makes the
split state equal the one-domain state bit for bit.  On B200 ranks the same DistSplit code
drives CUDA slab solvers over NCCL.
"""
import contextlib
import importlib
import math
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
F = np.array([1.0, 0.6, 0.0, 0.03, 2.0])


def split_module():
    sys.path.insert(0, ROOT)
    return importlib.import_module("3d_aero_lab_b200.split")


def test_slab_bounds_cover_the_planes_once():
    split = split_module()
    for NZ, n, align in [(61, 3, 16), (61, 2, 1), (200, 7, 16), (9, 4, 1), (50, 1, 1)]:
        b = split.slab_bounds(NZ, n, align=align)
        own = [x["own"] for x in b]
        assert own[0][0] == 0 and own[-1][1] == NZ
        assert all(own[i][1] == own[i + 1][0] for i in range(n - 1))
        for i, x in enumerate(b):
            (a, e), (lo, hi) = x["own"], x["stored"]
            assert e - a >= split.HALO and lo == max(0, a - 2) and hi == min(NZ, e + 2)
            if align > 1 and i > 0:
                assert a % align == 0
    with pytest.raises(ValueError):
        split.slab_bounds(5, 4)


class StandInSlab:
    """Slab protocol over a (5, nz, ny, nx) float64 state with a two-plane stencil."""

    def __init__(self, Q0, lo, hi, a, e):
        self.Q = Q0[:, lo:hi].copy()
        self.S1 = np.zeros_like(self.Q)
        self.own = (a - lo, e - lo)
        self.prev = None
        self.it = 0
        self.res_it = None

    def _R(self, X):
        far = np.broadcast_to(F[:, None, None, None], (5, 2) + X.shape[2:])
        P = np.concatenate([far, X, far], axis=1)
        return (0.1 * (P[:, 1:-3] + P[:, 3:-1] - 2 * X) + 0.02 * (P[:, 0:-4] - P[:, 4:])
                + 0.05 * (np.roll(X, 1, axis=3) - X) * X[0:1])

    def stage(self, which):
        if which == 1:
            self.S1 = self.Q + self._R(self.Q)
        else:
            self.Q = 0.5 * self.Q + 0.5 * (self.S1 + self._R(self.S1))
            self.it += 1

    def planes(self, which, c, k0, nk):
        import torch
        arr = self.S1 if which == 1 else self.Q
        return torch.from_numpy(arr[c, k0:k0 + nk].reshape(-1))

    def stream(self):
        return contextlib.nullcontext()

    def own_state(self):
        return self.Q[:, self.own[0]:self.own[1]]

    def force_sums(self, *args):
        X = self.own_state()
        return [float(X[0].sum()), float(X[4].sum()), float((X[1] * X[3]).sum()), 0.0]

    def residual_parts(self, stride):
        X = self.own_state()[0]
        first = self.prev is None
        n_it = self.it - (self.res_it or 0)
        out = [0.0, 0.0, float(n_it), 0.0] if first else [float(((X - self.prev) ** 2).sum()), float(X.size),
                                                          float(n_it), 1.0]
        self.prev, self.res_it = X.copy(), self.it
        return out

    def mach_max(self, stride):
        return float(np.abs(self.own_state()[1]).max())


def initial_state(NZ=23, NY=4, NX=6, seed=3):
    rng = np.random.default_rng(seed)
    return F[:, None, None, None] * (1 + 0.1 * rng.standard_normal((5, NZ, NY, NX)))


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def worker(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    import torch.distributed as dist
    from datetime import timedelta
    split = split_module()
    dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    Q0 = initial_state()
    b = split.slab_bounds(Q0.shape[1], ws)[rank]
    slab = StandInSlab(Q0, *b["stored"], *b["own"])
    d = split.DistSplit(slab, b)
    assert d.residual() is None
    d.step(7)
    f = d.forces(0.0, 0.0, None, 0.0)
    r = d.residual()
    m = d.mach_max()
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, b["own"], slab.own_state().copy(), f, r, m))


@pytest.mark.parametrize("ws", [2, 3])
def test_rank_slabs_reproduce_one_domain(ws):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    ps = [ctx.Process(target=worker, args=(r, ws, port, q)) for r in range(ws)]
    for p in ps:
        p.start()
    out = sorted([q.get(timeout=120) for _ in range(ws)], key=lambda x: x[0])
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    Q0 = initial_state()
    one = StandInSlab(Q0, 0, Q0.shape[1], 0, Q0.shape[1])
    one.residual_parts(1)
    for _ in range(7):
        one.stage(1)
        one.stage(2)
    for rank, (a, e), X, f, r, m in out:
        assert np.array_equal(X, one.Q[:, a:e]), rank         # bit for bit
        fs = one.force_sums()
        assert all(math.isclose(f[k], fs[i], rel_tol=1e-12) for i, k in enumerate(("CL", "CD", "Cm")))
        sq, cnt, n_it, _ = one.residual_parts(1) if rank == 0 else (sq, cnt, n_it, 1)
        assert math.isclose(r, math.sqrt(sq / cnt) / n_it, rel_tol=1e-12)
        assert m == one.mach_max(1)
