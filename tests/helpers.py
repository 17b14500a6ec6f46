"""Shared builders for the parity tests: the same aircraft shape and grid on the oracle and the GPU."""
import math

import numpy as np

README_CL, README_CD = 0.1927, 0.04406  # README.md:98, fighter 30k cells M0.6 a3 d3, 200 iterations


def rel_max_diff(a, b):
    """The reference's GPU/CPU metric (tools/gpucmp.mjs:19-21): max|a-b| / max|b| per variable."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / den) if den > 0 else float(np.max(np.abs(a - b)))


def freestream(M, alpha):
    a = alpha * math.pi / 180
    return [1.0, M * math.cos(a), 0.0, M * math.sin(a), 1 / (1.4 * 0.4) + 0.5 * M * M]


def oracle_case(aero, ref, typ, cells, delta, M=0.6, alpha=3.0, threads=8, prec=32, fix=None):
    ac = aero.build_aircraft(typ)
    sh = aero.shape_of(ac)
    g = ref.grid(sh, cells)
    geo = ref.geom(sh, g, delta)
    s = ref.CfdCPU(g, geo, prec=prec, threads=threads)
    F = freestream(M, alpha)
    s.setFree(F)
    s.setFix(fix if fix is not None else [F, F, F])
    s.reset()
    return ac, sh, g, geo, s


def box_geometry(rng, NX, NY, NZ, kinds=("fluid", "solid", "cut", "baffle", "fixed")):
    """Random cut-cell box: a valid geometry built like cfdGeom's final arrays, for per-cell tests."""
    N = NX * NY * NZ
    t = np.zeros(N, np.uint8)
    phi = np.ones(N, np.float32)
    ap = [np.ones(N, np.float32) for _ in range(3)] + [np.zeros(N, np.float32)]
    q = np.arange(N)
    i, j, k = q % NX, (q // NX) % NY, q // (NX * NY)
    if "cut" in kinds:
        cut = rng.random(N) < 0.15
        phi[cut] = (rng.integers(6, 27, cut.sum()) / 27.0).astype(np.float32)
        for d in range(3):
            m = rng.random(N) < 0.12
            ap[d][m] = (rng.integers(0, 10, m.sum()) / 9.0).astype(np.float32)
    if "solid" in kinds:
        sol = rng.random(N) < 0.06
        t[sol] = 1
        phi[sol] = 0.1
    if "fixed" in kinds:
        fx = rng.random(N) < 0.02
        t[fx & (t == 0)] = rng.integers(3, 6, (fx & (t == 0)).sum())
        phi[t >= 3] = 1
    if "baffle" in kinds:
        b = (rng.random(N) < 0.08) & (k + 1 < NZ)
        ap[3][b] = rng.uniform(-0.3, 0.3, b.sum()).astype(np.float32)
        ap[2][b] = np.minimum(ap[2][b], (rng.integers(0, 9, b.sum()) / 9.0).astype(np.float32))
    # clean-up as cfdGeom does (src/air_cfd.js:132-136)
    NXY = NX * NY
    for d, st, inside in ((0, 1, i + 1 < NX), (1, NX, j + 1 < NY), (2, NXY, k + 1 < NZ)):
        q2 = np.where(inside, q + st, q)
        close = inside & ((t == 1) | (t[q2] == 1))
        ap[d][close] = 0
        if d == 2:
            ap[3][close] = 0
            ap[3][~inside] = 0
    up = np.where(k + 1 < NZ, q + NXY, q)
    ap[3][(t >= 3) | ((k + 1 < NZ) & (t[up] >= 3))] = 0
    return t, phi, ap


class BoxGrid:
    """Grid object with the oracle's attribute names for a random stretched box."""

    def __init__(self, rng, NX, NY, NZ):
        self.xf = np.concatenate([[0.0], np.cumsum(rng.uniform(0.5, 1.5, NX))])
        self.yf = np.concatenate([[0.0], np.cumsum(rng.uniform(0.5, 1.5, NY))])
        self.zf = np.concatenate([[0.0], np.cumsum(rng.uniform(0.5, 1.5, NZ))])
        self.dims = np.array([NX, NY, NZ], np.int32)
        self.NX, self.NY, self.NZ, self.N = NX, NY, NZ, NX * NY * NZ
        self.h = 1.0
