"""Served solves: request streams for the continuous-batching server (a3d_server_*).

`requests(seed, n)` draws cases from the batched distribution (aircraft type uniform over the
three default aircraft, cells U[20k, 2M], M U[0.3, 0.85], alpha U[-2, 8] deg, delta U[-5, 5]
deg, free-stream fixed states or, with fix="cycle", the engine field model's states at sea level
and full dry throttle); `Server` wraps the C scheduler; `poisson_run` submits a request
list at seeded Poisson arrival times and collects results; `plain_loop` solves the same list
one request at a time with the plain solver (the reference's one-case controller), with the
same convergence rule.
"""
from __future__ import annotations

import ctypes as C
import math
import threading
import time

import numpy as np

from . import _lib
from .abi import a3d_request, a3d_result, a3d_server_config
from .aircraft import build_aircraft, shape_of, trefftz_x
from .cfd import CfdGPU, cfd_grid, freestream

TYPES = ("airliner", "interceptor", "fighter")
SERVED_KERNEL = 4  # the stage kernel the server configures its cases with (server.cpp configure_case)
_AIRCRAFT = {}


def aircraft(typ):
    if typ not in _AIRCRAFT:
        ac = build_aircraft(typ)
        _AIRCRAFT[typ] = (ac, shape_of(ac))
    return _AIRCRAFT[typ]


def requests(seed, n, cells=(20e3, 2.0e6), mach=(0.3, 0.85), alpha=(-2.0, 8.0), delta=(-5.0, 5.0),
             geometries=None, fix="free"):
    """Seeded case list.  `geometries` (optional) limits the distinct (type, cells, delta) draws
    so that repeated geometries exercise the warm start.  `fix`: "free" or "cycle" (see
    `request_fix`); it draws no random numbers, so both give the same cases."""
    rng = np.random.default_rng(seed)
    pool = None
    if geometries:
        pool = [(TYPES[rng.integers(3)], float(rng.uniform(*cells)), float(rng.uniform(*delta)))
                for _ in range(geometries)]
    out = []
    for _ in range(n):
        if pool:
            typ, c, d = pool[rng.integers(len(pool))]
        else:
            typ, c, d = TYPES[rng.integers(3)], float(rng.uniform(*cells)), float(rng.uniform(*delta))
        out.append({"type": typ, "cells": round(c), "M": float(rng.uniform(*mach)),
                    "alpha": float(rng.uniform(*alpha)), "delta": round(d, 3), "fix": fix})
    return out


def request_fix(r, ac, F):
    """Fixed states of a request: the free stream, or (fix="cycle") the engine field model sampled
    as applyCond does (src/air_cfd.js:526-533) at altitude h (default 0), throttle thr (default
    1) and afterburner ab (default off)."""
    if r.get("fix") == "cycle":
        from .field import fix_states
        return fix_states(ac, r.get("h", 0.0), r["M"], r["alpha"], r.get("thr", 1.0), r.get("ab", False))[1]
    return [F, F, F]


def to_request(r):
    ac, sh = aircraft(r["type"])
    q = a3d_request()
    q.shape = sh
    q.cells, q.M, q.alpha_deg, q.delta_deg = r["cells"], r["M"], r["alpha"], r["delta"]
    F = freestream(r["M"], r["alpha"])
    for i in range(5):
        q.F[i] = F[i]
    fx = request_fix(r, ac, F)
    for i in range(15):
        q.fix[i] = fx[i // 5][i % 5]
    q.ref_S, q.ref_xcg, q.ref_zcg, q.ref_c = ac.ref["S"], ac.ref["xcg"], ac.ref["zcg"], ac.ref["c"]
    q.xT = trefftz_x(ac)
    q.geometry_key = hash((r["type"], r["cells"], r["delta"])) & 0xFFFFFFFFFFFFFFFF
    return q


def result_dict(o):
    return {k: getattr(o, k) for k, _ in a3d_result._fields_}


class Server:
    def __init__(self, budget_gb=150.0, residual_drop=1e-3, max_active=64, chunk=50, max_iters=3000, device=0,
                 warm_start=True, kz=16, sequence=0, sequence_drop=0.05, sequence_max_iters=1500):
        """sequence: grid sequencing factor (a cold request first solves cells/sequence cells,
        until its residual dropped by sequence_drop or sequence_max_iters; 0 = off)."""
        cfg = a3d_server_config(budget_gb * 1e9, residual_drop, max_active, chunk, max_iters, device,
                                1 if warm_start else 0, kz, sequence, sequence_max_iters, sequence_drop)
        self._h = C.c_void_p()
        _lib.check(_lib.lib().a3d_server_create(C.byref(cfg), C.byref(self._h)))

    def submit(self, r):
        i = C.c_int64()
        _lib.check(_lib.lib().a3d_server_submit(self._h, C.byref(to_request(r)), C.byref(i)))
        return i.value

    def wait(self, i, timeout=600.0):
        o = a3d_result()
        _lib.check(_lib.lib().a3d_server_wait(self._h, int(i), float(timeout), C.byref(o)))
        return result_dict(o)

    def stats(self):
        a = np.zeros(6, np.int64)
        _lib.check(_lib.lib().a3d_server_stats(self._h, a))
        return dict(zip(("pending", "active", "completed", "warm_starts", "rounds", "resident_bytes"), a.tolist()))

    def close(self):
        if self._h:
            _lib.lib().a3d_server_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def arrivals(seed, n, rate):
    rng = np.random.default_rng(seed + 1)
    return np.cumsum(rng.exponential(1.0 / rate, n))


def poisson_run(server, reqs, rate, seed, timeout=1800.0):
    """Submits `reqs` at seeded Poisson times (mean `rate` per second); returns results and wall time."""
    times = arrivals(seed, len(reqs), rate)
    ids = [None] * len(reqs)
    t0 = time.perf_counter()

    def feeder():
        for k, r in enumerate(reqs):
            dt = times[k] - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
            ids[k] = server.submit(r)

    th = threading.Thread(target=feeder)
    th.start()
    th.join()
    res = [server.wait(i, timeout) for i in ids]
    wall = time.perf_counter() - t0
    return res, wall


def converged(r, residual_drop=1e-3):
    """True when a result stopped on the residual drop, False when it stopped at the cap."""
    return bool(r["res0"] and r["res0"] > 0 and r["residual"] is not None and r["residual"] / r["res0"] <= residual_drop)


def latency_stats(res, residual_drop=None):
    """p50/p99/mean/max latency (submit to result).  With residual_drop, also the fraction of
    requests that met the drop and the same statistics over converged and capped requests
    separately (None where a group is empty)."""
    def stats(rs):
        if not rs:
            return None
        lat = np.array([r["t_done"] - r["t_submit"] for r in rs])
        return {"n": len(rs), "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
                "mean_s": float(lat.mean()), "max_s": float(lat.max())}
    out = stats(res)
    if residual_drop is not None:
        conv = [r for r in res if converged(r, residual_drop)]
        capped = [r for r in res if not converged(r, residual_drop)]
        out.update({"converged_fraction": len(conv) / len(res), "converged": stats(conv), "capped": stats(capped)})
    return out


def solve_plain(r, residual_drop=1e-3, chunk=50, max_iters=3000, device=0, kernel=4, kz=0, chunks=0):
    """One request on its own solver, the same convergence rule as the server.  By default the
    lone case's fastest configuration (the default stage kernel, z run and z chunks picked from
    its size); with the server's per-case configuration (kernel=SERVED_KERNEL, kz=16, chunks=1)
    the results equal the served ones bit for bit."""
    ac, sh = aircraft(r["type"])
    g = cfd_grid(sh, r["cells"])
    s = CfdGPU(g, shape=sh, delta=r["delta"], device=device)
    s.set_kernel(kernel, kz)
    s.set_chunks(chunks)
    F = freestream(r["M"], r["alpha"])
    s.setFree(F)
    s.setFix(request_fix(r, ac, F))
    s.reset()
    s.residual(1)
    res0, its, res = None, 0, None
    while True:
        s.step(chunk)
        its += chunk
        res = s.residual(1)
        if res0 is None and res and res > 0:
            res0 = res
        if (res0 and res / res0 <= residual_drop) or its >= max_iters:
            break
    f = s.forces(r["alpha"], max(r["M"], 0.05), ac.ref["S"], ac.ref["xcg"], ac.ref["zcg"], ac.ref["c"])
    cdi = s.trefftz(trefftz_x(ac), r["alpha"], r["M"], ac.ref["S"])
    s.dispose()
    return {"CL": f["CL"], "CD": f["CD"], "Cm": f["Cm"], "CDi": cdi, "iterations": its, "residual": res,
            "res0": res0}


def plain_loop(reqs, rate, seed, **kw):
    """The same request list solved one at a time in arrival order (a single-case controller)."""
    times = arrivals(seed, len(reqs), rate)
    out, clock = [], 0.0
    t0 = time.perf_counter()
    for k, r in enumerate(reqs):
        start = max(clock, times[k])
        ts = time.perf_counter()
        o = solve_plain(r, **kw)
        clock = start + (time.perf_counter() - ts)
        o["t_submit"], o["t_done"] = float(times[k]), clock
        out.append(o)
    return out, time.perf_counter() - t0
