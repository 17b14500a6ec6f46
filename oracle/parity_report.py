"""Parity report: the GPU solver against the oracle's float32 and FP64 runs on the same inputs.

Test infrastructure (it runs the oracle); prints one JSON line per case.  Run from the
repository root on a machine with a GPU:

    python oracle/parity_report.py            # C1 (30k cells, 200 its, kernels 0-3) and C2 (4M, 2000 its)
    python oracle/parity_report.py --c1-only
    python oracle/parity_report.py --fix cycle --c2-fp64-only

--fix cycle: the engine cells hold the engine field model's states (sea level, full dry
throttle) instead of the free stream; --c2-fp64-only: C2 against the FP64 oracle run only
(the oracle's own float32 run does not depend on the GPU build).

Metrics per variable (rho, rho u, rho v, rho w, E): max|a - b| / max|b| (the reference's GPU/CPU
metric, tools/gpucmp.mjs:19-21), and the per-cell relative maximum and 99.9th percentile for
rho and E.
"""
import importlib
import json
import math
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle")]
aero = importlib.import_module("3d_aero_lab_b200")
import ref  # noqa: E402


def freestream(M, alpha):
    a = alpha * math.pi / 180
    return [1.0, M * math.cos(a), 0.0, M * math.sin(a), 1 / (1.4 * 0.4) + 0.5 * M * M]


def rel_max(a, b):
    den = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / den) if den > 0 else float(np.max(np.abs(a - b)))


def metrics(a, b):
    cell = [np.abs(a[c] - b[c]) / np.abs(b[c]) for c in (0, 4)]
    return {"gpucmp": [f"{rel_max(a[c], b[c]):.2e}" for c in range(5)],
            "percell_max_rho_E": [f"{float(np.max(x)):.2e}" for x in cell],
            "percell_p999_rho_E": [f"{float(np.quantile(x, 0.999)):.2e}" for x in cell]}


def oracle(sh, g, delta, F, fix, prec, threads):
    s = ref.CfdCPU(g, ref.geom(sh, g, delta), prec=prec, threads=threads)
    s.setFree(F)
    s.setFix(fix)
    s.reset()
    return s


def case(typ, cells, delta, its, kernels, M=0.6, alpha=3.0, fix_kind="free", with32=True):
    threads = ref.max_threads()
    ac = aero.build_aircraft(typ)
    sh = aero.shape_of(ac)
    S = ac.ref
    F = freestream(M, alpha)
    fix = aero.fix_states(ac, 0.0, M, alpha)[1] if fix_kind == "cycle" else [F, F, F]
    g = ref.grid(sh, cells)
    out = {"case": f"{typ} {g.NX}x{g.NY}x{g.NZ}={g.N} {its} its, M{M} a{alpha} d{delta}, fixed states {fix_kind}",
           "threads": threads}
    gpu = {}
    for k in kernels:
        s = aero.CfdGPU(aero.cfd_grid(sh, cells), shape=sh, delta=delta)
        s.set_kernel(k, 16)
        s.setFree(F)
        s.setFix(fix)
        s.reset()
        s.step(its)
        f = s.forces(alpha, M, S["S"], S["xcg"], 0, S["c"])
        gpu[k] = (s.read_array().astype(np.float64), [f["CL"], f["CD"]])
        s.dispose()
    t0 = time.time()
    a32 = None
    if with32:
        o32 = oracle(sh, g, delta, F, fix, 32, threads)
        o32.step(its)
        a32 = o32.read()
        del o32
    o64 = oracle(sh, g, delta, F, fix, 64, threads)
    o64.step(its)
    a64 = o64.read()
    f64 = o64.forces(alpha, M, S["S"], S["xcg"], 0, S["c"])
    out["oracle_cpu_s"] = round(time.time() - t0, 1)
    if a32 is not None:
        out["oracle32_vs_64"] = metrics(a32, a64)
    out["CL/CD oracle64"] = [f64["CL"], f64["CD"]]
    for k, (q, clcd) in gpu.items():
        r = {"vs_oracle64": metrics(q, a64), "CL/CD": clcd}
        if a32 is not None:
            r["vs_oracle32"] = metrics(q, a32)
        out[f"kernel{k}"] = r
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    fix_kind = sys.argv[sys.argv.index("--fix") + 1] if "--fix" in sys.argv else "free"
    case("fighter", 30000, 3.0, 200, [0, 1, 2, 3], fix_kind=fix_kind)
    if "--c1-only" not in sys.argv:
        case("fighter", 4.0e6, 3.0, 2000, [2], fix_kind=fix_kind, with32="--c2-fp64-only" not in sys.argv)
