"""Engine operating point, engine field model and the solver's fixed states.

The reference does not run its 3D solver with free-stream states in the engine cells: on
every condition change `CFD3.applyCond` (src/air_cfd.js:521-538) samples its axisymmetric
engine field model at three points and pushes the results with `setFix`:

* `sink`: just behind the fan face (station 2), mid-channel of the inlet stream;
* `jB`:   just inside the bypass nozzle exit, mid-annulus (podded turbofan only);
* `jC`:   just inside the core nozzle exit, mid-annulus.

This module restates that chain on the host:

* `EngineDeck` - the operating point at (h, M, throttle, afterburner) with the 105 %
  spool-speed limit (src/perf.js:7-47);
* `FieldModel` - the station knots and the sampled flow field (src/field.js:9-490): knot
  lists per stream, Mach numbers rescaled from the design point by corrected flow, combustor,
  mixer and afterburner temperature fields, the wall boundary layer, and outside the engine
  the intake sink, nacelle shoulder and the diffusing jets;
* `fix_states` - `applyCond`'s conversion of three samples into the solver's normalised
  conservative states (rho, rho u, 0, 0, E).

The throttle is an input.  The app obtains it from the performance context's trim point
(`PerfCtx.point`, src/perf.js:61-92): a numeric throttle passes straight through, and the
"level" setting searches the throttle whose installed thrust equals the drag.  The drag comes
from the panel method and the drag build-up, which this package does not carry, so
`level_throttle` takes the drag as an argument and restates only the throttle search.

Pure host arithmetic in IEEE double, in the reference's operation order.
"""
from __future__ import annotations

import math

from . import engine as E

DEG = math.pi / 180
CG = 1.4  # gamma of the 3D solver (src/air_cfd.js:11)

# installed-thrust loss per aircraft type (`aero.inst`, src/aircraft.js:17,31,45)
INSTALL_LOSS = {"airliner": 0.03, "interceptor": 0.05, "fighter": 0.05}


def _clamp(v, a, b):
    return a if v < a else (b if v > b else v)


def _lerp(a, b, t):
    return a + (b - a) * t


def _smooth(e0, e1, x):
    """Smoothstep (src/field.js:6)."""
    t = _clamp((x - e0) / (e1 - e0), 0, 1)
    return t * t * (3 - 2 * t)


def _jsdiv(a, b):
    """a / b with JavaScript's result for a zero divisor."""
    if b != 0:
        return a / b
    if a == 0 or a != a:
        return math.nan
    return math.copysign(math.inf, a) * math.copysign(1.0, b)


def _sign(v):
    """Math.sign."""
    return 1.0 if v > 0 else (-1.0 if v < 0 else v)


def inv_mfp(val, g, R, supersonic):
    """Mach number from the mass-flow parameter, by bisection (src/physics.js:32-42)."""
    vmax = E.mfp(1, g, R)
    if not (val > 0):
        return 0
    if val >= vmax:
        return 1
    lo, hi = (1, 6) if supersonic else (0, 1)
    for _ in range(48):
        mid = 0.5 * (lo + hi)
        v = E.mfp(mid, g, R)
        if (v > val) if supersonic else (v < val):
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def fs_state(h, M):
    """Free-stream static state used to normalise the solver's states (src/air_field.js:10-13)."""
    at = E.isa(h)
    V = M * at["a"]
    k = 1 + 0.2 * M * M
    return {"h": h, "M": M, "T": at["T"], "P": at["P"], "rho": at["rho"], "a": at["a"], "V": V,
            "Tt": at["T"] * k, "Pt": at["P"] * math.pow(k, 3.5), "q": 0.5 * at["rho"] * V * V}


def cfd_state(fs, W):
    """Nondimensional primitives (rho, u, v, w, p) of the solver -> dimensional state at the free
    stream fs (cfdState, src/air_cfd.js:484-490): P, T, rho, V, M, Tt, Pt, Cp, Taw, Vx, Vy, Vz."""
    T = CG * W[4] / W[0] * fs["T"]
    a = math.sqrt(1.4 * 287.05 * T)
    V = math.hypot(W[1], W[2], W[3]) * fs["a"]
    o = {"P": W[4] * CG * fs["P"], "T": T, "rho": W[0] * fs["rho"], "V": V, "M": V / a}
    o["Tt"] = T * (1 + 0.2 * o["M"] * o["M"])
    o["Pt"] = o["P"] * math.pow(1 + 0.2 * o["M"] * o["M"], 3.5)
    o["Cp"] = (o["P"] - fs["P"]) / fs["q"] if fs["q"] > 1 else 0
    o["Taw"] = T * (1 + 0.89 * 0.2 * o["M"] * o["M"])
    o["Vx"], o["Vy"], o["Vz"] = W[1] * fs["a"], W[2] * fs["a"], W[3] * fs["a"]
    return o


# ---------------------------------------------------------------------------
# engine deck  (src/perf.js:7-47)
# ---------------------------------------------------------------------------
class EngineDeck:
    """Operating points of one engine design, cached per (h, M, throttle, afterburner)."""

    def __init__(self, typ, design, eff, opt=None):
        self.type, self.design, self.eff = typ, design, eff
        self.opt = {"Tt7": 2000, "nozzleType": E.ENGINE_TYPES[typ]["nozzle"]}
        self.opt.update(opt or {})
        self.ref = E.run_cycle(self.p(0, 0, 1, False), None, E.flight_state(0, 0), design["Tt4max"])
        self.lim, self.cache = {}, {}

    @classmethod
    def for_engine(cls, P):
        """Deck of the engine parameters an aircraft was built with (src/app_air.js:269)."""
        return cls(P["type"], P["design"], P["eff"], {"Tt7": P["Tt7"], "nozzleType": P["nozzleType"]})

    def p(self, h, M, thr, ab):
        return {"type": self.type, "design": self.design, "eff": self.eff, "alt": h, "M0": M, "thr": thr,
                "ab": bool(ab), "Tt7": self.opt["Tt7"], "nozzleType": self.opt["nozzleType"]}

    def nrat(self, o):
        m = 0.0
        for k, v in o["spool"].items():
            m = max(m, v / self.ref["spool"][k])
        return m

    def tt4_limit(self, h, M):
        """Largest Tt4 within 105 % spool speed on a (250 m, 0.01) grid, regula falsi (perf.js:15-31)."""
        key = (E._jsround(h / 250), E._jsround(M * 100))
        if key in self.lim:
            return self.lim[key]
        hq = E._jsround(h / 250) * 250
        Mq = E._jsround(M * 100) / 100
        fl = E.flight_state(hq, Mq)
        p = self.p(hq, Mq, 1, False)
        T4 = self.design["Tt4max"]
        hi = T4
        oh = E.run_cycle(p, self.ref, fl, hi)
        res = T4
        if self.nrat(oh) > 1.05:
            lo = 0.45 * T4
            ol = E.run_cycle(p, self.ref, fl, lo)
            flo, fhi = self.nrat(ol) - 1.05, self.nrat(oh) - 1.05
            i = 0
            while i < 12 and hi - lo > 1:
                m = hi - fhi * (hi - lo) / (fhi - flo) if (flo < 0 and fhi > 0) else 0.5 * (lo + hi)
                fm = self.nrat(E.run_cycle(p, self.ref, fl, m)) - 1.05
                if fm > 0:
                    hi, fhi = m, fm
                else:
                    lo, flo = m, fm
                i += 1
            res = lo
        self.lim[key] = res
        return res

    def at(self, h, M, thr, ab):
        """Operating point, throttle = Tt4 / Tt4max capped by the speed limit (perf.js:33-45)."""
        h = max(0, min(20000, h))
        M = max(0, M)
        key = (E._jsround(h / 10), E._jsround(M * 1000), E._jsround(thr * 1000), bool(ab))
        if key in self.cache:
            return self.cache[key]
        Tl = self.tt4_limit(h, M)
        Tt4 = min(thr * self.design["Tt4max"], Tl)
        op = E.run_cycle(self.p(h, M, thr, ab), self.ref, E.flight_state(h, M), Tt4)
        r = {"F": op["F"], "mfuel": op["mfuel"], "op": op, "Tt4": Tt4,
             "limited": Tt4 < thr * self.design["Tt4max"] - 0.5,
             "N": {k: v / self.ref["spool"][k] for k, v in op["spool"].items()}}
        if len(self.cache) > 20000:
            self.cache.clear()
        self.cache[key] = r
        return r

    def thrust(self, h, M, thr, ab, n_eng, inst):
        """Installed thrust of all engines (PerfCtx.thrust, src/perf.js:55-59)."""
        e = self.at(h, M, thr, ab)
        return {"T": n_eng * e["F"] * (1 - inst), "ff": n_eng * e["op"]["mfuel"], "e": e}


def level_throttle(deck, h, M, D, ab, n_eng, inst):
    """Throttle whose installed thrust equals the drag D (the 'level' branch, src/perf.js:70-87).

    Returns (throttle, thrust record).  D [N] comes from the caller's drag model; n_eng and
    inst are the aircraft's engine count (`ac.T["nEng"]`) and `INSTALL_LOSS[type]`.
    """
    t_max = deck.thrust(h, M, 1, ab, n_eng, inst)
    if t_max["T"] <= D:
        return 1, t_max
    lo, hi = 0.35, 1
    tlo = deck.thrust(h, M, lo, ab, n_eng, inst)
    if tlo["T"] >= D:
        return lo, tlo
    thi = t_max
    i = 0
    while i < 16 and hi - lo > 2e-4:
        m = lo + (hi - lo) * (D - tlo["T"]) / max(1, thi["T"] - tlo["T"])
        mm = min(hi - 1e-4, max(lo + 1e-4, 0.5 * (lo + hi) if i % 3 == 2 else m))
        tm = deck.thrust(h, M, mm, ab, n_eng, inst)
        if tm["T"] >= D:
            hi, thi = mm, tm
        else:
            lo, tlo = mm, tm
        if abs(tm["T"] - D) < 2e-3 * D:
            break
        i += 1
    w = max(0, min(1, (D - tlo["T"]) / max(1e-6, thi["T"] - tlo["T"])))
    thr = lo + w * (hi - lo)
    return thr, {"T": D, "ff": tlo["ff"] + w * (thi["ff"] - tlo["ff"]), "e": thi["e"]}


# ---------------------------------------------------------------------------
# knots  (src/field.js:9-228)
# ---------------------------------------------------------------------------
class _Knots:
    """KnotList (src/field.js:10-16)."""

    def __init__(self):
        self.k = []

    def add(self, x, Tt, Pt, Md, sw, gas, mdot, extra=None):
        o = {"x": x, "Tt": Tt, "Pt": Pt, "Md": Md, "sw": sw or 0, "g": gas["g"], "cp": gas["cp"], "R": E.Rg(gas),
             "mdot": mdot, "noz": -1}
        if extra:
            o.update(extra)
        self.k.append(o)
        return o


def _rows_of(spec, comp):
    return sorted((r for r in spec["rows"] if r.get("comp") == comp), key=lambda r: r["x0"])


def _kb_compress(kb, rows, st, out, Min, Mout, gas, mdot, sw_rotor):
    """Compressor rows: total temperature rises rotor by rotor, polytropic Pt (field.js:20-35)."""
    nr = sum(1 for r in rows if r["rotor"]) or 1
    dT = (out["Tt"] - st["Tt"]) / nr
    ratio = out["Tt"] / st["Tt"]
    expo = _jsdiv(math.log(out["Pt"] / st["Pt"]), math.log(ratio or 1.0000001))
    x0, x1 = rows[0]["x0"], rows[-1]["x1"]
    Tt, sw = st["Tt"], 0

    def Mof(x):
        return _lerp(Min, Mout, _clamp((x - x0) / (x1 - x0), 0, 1))

    def PtOf(T):
        return st["Pt"] * math.pow(T / st["Tt"], expo if math.isfinite(expo) else 0)

    for r in rows:
        kb.add(r["x0"], Tt, PtOf(Tt), Mof(r["x0"]), sw, gas, mdot)
        if r["rotor"]:
            Tt += dT
            sw = sw_rotor
        else:
            sw = -8 if r.get("role") == "igv" else 0
        kb.add(r["x1"], Tt, PtOf(Tt), Mof(r["x1"]) * (1.04 if r["rotor"] else 1), sw, gas, mdot)
    return {"Tt": out["Tt"], "Pt": out["Pt"], "sw": sw}


def _kb_expand(kb, rows, st, out, gas, mdot, o):
    """Turbine rows: guide vanes add swirl, rotors extract work (src/field.js:37-58)."""
    nr = sum(1 for r in rows if r["rotor"]) or 1
    dT = (st["Tt"] - out["Tt"]) / nr
    expo = _jsdiv(math.log(out["Pt"] / st["Pt"]), math.log(out["Tt"] / st["Tt"]))
    Tt, Pt, sw, first = st["Tt"], st["Pt"], 0, True
    for r in rows:
        if not r["rotor"]:
            Tt_end = Tt - dT
            Pt_stage_end = st["Pt"] * math.pow(Tt_end / st["Tt"], expo)
            kb.add(r["x0"], Tt, Pt, o["Min"] if first else 0.42, sw, gas, mdot)
            Pt = Pt * math.pow(Pt_stage_end / Pt, 0.07)
            sw = 70 if first else 62
            kb.add(r["x0"] + (r["x1"] - r["x0"]) * 0.6, Tt, Pt, o["Mthroat"] if first else 0.62, sw, gas, mdot)
            kb.add(r["x1"], Tt, Pt, o["Mthroat"] * 0.9 if first else 0.6, sw, gas, mdot)
            first = False
        else:
            kb.add(r["x0"], Tt, Pt, 0.55, sw, gas, mdot)
            Tt -= dT
            Pt = st["Pt"] * math.pow(Tt / st["Tt"], expo)
            sw = 6
            kb.add(r["x1"], Tt, Pt, o["Mout"], sw, gas, mdot)
    return {"Tt": out["Tt"], "Pt": out["Pt"]}


def _comb_knots(kb, spec, c, Tt3, Pt3, Pt4, m3, m4):
    """Combustor knots (src/field.js:148-159)."""
    cb = spec["comb"]
    C, H = E.GAS["cold"], E.GAS["hot"]
    N = 7
    for i in range(N + 1):
        t = i / N
        x = _lerp(cb["xd"], cb["x1"], t)
        Tt = Tt3 + (c["Tt4"] - Tt3) * _smooth(0.04, 0.92, t)
        Pt = Pt3 + (Pt4 - Pt3) * _smooth(0, 0.9, t)
        gas = C if t < 0.35 else H
        kb.add(x, Tt, Pt, _lerp(0.07, 0.15, t * t), 0, gas, _lerp(m3, m4, t))


def _ab_knots(kb, spec, c, m6, m7, Tt6, Pt6, gas6, x_start):
    """Afterburner duct and C-D nozzle knots (src/field.js:160-180)."""
    ab = spec["ab"]
    gas7 = c["gas7"]
    kb.add(x_start, Tt6, Pt6, 0.34, 0, gas6, m6)
    kb.add(ab["xSpray"], Tt6, Pt6, 0.25, 0, gas6, m6)
    kb.add(ab["xFH"], Tt6, Pt6 * 0.998, 0.24, 0, gas6, m6)
    N = 6
    for i in range(1, N + 1):
        t = i / N
        x = _lerp(ab["xFH"], ab["x1"], t)
        Tt = Tt6 + (c["Tt7"] - Tt6) * _smooth(0, 0.85, t)
        Pt = Pt6 + (c["Pt7"] - Pt6) * t
        g = gas7 if (c["abOn"] and t > 0.3) else gas6
        kb.add(x, Tt, Pt, _lerp(0.24, 0.30, t), 0, g, _lerp(m6, m7, t), {"nozIn": True} if i == N else None)
    n = spec["nozzle"]
    P9 = c["S"]["9"]["Pt"]
    xs = [_lerp(n["x0"], n["xt"], 0.5), n["xt"], _lerp(n["xt"], n["xe"], 0.5), n["xe"]]
    fr = [0.35, 0.62, 0.81, 1]
    for i in range(len(xs)):
        kb.add(xs[i], c["Tt7"], _lerp(c["Pt7"], P9, fr[i]), 0, 0, gas7, m7,
               {"noz": fr[i], "exit": "core" if i == len(xs) - 1 else None, "throat": i == 1})


def build_knots(spec, c, P):
    """Knot list per stream for one cycle result (src/field.js:62-146)."""
    S, e, s = c["S"], P["eff"], spec["s"]
    C, H = E.GAS["cold"], E.GAS["hot"]
    fl = c["fl"]
    out = {}
    dPt = fl["Pt0"] - c["Pt2"]
    if spec["type"] == "hbtf":
        mT, mc, mb = c["mdot"], c["mcore"], c["mbyp"]
        m4 = mc * (1 + c["f"])
        kb = _Knots()
        kb.add(0, fl["Tt0"], fl["Pt0"] - dPt * 0.3, 0.46, 0, C, mT)
        kb.add(0.30 * s, fl["Tt0"], fl["Pt0"] - dPt * 0.7, 0.5, 0, C, mT)
        fan = _rows_of(spec, "fan")[0]
        kb.add(fan["x0"], c["Tt2"], c["Pt2"], 0.55, 0, C, mT)
        kb.add(fan["x1"], c["Tt13"], c["Pt13"], 0.5, 25, C, mT)
        kb.add(0.90 * s, c["Tt13"], c["Pt13"], 0.47, 22, C, mT)
        out["inlet"] = kb.k
        kb = _Knots()
        kb.add(0.90 * s, c["Tt13"], c["Pt13"], 0.45, 22, C, mb)
        kb.add(1.00 * s, c["Tt13"], c["Pt13"] * 0.998, 0.44, 20, C, mb)
        kb.add(1.10 * s, c["Tt13"], c["Pt13"] * 0.995, 0.40, 0, C, mb)
        kb.add(1.60 * s, c["Tt13"], c["Pt13"] * 0.993, 0.42, 0, C, mb)
        kb.add(1.90 * s, c["Tt13"], c["Pt13"] * 0.992, 0.46, 0, C, mb, {"nozIn": True})
        kb.add(2.05 * s, c["Tt13"], S["19"]["Pt"] * 1.001, 0, 0, C, mb, {"noz": 0.5})
        kb.add(2.2 * s, c["Tt13"], S["19"]["Pt"], 0, 0, C, mb, {"noz": 1, "exit": "bypass"})
        out["bypass"] = kb.k
        kb = _Knots()
        kb.add(0.90 * s, c["Tt13"], c["Pt13"], 0.48, 20, C, mc)
        _kb_compress(kb, _rows_of(spec, "lpc"), {"Tt": c["Tt13"], "Pt": c["Pt13"]},
                     {"Tt": c["Tt25"], "Pt": c["Pt25"]}, 0.5, 0.45, C, mc, 32)
        kb.add(1.30 * s, c["Tt25"], c["Pt25"], 0.44, 0, C, mc)
        kb.add(1.40 * s, c["Tt25"], c["Pt25"], 0.47, 0, C, mc)
        _kb_compress(kb, _rows_of(spec, "hpc"), {"Tt": c["Tt25"], "Pt": c["Pt25"]},
                     {"Tt": c["Tt3"], "Pt": c["Pt3"]}, 0.5, 0.30, C, mc, 34)
        kb.add(2.08 * s, c["Tt3"], c["Pt3"], 0.18, 0, C, mc)
        _comb_knots(kb, spec, c, c["Tt3"], c["Pt3"], c["Pt4"], mc, m4)
        _kb_expand(kb, _rows_of(spec, "hpt"), {"Tt": c["Tt4"], "Pt": c["Pt4"]},
                   {"Tt": c["Tt45"], "Pt": c["Pt45"]}, H, m4, {"Min": 0.15, "Mthroat": 0.95, "Mout": 0.45})
        kb.add(2.62 * s, c["Tt45"], c["Pt45"], 0.42, 0, H, m4)
        _kb_expand(kb, _rows_of(spec, "lpt"), {"Tt": c["Tt45"], "Pt": c["Pt45"]},
                   {"Tt": c["Tt5"], "Pt": c["Pt5"]}, H, m4, {"Min": 0.4, "Mthroat": 0.62, "Mout": 0.42})
        kb.add(3.10 * s, c["Tt5"], c["Pt5"], 0.40, 0, H, m4)
        kb.add(3.20 * s, c["Tt5"], c["Pt5"] * 0.999, 0.42, 0, H, m4, {"nozIn": True})
        kb.add(3.34 * s, c["Tt5"], S["9"]["Pt"] * 1.001, 0, 0, H, m4, {"noz": 0.55})
        kb.add(3.45 * s, c["Tt5"], S["9"]["Pt"], 0, 0, H, m4, {"noz": 1, "exit": "core"})
        out["core"] = kb.k
    elif spec["type"] == "tj":
        m0 = c["mdot"]
        m4 = m0 * (1 + c["f"])
        m7 = c["m7"]
        kb = _Knots()
        kb.add(0, fl["Tt0"], fl["Pt0"] - dPt * 0.3, 0.42, 0, C, m0)
        kb.add(0.2 * s, fl["Tt0"], fl["Pt0"] - dPt * 0.8, 0.47, 0, C, m0)
        _kb_compress(kb, _rows_of(spec, "comp"), {"Tt": c["Tt2"], "Pt": c["Pt2"]},
                     {"Tt": c["Tt3"], "Pt": c["Pt3"]}, 0.5, 0.30, C, m0, 30)
        kb.add(1.60 * s, c["Tt3"], c["Pt3"], 0.14, 0, C, m0)
        _comb_knots(kb, spec, c, c["Tt3"], c["Pt3"], c["Pt4"], m0, m4)
        _kb_expand(kb, _rows_of(spec, "turb"), {"Tt": c["Tt4"], "Pt": c["Pt4"]},
                   {"Tt": c["Tt5"], "Pt": c["Pt5"]}, H, m4, {"Min": 0.18, "Mthroat": 0.95, "Mout": 0.45})
        _ab_knots(kb, spec, c, m4, m7, c["Tt5"], c["Pt5"], H, 2.62 * s)
        out["core"] = kb.k
    else:
        mT, mc, mb = c["mdot"], c["mcore"], c["mbyp"]
        m4 = mc * (1 + c["f"])
        m6 = m4 + mb
        m7 = c["m7"]
        kb = _Knots()
        kb.add(0, fl["Tt0"], fl["Pt0"] - dPt * 0.3, 0.42, 0, C, mT)
        kb.add(0.2 * s, fl["Tt0"], fl["Pt0"] - dPt * 0.8, 0.47, 0, C, mT)
        _kb_compress(kb, _rows_of(spec, "fan"), {"Tt": c["Tt2"], "Pt": c["Pt2"]},
                     {"Tt": c["Tt13"], "Pt": c["Pt13"]}, 0.5, 0.42, C, mT, 28)
        kb.add(0.85 * s, c["Tt13"], c["Pt13"], 0.4, 0, C, mT)
        out["inlet"] = kb.k
        kb = _Knots()
        kb.add(0.85 * s, c["Tt13"], c["Pt13"], 0.3, 0, C, mb)
        kb.add(1.3 * s, c["Tt13"], c["Pt13"] * 0.995, 0.28, 0, C, mb)
        kb.add(1.8 * s, c["Tt13"], c["Pt13"] * 0.988, 0.4, 0, C, mb)
        kb.add(2.75 * s, c["Tt13"], c["Pt16"], 0.33, 0, C, mb)
        out["bypass"] = kb.k
        kb = _Knots()
        kb.add(0.85 * s, c["Tt13"], c["Pt13"], 0.45, 0, C, mc)
        _kb_compress(kb, _rows_of(spec, "hpc"), {"Tt": c["Tt25"], "Pt": c["Pt25"]},
                     {"Tt": c["Tt3"], "Pt": c["Pt3"]}, 0.5, 0.30, C, mc, 32)
        kb.add(1.58 * s, c["Tt3"], c["Pt3"], 0.16, 0, C, mc)
        _comb_knots(kb, spec, c, c["Tt3"], c["Pt3"], c["Pt4"], mc, m4)
        _kb_expand(kb, _rows_of(spec, "hpt"), {"Tt": c["Tt4"], "Pt": c["Pt4"]},
                   {"Tt": c["Tt45"], "Pt": c["Pt45"]}, H, m4, {"Min": 0.15, "Mthroat": 0.95, "Mout": 0.45})
        kb.add(2.17 * s, c["Tt45"], c["Pt45"], 0.42, 0, H, m4)
        _kb_expand(kb, _rows_of(spec, "lpt"), {"Tt": c["Tt45"], "Pt": c["Pt45"]},
                   {"Tt": c["Tt5"], "Pt": c["Pt5"]}, H, m4, {"Min": 0.4, "Mthroat": 0.6, "Mout": 0.42})
        kb.add(2.75 * s, c["Tt5"], c["Pt5"], 0.36, 0, H, m4)
        out["core"] = kb.k
        kb = _Knots()
        kb.add(2.75 * s, c["Tt6A"], c["Pt6A"] / e["piM"] * 0.995, 0.34, 0, c["mixGas"], m6)
        _ab_knots(kb, spec, c, m6, m7, c["Tt6A"], c["Pt6A"], c["mixGas"], 3.0 * s)
        out["ab"] = kb.k
    return out


def assign_mach(kn_ref, kn_op, cyc, stream_key):
    """Operating-point Mach numbers from the design point's effective areas (src/field.js:183-217)."""
    Min = 0.4
    for a, b in zip(kn_ref, kn_op):
        if b["noz"] >= 0:
            continue
        ratio = (b["mdot"] * math.sqrt(b["Tt"]) / b["Pt"]) / (a["mdot"] * math.sqrt(a["Tt"]) / a["Pt"])
        b["M"] = inv_mfp(E.mfp(a["Md"], a["g"], a["R"]) * ratio, b["g"], b["R"], False)
        if b["M"] > 0.999:
            b["choke"] = True
        if b.get("nozIn"):
            Min = b["M"]
    nz = cyc.get("nozB") if stream_key == "bypass" else cyc.get("noz")
    for b in kn_op:
        if b["noz"] < 0:
            continue
        f = b["noz"]
        if nz["type"] == "conv" or not nz["choked"]:
            b["M"] = Min + (nz["M"] - Min) * math.pow(f, 1.6)
        else:
            ft = 0.62
            if f <= ft:
                b["M"] = Min + (1 - Min) * math.pow(f / ft, 1.5)
            else:
                b["M"] = 1 + (nz["M"] - 1) * ((f - ft) / (1 - ft))
        if b.get("exit"):
            b["M"] = nz["M"]
    for b in kn_op:
        g = b["g"]
        k = 1 + 0.5 * (g - 1) * b["M"] * b["M"]
        b["T"] = b["Tt"] / k
        b["P"] = b["Pt"] / math.pow(k, g / (g - 1))
        b["a"] = math.sqrt(g * b["R"] * b["T"])
        b["V"] = b["M"] * b["a"]
        b["rho"] = b["P"] / (b["R"] * b["T"])


def knot_at(kn, x):
    """Knot state at x: linear in Tt, M, swirl and gas, geometric in Pt (src/field.js:218-232)."""
    lo, hi = 0, len(kn) - 1
    if x <= kn[0]["x"]:
        lo = hi = 0
    elif x >= kn[hi]["x"]:
        lo = hi
    else:
        while hi - lo > 1:
            m = (lo + hi) >> 1
            if kn[m]["x"] <= x:
                lo = m
            else:
                hi = m
    a, b = kn[lo], kn[hi]
    t = 0 if (hi == lo or b["x"] - a["x"] < 1e-9) else (x - a["x"]) / (b["x"] - a["x"])
    return {"Tt": _lerp(a["Tt"], b["Tt"], t), "Pt": a["Pt"] * math.pow(b["Pt"] / a["Pt"], t),
            "M": _lerp(a["M"], b["M"], t), "sw": _lerp(a["sw"], b["sw"], t), "g": _lerp(a["g"], b["g"], t),
            "cp": _lerp(a["cp"], b["cp"], t), "R": _lerp(a["R"], b["R"], t)}


# ---------------------------------------------------------------------------
# jets: diffusion of momentum and enthalpy flux  (src/field.js:234-258)
# ---------------------------------------------------------------------------
def _i0e(x):
    """exp(-|x|) I0(x), the polynomial fits of Abramowitz and Stegun 9.8.1-9.8.2."""
    ax = abs(x)
    if ax < 3.75:
        t = (x / 3.75) ** 2
        return math.exp(-ax) * (1 + t * (3.5156229 + t * (3.0899424 + t * (1.2067492 + t * (
            0.2659732 + t * (0.0360768 + t * 0.0045813))))))
    t = 3.75 / ax
    return (0.39894228 + t * (0.01328592 + t * (0.00225319 + t * (-0.00157565 + t * (0.00916281 + t * (
        -0.02057706 + t * (0.02635537 + t * (-0.01647633 + t * 0.00392377)))))))) / math.sqrt(ax)


# 10-point Gauss-Legendre nodes and weights
_GLX = [-0.9739065285, -0.8650633667, -0.6794095683, -0.4333953941, -0.1488743390,
        0.1488743390, 0.4333953941, 0.6794095683, 0.8650633667, 0.9739065285]
_GLW = [0.0666713443, 0.1494513492, 0.2190863625, 0.2692667193, 0.2955242247,
        0.2955242247, 0.2692667193, 0.2190863625, 0.1494513492, 0.0666713443]


def blur_disk(r, R, sig):
    """Disk of radius R convolved with a 2-D Gaussian of width sig, at radius r (field.js:245-258)."""
    if sig < 1e-5:
        return 1 if r < R else 0
    a, b = max(0, r - 6 * sig), min(R, r + 6 * sig)
    if b <= a:
        return 0
    hm, c, is2 = 0.5 * (b - a), 0.5 * (a + b), 1 / (sig * sig)
    s = 0.0
    for i in range(10):
        rho = c + hm * _GLX[i]
        d = r - rho
        s += _GLW[i] * rho * is2 * math.exp(-0.5 * d * d * is2) * _i0e(r * rho * is2)
    return min(1, s * hm)


# ---------------------------------------------------------------------------
# field model  (src/field.js:263-490)
# ---------------------------------------------------------------------------
class FieldModel:
    """Axisymmetric engine flow field rebuilt from the station-by-station cycle.

    `sol` = {"op": operating-point cycle, "fl": its flight state, "ref": design-point cycle};
    `P` = the engine parameters (only `eff` is read).
    """

    def __init__(self, spec, sol, P):
        self.spec, self.sol, self.P = spec, sol, P
        c, fl = sol["op"], sol["fl"]
        self.c, self.fl = c, fl
        k_ref, k_op = build_knots(spec, sol["ref"], P), build_knots(spec, c, P)
        for key in k_op:
            assign_mach(k_ref[key], k_op[key], c, key)
        self.kn = k_op
        self.bodies = [dict(b, bb=E.bbox(b["poly"])) for b in spec["bodies"]]
        U0 = fl["V0"]
        self.exits = []
        for g in spec["exitsGeom"]:
            n = c["nozB"] if g["key"] == "bypass" else c["noz"]
            Tt = n["Tt"]
            under = n["P"] > fl["P0"] * 1.02
            Mj = E.mach_from_npr(n["Pt"] / fl["P0"], n["gas"]["g"]) if under else n["M"]
            self.exits.append(dict(g, U=n["V"], Uex=n["V"] - U0, dTt=Tt - fl["Tt0"], Tt=Tt, Pt=n["Pt"], P=n["P"],
                                   T=n["T"], M=n["M"], gas=n["gas"], Mj=Mj,
                                   Ls=1.306 * math.sqrt(Mj * Mj - 1) * 2 * g["R"] if Mj > 1.02 else 0,
                                   under=under,
                                   spread=0.058 / (1 + 0.28 * max(0, Mj - 1)) * (1.12 if Tt > 600 else 1)))
        self.exits.sort(key=lambda e: -e["R"])
        self.maxdT = max(abs(e["dTt"]) for e in self.exits) + 1
        hot = None
        for e in self.exits:
            if e["dTt"] > (hot["dTt"] if hot else -1):
                hot = e
        self.hot_gas = hot["gas"] if (hot and hot["dTt"] > 50) else None
        for i, e in enumerate(self.exits):
            o = self.exits[i - 1] if i > 0 else None
            qm = e["Uex"] * abs(e["Uex"])
            qh = e["Uex"] * e["dTt"]
            e["Qm"] = qm - o["Uex"] * abs(o["Uex"]) if o else qm
            e["Qh"] = qh - o["Uex"] * o["dTt"] if o else qh
        k0 = (self.kn.get("inlet") or self.kn["core"])[0]
        self.Uface = k0["V"]
        self.chokes = [{"stream": key, "x": k["x"]} for key in self.kn for k in self.kn[key]
                       if k.get("choke") and k["noz"] < 0]

    def classify(self, x, r):
        """Flow stream, solid body or outside (src/field.js:306-319)."""
        sp = self.spec
        for key in sp["order"]:
            st = sp["streams"][key]
            if x < st["x0"] or x > st["x1"]:
                continue
            lo, hi = st["lo"].at(x), st["hi"].at(x)
            if lo <= r <= hi:
                return {"kind": "stream", "key": key, "lo": lo, "hi": hi}
        for b in self.bodies:
            bb = b["bb"]
            if x < bb[0] or x > bb[1] or r < bb[2] or r > bb[3]:
                continue
            if E.point_in_poly(x, r, b["poly"]):
                return {"kind": "solid", "key": b["key"], "mat": b["mat"]}
        return {"kind": "ext"}

    def sample(self, x, r, th=0.0):
        """All flow quantities at engine-frame (x, r, theta) (src/field.js:327-335)."""
        cl = self.classify(x, r)
        out = {"region": cl["kind"], "stream": cl["key"] if cl["kind"] == "stream" else None, "x": x, "r": r,
               "th": th, "mat": None, "zone": None}
        if cl["kind"] == "solid":
            out["solid"] = True
            out["mat"] = cl["mat"]
            return out
        out["solid"] = False
        if cl["kind"] == "stream":
            return self._sample_stream(x, r, th, cl, out)
        return self._sample_ext(x, r, th, out)

    def _sample_stream(self, x, r, th, cl, out):
        """Inside a stream: knots plus combustor, mixer, afterburner and wall layer (field.js:337-432)."""
        k = knot_at(self.kn[cl["key"]], x)
        c, sp = self.c, self.spec
        s = sp["s"]
        h = max(1e-6, cl["hi"] - cl["lo"])
        psi = (r - cl["lo"]) / h
        Tt, M = k["Tt"], k["M"]
        g, cp, R = k["g"], k["cp"], k["R"]
        zone = None
        cb = sp["comb"]
        if cb and cl["key"] == cb["stream"] and cb["x0"] <= x <= cb["turbEnd"]:
            Tt3, Tt4 = c["Tt3"], c["Tt4"]
            dT = max(0, Tt4 - Tt3)
            cosN = math.cos(cb["n"] * th)
            if x <= cb["x1"]:
                li, lo = cb["linerIn"].at(x), cb["linerOut"].at(x)
                if x < cb["xd"] or r < li or r > lo:
                    Tt = Tt3 * (1 + 0.012 * _smooth(cb["xd"], cb["x1"], x))
                    zone = "annulus"
                    M = 0.11
                else:
                    sN = (x - cb["xd"]) / (cb["x1"] - cb["xd"])
                    pl = (r - li) / max(1e-6, lo - li)
                    Tpz = min(Tt3 + 1.9 * dT, 2480, Tt3 + 1800)
                    if sN < 0.3:
                        Tline = Tt3 + (Tpz - Tt3) * _smooth(0.0, 0.26, sN)
                    else:
                        Tline = Tt4 + (Tpz - Tt4) * math.exp(-3.4 * (sN - 0.3) / 0.7)
                    amp = 0.55 if cb["cannular"] else 0.33
                    gP = (0.3 + 0.7 * math.exp(-(((pl - 0.5) / 0.24) ** 2))) * (1 + amp * cosN) / (1 + amp)
                    gE = 1 + 0.32 * (math.sin(math.pi * pl) - 2 / math.pi) + (0.14 if cb["cannular"] else 0.08) * cosN
                    G = _lerp(gP, gE, _smooth(0.28, 1, sN))
                    film = _smooth(0, 0.07, pl) * _smooth(0, 0.07, 1 - pl)
                    G *= 0.35 + 0.65 * film
                    Tt = Tt3 + (Tline - Tt3) * G
                    zone = "primary" if sN < 0.35 else "dilution"
                    M = _lerp(0.03, k["M"], _smooth(0, 0.7, sN))
            else:
                dec = math.exp(-(x - cb["x1"]) / (0.22 * s))
                pf = 0.32 * (math.sin(math.pi * psi) - 2 / math.pi) + (0.14 if cb["cannular"] else 0.08) * cosN
                Tt = k["Tt"] + dT * pf * dec * 0.9
        mx = sp["mixer"]
        if mx and cl["key"] == "ab":
            m = 1 - math.exp(-max(0, x - mx["x"]) / (0.5 * s))
            lo, hi = cl["lo"], cl["hi"]
            pa = (r * r - lo * lo) / max(1e-9, hi * hi - lo * lo)
            pc = mx["coreFrac"] + 0.13 * math.cos(mx["lobes"] * th) * (1 - m)
            w = 0.03 + 0.5 * m
            chi = 1 - _smooth(pc - w, pc + w, pa)
            Tloc = chi * c["Tt5"] + (1 - chi) * c["Tt13"]
            Tt = Tt + (1 - m) * (Tloc - c["Tt6A"])
            zone = zone or "mixer"
        ab = sp["ab"]
        if ab and cl["key"] == ab["stream"] and x > ab["xFH"] and c["abOn"]:
            Tt6 = c["Tt6A"] if sp["type"] == "lbtf" else c["Tt5"]
            L = ab["x1"] - ab["xFH"]
            t = (x - ab["xFH"]) / L
            F = 0
            spread = (x - ab["xFH"]) * math.tan(7 * DEG) + 0.004 * s
            for rg in ab["rings"]:
                F = max(F, 1 - _smooth(spread * 0.55, spread, abs(r - rg)))
            F = max(F, _smooth(0.45, 1.0, t))
            if x >= ab["x1"]:
                F = 1
            F *= _smooth(0, 0.035 * s, cl["hi"] - r) * 0.85 + 0.15
            meanT = k["Tt"]
            TtF = Tt6 + (c["Tt7"] - Tt6) * F
            Tt = meanT + (TtF - c["Tt7"]) if x >= ab["x1"] else TtF + (Tt - Tt6) * (1 - F)
            zone = "ab"
        kk = 1 + 0.5 * (g - 1) * M * M
        P = k["Pt"] / math.pow(1 + 0.5 * (g - 1) * k["M"] * k["M"], g / (g - 1))
        T = Tt / kk
        V = M * math.sqrt(g * R * T)
        d = min(psi, 1 - psi) * h
        dl = max(0.07 * h, 0.004 * s)
        if d < dl:
            u = math.pow(max(0, d) / dl, 1 / 7)
            V *= u
            T = Tt - V * V / (2 * cp)
        a = math.sqrt(g * R * T)
        sw = k["sw"] * DEG
        out.update(T=T, P=P, Tt=Tt, Pt=P * math.pow(Tt / T, g / (g - 1)), V=V, Vx=V * math.cos(sw),
                   Vth=V * math.sin(sw), M=V / a, a=a, rho=P / (R * T), g=g, cp=cp, R=R, psi=psi, zone=zone,
                   swirl=k["sw"])
        return out

    def _sample_ext(self, x, r, th, out):
        """Outside the engine: intake sink, nacelle shoulder, jets and shock cells (field.js:434-490)."""
        fl, sp = self.fl, self.spec
        C = E.GAS["cold"]
        g, cp, R = C["g"], C["cp"], E.Rg(C)
        U0, rl = fl["V0"], sp["lip"]["r"]
        U = U0
        lip = sp["lip"]
        dx = lip["x"] - x if x <= lip["x"] else (x - lip["x"]) * 4
        dr = max(0, r - rl)
        f = (1 - dx / math.sqrt(dx * dx + rl * rl)) * math.exp(-1.6 * (dr / rl) ** 2) * (
            1 if (r < lip["rOut"] * 1.02 or x < lip["x"]) else 0.4)
        U += (self.Uface - U0) * f
        if U0 > 1 and lip["x"] < x < sp["outerEnd"]:
            L = sp["outerEnd"] - lip["x"]
            dn = max(0, r - sp["outer"].at(x))
            U += 0.1 * U0 * math.sin(math.pi * (x - lip["x"]) / L) ** 2 * math.exp(-dn / (0.5 * rl))
        Tt, zone = fl["Tt0"], "free"
        qm = qh = 0.0
        wcore, shock = None, 0
        for e in self.exits:
            if x < e["x"]:
                continue
            dxe = x - e["x"]
            sig = 0.015 * e["R"] + e["spread"] * dxe
            w = blur_disk(r, e["R"], sig)
            if w <= 1e-6:
                continue
            qm += w * e["Qm"]
            qh += w * e["Qh"]
            if e["under"] and e["Ls"] > 0:
                env = math.exp(-dxe / (3.2 * e["Ls"])) * math.pow(w, 6)
                if env > 1e-3:
                    shock, wcore = env, e
        if qm != 0 or qh != 0:
            Uex = _sign(qm) * math.sqrt(abs(qm))
            sU = 2 * _sign(Uex or 1) if abs(Uex) < 2 else Uex
            dTt = _clamp(qh / sU, -self.maxdT, self.maxdT)
            U = U0 + Uex
            Tt = fl["Tt0"] + dTt
            zone = "jet"
        T = Tt - U * U / (2 * cp)
        P = fl["P0"]
        if zone == "free":
            P = fl["Pt0"] * math.pow(max(T, 1) / fl["Tt0"], g / (g - 1))
        if shock > 0:
            e = wcore
            dxe = x - e["x"]
            Pc = fl["P0"] * math.exp(math.log(e["P"] / fl["P0"]) * math.cos(2 * math.pi * dxe / e["Ls"])
                                     * math.exp(-dxe / (3.2 * e["Ls"])))
            ge, cpe = e["gas"]["g"], e["gas"]["cp"]
            Tiso = Tt * math.pow(min(1, Pc / e["Pt"]), (ge - 1) / ge)
            Uiso = math.sqrt(max(0, 2 * cpe * (Tt - Tiso)))
            b = min(1, shock)
            P = _lerp(P, Pc, b)
            U = _lerp(U, Uiso, b)
            T = Tt - U * U / (2 * cp)
            zone = "shock"
        T = max(T, 50)
        gg, cpp, RR = g, cp, R
        if zone != "free" and self.hot_gas:
            fr = _clamp((Tt - fl["Tt0"]) / self.maxdT, 0, 1)
            hg = self.hot_gas
            cpp = _lerp(cp, hg["cp"], fr)
            RR = _lerp(R, E.Rg(hg), fr)
            gg = cpp / (cpp - RR)
            T = max(50, Tt - U * U / (2 * cpp))
        a = math.sqrt(gg * RR * T)
        out.update(T=T, P=P, Tt=Tt, Pt=P * math.pow(Tt / T, gg / (gg - 1)), V=abs(U), Vx=U, Vth=0, M=abs(U) / a,
                   a=a, rho=P / (RR * T), g=gg, cp=cpp, R=RR, zone=zone, swirl=0)
        return out


# ---------------------------------------------------------------------------
# the solver's fixed states  (src/air_cfd.js:521-538)
# ---------------------------------------------------------------------------
def free_state(M, alpha_deg):
    """Normalised free stream (rho, rho u, rho v, rho w, E) (src/air_cfd.js:523-524)."""
    a = alpha_deg * DEG
    u, w = M * math.cos(a), M * math.sin(a)
    return [1, u, 0, w, 1 / (CG * (CG - 1)) + 0.5 * M * M]


def operating_point(ac, h, M, thr=1.0, ab=False, deck=None):
    """Field model of an aircraft's engine at (h, M, throttle) (src/app_air.js:349-354).

    `thr` is a number in (0, 1], as the app's manual and max settings give it (the 'level'
    setting: see `level_throttle`).  The afterburner is lit only on engines that have one.
    Returns (FieldModel, deck record); the model is None where the reference's constructor
    would throw.
    """
    eng = ac.eng
    deck = deck or EngineDeck.for_engine(eng["P"])
    ab = bool(ab) and ac.T["internal"]
    rop = deck.at(h, M, min(1, thr), ab)
    try:
        fm = FieldModel(ac.spec, {"op": rop["op"], "fl": E.flight_state(h, M), "ref": deck.ref},
                        deck.p(h, M, rop["op"].get("thr") or 1, ab))
    except (ArithmeticError, KeyError, TypeError, ValueError):
        fm = None
    return fm, rop


def fix_states(ac, h, M, alpha_deg, thr=1.0, ab=False, deck=None, fm=None):
    """The three fixed states [sink, jB, jC] that `applyCond` pushes (src/air_cfd.js:526-533).

    Each is (rho, rho u, 0, 0, E) in the solver's units (free-stream density 1, pressure 1/1.4):
    the field model's static state normalised by the free stream at altitude h.  A sample
    point that lands in a solid, or no field model, gives the free stream instead.
    Returns (F, [sink, jB, jC]).
    """
    F = free_state(M, alpha_deg)
    fs = fs_state(h, M)
    if fm is None:
        fm, _ = operating_point(ac, h, M, thr, ab, deck)
    sp = ac.spec
    s = sp["s"]

    def st(x, r):
        if fm is None:
            return None
        o = fm.sample(x, r, 0)
        if o["solid"]:
            return None
        rr = (o["P"] / fs["P"]) / (o["T"] / fs["T"])
        pp = (o["P"] / fs["P"]) / CG
        uu = o["Vx"] / fs["a"]
        return [rr, rr * uu, 0, 0, pp / (CG - 1) + 0.5 * rr * uu * uu]

    st2 = next((q for q in sp["stations"] if q["id"] == "2"), None)
    x2 = st2["x"] if st2 else sp["lip"]["x"] + 0.1 * s
    rin = sp["streams"].get("inlet") or sp["streams"].get("core")
    exB = next((q for q in sp["exitsGeom"] if q["key"] == "bypass"), None)
    exC = next((q for q in sp["exitsGeom"] if q["key"] != "bypass"), None)
    sink = st(x2 + 0.01 * s, 0.5 * (rin["lo"].at(x2) + rin["hi"].at(x2)) if rin else 0.3 * sp["lip"]["r"]) or F
    jB = (st(exB["x"] - 0.02 * s, 0.5 * (exB["R"] + exB["Rin"])) or F) if exB else F
    jC = (st(exC["x"] - 0.02 * s, 0.5 * (exC["R"] + (exC.get("Rin") or 0))) or F) if exC else F
    return F, [sink, jB, jC]
