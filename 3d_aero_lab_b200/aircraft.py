"""Parametric aircraft: the host-side geometry that the 3D solver is built from.

Restates the parts of the reference's aircraft model that reach the cut-cell grid:

* default dimensions of the three aircraft types (`src/aircraft.js:6-49`);
* NACA thickness and camber (`src/aircraft.js:58-59`);
* fuselage, lifting surfaces and `buildAircraft` (`src/aircraft.js:63-153`);
* the nacelle meridian of a podded engine (`src/aircraft.js:323-348`);
* the `AirGeom` attachment spans and bounding boxes (`src/air_field.js:104-114`).

`shape_of(ac)` packs everything the device-side inside tests need into the flat
`a3d_shape` record declared in `include/aero3d.h`.  In the reference this work
stays in the JavaScript host; here Python plays that role above the C ABI.
"""
from __future__ import annotations

import math

from . import engine as _engine

DEG = math.pi / 180  # src/field.js:7

AIRCRAFT_TYPES = {
    # default dimensions (src/aircraft.js:6-49); only entries that shape the body are kept
    "airliner": {"engine": "hbtf", "nEng": 2, "internal": False, "p": {
        "fusL": 37.6, "fusD": 3.95, "nose": 0.14, "tail": 0.30, "tailUp": 0.55, "noseP": 0.5,
        "wS": 122.6, "wB": 35.8, "wSweep": 27, "wTaper": 0.24, "wTcR": 0.15, "wTcT": 0.11, "wCamber": 0.02,
        "wDih": 5, "wInc": 2.0, "wX": 0.34, "wZ": -0.55,
        "hS": 31, "hB": 12.5, "hSweep": 32, "hTaper": 0.3, "hTc": 0.10, "hX": 0.80, "hZ": 0.15,
        "vS": 21.5, "vH": 5.9, "vSweep": 38, "vTaper": 0.3, "vTc": 0.10, "vX": 0.78,
        "engY": 0.34, "cg": 0.25}},
    "interceptor": {"engine": "tj", "nEng": 1, "internal": True, "p": {
        "fusL": 16.7, "fusD": 1.55, "nose": 0.28, "tail": 0.14, "tailUp": 0, "noseP": 0.85,
        "wS": 22, "wB": 7.4, "wSweep": 38, "wTaper": 0.35, "wTcR": 0.045, "wTcT": 0.04, "wCamber": 0,
        "wDih": -4, "wInc": 0, "wX": 0.47, "wZ": 0.0,
        "hS": 5.5, "hB": 3.9, "hSweep": 38, "hTaper": 0.35, "hTc": 0.045, "hX": 0.80, "hZ": -0.45,
        "vS": 4.6, "vH": 2.7, "vSweep": 42, "vTaper": 0.35, "vTc": 0.05, "vX": 0.72,
        "engY": 0, "cg": 0.20}},
    "fighter": {"engine": "lbtf", "nEng": 1, "internal": True, "p": {
        "fusL": 15.0, "fusD": 1.45, "nose": 0.26, "tail": 0.13, "tailUp": 0, "noseP": 0.75,
        "wS": 27.9, "wB": 9.45, "wSweep": 40, "wTaper": 0.23, "wTcR": 0.04, "wTcT": 0.04, "wCamber": 0,
        "wDih": 0, "wInc": 0, "wX": 0.40, "wZ": 0.0,
        "hS": 5.9, "hB": 5.6, "hSweep": 40, "hTaper": 0.3, "hTc": 0.04, "hX": 0.80, "hZ": -0.4,
        "vS": 5.1, "vH": 2.6, "vSweep": 47, "vTaper": 0.4, "vTc": 0.05, "vX": 0.70,
        "engY": 0, "cg": 0.30}},
}
NACELLE_NNX = 16  # 'medium' panel resolution used by tools/test_cfd3.js:5 (src/aircraft.js:52)


def naca_t(t, x):
    """NACA 4-digit half thickness, closed trailing edge (src/aircraft.js:58)."""
    x = max(0.0, min(1.0, x))
    return 5 * t * (0.2969 * math.sqrt(x) - 0.126 * x - 0.3516 * x * x + 0.2843 * x ** 3 - 0.1036 * x ** 4)


def naca_c(m, x, p=0.4):
    """NACA camber line (src/aircraft.js:59)."""
    if not m:
        return 0.0
    if x < p:
        return m / (p * p) * (2 * p * x - x * x)
    return m / ((1 - p) ** 2) * ((1 - 2 * p) + 2 * p * x - x * x)


class Fuselage:
    """Body of revolution with nose power law and cosine boat tail (src/aircraft.js:63-75)."""

    def __init__(self, p, end_r):
        self.L = p["fusL"]
        self.R0 = p["fusD"] / 2
        self.Ln = p["nose"] * self.L
        self.Lt = p["tail"] * self.L
        self.xt0 = self.L - self.Lt
        self.Re = min(end_r, self.R0 * 0.95)
        self.noseP = p["noseP"]
        self.tailUp = p["tailUp"]

    def R(self, x):
        if x <= 0:
            return 0.0
        if x < self.Ln:
            s = 1 - x / self.Ln
            return self.R0 * math.pow(max(0.0, 1 - s * s), self.noseP)
        if x <= self.xt0:
            return self.R0
        if x >= self.L:
            return self.Re
        t = (x - self.xt0) / self.Lt
        return self.Re + (self.R0 - self.Re) * 0.5 * (1 + math.cos(math.pi * t))

    def zc(self, x):
        return 0.0 if x <= self.xt0 else self.tailUp * self.R0 * ((x - self.xt0) / self.Lt) ** 2


class Surface:
    """Trapezoidal lifting surface (src/aircraft.js:78-102)."""

    def __init__(self, **o):
        self.o = o
        self.vertical = bool(o.get("vertical"))
        self.semi = o["b"] if self.vertical else o["b"] / 2
        self.cr = 2 * o["S"] / (o["b"] * (1 + o["taper"]))
        self.ct = self.cr * o["taper"]
        self.tanL = math.tan(o["sweep"] * math.pi / 180)
        self.tanD = math.tan((o.get("dih") or 0) * math.pi / 180)
        self.tanI = math.tan((o.get("inc") or 0) * math.pi / 180)
        t = o["taper"]
        self.mac = (2 / 3) * self.cr * (1 + t + t ** 2) / (1 + t)
        self.sMac = self.semi / 3 * (1 + 2 * t) / (1 + t)
        self.xMac = self.xLE(self.sMac)

    def chord(self, s):
        return self.cr + (self.ct - self.cr) * s / self.semi

    def xLE(self, s):
        return self.o["x0"] + s * self.tanL

    def tc(self, s):
        return self.o["tcR"] + (self.o["tcT"] - self.o["tcR"]) * s / self.semi

    def pt(self, s, xc, side, s_att=0, tip_zero=False):
        c = self.chord(s)
        x = self.xLE(s) + xc * c
        th = naca_t(self.tc(s), xc) * c
        if tip_zero:
            th = 0
        cam = naca_c(self.o.get("camber") or 0, xc) * c
        shear = -(xc - 0.25) * c * self.tanI
        if self.vertical:
            return [x, side * th, self.o["z0"] + s + 0 * cam]
        z = self.o["z0"] + (s - (s_att or 0)) * self.tanD + cam + shear + side * th
        return [x, s, z]


class Aircraft:
    """Assembled half model: the fields the CFD grid and geometry read."""


def build_aircraft(typ, p=None, eng=None):
    """Assemble fuselage, surfaces and engine installation (src/aircraft.js:108-153)."""
    T = AIRCRAFT_TYPES[typ]
    p = dict(T["p"], **(p or {}))
    if eng is None:
        eng = _engine.engine_for(typ, T["engine"])
    spec = eng["spec"]
    end_r = 0.06 * p["fusD"] / 2
    if T["internal"]:
        cas_r = max(q[1] for q in spec["outer"].pts)
        p["fusD"] = max(p["fusD"], 2 * (cas_r + 0.06))
        end_r = spec["outer"].at(spec["outerEnd"]) + 0.01
    fus = Fuselage(p, end_r)
    R0 = fus.R0
    wing = Surface(S=p["wS"], b=p["wB"], sweep=p["wSweep"], taper=p["wTaper"], tcR=p["wTcR"], tcT=p["wTcT"],
                   camber=p["wCamber"], dih=p["wDih"], inc=p["wInc"], x0=p["wX"] * fus.L, z0=p["wZ"] * R0)
    hx0 = p["hX"] * fus.L
    hz0 = fus.zc(hx0 + 1) + p["hZ"] * fus.R(hx0 + 1)
    htail = Surface(S=p["hS"], b=p["hB"], sweep=p["hSweep"], taper=p["hTaper"], tcR=p["hTc"], tcT=p["hTc"],
                    camber=0, dih=0, inc=0, x0=hx0, z0=hz0)
    vx0 = p["vX"] * fus.L
    vtail = Surface(S=p["vS"], b=p["vH"], sweep=p["vSweep"], taper=p["vTaper"], tcR=p["vTc"], tcT=p["vTc"],
                    vertical=True, x0=vx0, z0=0)
    vxm = vx0 + 0.5 * vtail.cr
    vtail.o["z0"] = fus.zc(vxm) + fus.R(vxm) * 0.85
    engines = []
    if T["internal"]:
        engines.append({"x0": fus.L - spec["outerEnd"], "y": 0.0, "z": 0.0, "internal": True})
    else:
        ye = p["engY"] * wing.semi
        Lnac, Rn = spec["outerEnd"], spec["view"]["Rmax"]
        x_lip = wing.xLE(ye) - Lnac + 0.35 * wing.chord(ye) * 0.25
        zw = wing.pt(ye, 0.02, -1, R0)[2]
        engines.append({"x0": x_lip, "y": ye, "z": zw - Rn - 0.28, "internal": False})
    ac = Aircraft()
    ac.type, ac.T, ac.p, ac.fus, ac.wing, ac.htail, ac.vtail = typ, T, p, fus, wing, htail, vtail
    ac.engines, ac.spec, ac.eng = engines, spec, eng
    xcg = wing.xMac + p["cg"] * wing.mac
    ac.ref = {"S": p["wS"], "b": p["wB"], "c": wing.mac, "xcg": xcg, "zcg": 0.0}
    for e in engines:
        if not e["internal"]:
            e["meridian"] = nacelle_meridian(spec)
    return ac


def nacelle_meridian(spec, nx=NACELLE_NNX):
    """Outer meridian of a podded nacelle, lip to plug tip (src/aircraft.js:325-336)."""
    hub, cowl, nac_out = spec["lines"]["hub"], spec["lines"]["cowl"], spec["lines"]["nacOut"]
    lip, xB = spec["lip"], spec["outerEnd"]
    exB, exC = spec["exitsGeom"][0], spec["exitsGeom"][1]
    mer = []

    def add_line(f, a, b, n):
        for k in range(1, n + 1):
            x = a + (b - a) * k / n
            mer.append([x, f(x)])

    mer.append([lip["x"], 0])
    mer.append([lip["x"], lip["r"] * 0.5])
    mer.append([lip["x"], lip["r"]])
    mer.append([lip["x"] + 0.02 * xB, lip["rOut"]])
    add_line(nac_out.at, lip["x"] + 0.02 * xB, xB, _js_round(nx * 0.55))
    mer.append([xB, 0.5 * (exB["R"] + exB["Rin"])])
    mer.append([xB, cowl.at(xB)])
    add_line(cowl.at, xB, exC["x"], _js_round(nx * 0.25))
    mer.append([exC["x"], hub.at(exC["x"])])
    add_line(hub.at, exC["x"], exC.get("plugTip") or exC["x"] + 0.3, _js_round(nx * 0.2))
    mer[-1][1] = 0
    return mer


def _js_round(v):
    """JavaScript Math.round: halves round toward +infinity."""
    return int(math.floor(v + 0.5))


def nacelle_envelope(mer, n=300):
    """Radius table of the nacelle outer envelope, stored in float32 (src/air_cfd.js:52-56)."""
    import numpy as np
    xmax = mer[-1][0]
    R = np.zeros(n + 1, dtype=np.float32)
    for k in range(n + 1):
        xe = xmax * k / n
        r = 0.0
        for q in range(len(mer) - 1):
            xa, ra = mer[q]
            xb, rb = mer[q + 1]
            if min(xa, xb) - 1e-9 <= xe <= max(xa, xb) + 1e-9:
                r = max(r, ra + (rb - ra) * (xe - xa) / (xb - xa) if xb > xa else max(ra, rb))
        R[k] = r
    return xmax, R


def attach_span(fus, S):
    """Span where a lifting surface leaves the fuselage (src/air_field.js:107)."""
    s_att = fus.R((S.xLE(fus.R0) * 2 + S.chord(fus.R0)) / 2) * 0.98
    return min(s_att, S.semi * 0.5)


def surface_bbox(S):
    """x/z bounding box of a lifting surface plus 20 % root chord (src/air_field.js:109)."""
    x0, x1, z0, z1 = math.inf, -math.inf, math.inf, -math.inf
    for k in range(11):
        s = S.semi * k / 10
        for xc in (0, 1):
            for sd in (-1, 1):
                q = S.pt(s, xc, sd, 0)
                x0, x1 = min(x0, q[0]), max(x1, q[0])
                z0, z1 = min(z0, q[2]), max(z1, q[2])
    return [x0, x1, z0 - 0.2 * S.cr, z1 + 0.2 * S.cr]


def trefftz_x(ac):
    """Trefftz plane station behind the tail (src/air_cfd.js:561)."""
    ht = ac.htail
    return max(ac.fus.L, ht.xLE(ht.semi) + ht.ct) + 0.12 * ac.fus.L


def shape_of(ac):
    """Pack the aircraft into the C `a3d_shape` record (include/aero3d.h)."""
    from .abi import a3d_shape
    sh = a3d_shape()
    f = ac.fus
    sh.fus_L, sh.fus_R0, sh.fus_Ln, sh.fus_Lt = f.L, f.R0, f.Ln, f.Lt
    sh.fus_xt0, sh.fus_Re, sh.fus_noseP, sh.fus_tailUp = f.xt0, f.Re, f.noseP, f.tailUp
    s_w, s_h = attach_span(f, ac.wing), attach_span(f, ac.htail)
    for dst, S, sA, bb in ((sh.wing, ac.wing, s_w, surface_bbox(ac.wing)),
                           (sh.htail, ac.htail, s_h, surface_bbox(ac.htail)),
                           (sh.vtail, ac.vtail, 0.0, [0.0, 0.0, 0.0, 0.0])):
        o = S.o
        dst.x0, dst.z0, dst.semi, dst.cr, dst.ct = o["x0"], o["z0"], S.semi, S.cr, S.ct
        dst.tanL, dst.tanD_pt, dst.tanI_pt = S.tanL, S.tanD, S.tanI
        dst.tanD_deg = math.tan((o.get("dih") or 0) * DEG)
        dst.tanI_deg = math.tan((o.get("inc") or 0) * DEG)
        dst.tcR, dst.tcT, dst.camber = o["tcR"], o["tcT"], float(o.get("camber") or 0)
        dst.sA = sA
        for i in range(4):
            dst.bb[i] = bb[i]
    sp = ac.spec
    sh.ref_b = ac.ref["b"]
    sh.view_Rmax = sp["view"]["Rmax"]
    sh.lip_x, sh.lip_r = sp["lip"]["x"], sp["lip"]["r"]
    sh.n_engines = len(ac.engines)
    for i, e in enumerate(ac.engines):
        de = sh.engines[i]
        de.x0, de.y, de.z, de.internal = e["x0"], e["y"], e["z"], 1 if e["internal"] else 0
        if not e["internal"] and e.get("meridian"):
            xmax, R = nacelle_envelope(e["meridian"])
            de.env_n, de.env_xmax = 300, xmax
            for k in range(301):
                de.env_R[k] = float(R[k])
        else:
            de.env_n, de.env_xmax = 0, 0.0
    sh.n_exits = len(sp["exitsGeom"])
    for i, ex in enumerate(sp["exitsGeom"]):
        dx = sh.exits[i]
        dx.type = 4 if ex["key"] == "bypass" else 5
        dx.x, dx.R, dx.Rin = ex["x"], ex["R"], ex.get("Rin") or 0.0
    return sh
