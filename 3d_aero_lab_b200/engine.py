"""Engine cycle and flow-path specification: the host-side inputs of the 3D solver.

The 3D Euler solver needs two things from the engine:

* geometry: the nozzle throat and exit radii r8/r9 (which size the casing of an internal
  engine and therefore the fuselage end radius), the exit rings that become fixed-state jet
  cells, the intake lip that becomes the inlet sink layer, and the outer casing/nacelle
  outline;
* the fixed states of those cells, which the reference samples from its engine field model
  at the current operating point (`field.py`); the field model reads the station table of
  the cycle and the full flow path (streams, blade rows, combustor, afterburner, bodies).

These come from the reference's 1-D cycle (`src/physics.js`) and from its flow-path
specification (`src/geometry.js`); the geometry is sized at the sea-level static design point
(`tools/airlib.js:6-11`).  Display-only parts of the specification (component names, chart
lists, view and plotting domains) are left out.

All arithmetic is IEEE double, in the same operation order as the reference so that
the outline coordinates agree to the last bit where the reference's own expression
order allows it.
"""
from __future__ import annotations

import math

# ---------------------------------------------------------------------------
# gas model and ISA  (src/physics.js:6-27)
# ---------------------------------------------------------------------------
GAS = {
    "cold": {"g": 1.4, "cp": 1004.5},
    "hot": {"g": 1.33, "cp": 1156.9},
    "ab": {"g": 1.30, "cp": 1243.0},
}


def Rg(gas):
    """Gas constant from cp and gamma (src/physics.js:11)."""
    return gas["cp"] * (gas["g"] - 1) / gas["g"]


def mix_gas(m1, g1, m2, g2):
    """Mass-weighted mixture of two gases (src/physics.js:12-16)."""
    cp = (m1 * g1["cp"] + m2 * g2["cp"]) / (m1 + m2)
    R = (m1 * Rg(g1) + m2 * Rg(g2)) / (m1 + m2)
    return {"g": cp / (cp - R), "cp": cp}


def isa(h):
    """ISA atmosphere 0-20 km (src/physics.js:19-26)."""
    h = max(0.0, min(20000.0, h))
    if h <= 11000:
        T = 288.15 - 0.0065 * h
        P = 101325 * math.pow(T / 288.15, 5.25588)
    else:
        T = 216.65
        P = 22632.06 * math.exp(-(h - 11000) / 6341.62)
    R, g = 287.05, 1.4
    return {"T": T, "P": P, "rho": P / (R * T), "a": math.sqrt(g * R * T)}


def mfp(M, g, R):
    """Mass-flow parameter mdot*sqrt(Tt)/(Pt*A) (src/physics.js:29-31)."""
    return M * math.sqrt(g / R) * math.pow(1 + 0.5 * (g - 1) * M * M, -(g + 1) / (2 * (g - 1)))


def area_ratio(M, g):
    """A/A* (src/physics.js:43-45)."""
    return (1 / M) * math.pow((2 / (g + 1)) * (1 + 0.5 * (g - 1) * M * M), (g + 1) / (2 * (g - 1)))


def mach_from_npr(npr, g):
    """Isentropic exit Mach for a pressure ratio (src/physics.js:46)."""
    return 0.0 if npr <= 1 else math.sqrt(2 / (g - 1) * (math.pow(npr, (g - 1) / g) - 1))


def crit_npr(g):
    """Critical (choking) pressure ratio (src/physics.js:47)."""
    return math.pow((g + 1) / 2, g / (g - 1))


def static_from_total(Tt, Pt, M, gas):
    """Static state from total state and Mach (src/physics.js:48-54)."""
    g, R = gas["g"], Rg(gas)
    k = 1 + 0.5 * (g - 1) * M * M
    T = Tt / k
    P = Pt / math.pow(k, g / (g - 1))
    a = math.sqrt(g * R * T)
    return {"T": T, "P": P, "a": a, "V": M * a, "rho": P / (R * T)}


def comp_pi(tau, gas, e):
    return math.pow(tau, gas["g"] * e / (gas["g"] - 1))


def comp_tau(pi, gas, e):
    return math.pow(pi, (gas["g"] - 1) / (gas["g"] * e))


def turb_pi(tau, gas, e):
    return math.pow(tau, gas["g"] / ((gas["g"] - 1) * e))


def turb_tau(pi, gas, e):
    return math.pow(pi, (gas["g"] - 1) * e / gas["g"])


def nozzle(mdot, Tt, Pt, P0, gas, typ, ar_max=None):
    """Nozzle exit state, area and throat area (src/physics.js:63-83)."""
    g, R = gas["g"], Rg(gas)
    npr = Pt / P0
    crit = crit_npr(g)
    choked = npr >= crit
    if npr <= 1.0005:
        M, P = 0.03, P0
    elif not choked:
        M, P = mach_from_npr(npr, g), P0
    elif typ == "conv":
        M, P = 1.0, Pt / crit
    else:
        M, P = mach_from_npr(npr, g), P0
        if ar_max and area_ratio(M, g) > ar_max:
            lo, hi = 1.0, M
            for _ in range(40):
                m = 0.5 * (lo + hi)
                if area_ratio(m, g) < ar_max:
                    lo = m
                else:
                    hi = m
            M = lo
            P = Pt / math.pow(1 + 0.5 * (g - 1) * M * M, g / (g - 1))
    s = static_from_total(Tt, Pt, M, gas)
    A = mdot / (s["rho"] * s["V"])
    Athroat = mdot * math.sqrt(Tt) / (Pt * mfp(1, g, R)) if choked else A
    return {"M": M, "P": P, "T": s["T"], "V": s["V"], "rho": s["rho"], "A": A,
            "Athroat": Athroat, "choked": choked, "npr": npr, "crit": crit, "Tt": Tt, "Pt": Pt,
            "gas": gas, "mdot": mdot, "type": typ}


ENGINE_TYPES = {
    # design-point tables (src/physics.js:86-105)
    "hbtf": {"design": {"mdot": 350, "opr": 32, "fpr": 1.6, "bpr": 5.5, "pibst": 1.8, "Tt4max": 1650},
             "hasAB": False, "nozzle": "conv", "arMax": None},
    "tj": {"design": {"mdot": 77, "opr": 13.5, "Tt4max": 1280},
           "hasAB": True, "nozzle": "cd", "arMax": 1.9},
    "lbtf": {"design": {"mdot": 110, "opr": 26, "fpr": 3.8, "Tt4max": 1680},
             "hasAB": True, "nozzle": "cd", "arMax": 1.8},
}
DEFAULT_EFF = {  # src/physics.js:106-110
    "ef": 0.89, "ec": 0.90, "et": 0.90, "etab": 0.99, "etb": 0.99, "pib": 0.96, "pidmax": 0.99,
    "pin": 0.99, "pifn": 0.99, "etam": 0.99, "LHV": 43.0e6, "pifd": 0.98, "piM": 0.98,
    "piabOn": 0.95, "piabOff": 0.98, "etaAB": 0.95,
}


def flight_state(alt, M0):
    """Free-stream totals (src/physics.js:113-120)."""
    a = isa(alt)
    g = GAS["cold"]["g"]
    k = 1 + 0.5 * (g - 1) * M0 * M0
    Tt0 = a["T"] * k
    Pt0 = a["P"] * math.pow(k, g / (g - 1))
    etaR = 1 if M0 <= 1 else 1 - 0.075 * math.pow(M0 - 1, 1.35)
    return {"alt": alt, "M0": M0, "T0": a["T"], "P0": a["P"], "rho0": a["rho"], "a0": a["a"],
            "V0": M0 * a["a"], "Tt0": Tt0, "Pt0": Pt0, "etaR": etaR}


def _afterburner_and_nozzle(r, p, fl, m6, Tt6, Pt6, gas6):
    """Afterburner and final nozzle (src/physics.js:320-335)."""
    e = p["eff"]
    Tt7, gas7, mfAB = Tt6, gas6, 0.0
    ab_on = bool(p["ab"] and ENGINE_TYPES[p["type"]]["hasAB"] and p["Tt7"] > Tt6 + 20)
    if ab_on:
        A = GAS["ab"]
        fab = (A["cp"] * p["Tt7"] - gas6["cp"] * Tt6) / (e["etaAB"] * e["LHV"] - A["cp"] * p["Tt7"])
        mfAB = m6 * fab
        Tt7 = p["Tt7"]
        Pt7 = Pt6 * e["piabOn"]
        gas7 = A
    else:
        Pt7 = Pt6 * e["piabOff"]
    m7 = m6 + mfAB
    S = r["S"]
    S.setdefault("6", {"Tt": Tt6, "Pt": Pt6, "gas": gas6})
    S["7"] = {"Tt": Tt7, "Pt": Pt7, "gas": gas7}
    S["9"] = {"Tt": Tt7, "Pt": Pt7 * e["pin"], "gas": gas7}
    r["noz"] = nozzle(m7, Tt7, Pt7 * e["pin"], fl["P0"], gas7, p.get("nozzleType") or "cd",
                      ENGINE_TYPES[p["type"]]["arMax"])
    r.update(abOn=ab_on, Tt7=Tt7, Pt7=Pt7, gas7=gas7, mfAB=mfAB, m7=m7, Tt6=Tt6, Pt6=Pt6)


def _finish_performance(r, p, fl, mdot, mfuel, nozzles):
    """Net thrust and fuel flow (src/physics.js:337-355)."""
    V0 = fl["V0"]
    F = -mdot * V0
    for n in nozzles:
        Fn = n["mdot"] * n["V"] + n["A"] * (n["P"] - fl["P0"])
        F += Fn
        n["F"] = Fn
    r["F"] = F
    r["mfuel"] = mfuel


def run_cycle(p, ref, fl, Tt4):
    """Station-by-station cycle, design point (ref None) or off-design (src/physics.js:127-318).

    Returns the station table `S` (total temperature, total pressure and gas per station id),
    the component ratios, mass flows, nozzles, thrust and fuel flow.  The warning strings of
    the reference are left out.
    """
    e, d, C, H = p["eff"], p["design"], GAS["cold"], GAS["hot"]
    cpc, cpt = C["cp"], H["cp"]
    Tt2 = fl["Tt0"]
    pid = e["pidmax"] * fl["etaR"]
    Pt2 = fl["Pt0"] * pid

    def fuel_air(Tt3):
        return (cpt * Tt4 - cpc * Tt3) / (e["etb"] * e["LHV"] - cpt * Tt4)

    S = {"0": {"Tt": fl["Tt0"], "Pt": fl["Pt0"], "gas": C}, "2": {"Tt": Tt2, "Pt": Pt2, "gas": C}}
    r = {"type": p["type"], "Tt4": Tt4, "Tt2": Tt2, "Pt2": Pt2, "pid": pid, "fl": fl, "S": S}

    if p["type"] == "tj":
        if ref is None:
            pic = d["opr"]
            tauc = comp_tau(pic, C, e["ec"])
            Tt3 = Tt2 * tauc
            f = fuel_air(Tt3)
            tauT = 1 - cpc * Tt2 * (tauc - 1) / (e["etam"] * (1 + f) * cpt * Tt4)
            piT = turb_pi(tauT, H, e["et"])
            mdot = d["mdot"]
        else:
            tauT, piT, f = ref["tauT"], ref["piT"], ref["f"]
            for _ in range(6):
                tauc = 1 + e["etam"] * (1 + f) * cpt * Tt4 * (1 - tauT) / (cpc * Tt2)
                Tt3 = Tt2 * tauc
                f = fuel_air(Tt3)
            pic = comp_pi(tauc, C, e["ec"])
        Pt3 = Pt2 * pic
        Pt4 = Pt3 * e["pib"]
        if ref is not None:
            mdot = ref["mdot"] * (Pt4 / ref["Pt4"]) * math.sqrt(ref["Tt4"] / Tt4) * (1 + ref["f"]) / (1 + f)
        Tt5 = Tt4 * tauT
        Pt5 = Pt4 * piT
        S.update({"3": {"Tt": Tt3, "Pt": Pt3, "gas": C}, "4": {"Tt": Tt4, "Pt": Pt4, "gas": H},
                  "5": {"Tt": Tt5, "Pt": Pt5, "gas": H}})
        r.update(tauc=tauc, pic=pic, opr=pic, f=f, tauT=tauT, piT=piT, mdot=mdot, mcore=mdot, bpr=0,
                 Tt3=Tt3, Pt3=Pt3, Pt4=Pt4, Tt5=Tt5, Pt5=Pt5, spool={"HP": math.sqrt(Tt2 * (tauc - 1))})
        _afterburner_and_nozzle(r, p, fl, mdot * (1 + f), Tt5, Pt5, H)
        _finish_performance(r, p, fl, mdot, mdot * f + r["mfAB"], [r["noz"]])
        return r

    mixed = p["type"] == "lbtf"
    if ref is None:
        pif = d["fpr"]
        tauf = comp_tau(pif, C, e["ef"])
        pibst = 1 if mixed else d["pibst"]
        taubst = comp_tau(pibst, C, e["ec"])
        picH = d["opr"] / (pif * pibst)
        if picH < 1.2:
            picH = max(1.2, picH)
        taucH = comp_tau(picH, C, e["ec"])
        Tt25 = Tt2 * tauf * taubst
        Tt3 = Tt25 * taucH
        f = fuel_air(Tt3)
        tautH = 1 - cpc * Tt25 * (taucH - 1) / (e["etam"] * (1 + f) * cpt * Tt4)
        pitH = turb_pi(tautH, H, e["et"])
        Pt4 = Pt2 * pif * pibst * picH * e["pib"]
        Tt45 = Tt4 * tautH
        Pt45 = Pt4 * pitH
        if mixed:
            Pt16 = Pt2 * pif * e["pifd"]
            pitL = Pt16 / Pt45
            if pitL >= 0.98:
                pitL = 0.9
            tautL = turb_tau(pitL, H, e["et"])
            W = e["etam"] * (1 + f) * cpt * Tt45 * (1 - tautL)
            alpha = W / (cpc * Tt2 * (tauf - 1)) - 1
            if alpha < 0.05:
                alpha = 0.05
            kb = 0
        else:
            alpha = d["bpr"]
            kb = (taubst - 1) * tauf / (tauf - 1)
            W = cpc * Tt2 * ((1 + alpha) * (tauf - 1) + tauf * (taubst - 1))
            tautL = 1 - W / (e["etam"] * (1 + f) * cpt * Tt45)
            if tautL < 0.25:
                tautL = 0.25
            pitL = turb_pi(tautL, H, e["et"])
        mcore = d["mdot"] / (1 + alpha)
    elif mixed:
        tautH, pitH, kb, taubst, pibst = ref["tautH"], ref["pitH"], 0, 1, 1

        def eval_tf(tf):
            ff, tcH, T3 = ref["f"], 1, Tt2
            pf = comp_pi(tf, C, e["ef"])
            T25 = Tt2 * tf
            for _ in range(6):
                tcH = 1 + e["etam"] * (1 + ff) * cpt * Tt4 * (1 - tautH) / (cpc * T25)
                T3 = T25 * tcH
                ff = fuel_air(T3)
            pcH = comp_pi(tcH, C, e["ec"])
            P4 = Pt2 * pf * pcH * e["pib"]
            mc = ref["mcore"] * (P4 / ref["Pt4"]) * math.sqrt(ref["Tt4"] / Tt4) * (1 + ref["f"]) / (1 + ff)
            m0 = ref["mdot"] * math.sqrt(max(1e-6, (tf - 1) / (ref["tauf"] - 1))) * (Pt2 / ref["Pt2"]) * math.sqrt(ref["Tt2"] / Tt2)
            al = max(0.02, m0 / mc - 1)
            T45 = Tt4 * tautH
            P45 = P4 * pitH
            tL = 1 - (1 + al) * cpc * Tt2 * (tf - 1) / (e["etam"] * (1 + ff) * cpt * T45)
            tL = max(0.3, min(0.995, tL))
            pL = turb_pi(tL, H, e["et"])
            res = Pt2 * pf * e["pifd"] - P45 * pL
            return {"res": res, "tf": tf, "pf": pf, "tcH": tcH, "pcH": pcH, "T3": T3, "ff": ff,
                    "mc": mc, "al": al, "tL": tL, "pL": pL}

        lo = 1.003
        hi = max(1.05, (ref["tauf"] - 1) * 2.2 + 1)
        a = eval_tf(lo)
        b = eval_tf(hi)
        mid = None
        if a["res"] > 0:
            mid = a
        elif b["res"] < 0:
            mid = b
        else:
            for _ in range(50):
                m = eval_tf(0.5 * (lo + hi))
                if m["res"] > 0:
                    hi = m["tf"]
                else:
                    lo = m["tf"]
                mid = m
                if hi - lo < 1e-7:
                    break
        tauf, pif, taucH, picH, Tt3, f = mid["tf"], mid["pf"], mid["tcH"], mid["pcH"], mid["T3"], mid["ff"]
        mcore, alpha, tautL, pitL = mid["mc"], mid["al"], mid["tL"], mid["pL"]
    else:
        tautH, pitH, tautL, pitL, kb = ref["tautH"], ref["pitH"], ref["tautL"], ref["pitL"], ref["kb"]
        tauf, alpha, f = ref["tauf"], ref["bpr"], ref["f"]
        for _ in range(80):
            pif = comp_pi(tauf, C, e["ef"])
            taubst = 1 + kb * (tauf - 1) / tauf
            pibst = comp_pi(taubst, C, e["ec"])
            Tt25 = Tt2 * tauf * taubst
            taucH = 1 + e["etam"] * (1 + f) * cpt * Tt4 * (1 - tautH) / (cpc * Tt25)
            picH = comp_pi(taucH, C, e["ec"])
            Tt3 = Tt25 * taucH
            f = fuel_air(Tt3)
            Pt4 = Pt2 * pif * pibst * picH * e["pib"]
            mcore = ref["mcore"] * (Pt4 / ref["Pt4"]) * math.sqrt(ref["Tt4"] / Tt4) * (1 + ref["f"]) / (1 + f)
            # fixed-area convergent core nozzle sets the LP turbine pressure ratio
            Pt45 = Pt4 * pitH
            Tt45 = Tt4 * tautH
            m5 = mcore * (1 + f)
            lo, hi = 0.03, 0.999
            for _ in range(44):
                mid = 0.5 * (lo + hi)
                tau = turb_tau(mid, H, e["et"])
                Pt9 = Pt45 * mid * e["pin"]
                n = nozzle(1, Tt45 * tau, Pt9, fl["P0"], H, "conv")
                cap = ref["A9core"] * Pt9 * mfp(n["M"], H["g"], Rg(H)) / math.sqrt(Tt45 * tau)
                if cap > m5:
                    hi = mid
                else:
                    lo = mid
            pitL = 0.5 * (lo + hi)
            tautL = turb_tau(pitL, H, e["et"])
            Tt13 = Tt2 * tauf
            Pt13 = Pt2 * pif
            n = nozzle(1, Tt13, Pt13 * e["pifn"], fl["P0"], C, "conv")
            mfp_ratio = mfp(n["M"], C["g"], Rg(C)) / ref["mfp19"]
            mbyp = ref["mbyp"] * (Pt13 / ref["Pt13"]) * math.sqrt(ref["Tt13"] / Tt13) * mfp_ratio
            a_new = max(0.02, mbyp / mcore)
            W = e["etam"] * (1 + f) * cpt * Tt4 * tautH * (1 - tautL)
            y = W / (cpc * Tt2 * (1 + a_new + kb))
            t_new = 1 + y
            dt = abs(t_new - tauf) + abs(a_new - alpha) * 0.01
            tauf = 0.5 * tauf + 0.5 * t_new
            alpha = 0.5 * alpha + 0.5 * a_new
            if dt < 1e-9:
                break
        pif = comp_pi(tauf, C, e["ef"])
        taubst = 1 + kb * (tauf - 1) / tauf
        pibst = comp_pi(taubst, C, e["ec"])

    Tt13 = Tt2 * tauf
    Pt13 = Pt2 * pif
    Tt25 = Tt13 * taubst
    Pt25 = Pt13 * pibst
    Tt3 = Tt25 * taucH
    Pt3 = Pt25 * picH
    Pt4 = Pt3 * e["pib"]
    Tt45 = Tt4 * tautH
    Pt45 = Pt4 * pitH
    Tt5 = Tt45 * tautL
    Pt5 = Pt45 * pitL
    mdot = mcore * (1 + alpha)
    mbyp = mcore * alpha
    S.update({"13": {"Tt": Tt13, "Pt": Pt13, "gas": C}, "21": {"Tt": Tt13, "Pt": Pt13, "gas": C},
              "25": {"Tt": Tt25, "Pt": Pt25, "gas": C}, "3": {"Tt": Tt3, "Pt": Pt3, "gas": C},
              "4": {"Tt": Tt4, "Pt": Pt4, "gas": H}, "45": {"Tt": Tt45, "Pt": Pt45, "gas": H},
              "5": {"Tt": Tt5, "Pt": Pt5, "gas": H}})
    r.update(tauf=tauf, pif=pif, taubst=taubst, pibst=pibst, taucH=taucH, picH=picH,
             opr=pif * pibst * picH, f=f, tautH=tautH, pitH=pitH, tautL=tautL, pitL=pitL, kb=kb,
             bpr=alpha, mdot=mdot, mcore=mcore, mbyp=mbyp, Tt3=Tt3, Pt3=Pt3, Pt4=Pt4, Tt13=Tt13,
             Pt13=Pt13, Tt25=Tt25, Pt25=Pt25, Tt45=Tt45, Pt45=Pt45, Tt5=Tt5, Pt5=Pt5,
             spool={"LP": math.sqrt(Tt2 * (tauf - 1)), "HP": math.sqrt(Tt25 * (taucH - 1))})
    m5 = mcore * (1 + f)
    if not mixed:
        nc = nozzle(m5, Tt5, Pt5 * e["pin"], fl["P0"], H, "conv")
        nb = nozzle(mbyp, Tt13, Pt13 * e["pifn"], fl["P0"], C, "conv")
        S["9"] = {"Tt": Tt5, "Pt": Pt5 * e["pin"], "gas": H}
        S["19"] = {"Tt": Tt13, "Pt": Pt13 * e["pifn"], "gas": C}
        r["noz"] = nc
        r["nozB"] = nb
        r["mfp19"] = mfp(nb["M"], C["g"], Rg(C))
        if ref is None:
            r["A9core"] = nc["A"]
        _finish_performance(r, p, fl, mdot, mcore * f, [nc, nb])
    else:
        Pt16 = Pt13 * e["pifd"]
        S["16"] = {"Tt": Tt13, "Pt": Pt16, "gas": C}
        mix = mix_gas(m5, H, mbyp, C)
        Tt6A = (m5 * H["cp"] * Tt5 + mbyp * C["cp"] * Tt13) / ((m5 + mbyp) * mix["cp"])
        Pt6A = (m5 * Pt5 + mbyp * Pt16) / (m5 + mbyp) * e["piM"]
        S["6A"] = {"Tt": Tt6A, "Pt": Pt6A, "gas": mix}
        r.update(Pt16=Pt16, Tt6A=Tt6A, Pt6A=Pt6A, mixGas=mix)
        _afterburner_and_nozzle(r, p, fl, m5 + mbyp, Tt6A, Pt6A, mix)
        _finish_performance(r, p, fl, mdot, mcore * f + r["mfAB"], [r["noz"]])
    return r


def solve_engine(p):
    """Design point, then the operating point with the 105 % spool-speed limit (src/physics.js:359-391)."""
    fl_ref = flight_state(0, 0)
    p_ref = dict(p, ab=False)
    ref = run_cycle(p_ref, None, fl_ref, p["design"]["Tt4max"])
    fl = flight_state(p["alt"], p["M0"])
    Tt4cmd = p["design"]["Tt4max"] * p["thr"]
    op = run_cycle(p, ref, fl, Tt4cmd)
    Nmax = 1.05
    op["limited"] = False

    def nrat(o):
        m = 0.0
        for k, v in o["spool"].items():
            m = max(m, v / ref["spool"][k])
        return m

    if nrat(op) > Nmax:
        lo, hi = 0.45 * p["design"]["Tt4max"], Tt4cmd
        for _ in range(40):
            mid = 0.5 * (lo + hi)
            o = run_cycle(p, ref, fl, mid)
            if nrat(o) > Nmax:
                hi = mid
            else:
                lo = mid
        op = run_cycle(p, ref, fl, lo)
        op["limited"] = True
    op["Tt4cmd"] = Tt4cmd
    op["N"] = {k: v / ref["spool"][k] for k, v in op["spool"].items()}
    return {"ref": ref, "op": op, "flRef": fl_ref, "fl": fl}


# ---------------------------------------------------------------------------
# flow-path outlines  (src/geometry.js)
# ---------------------------------------------------------------------------
def chaikin(pts, iters):
    """Corner-cutting smoothing (src/geometry.js:5-18)."""
    p = pts
    for _ in range(iters):
        q = [p[0]]
        for i in range(len(p) - 1):
            a, b = p[i], p[i + 1]
            q.append([0.75 * a[0] + 0.25 * b[0], 0.75 * a[1] + 0.25 * b[1]])
            q.append([0.25 * a[0] + 0.75 * b[0], 0.25 * a[1] + 0.75 * b[1]])
        q.append(p[-1])
        p = q
    return p


class Line:
    """Piecewise-linear r(x) outline with optional Chaikin smoothing (src/geometry.js:19-36).

    `smooth=None` means the reference's default of two smoothing passes, 0 means none.
    """

    def __init__(self, ctrl, s, smooth=None):
        pts = [[x * s, r * s] for x, r in ctrl]
        if smooth != 0:
            pts = chaikin(pts, smooth or 2)
        for i in range(1, len(pts)):
            if pts[i][0] < pts[i - 1][0]:
                pts[i][0] = pts[i - 1][0]
        self.pts = pts
        self.xs = [q[0] for q in pts]
        self.rs = [q[1] for q in pts]

    def at(self, x):
        xs, rs = self.xs, self.rs
        n = len(xs)
        if x <= xs[0]:
            return rs[0]
        if x >= xs[n - 1]:
            return rs[n - 1]
        lo, hi = 0, n - 1
        while hi - lo > 1:
            m = (lo + hi) >> 1
            if xs[m] <= x:
                lo = m
            else:
                hi = m
        dx = xs[hi] - xs[lo]
        return rs[hi] if dx < 1e-12 else rs[lo] + (rs[hi] - rs[lo]) * (x - xs[lo]) / dx


def _clamp(v, a, b):
    return a if v < a else (b if v > b else v)


def _jsround(v):
    """JavaScript Math.round (halves go up)."""
    return math.floor(v + 0.5)


def lip_arc(cx, cr, ax, ar, s, n):
    """Half-ellipse intake lip (src/geometry.js:37-44)."""
    out = []
    for i in range(n + 1):
        t = -math.pi / 2 + math.pi * i / n
        out.append([(cx - ax * math.cos(t)) * s, (cr + ar * math.sin(t)) * s])
    return out


def strip_poly(line, x0, x1, th):
    """Thin wall of thickness th along an outline (src/geometry.js:47-55)."""
    up, dn = [], []
    n = 24
    for i in range(n + 1):
        x = x0 + (x1 - x0) * i / n
        r = line.at(x)
        up.append([x, r + th / 2])
        dn.append([x, r - th / 2])
    return dn + up[::-1]


def bbox(poly):
    """[xmin, xmax, rmin, rmax] of a polygon (src/geometry.js:56-60)."""
    return [min(q[0] for q in poly), max(q[0] for q in poly), min(q[1] for q in poly), max(q[1] for q in poly)]


def point_in_poly(x, r, poly):
    """Even-odd crossing test (src/geometry.js:61-68)."""
    inside = False
    j = len(poly) - 1
    for i in range(len(poly)):
        xi, ri = poly[i]
        xj, rj = poly[j]
        if (ri > r) != (rj > r) and x < (xj - xi) * (r - ri) / (rj - ri) + xi:
            inside = not inside
        j = i
    return inside


def stage_rows(x0, x1, n_stages, o):
    """Equal-pitch rotor/stator rows of a compressor or turbine (src/geometry.js:70-95)."""
    rows = []
    n_rows = n_stages * 2 + (1 if o.get("igv") else 0)
    w = (x1 - x0) / n_rows
    x = x0
    if o.get("igv"):
        rows.append({"x0": x, "x1": x + w * 0.8, "rotor": False, "n": o.get("nIgv") or 30, "kind": "vane",
                     "role": "igv"})
        x += w
    for i in range(n_stages):
        nr = _jsround(o["nr0"] + (o["nr1"] - o["nr0"]) * (i / (n_stages - 1) if n_stages > 1 else 0))
        ns = _jsround(nr * (o.get("sRatio") or 1.15))
        if o.get("turbine"):
            rows.append({"x0": x, "x1": x + w * 0.82, "rotor": False, "n": ns, "kind": "ngv", "stage": i})
            x += w
            rows.append({"x0": x, "x1": x + w * 0.82, "rotor": True, "n": nr, "kind": "turb", "stage": i})
            x += w
        else:
            rows.append({"x0": x, "x1": x + w * 0.82, "rotor": True, "n": nr, "kind": o.get("kind") or "comp",
                         "stage": i})
            x += w
            rows.append({"x0": x, "x1": x + w * 0.82, "rotor": False, "n": ns, "kind": "vane", "stage": i})
            x += w
    for r in rows:
        r.update(stream=o.get("stream"), spool=o.get("spool"), comp=o.get("comp"))
    return rows


def _scale_rows(rows, s):
    """src/geometry.js:96"""
    for r in rows:
        r["x0"] *= s
        r["x1"] *= s
    return rows


def _row(x0, x1, stream, rotor, n, kind, comp, spool=None, role=None, stage=None):
    r = {"x0": x0, "x1": x1, "stream": stream, "rotor": rotor, "n": n, "kind": kind, "comp": comp}
    if spool is not None:
        r["spool"] = spool
    if role is not None:
        r["role"] = role
    if stage is not None:
        r["stage"] = stage
    return r


def v_gutter(x0, r, h):
    """Afterburner V-gutter flame holder, open downstream (src/geometry.js:329-331)."""
    return [[x0, r], [x0 + h * 1.1, r + h * 0.5], [x0 + h * 1.1, r + h * 0.38], [x0 + h * 0.18, r],
            [x0 + h * 1.1, r - h * 0.38], [x0 + h * 1.1, r - h * 0.5]]


def spec_hbtf(s, noz):
    """High-bypass turbofan flow path (src/geometry.js:108-188)."""
    hub = Line([[0.30, 0], [0.305, 0.03], [0.34, 0.085], [0.42, 0.155], [0.50, 0.207], [0.58, 0.24],
                [0.70, 0.262], [0.78, 0.272], [0.90, 0.29], [0.95, 0.305], [1.25, 0.33], [1.29, 0.322],
                [1.35, 0.228], [1.41, 0.162], [1.46, 0.145], [2.05, 0.212], [2.09, 0.20], [2.12, 0.19],
                [2.36, 0.19], [2.40, 0.225], [2.42, 0.238], [2.58, 0.242], [2.66, 0.25], [3.08, 0.24],
                [3.2, 0.232], [3.45, 0.16], [3.62, 0.09], [3.78, 0.028], [3.845, 0]], s)
    r9h = hub.at(3.45 * s) / s
    cowl_pts = [[0.90, 0.44], [0.96, 0.462], [1.1, 0.482], [1.4, 0.498], [1.8, 0.50], [2.05, 0.49],
                [2.2, 0.472], [2.6, 0.425], [2.9, 0.41], [3.2, 0.388]]
    A9 = noz.get("A9") if noz else None
    R9 = _clamp(math.sqrt(A9 / (math.pi * s * s) + r9h * r9h), 0.22, 0.33) if (A9 and A9 > 0) else 0.2853
    tip = Line([[0.90, 0.44], [0.95, 0.425], [1.25, 0.392], [1.29, 0.395], [1.35, 0.352], [1.41, 0.29],
                [1.46, 0.252], [1.55, 0.246], [2.05, 0.232], [2.08, 0.26], [2.12, 0.335], [2.15, 0.345],
                [2.34, 0.345], [2.39, 0.31], [2.42, 0.282], [2.58, 0.29], [2.66, 0.32], [3.08, 0.375],
                [3.2, 0.37], [3.45, R9]], s)
    cowl = Line(cowl_pts + [[3.45, R9 + 0.02]], s)
    r19c = cowl.at(2.2 * s) / s
    A19 = noz.get("A19") if noz else None
    R19 = _clamp(math.sqrt(A19 / (math.pi * s * s) + r19c * r19c), 0.62, 0.76) if (A19 and A19 > 0) else 0.7063
    nac_in = Line([[0.0, 0.843], [0.06, 0.822], [0.18, 0.804], [0.35, 0.80], [0.58, 0.80], [0.80, 0.80],
                   [1.1, 0.797], [1.5, 0.78], [1.9, 0.745 + 0.5 * (R19 - 0.70)], [2.2, R19]], s)
    nac_out = Line([[0.0, 0.905], [0.1, 0.94], [0.3, 0.968], [0.6, 0.978], [1.0, 0.97], [1.4, 0.93],
                    [1.8, 0.85], [2.1, 0.755 + 0.6 * (R19 - 0.70)], [2.2, R19 + 0.016]], s)
    lip = lip_arc(0, 0.874, 0.035, 0.031, s, 10)
    liner_in = Line([[2.15, 0.222], [2.20, 0.216], [2.30, 0.222], [2.42, 0.238]], s)
    liner_out = Line([[2.15, 0.308], [2.20, 0.318], [2.30, 0.305], [2.42, 0.282]], s)
    nac_poly = lip + nac_out.pts + [[2.2 * s, R19 * s]] + nac_in.pts[::-1]
    hub_poly = hub.pts + [[0.30 * s, 0]]
    cowl_poly = cowl.pts + tip.pts[::-1]
    rows = _scale_rows([
        _row(0.585, 0.775, "inlet", True, 24, "fan", "fan", spool="LP"),
        _row(1.00, 1.10, "bypass", False, 44, "vane", "byp", role="ogv"),
        *stage_rows(0.955, 1.25, 3, {"stream": "core", "spool": "LP", "nr0": 64, "nr1": 76, "comp": "lpc"}),
        *stage_rows(1.465, 2.05, 9, {"stream": "core", "spool": "HP", "nr0": 38, "nr1": 90, "igv": True,
                                     "nIgv": 40, "comp": "hpc"}),
        _row(2.425, 2.48, "core", False, 38, "ngv", "hpt", stage=0),
        _row(2.50, 2.572, "core", True, 72, "turb", "hpt", spool="HP", stage=0),
        *stage_rows(2.67, 3.07, 4, {"stream": "core", "spool": "LP", "nr0": 110, "nr1": 134, "turbine": True,
                                    "sRatio": 0.55, "comp": "lpt"}),
        _row(3.10, 3.16, "core", False, 14, "strut", "noz", role="trf"),
    ], s)
    return {
        "type": "hbtf", "s": s,
        "lines": {"hub": hub, "tip": tip, "cowl": cowl, "nacIn": nac_in, "nacOut": nac_out,
                  "linerIn": liner_in, "linerOut": liner_out},
        "streams": {
            "inlet": {"x0": 0, "x1": 0.90 * s, "lo": hub, "hi": nac_in, "gas": "cold"},
            "core": {"x0": 0.90 * s, "x1": 3.45 * s, "lo": hub, "hi": tip},
            "bypass": {"x0": 0.90 * s, "x1": 2.2 * s, "lo": cowl, "hi": nac_in, "gas": "cold"},
        },
        "order": ["inlet", "core", "bypass"],
        "bodies": [
            {"key": "nacelle", "poly": nac_poly, "mat": "nacelle"},
            {"key": "hub", "poly": hub_poly, "mat": "hub"},
            {"key": "cowl", "poly": cowl_poly, "mat": "cowl"},
            {"key": "linerIn", "poly": strip_poly(liner_in, 2.15 * s, 2.42 * s, 0.006 * s), "mat": "liner"},
            {"key": "linerOut", "poly": strip_poly(liner_out, 2.15 * s, 2.42 * s, 0.006 * s), "mat": "liner"},
            {"key": "dome", "poly": [[2.147 * s, 0.222 * s], [2.155 * s, 0.222 * s], [2.155 * s, 0.308 * s],
                                     [2.147 * s, 0.308 * s]], "mat": "liner"},
        ],
        "rows": rows,
        "comb": {"x0": 2.08 * s, "xd": 2.15 * s, "x1": 2.42 * s, "linerIn": liner_in, "linerOut": liner_out,
                 "n": 20, "cannular": False, "stream": "core", "turbEnd": 3.08 * s},
        "ab": None, "mixer": None, "nozzle": None,
        "stations": [
            {"id": "2", "x": 0.585 * s, "stream": "inlet"}, {"id": "13", "x": 0.93 * s, "stream": "bypass"},
            {"id": "21", "x": 0.955 * s, "stream": "core"}, {"id": "25", "x": 1.465 * s, "stream": "core"},
            {"id": "3", "x": 2.05 * s, "stream": "core"}, {"id": "4", "x": 2.425 * s, "stream": "core"},
            {"id": "45", "x": 2.62 * s, "stream": "core"}, {"id": "5", "x": 3.08 * s, "stream": "core"},
            {"id": "9", "x": 3.45 * s, "stream": "core"}, {"id": "19", "x": 2.2 * s, "stream": "bypass"},
        ],
        "lip": {"x": 0, "r": 0.843 * s, "rOut": 0.905 * s},
        "outer": nac_out, "outerEnd": 2.2 * s,
        "exitsGeom": [
            {"key": "bypass", "x": 2.2 * s, "R": R19 * s, "Rin": cowl.at(2.2 * s)},
            {"key": "core", "x": 3.45 * s, "R": R9 * s, "Rin": hub.at(3.45 * s), "plugTip": 3.845 * s},
        ],
        "view": {"Rmax": 0.98 * s},
    }


def spec_tj(s, noz):
    """Turbojet flow path (src/geometry.js:190-249)."""
    r8 = noz["r8"] if noz else 0.235 * s
    r9 = noz["r9"] if noz else 0.255 * s
    hub = Line([[0.08, 0], [0.085, 0.02], [0.13, 0.065], [0.22, 0.122], [0.35, 0.16], [0.6, 0.2], [1.0, 0.245],
                [1.55, 0.281], [1.58, 0.265], [1.62, 0.235], [1.66, 0.22], [2.12, 0.22], [2.17, 0.27],
                [2.20, 0.29], [2.62, 0.25], [2.9, 0.18], [3.1, 0.08], [3.2, 0.0]], s)
    cas_in = Line([[0.0, 0.445], [0.08, 0.415], [0.2, 0.402], [0.35, 0.40], [0.8, 0.37], [1.2, 0.335],
                   [1.55, 0.319], [1.59, 0.36], [1.63, 0.415], [1.66, 0.42], [2.10, 0.42], [2.16, 0.39],
                   [2.20, 0.37], [2.62, 0.37], [2.9, 0.40], [4.3, 0.40], [4.32, 0.398], [4.6, r8 / s],
                   [4.9, r9 / s]], s, 1)
    cas_out = Line([[0.0, 0.50], [0.12, 0.49], [0.35, 0.465], [1.5, 0.465], [1.66, 0.47], [2.2, 0.47],
                    [2.62, 0.445], [2.9, 0.45], [4.3, 0.45], [4.9, r9 / s + 0.025]], s, 1)
    lip = lip_arc(0, 0.4725, 0.03, 0.0275, s, 10)
    liner_in = Line([[1.67, 0.26], [1.8, 0.25], [2.0, 0.262], [2.2, 0.29]], s)
    liner_out = Line([[1.67, 0.38], [1.8, 0.395], [2.0, 0.385], [2.2, 0.37]], s)
    xe = 4.9 * s
    cas_poly = lip + cas_out.pts + [[xe, r9]] + cas_in.pts[::-1]
    hub_poly = hub.pts + [[0.08 * s, 0]]
    rows = _scale_rows([
        *stage_rows(0.36, 1.55, 12, {"stream": "core", "spool": "HP", "nr0": 30, "nr1": 72, "igv": True,
                                     "nIgv": 30, "comp": "comp"}),
        *stage_rows(2.205, 2.62, 3, {"stream": "core", "spool": "HP", "nr0": 80, "nr1": 96, "turbine": True,
                                     "sRatio": 0.6, "comp": "turb"}),
        _row(2.70, 2.78, "core", False, 12, "strut", "diff", role="trf"),
    ], s)
    ab_x0 = 3.25 * s
    fh_rings = [0.14 * s, 0.28 * s]
    bodies = [
        {"key": "casing", "poly": cas_poly, "mat": "casing"},
        {"key": "hub", "poly": hub_poly, "mat": "hub"},
        {"key": "linerIn", "poly": strip_poly(liner_in, 1.67 * s, 2.2 * s, 0.006 * s), "mat": "liner"},
        {"key": "linerOut", "poly": strip_poly(liner_out, 1.67 * s, 2.2 * s, 0.006 * s), "mat": "liner"},
        {"key": "dome", "poly": [[1.667 * s, 0.26 * s], [1.675 * s, 0.26 * s], [1.675 * s, 0.38 * s],
                                 [1.667 * s, 0.38 * s]], "mat": "liner"},
    ] + [{"key": "fh%d" % i, "poly": v_gutter(ab_x0, r, 0.035 * s), "mat": "fh"} for i, r in enumerate(fh_rings)]
    return {
        "type": "tj", "s": s, "r8": r8, "r9": r9,
        "lines": {"hub": hub, "tip": cas_in, "casIn": cas_in, "casOut": cas_out, "linerIn": liner_in,
                  "linerOut": liner_out},
        "streams": {"core": {"x0": 0, "x1": xe, "lo": hub, "hi": cas_in}},
        "order": ["core"],
        "bodies": bodies, "rows": rows,
        "comb": {"x0": 1.58 * s, "xd": 1.67 * s, "x1": 2.2 * s, "linerIn": liner_in, "linerOut": liner_out,
                 "n": 10, "cannular": True, "stream": "core", "turbEnd": 2.62 * s},
        "ab": {"stream": "core", "xSpray": 2.95 * s, "xFH": ab_x0, "x1": 4.3 * s, "rings": fh_rings,
               "xNoz": 4.3 * s, "xt": 4.6 * s, "xe": xe},
        "mixer": None,
        "stations": [
            {"id": "2", "x": 0.36 * s, "stream": "core"}, {"id": "3", "x": 1.55 * s, "stream": "core"},
            {"id": "4", "x": 2.205 * s, "stream": "core"}, {"id": "5", "x": 2.62 * s, "stream": "core"},
            {"id": "6", "x": 2.95 * s, "stream": "core"}, {"id": "7", "x": 4.3 * s, "stream": "core"},
            {"id": "8", "x": 4.6 * s, "stream": "core"}, {"id": "9", "x": 4.9 * s, "stream": "core"},
        ],
        "lip": {"x": 0, "r": 0.445 * s, "rOut": 0.50 * s},
        "outer": cas_out, "outerEnd": xe,
        "exitsGeom": [{"key": "core", "x": xe, "R": r9, "Rin": 0}],
        "nozzle": {"x0": 4.3 * s, "xt": 4.6 * s, "xe": xe, "r8": r8, "r9": r9, "rDuct": 0.40 * s},
        "view": {"Rmax": 0.5 * s},
    }


def spec_lbtf(s, noz):
    """Low-bypass afterburning turbofan flow path (src/geometry.js:251-328)."""
    r8 = noz["r8"] if noz else 0.265 * s
    r9 = noz["r9"] if noz else 0.29 * s
    hub = Line([[0.05, 0], [0.055, 0.02], [0.10, 0.055], [0.2, 0.105], [0.30, 0.14], [0.45, 0.19], [0.60, 0.23],
                [0.75, 0.25], [0.85, 0.255], [0.95, 0.265], [1.55, 0.287], [1.58, 0.26], [1.62, 0.24],
                [1.95, 0.24], [1.99, 0.275], [2.00, 0.285], [2.15, 0.285], [2.55, 0.27], [2.75, 0.25],
                [3.0, 0.17], [3.2, 0.07], [3.28, 0]], s)
    cas_in = Line([[0.0, 0.49], [0.06, 0.47], [0.18, 0.463], [0.30, 0.462], [0.52, 0.43], [0.75, 0.40],
                   [0.85, 0.43], [1.0, 0.44], [1.6, 0.45], [2.0, 0.45], [2.4, 0.44], [2.75, 0.44], [4.3, 0.44],
                   [4.32, 0.438], [4.6, r8 / s], [4.95, r9 / s]], s, 1)
    tip = Line([[0.85, 0.345], [0.95, 0.335], [1.55, 0.305], [1.58, 0.35], [1.62, 0.395], [1.95, 0.395],
                [1.99, 0.345], [2.00, 0.335], [2.15, 0.342], [2.20, 0.345], [2.55, 0.37], [2.75, 0.38]], s)
    core_cas = Line([[0.85, 0.345], [0.92, 0.36], [1.2, 0.37], [1.5, 0.375], [1.62, 0.41], [1.95, 0.41],
                     [2.05, 0.39], [2.4, 0.39], [2.75, 0.385]], s)
    cas_out = Line([[0.0, 0.54], [0.1, 0.525], [0.3, 0.515], [2.75, 0.515], [4.3, 0.515],
                    [4.95, r9 / s + 0.03]], s, 1)
    lip = lip_arc(0, 0.515, 0.03, 0.025, s, 10)
    liner_in = Line([[1.66, 0.262], [1.8, 0.255], [2.0, 0.285]], s)
    liner_out = Line([[1.66, 0.375], [1.8, 0.385], [2.0, 0.335]], s)
    xe = 4.95 * s
    cas_poly = lip + cas_out.pts + [[xe, r9]] + cas_in.pts[::-1]
    hub_poly = hub.pts + [[0.05 * s, 0]]
    core_poly = core_cas.pts + tip.pts[::-1]
    rows = _scale_rows([
        *stage_rows(0.30, 0.75, 3, {"stream": "inlet", "spool": "LP", "nr0": 28, "nr1": 44, "igv": True,
                                    "nIgv": 22, "kind": "fan", "sRatio": 1.1, "comp": "fan"}),
        *stage_rows(0.955, 1.55, 7, {"stream": "core", "spool": "HP", "nr0": 34, "nr1": 72, "igv": True,
                                     "nIgv": 36, "comp": "hpc"}),
        _row(2.005, 2.055, "core", False, 34, "ngv", "hpt", stage=0),
        _row(2.07, 2.14, "core", True, 66, "turb", "hpt", spool="HP", stage=0),
        *stage_rows(2.20, 2.55, 2, {"stream": "core", "spool": "LP", "nr0": 72, "nr1": 80, "turbine": True,
                                    "sRatio": 0.6, "comp": "lpt"}),
    ], s)
    ab_x0 = 3.35 * s
    fh_rings = [0.16 * s, 0.32 * s]
    return {
        "type": "lbtf", "s": s, "r8": r8, "r9": r9,
        "lines": {"hub": hub, "tip": tip, "casIn": cas_in, "casOut": cas_out, "coreCas": core_cas,
                  "linerIn": liner_in, "linerOut": liner_out},
        "streams": {
            "inlet": {"x0": 0, "x1": 0.85 * s, "lo": hub, "hi": cas_in, "gas": "cold"},
            "core": {"x0": 0.85 * s, "x1": 2.75 * s, "lo": hub, "hi": tip},
            "bypass": {"x0": 0.85 * s, "x1": 2.75 * s, "lo": core_cas, "hi": cas_in, "gas": "cold"},
            "ab": {"x0": 2.75 * s, "x1": xe, "lo": hub, "hi": cas_in},
        },
        "order": ["inlet", "core", "bypass", "ab"],
        "bodies": [
            {"key": "casing", "poly": cas_poly, "mat": "casing"},
            {"key": "hub", "poly": hub_poly, "mat": "hub"},
            {"key": "coreCase", "poly": core_poly, "mat": "cowl"},
            {"key": "linerIn", "poly": strip_poly(liner_in, 1.66 * s, 2.0 * s, 0.006 * s), "mat": "liner"},
            {"key": "linerOut", "poly": strip_poly(liner_out, 1.66 * s, 2.0 * s, 0.006 * s), "mat": "liner"},
            {"key": "dome", "poly": [[1.657 * s, 0.262 * s], [1.665 * s, 0.262 * s], [1.665 * s, 0.375 * s],
                                     [1.657 * s, 0.375 * s]], "mat": "liner"},
        ] + [{"key": "fh%d" % i, "poly": v_gutter(ab_x0, r, 0.035 * s), "mat": "fh"}
             for i, r in enumerate(fh_rings)],
        "rows": rows,
        "comb": {"x0": 1.58 * s, "xd": 1.66 * s, "x1": 2.0 * s, "linerIn": liner_in, "linerOut": liner_out,
                 "n": 18, "cannular": False, "stream": "core", "turbEnd": 2.55 * s},
        "ab": {"stream": "ab", "xSpray": 3.15 * s, "xFH": ab_x0, "x1": 4.3 * s, "rings": fh_rings,
               "xNoz": 4.3 * s, "xt": 4.6 * s, "xe": xe},
        "mixer": {"x": 2.75 * s, "lobes": 16, "coreFrac": 0.625},
        "stations": [
            {"id": "2", "x": 0.30 * s, "stream": "inlet"}, {"id": "13", "x": 0.88 * s, "stream": "bypass"},
            {"id": "25", "x": 0.955 * s, "stream": "core"}, {"id": "3", "x": 1.55 * s, "stream": "core"},
            {"id": "4", "x": 2.005 * s, "stream": "core"}, {"id": "45", "x": 2.17 * s, "stream": "core"},
            {"id": "5", "x": 2.55 * s, "stream": "core"}, {"id": "16", "x": 2.7 * s, "stream": "bypass"},
            {"id": "6A", "x": 3.0 * s, "stream": "ab"}, {"id": "7", "x": 4.3 * s, "stream": "ab"},
            {"id": "8", "x": 4.6 * s, "stream": "ab"}, {"id": "9", "x": xe, "stream": "ab"},
        ],
        "lip": {"x": 0, "r": 0.49 * s, "rOut": 0.54 * s},
        "outer": cas_out, "outerEnd": xe,
        "exitsGeom": [{"key": "core", "x": xe, "R": r9, "Rin": 0}],
        "nozzle": {"x0": 4.3 * s, "xt": 4.6 * s, "xe": xe, "r8": r8, "r9": r9, "rDuct": 0.44 * s},
        "view": {"Rmax": 0.54 * s},
    }


def build_spec(typ, s, noz):
    """Dispatch on engine type (src/geometry.js:101-105)."""
    if typ == "hbtf":
        return spec_hbtf(s, noz)
    if typ == "tj":
        return spec_tj(s, noz)
    return spec_lbtf(s, noz)


def engine_for(aircraft_type, engine_type):
    """Sea-level static design-point engine that sizes the nozzle (tools/airlib.js:6-11)."""
    E = ENGINE_TYPES[engine_type]
    P = {"type": engine_type, "design": dict(E["design"]), "eff": dict(DEFAULT_EFF), "alt": 0, "M0": 0,
         "thr": 1, "ab": False, "Tt7": 2100 if engine_type == "lbtf" else 2000, "nozzleType": E["nozzle"]}
    sol = solve_engine(P)
    nz = sol["op"]["noz"]
    ref = sol["ref"]
    noz = {"r8": math.sqrt(nz["Athroat"] / math.pi),
           "r9": math.sqrt(max(nz["A"], nz["Athroat"]) / math.pi),
           "A9": ref["noz"]["A"] if ref.get("noz") else None,
           "A19": ref["nozB"]["A"] if ref.get("nozB") else None}
    spec = build_spec(engine_type, 1, noz)
    return {"spec": spec, "sol": sol, "P": P, "noz": noz}
