"""Engine cycle, engine deck and field model: the host chain behind the fixed states.

Pins from the reference's own published numbers:
  * README.md:73-75 - 1-D net thrust at sea level, M0.25, full dry throttle: TJ 55.4 kN,
    HBTF 95.8 kN, LBTF 70.2 kN (solveEngine);
  * README.md:97 - airliner cruise at 11 km, M0.78, 72.6 t, L/D 17.8: TSFC 19.4 g/(kN s)
    (EngineDeck + the level-flight throttle search).
The field model's samples have no published values and no JavaScript runtime exists here to
produce them; they are checked through properties of the model instead (design-point knot
Mach numbers, the undisturbed far field, knot states mid-stream, conservation of the jet
blur, physical fixed states).
"""
import importlib
import math

import numpy as np
import pytest

E = importlib.import_module("3d_aero_lab_b200.engine")
Fm = importlib.import_module("3d_aero_lab_b200.field")
A = importlib.import_module("3d_aero_lab_b200.aircraft")

TYPES = {"airliner": "hbtf", "interceptor": "tj", "fighter": "lbtf"}


def engine_params(et, alt=0.0, M0=0.0, thr=1.0, ab=False):
    T = E.ENGINE_TYPES[et]
    return {"type": et, "design": dict(T["design"]), "eff": dict(E.DEFAULT_EFF), "alt": alt, "M0": M0, "thr": thr,
            "ab": ab, "Tt7": 2100 if et == "lbtf" else 2000, "nozzleType": T["nozzle"]}


@pytest.fixture(scope="module")
def aircraft():
    return {t: A.build_aircraft(t) for t in TYPES}


@pytest.mark.parametrize("et,kN", [("tj", 55.4), ("hbtf", 95.8), ("lbtf", 70.2)])
def test_cycle_thrust_matches_readme(et, kN):
    sol = E.solve_engine(engine_params(et, 0.0, 0.25))
    assert round(sol["op"]["F"] / 1000, 1) == kN
    assert not sol["op"]["limited"]


def test_cruise_tsfc_matches_readme(aircraft):
    ac = aircraft["airliner"]
    deck = Fm.EngineDeck.for_engine(ac.eng["P"])
    D = 72600 * 9.80665 / 17.8
    thr, th = Fm.level_throttle(deck, 11000, 0.78, D, False, ac.T["nEng"], Fm.INSTALL_LOSS["airliner"])
    assert 0.35 < thr < 1
    assert round(th["ff"] / th["T"] * 1e6, 1) == 19.4


@pytest.mark.parametrize("D", [2.0e4, 4.0e4, 6.0e4])
def test_level_throttle_balances_drag(aircraft, D):
    ac = aircraft["airliner"]
    deck = Fm.EngineDeck.for_engine(ac.eng["P"])
    n, inst = ac.T["nEng"], Fm.INSTALL_LOSS["airliner"]
    thr, th = Fm.level_throttle(deck, 11000, 0.78, D, False, n, inst)
    lo = deck.thrust(11000, 0.78, 0.35, False, n, inst)["T"]
    hi = deck.thrust(11000, 0.78, 1, False, n, inst)["T"]
    if lo < D < hi:
        got = deck.thrust(11000, 0.78, thr, False, n, inst)["T"]
        assert abs(got - D) < 3e-3 * D


def test_station_table_feeds_the_nozzles():
    for et in ("tj", "hbtf", "lbtf"):
        for ab in (False, True):
            op = E.solve_engine(engine_params(et, 3000, 0.7, 1.0, ab))["op"]
            S = op["S"]
            assert S["9"]["Pt"] == op["noz"]["Pt"] and S["9"]["Tt"] == op["noz"]["Tt"]
            if et == "hbtf":
                assert S["19"]["Pt"] == op["nozB"]["Pt"] and S["19"]["Tt"] == op["nozB"]["Tt"]
            else:
                assert op["abOn"] == ab


def test_deck_respects_spool_speed_limit(aircraft):
    for t in TYPES:
        deck = Fm.EngineDeck.for_engine(aircraft[t].eng["P"])
        for h in (0, 5000, 11000, 16000):
            for M in (0.0, 0.5, 0.9, 1.5):
                r = deck.at(h, M, 1.0, False)
                assert max(r["N"].values()) < 1.06, (t, h, M, r["N"])
                assert r["Tt4"] <= deck.design["Tt4max"]
                assert deck.at(h, M, 1.0, False) is r  # cached


def test_design_point_knots_keep_design_mach(aircraft):
    """At the design point the corrected-flow rescaling must return every knot's design Mach."""
    for t in TYPES:
        ac = aircraft[t]
        fm, rop = Fm.operating_point(ac, 0.0, 0.0, 1.0, False)
        assert fm is not None and not rop["limited"]
        for key, kn in fm.kn.items():
            for k in kn:
                if k["noz"] < 0:
                    assert abs(k["M"] - k["Md"]) < 1e-4, (t, key, k["x"], k["M"], k["Md"])


def test_far_field_is_undisturbed(aircraft):
    for t, (h, M) in zip(TYPES, [(0.0, 0.6), (11000.0, 0.78), (11000.0, 1.6)]):
        ac = aircraft[t]
        fm, _ = Fm.operating_point(ac, h, M, 1.0, False)
        s = ac.spec["s"]
        o = fm.sample(-500 * s, 0.5 * s)
        fl = E.flight_state(h, M)
        assert o["region"] == "ext" and o["zone"] == "free"
        assert o["Tt"] == fl["Tt0"]
        assert abs(o["Vx"] / fl["V0"] - 1) < 1e-6
        # the static state comes back through cp = 1004.5 (R = 287.0) while the atmosphere uses
        # R = 287.05, so it differs from (T0, P0) by 3.5e-5 M^2 (T) and 1.2e-4 M^2 (P): compare
        # with the isentropic state of the undisturbed speed instead
        T = fl["Tt0"] - fl["V0"] ** 2 / (2 * 1004.5)
        assert abs(o["T"] / T - 1) < 1e-6 and abs(o["P"] / (fl["Pt0"] * (T / fl["Tt0"]) ** 3.5) - 1) < 1e-5
        assert abs(o["T"] / fl["T0"] - 1) < 4e-5 * M * M and abs(o["P"] / fl["P0"] - 1) < 1.3e-4 * M * M


def test_stream_sample_mid_channel_is_the_knot_state(aircraft):
    """Away from the walls, combustor and afterburner a stream sample is its knot state."""
    ac = aircraft["airliner"]
    fm, _ = Fm.operating_point(ac, 0.0, 0.6, 1.0, False)
    s = ac.spec["s"]
    st = ac.spec["streams"]["bypass"]
    x = 1.60 * s
    r = 0.5 * (st["lo"].at(x) + st["hi"].at(x))
    o = fm.sample(x, r)
    k = next(k for k in fm.kn["bypass"] if k["x"] == x)
    assert o["region"] == "stream" and o["stream"] == "bypass"
    assert o["Tt"] == k["Tt"] == fm.c["Tt13"]
    assert math.isclose(o["P"], k["P"], rel_tol=1e-13)
    assert math.isclose(o["V"], k["V"], rel_tol=1e-12)


@pytest.mark.parametrize("R,sig", [(1.0, 0.05), (1.0, 0.3), (0.4, 0.2)])
def test_jet_blur_conserves_the_disk_area(R, sig):
    """The blurred disk is a convolution: its area integral stays pi R^2 (to the 0.3 % that the
    reference's 10-point quadrature and its clip at 1 leave)."""
    r = np.linspace(0.0, R + 8 * sig, 4001)
    w = np.array([Fm.blur_disk(x, R, sig) for x in r])
    area = np.trapezoid(w * 2 * np.pi * r, r)
    assert abs(area / (np.pi * R * R) - 1) < 5e-3
    assert Fm.blur_disk(0.0, R, sig) <= 1 and Fm.blur_disk(R + 7 * sig, R, sig) < 1e-6


def test_i0e_matches_series():
    for x in (0.0, 0.5, 2.0, 3.74, 3.76, 8.0, 40.0):
        s = sum((x / 2) ** (2 * k) / math.factorial(k) ** 2 for k in range(80))
        assert abs(Fm._i0e(x) - math.exp(-x) * s) < 2e-7 * max(1.0, math.exp(-x) * s)


def prim(U):
    rho, ru, rv, rw, En = U
    u, v, w = ru / rho, rv / rho, rw / rho
    return rho, u, (1.4 - 1) * (En - 0.5 * rho * (u * u + v * v + w * w))


@pytest.mark.parametrize("t", list(TYPES))
@pytest.mark.parametrize("h,M", [(0.0, 0.6), (11000.0, 0.78)])
@pytest.mark.parametrize("ab", [False, True])
def test_fix_states_are_physical(aircraft, t, h, M, ab):
    ac = aircraft[t]
    fm, rop = Fm.operating_point(ac, h, M, 1.0, ab)
    assert fm is not None
    F, fx = Fm.fix_states(ac, h, M, 3.0, fm=fm)
    assert F == Fm.free_state(M, 3.0)
    sink, jB, jC = fx
    for U in fx:
        assert all(math.isfinite(v) for v in U)
        rho, u, p = prim(U)
        assert rho > 0 and p > 0
    assert prim(sink)[1] > 0 and prim(jC)[1] > 0
    assert sink != F and jC != F  # both sample points lie in a flow stream
    if TYPES[t] == "hbtf":
        assert jB != F and prim(jB)[1] > 0
        assert rop["op"].get("abOn") is None  # no afterburner on a podded turbofan
    else:
        assert jB == F  # no bypass exit: the reference pushes the free stream
        assert rop["op"]["abOn"] == ab


@pytest.mark.parametrize("t", ["interceptor", "fighter"])
def test_afterburner_heats_the_core_jet(aircraft, t):
    ac = aircraft[t]
    T = []
    for ab in (False, True):
        _, fx = Fm.fix_states(ac, 0.0, 0.6, 3.0, 1.0, ab)
        rho, u, p = prim(fx[2])
        T.append(p / rho)
    assert T[1] > 1.5 * T[0]


def test_throttle_lowers_the_jet_speed(aircraft):
    ac = aircraft["airliner"]
    u = [prim(Fm.fix_states(ac, 0.0, 0.6, 3.0, thr)[1][2])[1] for thr in (0.6, 0.8, 1.0)]
    assert u[0] < u[1] < u[2]


def test_fix_states_match_the_committed_record():
    """Regression record of fix_states (tests/golden/make_field_golden.py)."""
    import json
    import os
    import sys
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    rec = json.load(open(os.path.join(here, "field_fix_states.json")))
    sys.path.insert(0, here)
    import make_field_golden
    now = make_field_golden.states()
    assert len(now) == len(rec["cases"]) == 24
    for a, b in zip(now, rec["cases"]):
        assert (a["type"], a["h"], a["M"], a["thr"], a["ab"]) == (b["type"], b["h"], b["M"], b["thr"], b["ab"])
        for u, v in zip(a["fix"], b["fix"]):
            assert all(math.isclose(x, y, rel_tol=1e-12, abs_tol=1e-15) for x, y in zip(u, v)), a


def test_cfd_state_of_the_free_stream_is_the_free_stream():
    """cfdState (src/air_cfd.js:484-490) of the solver's free stream gives back the atmosphere."""
    for h, M in ((0.0, 0.6), (11000.0, 0.78)):
        fs = Fm.fs_state(h, M)
        F = Fm.free_state(M, 0.0)
        W = [F[0], F[1] / F[0], F[2] / F[0], F[3] / F[0], (1.4 - 1) * (F[4] - 0.5 * F[1] ** 2 / F[0])]
        o = Fm.cfd_state(fs, W)
        assert math.isclose(o["P"], fs["P"], rel_tol=1e-12) and math.isclose(o["T"], fs["T"], rel_tol=1e-12)
        assert math.isclose(o["rho"], fs["rho"], rel_tol=1e-12) and math.isclose(o["M"], M, rel_tol=1e-12)
        assert abs(o["Cp"]) < 1e-12 and math.isclose(o["Vx"], fs["V"], rel_tol=1e-12)


def test_app_convergence_rule():
    """CFD3.readback's test (src/air_cfd.js:575): res/res0 < 2e-3 and the last four C_L within
    2e-3, with more than six readbacks."""
    ctl = importlib.import_module("3d_aero_lab_b200.controller")
    h = [{"CL": 0.3}] * 6
    assert not ctl.converged(h, 1e-6, 1.0)                       # six readbacks are not enough
    h = h + [{"CL": 0.3}]
    assert ctl.converged(h, 1e-3, 1.0)
    assert not ctl.converged(h, 3e-3, 1.0)                       # residual not low enough
    assert not ctl.converged(h, 1e-3, None)                      # no first residual yet
    h2 = h[:-1] + [{"CL": 0.3021}]
    assert not ctl.converged(h2, 1e-3, 1.0)                      # C_L still moving
    h3 = [{"CL": 0.5}] * 3 + [{"CL": 0.3}, {"CL": 0.301}, {"CL": 0.3005}, {"CL": 0.3015}]
    assert ctl.converged(h3, 1e-3, 1.0)                          # only the last four count


class _FakeSolver:
    """Stands in for CfdGPU in the controller loop: the residual decays geometrically with the
    iterations and C_L settles towards 0.3."""

    def __init__(self, decay):
        self.it = 0
        self.decay = decay
        self.snap = False

    def step(self, n):
        self.it += n

    def residual(self, stride=3):
        if not self.snap:  # the first call only snapshots, as the device residual does
            self.snap = True
            return None
        return 1e-2 * self.decay ** self.it

    def mach_max(self, stride=2):
        return 0.9


class _FakeCase:
    def __init__(self, decay):
        self.solver = _FakeSolver(decay)

    def forces(self):
        return {"CL": 0.3 + 0.2 * math.exp(-self.solver.it / 300.0), "CD": 0.04, "Cm": -0.1}

    def trefftz(self):
        return 0.01


def test_controller_loop_stops_by_the_app_rule():
    """Controller.run on a case whose residual falls 100x per 1000 iterations: it stops at the
    first readback where res/res0 < 2e-3 and the last four C_L lie within 2e-3."""
    ctl = importlib.import_module("3d_aero_lab_b200.controller")
    c = ctl.Controller(_FakeCase(0.01 ** (1 / 1000)), check_every=200)
    rec = c.run()
    assert c.conv and rec["it"] == c.it and c.it % 200 == 0
    assert c.res / c.res0 < ctl.Controller.RES_DROP
    cl = [h["CL"] for h in c.hist[-4:]]
    assert max(cl) - min(cl) < ctl.Controller.CL_TOL
    # the readback before did not yet meet the rule
    assert not ctl.converged(c.hist[:-1], c.hist[-2]["res"], c.res0)
    assert c.res0 == c.hist[0]["res"] and len(c.hist) == c.it // 200


def test_controller_loop_stops_at_the_iteration_cap():
    """A case whose residual never drops stops on the first readback past 30,000 iterations
    (the app's `it > 30000`)."""
    ctl = importlib.import_module("3d_aero_lab_b200.controller")
    c = ctl.Controller(_FakeCase(1.0), check_every=1000)
    c.run()
    assert c.conv and c.it == ctl.Controller.MAX_ITERS + 1
    assert not ctl.converged(c.hist, c.res, c.res0)  # the cap, not the residual rule
    c2 = ctl.Controller(_FakeCase(1.0), check_every=1000)
    c2.run(max_iters=2500)  # a bounded run stops at its own limit, not converged
    assert not c2.conv and c2.it == 2500
