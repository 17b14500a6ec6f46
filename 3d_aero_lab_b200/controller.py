"""The app's per-case solve loop (CFD3, src/air_cfd.js:495-586) on the GPU solver.

The reference app steps its solver every animation frame and, every 1.4 s of wall time, reads
the state back to compute the density residual (every third cell), the forces, the Trefftz
induced drag and the largest Mach number.  It keeps a history and declares the case converged
when both hold (`readback`, src/air_cfd.js:550-578):

* the residual has dropped below 2e-3 of the first one;
* the last four C_L values lie within 2e-3, with more than six readbacks in the history.

It also stops after 30,000 iterations.  `Controller` keeps those rules but reads back every
`check_every` iterations instead of every 1.4 s, and the reductions run on the device, so no
full state crosses to the host.
"""
from __future__ import annotations


class Controller:
    """Convergence loop of one case (a `cfd.Case`) with the reference app's rules."""

    RES_DROP = 2e-3      # res / res0 (src/air_cfd.js:575)
    CL_WINDOW = 4        # readbacks whose C_L spread is tested
    CL_TOL = 2e-3
    MIN_HISTORY = 7      # hist.length > 6
    MAX_ITERS = 30000    # src/air_cfd.js:576

    def __init__(self, case, check_every=200, residual_stride=3):
        self.case = case
        self.check_every = int(check_every)
        self.stride = int(residual_stride)
        self.res = None
        self.res0 = None
        self.hist = []
        self.conv = False
        self.case.solver.residual(self.stride)  # first snapshot, as the first readback does

    @property
    def it(self):
        return self.case.solver.it

    def readback(self):
        """Residual, forces, Trefftz CD_i and Mach maximum; updates the history and `conv`."""
        s = self.case.solver
        res = s.residual(self.stride)
        if res is not None:
            self.res = res
            if not (self.res0 and self.res0 > 0) and res > 0:
                self.res0 = res
        f = self.case.forces()
        rec = {"it": s.it, "res": self.res, "CL": f["CL"], "CD": f["CD"], "Cm": f["Cm"],
               "CDi": self.case.trefftz(), "Mmax": s.mach_max(2)}
        self.hist.append(rec)
        if len(self.hist) > 400:
            del self.hist[:len(self.hist) - 400]
        self.conv = self.conv or converged(self.hist, self.res, self.res0)
        if s.it > self.MAX_ITERS:
            self.conv = True
        return rec

    def run(self, max_iters=None):
        """Step and read back until converged (or max_iters more iterations); returns the last record."""
        limit = self.it + (max_iters if max_iters is not None else self.MAX_ITERS + 1)
        rec = None
        while not self.conv and self.it < limit:
            self.case.solver.step(min(self.check_every, limit - self.it))
            rec = self.readback()
        return rec


def converged(hist, res, res0, drop=Controller.RES_DROP, window=Controller.CL_WINDOW, tol=Controller.CL_TOL,
              min_history=Controller.MIN_HISTORY):
    """The app's convergence test on a readback history (src/air_cfd.js:575)."""
    if len(hist) < min_history or not (res0 and res0 > 0) or res is None or not (res / res0 < drop):
        return False
    cl = [h["CL"] for h in hist[-window:]]
    return max(cl) - min(cl) < tol
