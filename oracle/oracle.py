"""ctypes front end of the CPU FP64 oracle -- TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, as the checker; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build
from . import formats as F

MAXV = 16
_lib = None


class OracleInput(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("bx", C.c_double), ("by", C.c_double), ("bz", C.c_double),
        ("natv", C.c_int),
        ("rhov", C.POINTER(C.c_double)), ("qv", C.POINTER(C.c_double)),
        ("sigv", C.POINTER(C.c_double)), ("epsv", C.POINTER(C.c_double)),
        ("temper", C.c_double), ("xt", C.c_double),
        ("ntab", C.c_int), ("dr", C.c_double),
        ("xvv", C.POINTER(C.c_double)),
        ("natom", C.c_int),
        ("sig", C.POINTER(C.c_double)), ("eps", C.POINTER(C.c_double)),
        ("q", C.POINTER(C.c_double)), ("xyz", C.POINTER(C.c_double)),
        ("closure", C.c_int), ("conv", C.c_double), ("maxstep", C.c_int),
        ("count", C.c_int), ("m", C.c_double), ("mp", C.c_double),
        ("chargeup", C.c_int),
        ("t_init", C.POINTER(C.c_double)),
        ("verbose", C.c_int),
        ("esp", C.POINTER(C.c_double)),
        ("cvv", C.POINTER(C.c_double)),
        ("ntab2", C.c_int),
        ("ttab2", C.POINTER(C.c_double)), ("chs", C.POINTER(C.c_double)),
        ("wfk", C.POINTER(C.c_double)),
        ("pfhs", C.c_double), ("wfk0", C.c_double),
    ]


class OracleResult(C.Structure):
    _fields_ = [
        ("xmu_sc", C.c_double * MAXV), ("xmu_sc_hnc", C.c_double * MAXV),
        ("xmu_gf", C.c_double * MAXV), ("ibeta", C.c_double),
        ("sfe_sc", C.c_double), ("sfe_sc_hnc", C.c_double), ("sfe_gf", C.c_double),
        ("pmv", C.c_double), ("pressure", C.c_double), ("cuv", C.c_double),
        ("se", C.c_double), ("se_lj", C.c_double), ("se_es", C.c_double),
        ("correction", C.c_double), ("rms", C.c_double),
        ("iterations", C.c_int), ("status", C.c_int),
        ("t_setup", C.c_double), ("t_iter", C.c_double), ("t_obs", C.c_double),
        ("sfe_rmdft", C.c_double),
    ]


def lib():
    global _lib
    if _lib is None:
        path = _build.build_oracle()
        _lib = C.CDLL(path)
        d = C.POINTER(C.c_double)
        _lib.oracle_solve.argtypes = [C.POINTER(OracleInput), C.POINTER(OracleResult),
                                      d, d, d, d, d, d, d]
        _lib.oracle_potentials.argtypes = [C.POINTER(OracleInput), d, d, d, d]
        _lib.oracle_fft3d.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double,
                                      C.c_double, C.c_double, d, C.c_int]
        _lib.oracle_chi_grid.argtypes = [C.POINTER(OracleInput), d]
        _lib.oracle_spline_eval.argtypes = [C.c_int, d, d, C.c_int, d, d]
    return _lib


def _p(a):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Case:
    """One solve: cell, solvent, solute and control, as contiguous arrays."""

    def __init__(self, grid, box, solvent: F.Solvent, sig, eps, q, xyz,
                 closure=0, conv=1e-6, maxstep=10000, count=2, m=0.6, mp=0.2,
                 chargeup=0, t_init=None, esp=None, cvv=None, hs=None):
        self.grid = tuple(int(g) for g in grid)
        self.box = tuple(float(b) for b in box)
        self.sv = solvent
        self.sig, self.eps, self.q = _f64(sig), _f64(eps), _f64(q)
        self.xyz = _f64(np.asarray(xyz).reshape(-1, 3))
        self.closure, self.conv, self.maxstep = closure, conv, maxstep
        self.count, self.m, self.mp, self.chargeup = count, m, mp, chargeup
        self.t_init = None if t_init is None else _f64(t_init)
        self.esp = None if esp is None else _f64(esp).ravel()
        self.cvv = None if cvv is None else _f64(cvv)     # RMDFT: .cvk table
        self.hs = hs                                       # RMDFT: F.HardSphere
        self._keep = []

    @property
    def n(self):
        return self.grid[0] * self.grid[1] * self.grid[2]

    def cstruct(self, verbose=0) -> OracleInput:
        sv = self.sv
        arrs = [_f64(sv.rhov), _f64(sv.qv), _f64(sv.sigv), _f64(sv.epsv), _f64(sv.xvv)]
        self._keep = arrs
        s = OracleInput()
        s.nx, s.ny, s.nz = self.grid
        s.bx, s.by, s.bz = self.box
        s.natv = sv.natv
        s.rhov, s.qv, s.sigv, s.epsv, s.xvv = [_p(a) for a in arrs]
        s.temper, s.xt, s.ntab, s.dr = sv.temper, sv.xt, sv.ntab, sv.dr
        s.natom = len(self.q)
        s.sig, s.eps, s.q, s.xyz = _p(self.sig), _p(self.eps), _p(self.q), _p(self.xyz)
        s.closure, s.conv, s.maxstep = self.closure, self.conv, self.maxstep
        s.count, s.m, s.mp, s.chargeup = self.count, self.m, self.mp, self.chargeup
        s.t_init = _p(self.t_init)
        s.verbose = verbose
        s.esp = _p(self.esp)
        if self.cvv is not None and self.hs is not None:
            hs = [_f64(self.hs.k), _f64(self.hs.chs), _f64(self.hs.w)]
            self._keep += hs
            s.cvv = _p(self.cvv)
            s.ntab2 = self.hs.ntab2
            s.ttab2, s.chs, s.wfk = [_p(a) for a in hs]
            s.pfhs, s.wfk0 = self.hs.pfhs, self.hs.wfk0
        return s


def case_from_inp(inp, structure=None, centering=True, zero=False, xvk=None,
                  chargeup=0):
    ctrl, sol = F.read_control(inp, structure, centering, zero)
    path = xvk or os.path.join(os.path.dirname(os.path.abspath(inp)), ctrl.fsolvent)
    sv = F.read_xvk(path)
    return Case(ctrl.grid, ctrl.box, sv, sol.sig, sol.eps, sol.q, sol.xyz,
                ctrl.closure, ctrl.conv, ctrl.maxstep, ctrl.count, ctrl.m,
                ctrl.mp, chargeup), ctrl, sol


def solve(case: Case, want_grids=False, verbose=0):
    L = lib()
    s = case.cstruct(verbose)
    r = OracleResult()
    nv, n, na = case.sv.natv, case.n, len(case.q)
    g = h = t = None
    if want_grids:
        g = np.zeros((nv, n)); h = np.zeros((nv, n)); t = np.zeros((nv, n))
    euv = np.zeros((2, nv, na)); dulj = np.zeros((na, 3)); due = np.zeros((na, 3))
    trace = np.zeros(max(1, case.maxstep * (case.chargeup + 1)))
    rc = L.oracle_solve(C.byref(s), C.byref(r), _p(g), _p(h), _p(t), _p(euv),
                        _p(dulj), _p(due), _p(trace))
    if rc == -4:
        raise ValueError("insufficient maximal T tabulated (hard-sphere table)")
    if rc != 0:
        raise RuntimeError("oracle_solve failed: %d" % rc)
    res = {k: getattr(r, k) for k, _ in OracleResult._fields_
           if not k.startswith("xmu")}
    res["xmu_sc"] = np.array(r.xmu_sc[:nv])
    res["xmu_sc_hnc"] = np.array(r.xmu_sc_hnc[:nv])
    res["xmu_gf"] = np.array(r.xmu_gf[:nv])
    res["euv"], res["dulj"], res["due"] = euv, dulj, due
    res["trace"] = trace[:r.iterations]
    if want_grids:
        res["g"], res["h"], res["t"] = g, h, t
    return res


def potentials(case: Case):
    L = lib()
    s = case.cstruct()
    nv, n = case.sv.natv, case.n
    u = np.zeros((nv, n)); e = np.zeros(n); fr = np.zeros(n); fk = np.zeros(2 * n)
    L.oracle_potentials(C.byref(s), _p(u), _p(e), _p(fr), _p(fk))
    return u, e, fr, fk[0::2] + 1j * fk[1::2]


def chi_grid(case: Case):
    L = lib()
    s = case.cstruct()
    nv, n = case.sv.natv, case.n
    x = np.zeros((nv, nv, n))
    if L.oracle_chi_grid(C.byref(s), _p(x)) != 0:
        raise ValueError("insufficient maximal T tabulated")
    return x


def fft3d(a: np.ndarray, grid, box, key: int) -> np.ndarray:
    L = lib()
    buf = np.empty(2 * a.size)
    buf[0::2] = a.real.ravel(); buf[1::2] = a.imag.ravel()
    L.oracle_fft3d(grid[0], grid[1], grid[2], box[0], box[1], box[2], _p(buf), key)
    return buf[0::2] + 1j * buf[1::2]


def spline_eval(xp, yp, xq):
    L = lib()
    xp, yp, xq = _f64(xp), _f64(yp), _f64(xq)
    yq = np.zeros_like(xq)
    L.oracle_spline_eval(len(xp), _p(xp), _p(yp), len(xq), _p(xq), _p(yq))
    return yq


def write_xmu(res: dict, path: str, closure: int, natv: int, rmdft: bool = False):
    """output_xmu.cu:7-111 (fixed, 5 decimals)."""
    ib = res["ibeta"]
    L = [" $RESULT"]
    if rmdft:                                        # output_xmu.cu:25-28
        L.append("SFE_RMDFT= %.5f !(J/mol)" % res["sfe_rmdft"])
        L.append("")
    L.append("SFE_SC= %.5f !(J/mol)" % (ib * res["xmu_sc"].sum()))
    L += ["  SFEC_SC(%d)= %.5f" % (i, ib * res["xmu_sc"][i]) for i in range(natv)]
    L.append("")
    if closure == 0:
        L.append("SFE_SC_HNC= %.5f !(J/mol)" % (ib * res["xmu_sc_hnc"].sum()))
        L += ["  SFEC_SC_HNC(%d)= %.5f" % (i, ib * res["xmu_sc_hnc"][i]) for i in range(natv)]
        L.append("")
    L.append("SFE_GF= %.5f !(J/mol)" % (ib * res["xmu_gf"].sum()))
    L += ["  SFEC_GF(%d)= %.5f" % (i, ib * res["xmu_gf"][i]) for i in range(natv)]
    L.append("")
    L.append("SE= %.5f !(J/mol)" % res["se"])
    L.append("  SE_LJ= %.5f" % res["se_lj"])
    L.append("  SE_ES= %.5f" % res["se_es"])
    L.append("")
    L.append("PMV= %.5f !(L/mol)" % (res["pmv"] * 1000))
    L.append("Pressure= %.5f !(J/m^3)" % (ib * res["pressure"]))
    L.append("Correction_Term= %.5f !(J/mol)" % res["correction"])
    L.append(" $END")
    with open(path, "w") as f:
        f.write("\n".join(L) + "\n")
