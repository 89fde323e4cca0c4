"""1D XRISM solvent tables through the library's C ABI (rism1d_solve,
rism1d_write_xvk): site-site susceptibilities X_ab(k) of a molecular
solvent for the 3D solver's .xvk input."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import KH, HNC, RismError, lib  # noqa: F401


class Params(C.Structure):
    _fields_ = [("temperature", C.c_double), ("ntab", C.c_int), ("dr", C.c_double),
                ("closure", C.c_int), ("convergence", C.c_double), ("maxstep", C.c_int),
                ("mixing", C.c_double), ("verbose", C.c_int),
                ("dielectric", C.c_double), ("smear", C.c_double)]


class Site(C.Structure):
    _fields_ = [("name", C.c_char * 8), ("spc", C.c_int), ("sym", C.c_int),
                ("sigma", C.c_double), ("epsilon", C.c_double), ("charge", C.c_double),
                ("x", C.c_double), ("y", C.c_double), ("z", C.c_double),
                ("density", C.c_double)]


def _bind():
    L = lib()
    if not getattr(L, "_rism1d_bound", False):
        d = C.POINTER(C.c_double)
        L.rism1d_solve.argtypes = [C.POINTER(Params), C.c_int, C.POINTER(Site), d, d,
                                   C.POINTER(C.c_int)]
        L.rism1d_write_xvk.argtypes = [C.c_char_p, C.POINTER(Params), C.c_int,
                                       C.POINTER(Site), d, C.c_double]
        L.rism1d_last_error.restype = C.c_char_p
        L._rism1d_bound = True
    return L


def make_sites(rows):
    """rows: (name, spc, sym, sigma, eps [J/mol], q, x, y, z, density [M])."""
    arr = (Site * len(rows))()
    for s, r in zip(arr, rows):
        s.name = r[0].encode()[:7]
        s.spc, s.sym = int(r[1]), int(r[2])
        s.sigma, s.epsilon, s.charge = float(r[3]), float(r[4]), float(r[5])
        s.x, s.y, s.z, s.density = float(r[6]), float(r[7]), float(r[8]), float(r[9])
    return arr


def read_sites(path):
    """Site rows and grid of an .xvk header (solvent_read.cc:31-47)."""
    lines = open(path).read().split("\n")
    f = lines[1].split()
    num, ntab, dr = int(f[1]), int(f[3]), float(f[4])
    temper = float(lines[2].split()[2])
    rows = []
    for ln in lines[4:4 + num]:
        t = ln.split()
        rows.append((t[1], int(t[2]), int(t[3])) + tuple(float(v) for v in t[4:11]))
    return rows, temper, ntab, dr


def solve(rows, temperature, ntab=4096, dr=0.05, closure=KH, convergence=1e-12,
          maxstep=10000, mixing=0.0, verbose=0, dielectric=0.0, smear=0.0):
    """Returns (xvv [ntype, ntype, ntab], xt [1/Pa], iterations).
    dielectric > 0 selects DRISM with that dielectric constant (smear: the
    bridge's damping length in A, 0 = 2.0); mixing 0 takes the solver's
    default (0.3 for XRISM, 0.1 for DRISM)."""
    L = _bind()
    p = Params(temperature, ntab, dr, closure, convergence, maxstep, mixing, verbose,
               dielectric, smear)
    sites = make_sites(rows)
    nt = max(abs(int(r[2])) for r in rows)
    xvv = np.zeros((nt, nt, ntab))
    xt = C.c_double()
    it = C.c_int()
    rc = L.rism1d_solve(C.byref(p), len(rows), sites,
                        xvv.ctypes.data_as(C.POINTER(C.c_double)), C.byref(xt), C.byref(it))
    if rc != 0:
        raise RismError(rc, L.rism1d_last_error().decode())
    return xvv, xt.value, it.value


def write_xvk(path, rows, temperature, xvv, xt, ntab=4096, dr=0.05, closure=KH):
    L = _bind()
    p = Params(temperature, ntab, dr, closure, 0.0, 0, 0.0, 0)
    sites = make_sites(rows)
    x = np.ascontiguousarray(xvv, dtype=np.float64)
    rc = L.rism1d_write_xvk(path.encode(), C.byref(p), len(rows), sites,
                            x.ctypes.data_as(C.POINTER(C.c_double)), float(xt))
    if rc != 0:
        raise RismError(rc, L.rism1d_last_error().decode())
