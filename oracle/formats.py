"""Readers for the reference's input files -- TEST INFRASTRUCTURE (oracle).

Independent Python restatement of the reference parsers, used by the tests
to feed identical arrays to the oracle and to check the product's C++
parsers:

* control file ``.inp`` / structure file   -- read_input.cu:21-89
* solute centring                          -- solute.cu:13-43
* solvent susceptibility file ``.xvk``     -- solvent_read.cc:10-86
* ESP cube ``-e``                          -- cal_Coulomb.cu:41-88
* physical constants                       -- physical.h:4-17
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

AVOGADRO = 6.02214076e23
BOHR = 0.5291771500001
BOLTZMANN = 1.380649e-23
HARTREE = 4.359744722207185e-18
KCAL2J = 4184.0
VERSION = "20220301"


def c_round(x: float) -> float:
    """C ``round()``: halves away from zero (Python's round is half-even)."""
    return math.copysign(math.floor(abs(x) + 0.5), x)


@dataclass
class Control:
    outlist: str
    ksave: int
    closure: int            # 0 KH, 1 HNC
    fsolvent: str
    conv: float
    maxstep: int
    count: int
    m: float
    mp: float
    box: tuple
    grid: tuple


@dataclass
class Solute:
    sig: np.ndarray
    eps: np.ndarray
    q: np.ndarray
    xyz: np.ndarray          # (natom, 3)
    shift: tuple = (0.0, 0.0, 0.0)


@dataclass
class Solvent:
    natv: int
    rhov: np.ndarray         # molecules / A^3
    qv: np.ndarray
    sigv: np.ndarray
    epsv: np.ndarray
    temper: float
    xt: float
    ntab: int
    dr: float
    xvv: np.ndarray          # (natv, natv, ntab)
    sites: list = field(default_factory=list)


def read_control(path: str, structure: str | None = None,
                 centering: bool = True, zero: bool = False):
    """read_input.cu:21-89: whitespace tokens, version check, atoms."""
    with open(path) as f:
        tok = f.read().split()
    it = iter(tok)
    outlist = next(it)
    ksave = int(next(it))
    if next(it) != VERSION:
        raise ValueError("This input file is for old version.")
    clos = next(it)
    if clos not in ("KH", "HNC"):
        raise ValueError("Unexpected closure switch")
    fsolvent = next(it)
    conv = float(next(it)); maxstep = int(next(it))
    count = int(next(it)); m = float(next(it)); mp = float(next(it))
    box = tuple(float(next(it)) for _ in range(3))
    grid = tuple(int(next(it)) for _ in range(3))
    ctrl = Control(outlist, ksave, 0 if clos == "KH" else 1, fsolvent, conv,
                   maxstep, count, m, mp, box, grid)
    if structure:
        with open(structure) as f:
            it = iter(f.read().split())
    num_s = next(it)
    if not num_s.isdigit():
        raise ValueError("Number of solute atom is not a natural number.")
    num = int(num_s)
    vals = np.array([float(next(it)) for _ in range(6 * num)]).reshape(num, 6)
    sol = Solute(sig=vals[:, 0].copy(), eps=vals[:, 1].copy(),
                 q=vals[:, 2].copy(), xyz=vals[:, 3:6].copy())
    if centering:
        sol.shift = centre(sol.xyz)
    if zero:
        sol.q[:] = 0.0
    return ctrl, sol


def centre(xyz: np.ndarray) -> tuple:
    """solute.cu:13-43: integer shift putting the bounding box at the origin."""
    lo = xyz.min(axis=0); hi = xyz.max(axis=0)
    shift = tuple(c_round(-(hi[d] - lo[d]) / 2 - lo[d]) for d in range(3))
    xyz += np.array(shift)
    return shift


def read_xvk(path: str) -> Solvent:
    """solvent_read.cc:10-86 (site table, merge by |SYM|, chi table)."""
    with open(path) as f:
        lines = f.read().split("\n")
    h1 = lines[1].split()
    num, natv, ntab, dr = int(h1[1]), int(h1[2]), int(h1[3]), float(h1[4])
    h2 = lines[2].split()
    temper, xt = float(h2[2]), float(h2[3])
    sigv = np.zeros(natv); epsv = np.zeros(natv); qv = np.zeros(natv)
    rhov = np.zeros(natv)
    sites = []
    for i in range(num):
        tk = lines[4 + i].split()
        sym = int(tk[3])
        i2 = abs(sym) - 1
        sigv[i2] = float(tk[4]); epsv[i2] = float(tk[5]); qv[i2] = float(tk[6])
        rhov[i2] += float(tk[10])
        sites.append((tk[1], int(tk[2]), sym, float(tk[4]), float(tk[5]),
                      float(tk[6]), float(tk[7]), float(tk[8]), float(tk[9]),
                      float(tk[10])))
    rhov *= AVOGADRO * 1.0e-27
    data = " ".join(lines[num + 5:]).split()
    need = ntab * natv * natv
    if len(data) < need:
        raise ValueError("short chi table in %s" % path)
    xvv = np.array([float(x) for x in data[:need]]).reshape(ntab, natv, natv)
    xvv = np.ascontiguousarray(xvv.transpose(1, 2, 0))
    return Solvent(natv, rhov, qv, sigv, epsv, temper, xt, ntab, dr, xvv, sites)


def read_esp_cube(path: str, grid) -> np.ndarray:
    """cal_Coulomb.cu:41-88: two comment lines; natom, origin and one more
    number; three axis lines whose counts must equal the cell grid; natom
    atom lines (skipped); then the values with z fastest.  Returns the
    values [N] in the solver's layout (x fastest), in Hartree/e."""
    with open(path) as f:
        f.readline(); f.readline()
        tok = f.read().split()
    natom = int(tok[0])
    pos = 5                                          # natom x0 y0 z0 di
    counts = []
    for _ in range(3):
        counts.append(int(tok[pos])); pos += 4
    if tuple(counts) != tuple(int(g) for g in grid):
        raise ValueError("cube file doesn't match input")
    pos += 5 * natom
    nx, ny, nz = counts
    vals = np.array([float(v) for v in tok[pos:pos + nx * ny * nz]])
    if vals.size != nx * ny * nz:
        raise ValueError("short ESP cube %s" % path)
    return np.ascontiguousarray(vals.reshape(nx, ny, nz).transpose(2, 1, 0)).ravel()


@dataclass
class HardSphere:
    """RMDFT hard-sphere table (solvent_read.cc:118-140): site 0's packing
    fraction and w(0), then rows k, chi_hs(k), w(k)."""
    ntab2: int
    pfhs: float
    wfk0: float
    k: np.ndarray
    chs: np.ndarray
    w: np.ndarray


def read_hard_sphere(path: str) -> HardSphere:
    with open(path) as f:
        lines = f.read().split("\n")
    ntab2 = int(lines[0].split()[0])
    pf, w0 = (float(x) for x in lines[1].split()[:2])
    rows = np.array([[float(x) for x in ln.split()[:3]] for ln in lines[2:2 + ntab2]])
    if rows.shape != (ntab2, 3):
        raise ValueError("short hard-sphere table %s" % path)
    return HardSphere(ntab2, pf, w0, rows[:, 0].copy(), rows[:, 1].copy(), rows[:, 2].copy())


def read_cvk(xvk_path: str) -> np.ndarray:
    """solvent_read.cc:94-116: the solvent c(k) table next to the .xvk (same
    stem, extension .cvk, same layout as the chi table); [natv][natv][ntab]."""
    stem = xvk_path[:xvk_path.rfind(".")] if "." in xvk_path else xvk_path
    return read_xvk(stem + ".cvk").xvv


def parse_xmu(path: str) -> dict:
    """Key = value lines of an .xmu file (output_xmu.cu:7-111)."""
    out = {}
    with open(path) as f:
        for line in f:
            s = line.strip()
            if "=" not in s:
                continue
            k, v = s.split("=", 1)
            out[k.strip()] = float(v.split()[0])
    return out
