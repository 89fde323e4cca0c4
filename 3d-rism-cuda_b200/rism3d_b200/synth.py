"""Seeded synthetic solutes for the benchmark workloads.

The reference publishes no benchmark suite; its only protein-scale input is
ProteinG (846 atoms, 128 A cell, 256^3 grid).  These generators stand in for
it with seeded synthetic molecules of the stated shapes:

* ``small_chain``  -- 12-atom bonded chain, bonds U[1.0, 1.5] A (64^3, 32 A)
* ``globule``      -- 300 atoms uniform in a 12 A sphere, d_min 1.2 A (128^3, 64 A)
* ``protein_like`` -- 846-atom compact random chain, 3.8 A steps, confined so
                      that the radius of gyration is ~15 A (256^3, 128 A)
* ``small_batch``  -- 256 molecules of 8-40 atoms on 48^3 / 64^3 / 96^3 grids
                      at 0.5 A spacing

Charges are U[-0.8, 0.8] (chains, globule) or N(0, 0.3) (protein-like),
shifted to net zero; epsilon U[0.05, 0.2] kcal/mol, stored in J/mol (x4184)
as the reference's solute format expects (read_input.cu:72-76).
"""
from __future__ import annotations

import numpy as np

KCAL2J = 4184.0


class Solute:
    def __init__(self, sig, eps, q, xyz, grid, box, name):
        self.sig = np.asarray(sig, float)
        self.eps = np.asarray(eps, float)
        self.q = np.asarray(q, float)
        self.xyz = np.asarray(xyz, float).reshape(-1, 3)
        self.grid = tuple(grid)
        self.box = tuple(float(b) for b in box)
        self.name = name

    @property
    def natom(self):
        return len(self.q)

    def rg(self):
        c = self.xyz.mean(axis=0)
        return float(np.sqrt(((self.xyz - c) ** 2).sum(axis=1).mean()))

    def write_inp(self, path, xvk="h2o_vv.xvk", closure="KH", conv=1.0e-6,
                  maxstep=10000, an2=(2, 0.6, 0.2), outlist="m"):
        """Control file in the reference's format (read_input.cu:29-76)."""
        L = [" %s    0  20220301" % outlist, " %s" % closure, " %s" % xvk,
             " %.1e   %d" % (conv, maxstep), " %d   %g   %g" % an2,
             "  %g  %g  %g" % self.box, "  %d  %d  %d" % self.grid,
             "%d" % self.natom]
        for i in range(self.natom):
            L.append("%.10f %.6f %.10f %.6f %.6f %.6f" % (
                self.sig[i], self.eps[i], self.q[i], *self.xyz[i]))
        with open(path, "w") as f:
            f.write("\n".join(L) + "\n")


def _chain(rng, n, lo, hi, min_sep=0.0, max_tries=200):
    xyz = np.zeros((n, 3))
    for i in range(1, n):
        for _ in range(max_tries):
            d = rng.normal(size=3)
            d /= np.linalg.norm(d)
            p = xyz[i - 1] + d * rng.uniform(lo, hi)
            if i < 2 or min_sep <= 0 or np.min(np.linalg.norm(xyz[:i - 1] - p, axis=1)) >= min_sep:
                break
        xyz[i] = p
    return xyz


def _params(rng, n, sig_lo, sig_hi, qmode):
    sig = rng.uniform(sig_lo, sig_hi, n)
    eps = rng.uniform(0.05, 0.2, n) * KCAL2J
    if qmode == "uniform":
        q = rng.uniform(-0.8, 0.8, n)
    else:
        q = rng.normal(0.0, 0.3, n)
    q = q - q.mean()
    return sig, eps, q


def small_chain(seed=0, natom=12, grid=(64, 64, 64), box=(32.0, 32.0, 32.0)):
    rng = np.random.default_rng(seed)
    xyz = _chain(rng, natom, 1.0, 1.5, min_sep=1.0)
    sig, eps, q = _params(rng, natom, 2.5, 3.8, "uniform")
    return Solute(sig, eps, q, xyz, grid, box, "chain%d_s%d" % (natom, seed))


def globule(seed=1, natom=300, radius=12.0, dmin=1.2, grid=(128, 128, 128),
            box=(64.0, 64.0, 64.0)):
    rng = np.random.default_rng(seed)
    pts = []
    while len(pts) < natom:
        p = rng.uniform(-radius, radius, 3)
        if np.linalg.norm(p) > radius:
            continue
        if pts and np.min(np.linalg.norm(np.array(pts) - p, axis=1)) < dmin:
            continue
        pts.append(p)
    sig, eps, q = _params(rng, natom, 2.5, 3.8, "uniform")
    return Solute(sig, eps, q, np.array(pts), grid, box, "globule%d_s%d" % (natom, seed))


def protein_like(seed=2, natom=846, step=3.8, rg=15.0, dmin=2.6,
                 grid=(256, 256, 256), box=(128.0, 128.0, 128.0)):
    """Random chain with fixed 3.8 A steps inside a sphere of radius
    sqrt(5/3)*rg (a uniformly filled sphere has that radius of gyration)."""
    rng = np.random.default_rng(seed)
    R = np.sqrt(5.0 / 3.0) * rg
    xyz = np.zeros((natom, 3))
    i = 1
    while i < natom:
        placed = False
        for _ in range(500):
            d = rng.normal(size=3)
            d /= np.linalg.norm(d)
            p = xyz[i - 1] + step * d
            if np.linalg.norm(p) > R:
                continue
            if i >= 2 and np.min(np.linalg.norm(xyz[:i - 1] - p, axis=1)) < dmin:
                continue
            placed = True
            break
        if not placed:          # dead end: back off a few residues
            i = max(1, i - 5)
            continue
        xyz[i] = p
        i += 1
    sig, eps, q = _params(rng, natom, 3.0, 3.8, "normal")
    return Solute(sig, eps, q, xyz, grid, box, "protein%d_s%d" % (natom, seed))


def small_batch(seed=3, nmol=256, spacing=0.5, grids=(48, 64, 96)):
    rng = np.random.default_rng(seed)
    mols = []
    for k in range(nmol):
        n = int(rng.integers(8, 41))
        g = int(grids[rng.integers(0, len(grids))])
        L = g * spacing
        s = small_chain(seed=int(rng.integers(0, 2**31 - 1)), natom=n,
                        grid=(g, g, g), box=(L, L, L))
        s.name = "mol%03d" % k
        mols.append(s)
    return mols
