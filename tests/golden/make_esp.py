"""ESP cube for the -e parity case (the reference reads it in
cal_Coulomb.cu:41-96): the potential of the solute's charges smeared as
Gaussians of width a = 1 bohr, phi(r) = sum_u q_u erf(|r - R_u| / a) / |r - R_u|
in Hartree/e (distances in bohr), at the cell's grid points
r = ((i - n/2) d) with the control file's coordinates (-e also switches
centring off, main.cu:37-41).  The smearing makes it differ from the
point-charge potential near every atom, so a solve that ignored the cube
would not match.

    python tests/golden/make_esp.py CONTROL.inp OUT.cube

The cube is regenerated wherever it is needed (a few MB of text); the same
function feeds the reference run (run_reference.py) and the tests.
"""
import os
import sys

import numpy as np
from scipy.special import erf

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import formats as F  # noqa: E402

WIDTH = 1.0          # bohr


def esp_values(inp):
    """(grid, box, values) with values [N] x fastest, Hartree/e."""
    ctrl, sol = F.read_control(inp, None, centering=False, zero=False)
    nx, ny, nz = ctrl.grid
    d = [ctrl.box[k] / ctrl.grid[k] for k in range(3)]
    ax = [(np.arange(n) - n // 2) * dd for n, dd in zip(ctrl.grid, d)]
    X, Y, Z = np.meshgrid(ax[0], ax[1], ax[2], indexing="ij")      # [nx][ny][nz]
    phi = np.zeros(X.shape)
    for q, (x, y, z) in zip(sol.q, np.asarray(sol.xyz).reshape(-1, 3)):
        r = np.sqrt((X - x) ** 2 + (Y - y) ** 2 + (Z - z) ** 2) / F.BOHR
        with np.errstate(divide="ignore", invalid="ignore"):
            v = np.where(r > 1e-12, erf(r / WIDTH) / r, 2.0 / (WIDTH * np.sqrt(np.pi)))
        phi += q * v
    return ctrl.grid, ctrl.box, np.ascontiguousarray(phi.transpose(2, 1, 0)).ravel()


def write_cube(inp, path):
    grid, box, vals = esp_values(inp)
    _, sol = F.read_control(inp, None, centering=False, zero=False)
    nx, ny, nz = grid
    d = [box[k] / grid[k] / F.BOHR for k in range(3)]
    org = [-(grid[k] // 2) * d[k] for k in range(3)]
    xyz = np.asarray(sol.xyz).reshape(-1, 3) / F.BOHR
    L = ["ESP of Gaussian-smeared solute charges (width %.1f bohr)" % WIDTH,
         "values in Hartree/e, z fastest",
         "%5d%12.6f%12.6f%12.6f%5d" % (len(sol.q), org[0], org[1], org[2], 1)]
    for k, n in enumerate(grid):
        v = [0.0, 0.0, 0.0]
        v[k] = d[k]
        L.append("%5d%12.6f%12.6f%12.6f" % (n, v[0], v[1], v[2]))
    for q, p in zip(sol.q, xyz):
        L.append("%5d%12.6f%12.6f%12.6f%12.6f" % (1, q, p[0], p[1], p[2]))
    cube = vals.reshape(nz, ny, nx).transpose(2, 1, 0)               # [ix][iy][iz]
    with open(path, "w") as f:
        f.write("\n".join(L) + "\n")
        for ix in range(nx):
            for iy in range(ny):
                row = cube[ix, iy]
                for s in range(0, nz, 6):
                    f.write("".join("%13.5E" % v for v in row[s:s + 6]) + "\n")


if __name__ == "__main__":
    write_cube(sys.argv[1], sys.argv[2])
