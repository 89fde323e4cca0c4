"""1D XRISM solvent tables (rism1d_solve): the reference ships water
susceptibility tables made by a program it does not include; the library's
own 1D solver reproduces them from the model in their headers.  Runs on the
CPU (host code of the library; no GPU involved)."""
import os

import numpy as np

from conftest import GOLDEN
from oracle import formats as F


def _solve_shipped_water():
    from rism3d_b200 import xrism1d as X
    rows, T, ntab, dr = X.read_sites(os.path.join(GOLDEN, "h2o_vv.xvk"))
    return X, rows, T, ntab, dr, X.solve(rows, T, ntab, dr, convergence=1e-10)


def test_water_table_matches_the_shipped_xvk():
    """example/h2o_vv.xvk (TIP3P-like water, 298 K, 54 M, 4096 x 0.05 A):
    X_ab(k) to 2e-5 absolute at every k, chi_T to 2e-5 relative."""
    X, rows, T, ntab, dr, (xvv, xt, it) = _solve_shipped_water()
    ref = F.read_xvk(os.path.join(GOLDEN, "h2o_vv.xvk"))
    assert xvv.shape == ref.xvv.shape
    assert np.abs(xvv - ref.xvv).max() < 2e-5
    assert abs(xt - ref.xt) < 2e-5 * ref.xt
    # k -> pi/dr: the intramolecular terms alone (h vanishes on this grid)
    assert xvv[0, 0, -1] == 1.0


def test_written_table_reads_back(tmp_path):
    X, rows, T, ntab, dr, (xvv, xt, it) = _solve_shipped_water()
    path = str(tmp_path / "w.xvk")
    X.write_xvk(path, rows, T, xvv, xt, ntab, dr)
    back = F.read_xvk(path)
    ref = F.read_xvk(os.path.join(GOLDEN, "h2o_vv.xvk"))
    assert back.natv == ref.natv and back.ntab == ref.ntab
    assert np.allclose(back.rhov, ref.rhov) and np.allclose(back.qv, ref.qv)
    assert np.allclose(back.sigv, ref.sigv) and np.allclose(back.epsv, ref.epsv)
    assert abs(back.temper - T) < 1e-9 and abs(back.xt - xt) < 1e-9 * xt
    assert np.abs(back.xvv - xvv).max() < 1e-14


def test_bad_input_is_an_error():
    import pytest
    from rism3d_b200 import RismError
    from rism3d_b200 import xrism1d as X
    rows = [("O", 1, 1, 3.15, 636.0, 0.0, 0.0, 0.0, 0.0, 54.0)]
    with pytest.raises(RismError):
        X.solve(rows, 298.0, ntab=1000, dr=0.05)          # not a power of two
    with pytest.raises(RismError):
        X.solve([rows[0][:9] + (-1.0,)], 298.0, ntab=256)  # negative density


def test_cli_writes_a_table_the_3d_reader_accepts(tmp_path):
    """bin/rism1d-b200 on a sites file: the written .xvk parses with the
    reference's reader layout and equals the library call's table."""
    import subprocess
    from conftest import ROOT
    from rism3d_b200 import xrism1d as X
    rows, T, ntab, dr = X.read_sites(os.path.join(GOLDEN, "h2o_vv.xvk"))
    sites = tmp_path / "water.sites"
    sites.write_text("# name spc sym sigma eps q x y z density\n" +
                     "\n".join(" ".join(str(v) for v in r) for r in rows) + "\n")
    out = tmp_path / "water_vv.xvk"
    exe = os.path.join(ROOT, "3d-rism-cuda_b200", "bin", "rism1d-b200")
    p = subprocess.run([exe, "-T", str(T), "-n", "1024", "-r", "0.1", "-e", "1e-10",
                        str(sites), str(out)], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    back = F.read_xvk(str(out))
    xvv, xt, _ = X.solve(rows, T, 1024, 0.1, convergence=1e-10)
    assert back.ntab == 1024 and back.natv == 2
    assert np.abs(back.xvv - xvv).max() < 1e-12
    assert abs(back.xt - xt) < 1e-8 * xt


def test_hnc_closure_converges_for_water():
    """The HNC closure (no linearisation of exp) on the same water model:
    converges, and its X(k) differs from KH only where g is large."""
    from rism3d_b200 import xrism1d as X
    rows, T, ntab, dr = X.read_sites(os.path.join(GOLDEN, "h2o_vv.xvk"))
    kh, xt_kh, _ = X.solve(rows, T, 1024, 0.1, closure=X.KH, convergence=1e-9)
    hnc, xt_hnc, _ = X.solve(rows, T, 1024, 0.1, closure=X.HNC, convergence=1e-9)
    assert np.all(np.isfinite(hnc)) and xt_hnc > 0
    assert np.abs(hnc[:, :, -200:] - kh[:, :, -200:]).max() < 1e-2   # large k: intramolecular


def test_drism_salt_solution_against_the_shipped_table():
    """The reference ships a salt-solution table, example/naclaq_vv.xvk
    (3-site water at 54 M with Na+ and Cl- at 0.1 M, 298 K, 4096 x 0.05 A;
    every 4th k row is kept in tests/golden/naclaq_sub4_vv.xvk), without the
    program that made it.  DRISM (dielectric 78.44, the bridge damped over
    2 A) reproduces, relative to each block's largest entry:
    - the water-water block to 4e-4 at every k, and chi_T to 3e-4;
    - every block with an ion to 3-8 % below k = 0.6 1/A and to 1 % above.
    The ion residual is a difference in the table's generator that the
    dielectric constant barely moves, so these bounds hold the measured
    agreement; they are not a pin.  Plain XRISM on this model lands on a
    negative concentration structure factor (ion entries off by ~0.7) and is
    refused by rism1d_solve's k -> 0 check."""
    from rism3d_b200 import xrism1d as X
    path = os.path.join(GOLDEN, "naclaq_sub4_vv.xvk")
    rows, T, _, dr = X.read_sites(path)
    ref = F.read_xvk(path)
    xvv, xt, it = X.solve(rows, T, 4096, dr, convergence=1e-6, dielectric=78.44)
    ours = xvv[:, :, 3::4]                   # the rows the fixture kept
    k = (4.0 * np.arange(1, 1025)) * np.pi / (4096 * dr)
    small = k < 0.6
    for a in range(4):
        for b in range(4):
            d = np.abs(ours[a, b] - ref.xvv[a, b]) / np.abs(ref.xvv[a, b]).max()
            if a < 2 and b < 2:              # water-water
                assert d.max() < 6e-4, (a, b, d.max())
            else:
                assert d[small].max() < 0.1 and d[~small].max() < 1.5e-2, (a, b)
    assert abs(xt / ref.xt - 1.0) < 5e-4
    assert ours[2, 2, 0] > 0.6 and ours[2, 3, 0] > 0.5   # the physical branch


def test_drism_needs_the_dipole_along_z():
    import pytest
    from rism3d_b200 import RismError
    from rism3d_b200 import xrism1d as X
    water = [("O", 1, 1, 3.15, 636.0, -0.834, 0.0, 0.0, 0.0, 54.0),
             ("H", 1, 2, 0.4, 192.5, 0.417, 0.58588, 0.7567, 0.0, 54.0),
             ("H", 1, -2, 0.4, 192.5, 0.417, 0.58588, -0.7567, 0.0, 54.0)]   # dipole along x
    with pytest.raises(RismError):
        X.solve(water, 298.0, ntab=256, dielectric=78.44)
