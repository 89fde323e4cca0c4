"""Host logic on CPU: file readers, centring, the half-shifted transform
and the natural spline of the oracle, and the product's C++ readers (via
the CLI-free C ABI is impossible without a GPU, so the product readers are
exercised in the GPU tests)."""
import os

import numpy as np
import pytest
from scipy.interpolate import CubicSpline

from conftest import GOLDEN
from oracle import formats as F
from oracle import oracle as O


def test_read_xvk_merges_sites(golden):
    sv = F.read_xvk(os.path.join(golden, "h2o_vv.xvk"))
    assert sv.natv == 2 and sv.ntab == 4096 and sv.dr == 0.05
    assert sv.temper == 298.0
    # H sites (SYM 2 and -2) merged: density doubles (solvent_read.cc:71-77)
    assert np.isclose(sv.rhov[1], 2 * sv.rhov[0])
    assert np.isclose(sv.rhov[0], 54.0 * F.AVOGADRO * 1e-27)
    assert sv.qv[0] == -0.834 and sv.qv[1] == 0.417
    # last row of the file: X[H][H] -> ~1.0078 at high k, X[O][H] ~ 2 X[H][O]
    assert abs(sv.xvv[1, 1, -1] - 1.00784025240904) < 1e-12
    assert abs(sv.xvv[0, 1, -1] - 2 * sv.xvv[1, 0, -1]) < 1e-9


def test_read_control_and_split_form(golden):
    c1, s1 = F.read_control(os.path.join(golden, "test1.inp"))
    c2, s2 = F.read_control(os.path.join(golden, "test1_c"), os.path.join(golden, "test1_s"))
    assert c1.grid == c2.grid == (64, 64, 64)
    assert c1.closure == 0 and c1.count == 2 and c1.m == 0.6 and c1.mp == 0.2
    assert np.array_equal(s1.xyz, s2.xyz) and np.array_equal(s1.q, s2.q)


def test_bad_control_rejected(tmp_path, golden):
    txt = open(os.path.join(golden, "test1.inp")).read().replace("20220301", "20210101")
    p = tmp_path / "old.inp"
    p.write_text(txt)
    with pytest.raises(ValueError):
        F.read_control(str(p))
    txt = open(os.path.join(golden, "test1.inp")).read().replace("KH", "PY")
    p.write_text(txt)
    with pytest.raises(ValueError):
        F.read_control(str(p))


def test_centre_rounds_half_away_from_zero():
    xyz = np.array([[0.0, 0.0, 0.0], [3.0, 1.0, -5.0]])
    shift = F.centre(xyz)
    # -(3-0)/2 - 0 = -1.5 -> -2 (C round), y: -0.5 -> -1, z: -(0+5)/2+5 = 2.5 -> 3
    assert shift == (-2.0, -1.0, 3.0)


def test_half_shifted_fft_matches_direct_sum():
    n, L = 8, 4.0
    rng = np.random.default_rng(0)
    f = rng.normal(size=(n, n, n))          # [z][y][x]
    F_or = O.fft3d(f.astype(complex).ravel(), (n, n, n), (L, L, L), -1).reshape(n, n, n)
    dr = L / n
    r = (np.arange(n) - n // 2) * dr
    k = 2 * np.pi * (np.arange(n) - n / 2 + 0.5) / L
    ph = np.exp(-1j * np.outer(k, r))        # [k][r]
    direct = np.einsum("az,by,cx,zyx->abc", ph, ph, ph, f) * dr ** 3
    assert np.allclose(F_or, direct, atol=1e-12 * np.abs(direct).max())
    # inverse round trip
    back = O.fft3d(F_or.ravel(), (n, n, n), (L, L, L), +1).reshape(n, n, n)
    assert np.allclose(back.real, f, atol=1e-12) and np.abs(back.imag).max() < 1e-12
    # F(-k) = conj F(k): the mirror of linear index j is N-1-j
    flat = F_or.ravel()
    assert np.allclose(flat[::-1], np.conj(flat), atol=1e-12 * np.abs(flat).max())


@pytest.mark.parametrize("n", [12, 48, 96])
def test_oracle_fft_mixed_radix(n):
    rng = np.random.default_rng(n)
    a = rng.normal(size=(4, 4, n)) + 1j * rng.normal(size=(4, 4, n))
    L = 1.0
    got = O.fft3d(a.ravel(), (n, 4, 4), (L, L, L), -1).reshape(4, 4, n)
    # undo the oracle's twiddles with the definition, compare to numpy
    idx = [np.arange(m) for m in (4, 4, n)]
    iz, iy, ix = np.meshgrid(*idx, indexing="ij")
    dirs = np.where((ix + iy + iz) % 2 == 0, 1.0, -1.0)
    dkr = np.pi / n * (ix - n // 2) + np.pi / 4 * (iy - 2) + np.pi / 4 * (iz - 2)
    dkf = np.cos(dkr) - 1j * np.sin(dkr)
    dv = L ** 3 / (16 * n)
    want = dv * dirs * np.fft.fftn(dirs * dkf * a)
    assert np.allclose(got, want, atol=1e-12 * np.abs(want).max())


def test_spline_is_natural_cubic():
    x = np.linspace(0.1, 5.0, 60)
    y = np.sin(x) * np.exp(-0.3 * x)
    q = np.linspace(0.05, 5.2, 333)
    got = O.spline_eval(x, y, q)
    cs = CubicSpline(x, y, bc_type="natural", extrapolate=True)
    assert np.allclose(got, cs(q), atol=1e-12)


def test_oracle_chi_grid_uses_unique_k(golden):
    sv = F.read_xvk(os.path.join(golden, "h2o_vv.xvk"))
    case = O.Case((8, 8, 8), (6.0, 6.0, 6.0), sv, [3.0], [500.0], [0.0], [[0, 0, 0]])
    x = O.chi_grid(case).reshape(2, 2, 8, 8, 8)
    # chi depends on |k| only: symmetric under x<->y<->z permutations
    assert np.allclose(x, x.transpose(0, 1, 2, 4, 3))
    assert np.allclose(x, x.transpose(0, 1, 4, 3, 2))


def test_esp_cube_reader_orders_values_x_fastest(tmp_path):
    """cal_Coulomb.cu:41-88: two comment lines, natom / origin / one more
    number, three axis lines, natom atom lines, then values with z fastest;
    the reader returns them x fastest and refuses a cube on another grid."""
    nx, ny, nz = 4, 3, 2
    vals = np.arange(nx * ny * nz, dtype=float) * 0.5          # cube order: ix, iy, iz
    lines = ["comment", "comment", "    1    0.0    0.0    0.0    1",
             "%5d 0.5 0.0 0.0" % nx, "%5d 0.0 0.5 0.0" % ny, "%5d 0.0 0.0 0.5" % nz,
             "    8   -0.5   0.0   0.0   0.0"]
    lines += [" ".join("%13.5E" % v for v in vals[i:i + 6]) for i in range(0, vals.size, 6)]
    p = tmp_path / "t.cube"
    p.write_text("\n".join(lines) + "\n")
    got = F.read_esp_cube(str(p), (nx, ny, nz))
    cube = vals.reshape(nx, ny, nz)
    for ix, iy, iz in ((0, 0, 0), (3, 0, 1), (1, 2, 0), (3, 2, 1)):
        assert got[ix + nx * (iy + ny * iz)] == cube[ix, iy, iz]
    with pytest.raises(ValueError):
        F.read_esp_cube(str(p), (4, 4, 2))


def test_hard_sphere_table_and_cvk_beside_the_xvk(tmp_path):
    """solvent_read.cc:88-140: the .cvk (same layout as the .xvk, same stem)
    and the -r table (ntab2; packing fraction and w(0); rows k chs w)."""
    p = tmp_path / "hs.xsv"
    p.write_text("3\n0.4 1.05\n0 -700.0 1.05\n0.1 -690.5 1.04\n0.2 -680.25 1.02\n")
    hs = F.read_hard_sphere(str(p))
    assert hs.ntab2 == 3 and hs.pfhs == 0.4 and hs.wfk0 == 1.05
    assert np.array_equal(hs.k, [0.0, 0.1, 0.2]) and hs.chs[2] == -680.25 and hs.w[1] == 1.04
    p.write_text("4\n0.4 1.05\n0 -700.0 1.05\n")
    with pytest.raises(ValueError):
        F.read_hard_sphere(str(p))
    xvk = os.path.join(GOLDEN, "rmdft_h2o_vv.xvk")
    cvk = F.read_cvk(xvk)
    sv = F.read_xvk(xvk)
    assert cvk.shape == sv.xvv.shape
    assert not np.allclose(cvk, sv.xvv)
