"""The SE totals the solver takes from the potential grids equal the
reference's per-(site, atom) pair sums (cal_euv.cu:7-76), checked on the CPU
oracle: sum over the grid of g u_v and g e (the grids of cal_LJ.cu and
cal_Coulomb.cu, r^2 clamped at 1e-4 and r < 1e-5 skipped) minus each atom's
own terms at the points with r < sigma_uv / 2 reproduces SE_LJ and SE_ES."""
import numpy as np

from helpers import load_case
from oracle import formats as F
from oracle import oracle as O


def test_grid_form_of_se_matches_pair_sums():
    case, _, _ = load_case("cfg0_chain12")
    res = O.solve(case, want_grids=True)
    u, e, _, _ = O.potentials(case)
    g = res["g"]
    sv = case.sv
    nx, ny, nz = case.grid
    d = [case.box[k] / case.grid[k] for k in range(3)]
    dv = d[0] * d[1] * d[2]
    T = sv.temper
    ibeta = F.AVOGADRO * F.BOLTZMANN * T
    ubeta = F.HARTREE * F.BOHR / (F.BOLTZMANN * T)
    cc = F.HARTREE * F.BOHR * F.AVOGADRO
    ax = [(np.arange(n) - n // 2) * dd for n, dd in zip(case.grid, d)]
    X, Y, Z = np.meshgrid(ax[0], ax[1], ax[2], indexing="ij")
    slj = ses = 0.0
    for v in range(sv.natv):
        gv = g[v].reshape(nz, ny, nx).transpose(2, 1, 0)          # [ix][iy][iz]
        sg_lj = float(np.sum(g[v] * u[v]))
        sg_es = float(np.sum(g[v] * e)) / ubeta
        c_lj = c_es = 0.0
        for iu in range(len(case.q)):
            sig = (case.sig[iu] + sv.sigv[v]) * 0.5
            r2 = (X - case.xyz[iu, 0]) ** 2 + (Y - case.xyz[iu, 1]) ** 2 + (Z - case.xyz[iu, 2]) ** 2
            r = np.sqrt(r2)
            core = r < sig * 0.5
            ir2 = np.where(r2 < 1e-4, 1e4, 1.0 / np.maximum(r2, 1e-300))
            s6 = (sig * sig * ir2) ** 3
            e4 = 4.0 * np.sqrt(case.eps[iu] * sv.epsv[v]) / ibeta
            c_lj += float(np.sum(np.where(core, gv * e4 * s6 * (s6 - 1.0), 0.0)))
            c_es += float(np.sum(np.where(core & (r >= 1e-5), gv * case.q[iu] / np.maximum(r, 1e-300), 0.0)))
        slj += sv.rhov[v] * ibeta * (sg_lj - c_lj) * dv
        ses += sv.rhov[v] * sv.qv[v] * cc * (sg_es - c_es) * dv
    assert abs(slj - res["se_lj"]) <= 1e-9 * abs(res["se_lj"]) + 1e-9, (slj, res["se_lj"])
    assert abs(ses - res["se_es"]) <= 1e-9 * abs(res["se_es"]) + 1e-9, (ses, res["se_es"])
