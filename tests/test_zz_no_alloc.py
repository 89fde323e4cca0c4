"""rism3d_exchem_noalloc: the allocation-free mu_ex / PMV integrals, for
callers that cannot call cudaMalloc (their own pool allocator holds the
free device memory, or they cannot afford cudaMalloc's implicit device
synchronisation).  Checked through the C ABI against the integrals that
rism3d_solve reports for the same solution, on two calls in a row (the
calls share one static scratch array).  Collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

from helpers import MU_TOL, load_case, product_solver

pytestmark = pytest.mark.gpu


def test_noalloc_exchem_matches_solve_twice():
    import torch
    import rism3d_b200 as R
    case, _, _ = load_case("test1")
    s = product_solver(case)
    r = s.solve()
    V, n = case.sv.natv, case.n
    dv = case.box[0] * case.box[1] * case.box[2] / n
    h = torch.tensor(s.grid_array(R.GRID_H), dtype=torch.float64, device="cuda")
    t = torch.tensor(s.grid_array(R.GRID_T), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    L = R.lib()
    f = L.rism3d_exchem_noalloc
    dp = C.POINTER(C.c_double)
    f.argtypes = [C.c_int, C.c_int, C.c_longlong, C.c_double, C.c_double, dp,
                  C.c_void_p, C.c_void_p, C.c_void_p, dp]
    rho = np.ascontiguousarray(case.sv.rhov, dtype=np.float64)
    ibeta = 6.02214076e23 * 1.380649e-23 * case.sv.temper
    for call in range(2):
        out = np.zeros(3 * V + 1)
        rc = f(case.closure, V, n, dv, case.sv.temper, rho.ctypes.data_as(dp),
               h.data_ptr(), t.data_ptr(), None, out.ctypes.data_as(dp))
        assert rc == R.OK, L.rism3d_last_error(None)
        assert np.all(np.abs(out[:V] - r["sfec_sc"]) < MU_TOL), call
        assert np.all(np.abs(out[V:2 * V] - r["sfec_sc_hnc"]) < MU_TOL), call
        assert np.all(np.abs(out[2 * V:3 * V] - r["sfec_gf"]) < MU_TOL), call
        pmv = case.sv.xt * (1.0 - out[3 * V]) * ibeta * 1000.0
        assert abs(pmv - r["pmv"]) < 1e-4, call
    # beyond the stated limit: a clear error, nothing launched
    rc = f(case.closure, R.MAX_SITES + 1, n, dv, case.sv.temper, rho.ctypes.data_as(dp),
           h.data_ptr(), t.data_ptr(), None, out.ctypes.data_as(dp))
    assert rc == R.UNSUPPORTED_SHAPE
    assert b"natv" in L.rism3d_last_error(None)
    s.close()
