"""ctypes binding of the rism3d_b200 C ABI (include/rism3d_b200.h).

The shared library is built in-tree by ``build.py`` (sm_100a).  Loading it
requires no GPU; every compute call does, and fails with a RismError when
the device or the library is missing -- there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librism3d_b200.so")
MAX_SITES = 8

OK, BAD_INPUT, UNSUPPORTED_SHAPE, CUDA_ERROR, CUFFT_ERROR, DIVERGED, NOT_CONVERGED, \
    NO_DEVICE, BAD_STATE = range(9)
KH, HNC = 0, 1
FP64, MIXED = 0, 1
GRID_G, GRID_H, GRID_C, GRID_T, GRID_U, GRID_E, GRID_FR, GRID_QV = range(8)

EXPORTS = ["rism3d_create", "rism3d_set_solvent", "rism3d_set_solute", "rism3d_set_tuv",
           "rism3d_solve", "rism3d_euv", "rism3d_forces", "rism3d_grad", "rism3d_grad_precision", "rism3d_get_grid",
           "rism3d_solve_batch", "rism3d_destroy", "rism3d_last_error",
           "rism3d_initialize", "rism3d_iterate", "rism3d_output",
           "rism3d_refresh_potentials", "rism3d_kernel_launches", "rism3d_time_kernel",
           "rism3d_set_esp", "rism3d_set_rmdft", "rism3d_get_grid_device"]


class RismError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("rism3d error %d: %s" % (code, msg))
        self.code = code


class Params(C.Structure):
    _fields_ = [("grid", C.c_int * 3), ("box", C.c_double * 3), ("closure", C.c_int),
                ("convergence", C.c_double), ("maxstep", C.c_int), ("an2_count", C.c_int),
                ("an2_m", C.c_double), ("an2_mp", C.c_double), ("precision", C.c_int),
                ("mixed_switch", C.c_double), ("device", C.c_int), ("verbose", C.c_int),
                ("stream", C.c_void_p), ("batch_chunk_points", C.c_longlong)]


class Result(C.Structure):
    _fields_ = [("natv", C.c_int), ("natom", C.c_int), ("sfe_sc", C.c_double),
                ("sfe_sc_hnc", C.c_double), ("sfe_gf", C.c_double),
                ("sfec_sc", C.c_double * MAX_SITES), ("sfec_sc_hnc", C.c_double * MAX_SITES),
                ("sfec_gf", C.c_double * MAX_SITES), ("pmv", C.c_double),
                ("pressure", C.c_double), ("correction", C.c_double), ("se", C.c_double),
                ("se_lj", C.c_double), ("se_es", C.c_double), ("rms", C.c_double),
                ("iterations", C.c_int), ("iterations_fp32", C.c_int), ("status", C.c_int),
                ("ms_setup", C.c_double), ("ms_iterate", C.c_double), ("ms_observe", C.c_double),
                ("sfe_rmdft", C.c_double)]

    def as_dict(self):
        d = {}
        for k, _ in self._fields_:
            v = getattr(self, k)
            if k.startswith("sfec"):
                v = np.array(v[:self.natv])
            d[k] = v
        return d


_lib = None


def lib():
    """Load the in-tree library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RismError(CUDA_ERROR, "librism3d_b200.so not built (run build.py)")
        L = C.CDLL(LIB_PATH)
        d = C.POINTER(C.c_double)
        i = C.POINTER(C.c_int)
        vp = C.c_void_p
        L.rism3d_create.argtypes = [C.POINTER(Params), C.POINTER(vp)]
        L.rism3d_set_solvent.argtypes = [vp, C.c_int, d, d, d, d, C.c_double, C.c_double,
                                         C.c_int, C.c_double, d]
        L.rism3d_set_solute.argtypes = [vp, C.c_int, d, d, d, d]
        L.rism3d_set_tuv.argtypes = [vp, d]
        L.rism3d_solve.argtypes = [vp, C.c_int, C.POINTER(Result)]
        L.rism3d_euv.argtypes = [vp, d]
        L.rism3d_forces.argtypes = [vp, d, d]
        L.rism3d_grad.argtypes = [vp, d, d, d, d]
        L.rism3d_grad_precision.argtypes = [vp, C.c_int, d, d, d, d]
        L.rism3d_get_grid.argtypes = [vp, C.c_int, d]
        L.rism3d_solve_batch.argtypes = [vp, C.c_int, i, i, d, d, d, d, d, C.POINTER(Result)]
        L.rism3d_destroy.argtypes = [vp]
        L.rism3d_last_error.argtypes = [vp]
        L.rism3d_last_error.restype = C.c_char_p
        L.rism3d_initialize.argtypes = [C.POINTER(vp), C.c_char_p, C.c_char_p, C.c_char_p,
                                        C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int]
        L.rism3d_iterate.argtypes = [vp, C.c_int]
        L.rism3d_output.argtypes = [vp]
        L.rism3d_refresh_potentials.argtypes = [vp]
        L.rism3d_set_esp.argtypes = [vp, d]
        L.rism3d_get_grid_device.argtypes = [vp, C.c_int, vp]
        L.rism3d_set_rmdft.argtypes = [vp, d, C.c_int, d, d, d, C.c_double, C.c_double]
        L.rism3d_kernel_launches.argtypes = [vp]
        L.rism3d_kernel_launches.restype = C.c_longlong
        L.rism3d_time_kernel.argtypes = [vp, C.c_int, C.c_int, d]
        _lib = L
    return _lib


def _dp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Solver:
    """One solve context on one GPU (array-level API)."""

    def __init__(self, grid, box, closure=KH, convergence=1e-6, maxstep=10000,
                 an2=(2, 0.6, 0.2), precision=FP64, mixed_switch=0.0, device=0,
                 verbose=0, stream=None, batch_chunk_points=0):
        L = lib()
        p = Params()
        p.grid[:] = [int(g) for g in grid]
        p.box[:] = [float(b) for b in box]
        p.closure, p.convergence, p.maxstep = closure, convergence, maxstep
        p.an2_count, p.an2_m, p.an2_mp = int(an2[0]), float(an2[1]), float(an2[2])
        p.precision, p.mixed_switch, p.device, p.verbose = precision, mixed_switch, device, verbose
        p.stream = stream
        p.batch_chunk_points = int(batch_chunk_points)
        h = C.c_void_p()
        rc = L.rism3d_create(C.byref(p), C.byref(h))
        if rc != OK:
            raise RismError(rc, L.rism3d_last_error(None).decode())
        self.h = h
        self.device = device
        self.grid = tuple(p.grid)
        self.n = self.grid[0] * self.grid[1] * self.grid[2]
        self.natv = 0
        self.natom = 0

    def _check(self, rc, allow=(OK,)):
        if rc not in allow:
            raise RismError(rc, lib().rism3d_last_error(self.h).decode())
        return rc

    def set_solvent(self, natv, rho, q, sig, eps, temperature, xt, ntab, dr, xvv):
        self._keep_sv = [_f64(rho), _f64(q), _f64(sig), _f64(eps), _f64(xvv)]
        a = self._keep_sv
        self._check(lib().rism3d_set_solvent(self.h, natv, _dp(a[0]), _dp(a[1]), _dp(a[2]),
                                             _dp(a[3]), temperature, xt, ntab, dr, _dp(a[4])))
        self.natv = natv

    def set_solvent_obj(self, sv):
        """From any object with the fields of oracle.formats.Solvent."""
        self.set_solvent(sv.natv, sv.rhov, sv.qv, sv.sigv, sv.epsv, sv.temper, sv.xt,
                         sv.ntab, sv.dr, sv.xvv)

    def set_solute(self, sig, eps, q, xyz):
        sig, eps, q, xyz = _f64(sig), _f64(eps), _f64(q), _f64(np.asarray(xyz).reshape(-1, 3))
        self._check(lib().rism3d_set_solute(self.h, len(q), _dp(sig), _dp(eps), _dp(q), _dp(xyz)))
        self.natom = len(q)

    def set_esp(self, esp):
        """ESP cube values [N] (Hartree/e, x fastest) replacing the point-charge
        potential in the closure; None removes it (rism3d_set_esp)."""
        self._keep_esp = None if esp is None else _f64(np.asarray(esp).ravel())
        self._check(lib().rism3d_set_esp(self.h, _dp(self._keep_esp)))

    def set_rmdft(self, cvk, k=None, chs=None, w=None, pfhs=0.0, w0=0.0):
        """RMDFT tables (rism3d_set_rmdft): cvk [natv][natv][ntab] on the chi
        knots and site 0's hard-sphere table k, chs, w with its packing
        fraction and w(0); cvk None switches the correction off."""
        if cvk is None:
            self._check(lib().rism3d_set_rmdft(self.h, None, 0, None, None, None, 0.0, 0.0))
            return
        self._keep_rm = [_f64(cvk), _f64(k), _f64(chs), _f64(w)]
        cv, kk, cs, ww = self._keep_rm
        self._check(lib().rism3d_set_rmdft(self.h, _dp(cv), len(kk), _dp(kk), _dp(cs), _dp(ww),
                                           float(pfhs), float(w0)))

    def set_tuv(self, t):
        self._keep_t = None if t is None else _f64(t)
        self._check(lib().rism3d_set_tuv(self.h, _dp(self._keep_t)))

    def solve(self, chargeup=0, allow_unconverged=False):
        r = Result()
        allow = (OK, DIVERGED, NOT_CONVERGED) if allow_unconverged else (OK,)
        self._check(lib().rism3d_solve(self.h, chargeup, C.byref(r)), allow)
        return r.as_dict()

    def grid_array(self, which):
        nsite = self.natv if which in (GRID_G, GRID_H, GRID_C, GRID_T, GRID_U) else 1
        out = np.zeros((nsite, self.n))
        self._check(lib().rism3d_get_grid(self.h, which, _dp(out)))
        return out

    def grid_tensor(self, which):
        """The grid as a torch float64 tensor on the solver's GPU, formed on the
        device with no host copy (rism3d_get_grid_device)."""
        import torch
        nsite = self.natv if which in (GRID_G, GRID_H, GRID_C, GRID_T, GRID_U) else 1
        out = torch.empty((nsite, self.n), dtype=torch.float64, device="cuda:%d" % self.device)
        self._check(lib().rism3d_get_grid_device(self.h, which, C.c_void_p(out.data_ptr())))
        return out

    def euv(self):
        out = np.zeros((2, self.natv, self.natom))
        self._check(lib().rism3d_euv(self.h, _dp(out)))
        return out

    def forces(self):
        a = np.zeros((self.natom, 3)); b = np.zeros((self.natom, 3))
        self._check(lib().rism3d_forces(self.h, _dp(a), _dp(b)))
        return a, b

    def grad(self, precision=FP64):
        """d(SFE_SC)/d(q, sigma, eps, xyz) of every atom (J/mol per unit):
        rism3d_grad (FP64), or with precision=MIXED the FP32 variant
        (rism3d_grad_precision)."""
        dq = np.zeros(self.natom); ds = np.zeros(self.natom); de = np.zeros(self.natom)
        dR = np.zeros((self.natom, 3))
        if precision == FP64:
            self._check(lib().rism3d_grad(self.h, _dp(dq), _dp(ds), _dp(de), _dp(dR)))
        else:
            self._check(lib().rism3d_grad_precision(self.h, precision, _dp(dq), _dp(ds),
                                                    _dp(de), _dp(dR)))
        return dq, ds, de, dR

    def solve_batch(self, mols):
        """mols: list of (sig, eps, q, xyz, grid, box), cubic cells; returns a
        list of result dicts (rism3d_solve_batch)."""
        natoms = np.array([len(m[2]) for m in mols], dtype=np.int32)
        grids = np.array([int(m[4]) for m in mols], dtype=np.int32)
        boxes = _f64([float(m[5]) for m in mols])
        sig = _f64(np.concatenate([np.asarray(m[0], float) for m in mols]))
        eps = _f64(np.concatenate([np.asarray(m[1], float) for m in mols]))
        q = _f64(np.concatenate([np.asarray(m[2], float) for m in mols]))
        xyz = _f64(np.concatenate([np.asarray(m[3], float).reshape(-1, 3) for m in mols]))
        res = (Result * len(mols))()
        ip = C.POINTER(C.c_int)
        self._check(lib().rism3d_solve_batch(
            self.h, len(mols), natoms.ctypes.data_as(ip), grids.ctypes.data_as(ip),
            _dp(boxes), _dp(sig), _dp(eps), _dp(q), _dp(xyz), res),
            (OK, DIVERGED, NOT_CONVERGED))
        return [r.as_dict() for r in res]

    def refresh_potentials(self):
        self._check(lib().rism3d_refresh_potentials(self.h))

    def kernel_launches(self):
        return int(lib().rism3d_kernel_launches(self.h))

    def time_kernel(self, which, reps):
        ms = np.zeros(1)
        self._check(lib().rism3d_time_kernel(self.h, which, reps, _dp(ms)))
        return float(ms[0])

    def close(self):
        if getattr(self, "h", None):
            lib().rism3d_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
