"""Adjoint gradients of SFE_SC (rism3d_grad) against central finite
differences of the solve itself and against cal_grad-style forces, plus a
torch.autograd.Function wrapper that routes backward() through the adjoint.

The finite differences re-solve at tight convergence (1e-10) so that the
difference quotient (signal ~1e-2 J/mol at the steps used) is not buried in
the convergence noise of mu_ex."""
import numpy as np
import pytest

from helpers import load_case, product_solver

pytestmark = pytest.mark.gpu


def _solver(case):
    s = product_solver(case)
    return s


def _mu(s, case, q=None, sig=None, eps=None, xyz=None):
    s.set_solute(case.sig if sig is None else sig, case.eps if eps is None else eps,
                 case.q if q is None else q, case.xyz if xyz is None else xyz)
    return s.solve()["sfe_sc"]


@pytest.fixture(scope="module")
def tight():
    case, _, _ = load_case("cfg0_chain12", conv=1e-10)
    s = _solver(case)
    s.solve()
    grads = s.grad()
    yield case, s, grads
    s.close()


def _check(fd, ad, rel=1e-4, floor=1e-6):
    fd, ad = np.asarray(fd), np.asarray(ad)
    scale = max(np.abs(fd).max(), floor)
    assert np.abs(fd - ad).max() <= rel * scale, (fd, ad)


def test_charge_gradient_matches_central_differences(tight):
    case, s, (dq, _, _, _) = tight
    h = 1e-4
    fd = []
    for u in range(len(case.q)):
        qp, qm = case.q.copy(), case.q.copy()
        qp[u] += h; qm[u] -= h
        fd.append((_mu(s, case, q=qp) - _mu(s, case, q=qm)) / (2 * h))
    _check(fd, dq)


def test_position_gradient_matches_central_differences(tight):
    case, s, (_, _, _, dR) = tight
    h = 1e-3
    for k in range(3):
        fd = []
        for u in range(len(case.q)):
            xp, xm = case.xyz.copy(), case.xyz.copy()
            xp[u, k] += h; xm[u, k] -= h
            fd.append((_mu(s, case, xyz=xp) - _mu(s, case, xyz=xm)) / (2 * h))
        _check(fd, dR[:, k])


def test_lj_parameter_gradients_match_central_differences(tight):
    case, s, (_, dsig, deps, _) = tight
    fds, fde = [], []
    for u in range(len(case.q)):
        h = 1e-4
        sp, sm = case.sig.copy(), case.sig.copy()
        sp[u] += h; sm[u] -= h
        fds.append((_mu(s, case, sig=sp) - _mu(s, case, sig=sm)) / (2 * h))
        he = 1e-4 * case.eps[u]
        ep, em = case.eps.copy(), case.eps.copy()
        ep[u] += he; em[u] -= he
        fde.append((_mu(s, case, eps=ep) - _mu(s, case, eps=em)) / (2 * he))
    _check(fds, dsig)
    _check(fde, deps)


def test_position_gradient_agrees_with_cal_grad_forces(tight):
    """cal_grad (cal_grad.cu:51-145) integrates rho g grad_R u outside
    r < sigma/2.  That is the derivative of mu_ex only when the analytic
    long-range transform fk equals the discrete transform of fr; the exact
    gradient adds the mismatch term (about 0.5% here, and the finite-difference
    tests above show it belongs to the derivative), so the two agree to 1%."""
    case, s, (_, _, _, dR) = tight
    s.set_solute(case.sig, case.eps, case.q, case.xyz)
    s.solve()
    dulj, due = s.forces()
    tot = dulj + due
    assert np.abs(tot - dR).max() <= 1e-2 * np.abs(dR).max()


def test_autograd_function_routes_backward_through_the_adjoint(tight):
    import torch
    case, s, (dq, dsig, deps, dR) = tight

    class SolvationFreeEnergy(torch.autograd.Function):
        @staticmethod
        def forward(ctx, q, sig, eps, xyz):
            s.set_solute(sig.numpy(), eps.numpy(), q.numpy(), xyz.numpy())
            mu = s.solve()["sfe_sc"]
            g = s.grad()
            ctx.save_for_backward(*[torch.from_numpy(np.ascontiguousarray(a)) for a in g])
            return torch.tensor(mu, dtype=torch.float64)

        @staticmethod
        def backward(ctx, gout):
            gq, gs, ge, gR = ctx.saved_tensors
            return gout * gq, gout * gs, gout * ge, gout * gR

    args = [torch.tensor(a, dtype=torch.float64, requires_grad=True)
            for a in (case.q, case.sig, case.eps, case.xyz)]
    mu = SolvationFreeEnergy.apply(*args)
    (2.0 * mu).backward()
    assert np.allclose(args[0].grad.numpy(), 2 * dq)
    assert np.allclose(args[3].grad.numpy(), 2 * dR)


def _fd_check(fd, ad, rel, scale):
    """|fd - ad| <= rel * max(|fd|, scale) per entry (scale keeps a
    component that happens to be near zero from demanding more than the
    difference quotient can resolve)."""
    fd, ad = np.asarray(fd), np.asarray(ad)
    bound = rel * np.maximum(np.abs(fd), scale)
    bad = np.abs(fd - ad) > bound
    assert not bad.any(), (np.flatnonzero(bad), fd[bad], ad[bad])


def test_config4_gradients_on_32_atoms_match_central_differences():
    """Config 4: the 846-atom solute at 256^3 (KH).  The adjoint gradients of
    all atoms in FP64 and in the FP32 variant (FP32 transposed solve and LJ
    pair factors, FP64 sums) agree with each other; on 32 seeded atoms they
    agree with central finite differences of the solve: charges (step 1e-4 e)
    to 1e-4 relative, all three position components to 2e-4.  The KH
    closure switches from e^x to 1 + x at x = 0, so mu is only once
    differentiable in the positions and a central difference carries an
    error linear in the step (measured ~5x larger at 5e-3 A than at 1e-3 A);
    the extrapolation 2 D(h) - D(2h) removes its mean, and the steps are
    h = 2.5e-4 A and 5e-4 A (with 1e-3 A and 2e-3 A, 2 of the 96 components
    were 2.4e-4 and 4.8e-4 off).  LJ sigma (step 1e-4 A) and epsilon (step
    5e-4 of each epsilon) are checked on 4 of the atoms.  The epsilon step
    is not 1e-4: mu is resolved to ~1e-6 J/mol, and for the atom with the
    smallest epsilon gradient (-0.0118) a 1e-4 step moves mu by only a few
    times that, so its difference quotient was 1 % off, against 1e-5 at
    5e-4 (2e-4: 1.3e-3; 1e-3: 3e-4, the step's truncation).  The differences re-solve in FP64 to a 1e-11
    residual, each started from the unperturbed solution (a mixed-precision
    context evaluates the LJ grid in FP32, whose rounding moves mu by more
    than the 1e-3 A position steps resolve).
    Every atom's position gradient is also checked against cal_grad forces
    (1 %: the long-range mismatch term)."""
    import rism3d_b200 as R
    case, _, _ = load_case("cfg2_protein846_kh", conv=1e-11)
    s = _solver(case)
    s.solve()
    dq, dsig, deps, dR = s.grad()
    dq32, dsig32, deps32, dR32 = s.grad(precision=R.MIXED)
    for a64, a32 in ((dq, dq32), (dsig, dsig32), (deps, deps32), (dR, dR32)):
        assert np.abs(a32 - a64).max() <= 1e-4 * np.abs(a64).max(), np.abs(a32 - a64).max()
    dulj, due = s.forces()
    assert np.abs(dulj + due - dR).max() <= 1e-2 * np.abs(dR).max()
    t0 = s.grid_array(R.GRID_T)
    s.close()
    fdsolver = product_solver(case)
    fdsolver.set_tuv(t0)
    rng = np.random.default_rng(4)
    atoms = rng.choice(len(case.q), 32, replace=False)

    def mu(**kw):
        return _mu(fdsolver, case, **kw)

    def dpos(u, k, h):
        xp, xm = case.xyz.copy(), case.xyz.copy()
        xp[u, k] += h; xm[u, k] -= h
        return (mu(xyz=xp) - mu(xyz=xm)) / (2 * h)

    fdq, fdR = [], []
    for u in atoms:
        qp, qm = case.q.copy(), case.q.copy()
        qp[u] += 1e-4; qm[u] -= 1e-4
        fdq.append((mu(q=qp) - mu(q=qm)) / 2e-4)
        fdR.append([2.0 * dpos(u, k, 2.5e-4) - dpos(u, k, 5e-4) for k in range(3)])
    _fd_check(fdq, dq[atoms], 1e-4, 1e-2 * np.abs(dq).max())
    _fd_check(np.array(fdR), dR[atoms], 2e-4, 1e-2 * np.abs(dR).max())
    fds, fde = [], []
    for u in atoms[:4]:
        sp, sm = case.sig.copy(), case.sig.copy()
        sp[u] += 1e-4; sm[u] -= 1e-4
        fds.append((mu(sig=sp) - mu(sig=sm)) / 2e-4)
        he = 5e-4 * case.eps[u]
        ep, em = case.eps.copy(), case.eps.copy()
        ep[u] += he; em[u] -= he
        fde.append((mu(eps=ep) - mu(eps=em)) / (2 * he))
    _fd_check(fds, dsig[atoms[:4]], 1e-4, 1e-2 * np.abs(dsig).max())
    _fd_check(fde, deps[atoms[:4]], 1e-4, 1e-2 * np.abs(deps).max())
    fdsolver.close()


def test_fp32_adjoint_variant_matches_fp64_on_the_small_chain(tight):
    """The FP32 variant of the adjoint (rism3d_grad_precision, MIXED) on the
    12-atom chain agrees with the FP64 adjoint (and so with the finite
    differences above) to 1e-5 of each gradient's largest entry."""
    import rism3d_b200 as R
    case, s, g64 = tight
    s.set_solute(case.sig, case.eps, case.q, case.xyz)
    s.solve()
    g32 = s.grad(precision=R.MIXED)
    for a64, a32 in zip(g64, g32):
        assert np.abs(a32 - a64).max() <= 1e-5 * np.abs(a64).max()
