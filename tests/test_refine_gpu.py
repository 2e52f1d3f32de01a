"""GPU: mixed-precision trailing updates and FP64 iterative refinement (no
reference counterpart: the reference is FP64 only and has no solve).  The
target: backward error <= 1e-12 from factors whose trailing updates ran in
FP32 or BF16, with the residual always in FP64."""
import numpy as np
import pytest

from common import backward_error, relative_error, reconstruct, spectral_matrix, uniform_symmetric

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _factor(bbk, cuda, a, b, mode):
    import torch
    f = torch.from_numpy(a).to(cuda)
    perm, pt, _ = bbk.factor_device(f, b, mode=mode)
    return f, perm, pt


@pytest.mark.parametrize("mode,bound", [("fp32", 1e-5), ("bf16x3", 1e-5), ("bf16", 0.25)])
def test_low_precision_update_factorization(cuda, bbk, mode, bound):
    # the factors of a perturbed matrix: residual on the order of the update's unit roundoff
    a = uniform_symmetric(600, 5)
    f, perm, pt = _factor(bbk, cuda, a, 64, mode)
    res = relative_error(reconstruct(f.cpu().numpy(), perm.cpu().numpy(), pt.cpu().numpy()), a)
    assert res < bound, res
    exact = bbk.factor_host(a, 64, mode="fp64")
    assert relative_error(reconstruct(exact.factors, exact.perm, exact.pivot_types), a) < 1e-13


def test_residual_kernel_and_fp64_refinement(cuda, bbk):
    import torch
    n = 700
    a = uniform_symmetric(n, 9)
    rhs = np.random.default_rng(1).standard_normal((3, n))
    f, perm, pt = _factor(bbk, cuda, a, 64, "fp64")
    x, info = bbk.solve_refined_device(torch.from_numpy(a).to(cuda), f, perm, pt,
                                       torch.from_numpy(rhs).to(cuda), tol=TOL, method="classical")
    assert info.converged == 1 and info.iterations <= 1
    assert backward_error(a, x.cpu().numpy().T, rhs.T) <= TOL


@pytest.mark.parametrize("mode,lo,hi", [("fp32", 1e-4, 1e4), ("bf16x3", 1e-4, 1e4), ("bf16", 1e-1, 1e1)])
def test_gmres_ir_ill_conditioned(cuda, bbk, mode, lo, hi):
    """GMRES-IR reaches 1e-12 from low-precision-update factors: FP32 and
    three-term BF16 updates at kappa ~ 1e8 (the mixed-precision workload's
    spectrum at small n); single-term BF16 updates only at kappa ~ 1e2 (its
    factor error times kappa must stay small)."""
    import torch
    n = 1200
    a = spectral_matrix(n, 3, lo=lo, hi=hi)
    rhs = np.random.default_rng(2).standard_normal((4, n))
    f, perm, pt = _factor(bbk, cuda, a, 64, mode)
    x, info = bbk.solve_refined_device(torch.from_numpy(a).to(cuda), f, perm, pt,
                                       torch.from_numpy(rhs).to(cuda), tol=TOL, max_iter=20,
                                       method="gmres", restart=30)
    be = backward_error(a, x.cpu().numpy().T, rhs.T)
    assert info.converged == 1, (info.backward_error, info.iterations, info.inner_iterations)
    assert be <= 2 * TOL, be
    # forward error against the FP64 factorization's solution: a backward error
    # of TOL allows up to about kappa * TOL
    f64 = bbk.factor_host(a, 64, mode="fp64")
    x64 = bbk.solve_host(f64, rhs.T)
    fe = np.abs(x.cpu().numpy().T - x64).max() / np.abs(x64).max()
    assert fe < 10 * (hi / lo) * TOL, fe


def test_classical_ir_fp32_well_conditioned(cuda, bbk):
    import torch
    n = 800
    a = spectral_matrix(n, 4, lo=1e-1, hi=1e1)  # kappa ~ 100
    rhs = np.random.default_rng(7).standard_normal((2, n))
    f, perm, pt = _factor(bbk, cuda, a, 64, "fp32")
    x, info = bbk.solve_refined_device(torch.from_numpy(a).to(cuda), f, perm, pt,
                                       torch.from_numpy(rhs).to(cuda), tol=TOL, max_iter=20,
                                       method="classical")
    assert info.converged == 1 and info.initial_backward_error > TOL
    assert backward_error(a, x.cpu().numpy().T, rhs.T) <= 2 * TOL
