"""GPU: the compact-factor solve (no reference counterpart; checked against
the oracle's restatement of the reference's compact-storage reading rules and
by backward error)."""
import numpy as np
import pytest

from common import kkt_matrix, uniform_symmetric

pytestmark = pytest.mark.gpu


def backward_error(a, x, b):
    r = b - a @ x
    return np.max(np.abs(r), axis=0).max() / (np.abs(a).sum(1).max() * np.abs(x).max() + np.abs(b).max())


@pytest.mark.parametrize("n,b,nrhs", [(7, 2, 1), (64, 8, 3), (300, 32, 16), (1000, 64, 1)])
def test_solve_matches_oracle(cuda, bbk, port, n, b, nrhs):
    a = uniform_symmetric(n, n)
    rhs = np.random.default_rng(n).standard_normal((n, nrhs))
    fac = bbk.factor_host(a, b, mode="fp64_ordered")
    want = port.solve(port.factor(a, b), rhs)
    got = bbk.solve_host(fac, rhs)
    assert np.max(np.abs(got - want)) <= 1e-9 * max(1.0, np.max(np.abs(want)))
    assert backward_error(a, got, rhs) < 1e-14


def test_factor_solve_one_call_kkt(cuda, bbk):
    a = kkt_matrix(1200, 960, seed=5)
    rhs = np.random.default_rng(1).standard_normal(1200)
    fac, x = bbk.factor_solve_host(a, 128, rhs)
    assert backward_error(a, x[:, None], rhs[:, None]) < 1e-14


def test_zero_pivot_gives_zero_component(cuda, bbk, port):
    a = np.diag([2.0, -3.0, 0.0, 5.0])
    rhs = np.array([2.0, 3.0, 1.0, 10.0])
    fac = bbk.factor_host(a, 2)
    x = bbk.solve_host(fac, rhs)
    assert np.allclose(x, port.solve(port.factor(a, 2), rhs))
    assert x[2] == 0.0
