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


@pytest.mark.parametrize("n,b", [(9600, 64), (20000, 128)])
def test_pull_sweep_agrees_with_streaming_sweep(cuda, bbk, n, b):
    # Up to 32 right-hand sides go through the pull sweep (8 per launch: each
    # CTA gathers the solved blocks' contributions for its next block); more
    # go through the streaming sweep (each solved block pushed into every
    # later block).  The two sum in different orders, so they agree to
    # rounding: columns solved among 160 against the same columns solved
    # among 4 (one launch) and 12 (two launches), each with a backward error
    # at the FP64 level.  n=9600 and 20000 give 2 and 3 blocks per CTA.
    import torch
    g = torch.Generator(device=cuda).manual_seed(n)
    a = torch.rand(n, n, device=cuda, dtype=torch.float64, generator=g) * 2 - 1
    a = a + a.T
    f = a.clone()
    perm, pt, _ = bbk.factor_device(f, b, mode="fp64")
    rhs = torch.randn(160, n, device=cuda, dtype=torch.float64, generator=g)
    many = bbk.solve_device(f, perm, pt, rhs.clone())

    def berr(x, r):
        res = a @ x.T - r.T
        return float(res.abs().max() / (a.abs().sum(1).max() * x.abs().max() + r.abs().max()))

    assert berr(many[:12], rhs[:12]) < 1e-14
    for k in (4, 12):
        few = bbk.solve_device(f, perm, pt, rhs[:k].clone())
        assert berr(few, rhs[:k]) < 1e-14, k
        diff = float((many[:k] - few).abs().max() / many[:k].abs().max())
        assert diff < 1e-9, (k, diff)


def test_factor_solve_one_call_kkt(cuda, bbk):
    a = kkt_matrix(1200, 960, seed=5)
    rhs = np.random.default_rng(1).standard_normal(1200)
    fac, x = bbk.factor_solve_host(a, 128, rhs)
    assert backward_error(a, x[:, None], rhs[:, None]) < 1e-14


@pytest.mark.parametrize("kind", ["kkt", "uniform"])
def test_factor_solve_one_call_returns_the_factors(cuda, bbk, kind):
    # the one-call entry point copies the factors back on a second stream
    # while it solves: they must be exactly the factorization's, with the
    # strict lower triangle of the caller's matrix untouched
    n, b = 1500, 64
    a = kkt_matrix(n, 1200, seed=7) if kind == "kkt" else uniform_symmetric(n, 8)
    a = a + np.tril(np.full((n, n), 3.25), -1)  # lower part the factorization must not touch
    rhs = np.random.default_rng(2).standard_normal((n, 3))
    fac, x = bbk.factor_solve_host(a, b, rhs)
    ref = bbk.factor_host(a, b)
    assert np.array_equal(np.triu(fac.factors), np.triu(ref.factors))
    assert np.array_equal(np.tril(fac.factors, -1), np.tril(a, -1))
    assert np.array_equal(fac.perm, ref.perm) and np.array_equal(fac.pivot_types, ref.pivot_types)
    assert np.array_equal(fac.panel_end, ref.panel_end)
    sym = np.triu(a) + np.triu(a, 1).T
    assert backward_error(sym, x, rhs) < 1e-13


def test_zero_pivot_gives_zero_component(cuda, bbk, port):
    a = np.diag([2.0, -3.0, 0.0, 5.0])
    rhs = np.array([2.0, 3.0, 1.0, 10.0])
    fac = bbk.factor_host(a, 2)
    x = bbk.solve_host(fac, rhs)
    assert np.allclose(x, port.solve(port.factor(a, 2), rhs))
    assert x[2] == 0.0


def test_solve_reports_an_expired_wait_and_the_context_survives(cuda, bbk):
    # With a 1 ns bound every sweep block that has to wait for an earlier one
    # gives up (n = 4096: 64 blocks, most of them wait): the synchronous solve
    # must return BBK_ERR_TIMEOUT instead of partly solved right-hand sides
    # with BBK_OK, and the next solve with the normal bound must succeed.
    import torch
    n, blk = 4096, 64
    a = uniform_symmetric(n, 4096)
    f = torch.from_numpy(a).to(cuda)
    perm, pt, _ = bbk.factor_device(f, blk)
    rhs = np.random.default_rng(7).standard_normal((2, n))
    try:
        bbk.set_wait_timeout_ns(1)
        with pytest.raises(bbk.BbkError) as err:
            bbk.solve_device(f, perm, pt, torch.from_numpy(rhs).to(cuda))
        assert err.value.status == bbk.BBK_ERR_TIMEOUT
    finally:
        bbk.set_wait_timeout_ns(5_000_000_000)
    x = bbk.solve_device(f, perm, pt, torch.from_numpy(rhs).to(cuda)).cpu().numpy()
    assert backward_error(a, x.T, rhs.T) < 1e-14
