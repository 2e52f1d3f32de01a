"""GPU: the benchmark configurations at their full sizes, checked through
properties that hold at any size (the reference itself is far too slow to run
there): the permutation is a permutation, the pivot types form valid 1x1 /
2x2 blocks, the panel ends are increasing, the factors reproduce the matrix
(P^T L D L^T P = A, where the n x n reconstruction fits), and solves with them
have small backward error.

Inputs are generated on the device from fixed seeds with the structure each
configuration names: KKT n=10000 (block 128, 1 RHS), the spectral matrix
n=20000 with condition ~1e8 (16 RHS) and the random indefinite n=40000
(block 256, 4 RHS, ~13 GB in HBM)."""
import pytest

pytestmark = pytest.mark.gpu

TOLERANCE = 1e-10  # reconstruction, the reference tests' relative Frobenius bound


def _kkt(n, h, seed, device):
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    gm = torch.randn(h, h, generator=g, dtype=torch.float64, device=device)
    a = torch.zeros(n, n, dtype=torch.float64, device=device)
    a[:h, :h] = gm @ gm.T / h
    a[:h, :h] += 1e-2 * torch.eye(h, dtype=torch.float64, device=device)
    del gm
    bm = torch.randn(n - h, h, generator=g, dtype=torch.float64, device=device)
    a[h:, :h] = bm
    a[:h, h:] = bm.T
    return a, g


def _spectral(n, seed, device, lo=1e-4, hi=1e4):
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    q, _ = torch.linalg.qr(torch.randn(n, n, generator=g, dtype=torch.float64, device=device))
    mag = torch.exp(torch.empty(n, dtype=torch.float64, device=device).uniform_(
        float(torch.log(torch.tensor(lo))), float(torch.log(torch.tensor(hi))), generator=g))
    sign = torch.ones(n, dtype=torch.float64, device=device)
    sign[torch.randperm(n, generator=g, device=device)[: n // 2]] = -1.0
    a = (q * (sign * mag)) @ q.T
    del q
    return (a + a.T) * 0.5, g


def _random_indefinite(n, seed, device):
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    a = torch.empty(n, n, dtype=torch.float64, device=device).uniform_(-1.0, 1.0, generator=g)
    a = torch.triu(a)
    a = a + torch.triu(a, 1).T
    a.diagonal().add_(torch.randn(n, generator=g, dtype=torch.float64, device=device) * 0.1)
    return a, g


def _check_structure(perm, pt, pe, n):
    import torch
    assert torch.equal(torch.sort(perm.long()).values, torch.arange(n, device=perm.device))
    p = pt.long().cpu()
    assert bool(((p == 1) | (p == 2) | (p == -2)).all())
    two = (p == 2).nonzero().flatten()
    assert bool((two + 1 < n).all()) and bool((p[two + 1] == -2).all())
    minus = (p == -2).nonzero().flatten()
    assert bool((minus > 0).all()) and bool((p[minus - 1] == 2).all())
    e = pe.long().cpu()
    assert bool((e[1:] > e[:-1]).all()) and int(e[-1]) == n


def _backward_error(a, x, b):
    """max over right-hand sides of ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf);
    a is n x n, x and b are (nrhs, n)."""
    r = b - x @ a  # A symmetric: (A x_k)^T = x_k^T A
    an = a.abs().sum(1).max()
    return float((r.abs().amax(1) / (an * x.abs().amax(1) + b.abs().amax(1))).max())


SAMPLED_TOLERANCE = 1e-8  # tests/block_ldlt_large_stress_test.cc:26, kResidualTolerance


def _factor_and_check(bbk, a0, block, nrhs, g, reconstruct, be_tol, mode="fp64", sampled=False):
    import torch
    n = a0.shape[0]
    f = a0.clone()
    perm, pt, pe = bbk.factor_device(f, block, mode=mode)
    torch.cuda.synchronize()
    _check_structure(perm, pt, pe, n)
    if sampled:
        # the reference's own large-matrix check: 4096 sampled entries of
        # P^T L D L^T P from the compact factors, on the device
        from oracle.oracle import Port
        rows, cols = Port().residual_samples(n, 11, 4096)
        res = bbk.sampled_residual_device(a0, f, perm, pt, torch.from_numpy(rows).to(a0.device),
                                          torch.from_numpy(cols).to(a0.device))
        assert res < SAMPLED_TOLERANCE, (mode, res)
    rhs = torch.randn(nrhs, n, generator=g, dtype=torch.float64, device=a0.device)
    x = bbk.solve_device(f, perm, pt, rhs.clone())
    be = _backward_error(a0, x, rhs)
    assert be <= be_tol, (mode, be)
    if reconstruct:
        rec = bbk.reconstruct_device(f, perm, pt)
        err = float(torch.linalg.norm(rec - a0) / max(float(torch.linalg.norm(a0)), 1.0))
        del rec
        assert err < TOLERANCE, (mode, err)
    del f
    return pt.cpu()


def test_kkt_n10000_block128(cuda, bbk):
    import torch
    dev = torch.device("cuda", 0)
    a0, g = _kkt(10000, 8000, 20240, dev)
    pt_fast = _factor_and_check(bbk, a0, 128, 1, g, True, 1e-14)
    pt_exact = _factor_and_check(bbk, a0, 128, 1, g, True, 1e-14, mode="fp64_ordered")
    # the zero (2,2) block forces 2x2 pivots in both update modes
    assert int((pt_fast == 2).sum()) > 0 and int((pt_exact == 2).sum()) > 0
    del a0
    torch.cuda.empty_cache()


def test_spectral_n20000_16rhs(cuda, bbk):
    import torch
    dev = torch.device("cuda", 0)
    a0, g = _spectral(20000, 7, dev)
    _factor_and_check(bbk, a0, 128, 16, g, False, 1e-13, sampled=True)
    del a0
    torch.cuda.empty_cache()


def test_random_indefinite_n40000_block256(cuda, bbk):
    import torch
    dev = torch.device("cuda", 0)
    free, _ = torch.cuda.mem_get_info()
    if free < 40e9:
        pytest.skip(f"needs ~40 GB free device memory, {free / 1e9:.0f} GB free")
    a0, g = _random_indefinite(40000, 11, dev)
    _factor_and_check(bbk, a0, 256, 4, g, False, 1e-12, sampled=True)
    del a0
    torch.cuda.empty_cache()
