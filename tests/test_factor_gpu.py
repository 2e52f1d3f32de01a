"""GPU parity of the factorization against the oracle.

Bar: the plain FP64 path reproduces the reference's pivot
sequence (pivot types and permutation) exactly unless a decision was a near
tie, and its relative reconstruction residual is within 10x of the
reference's and at most n * eps64 (on the reference's relative-error metric,
with the reference's own tolerance 1e-10 for its unit cases).  The
reference-ordered update mode must be bitwise identical to the reference.
"""
import numpy as np
import pytest

from common import (FIXED, GOLDEN_4x4, GOLDEN_4x4_COMPACT, GOLDEN_4x4_PIVOTS, TOLERANCE, kkt_matrix,
                    load_large_cases, load_small_cases, reconstruct, relative_error, uniform_symmetric,
                    upper_hash)

pytestmark = pytest.mark.gpu
EPS = np.finfo(np.float64).eps


@pytest.mark.parametrize("mode", ["fp64", "fp64_ordered", "fp32"])
def test_golden_compact_storage(cuda, bbk, mode):
    d = bbk.BlockLdltDecomposition(GOLDEN_4x4, 2, mode=mode)
    d.factorize()
    assert relative_error(d.compact_factors(), GOLDEN_4x4_COMPACT) < TOLERANCE
    assert d.pivot_types().tolist() == GOLDEN_4x4_PIVOTS
    assert relative_error(d.reconstruct_original(), GOLDEN_4x4) < TOLERANCE


@pytest.mark.parametrize("ci", range(3))
@pytest.mark.parametrize("b", range(1, 5))
def test_fixed_factorizations(cuda, bbk, ci, b):
    d = bbk.BlockLdltDecomposition(FIXED[ci], b)
    d.factorize()
    assert relative_error(d.reconstruct_original(), FIXED[ci]) < TOLERANCE


def test_triangular_input(cuda, bbk):
    # tests/block_ldlt_decomposition_test.cc:387-419: only one triangle is read
    for b in range(1, 5):
        up = np.triu(GOLDEN_4x4) + np.tril(np.full((4, 4), 12345.0), -1)
        lo = np.tril(GOLDEN_4x4) + np.triu(np.full((4, 4), 12345.0), 1)
        for m, lower in ((up, False), (lo, True)):
            d = bbk.BlockLdltDecomposition(m, b, lower=lower)
            d.factorize()
            assert relative_error(d.reconstruct_original(), GOLDEN_4x4) < TOLERANCE


def test_small_fixtures_bitwise_ordered(cuda, bbk):
    for c in load_small_cases():
        r = bbk.factor_host(c["a"], c["b"], mode="fp64_ordered")
        assert np.array_equal(np.triu(r.factors), c["f"], equal_nan=True), c["name"]
        assert np.array_equal(r.perm, c["perm"]), c["name"]
        assert np.array_equal(r.pivot_types, c["pt"]), c["name"]
        assert np.array_equal(r.panel_end, c["ends"]), c["name"]


def test_small_fixtures_tensor_core(cuda, bbk):
    for c in load_small_cases():
        r = bbk.factor_host(c["a"], c["b"], mode="fp64")
        a = c["a"]
        assert np.array_equal(r.pivot_types, c["pt"]), c["name"]
        assert np.array_equal(r.perm, c["perm"]), c["name"]
        res = relative_error(reconstruct(r.factors, r.perm, r.pivot_types), a)
        assert res < TOLERANCE, (c["name"], res)


def test_random_factorizations_bitwise_ordered(cuda, bbk, port):
    # the reference's TestRandomFactorizations grid (sizes 3..16, every block size)
    for n in range(3, 17):
        for b in range(1, n + 1):
            a = port.random_symmetric(n, 10000 * n + 100 * b)
            want = port.factor(a, b)
            got = bbk.factor_host(a, b, mode="fp64_ordered")
            assert np.array_equal(np.triu(got.factors), np.triu(want.factors)), (n, b)
            assert np.array_equal(got.perm, want.perm) and np.array_equal(got.pivot_types, want.pivot_types)


def test_non_finite_entries_bitwise_ordered(cuda, bbk, port):
    # NaN / inf entries: the argmax never picks a NaN (strict '>' in the
    # reference's scans), so factors (NaN where NaN), pivots and permutation
    # follow the reference exactly.
    for k, (i, j, v) in enumerate(((3, 7, np.nan), (0, 5, np.inf), (4, 4, np.nan), (1, 9, -np.inf))):
        a = port.random_symmetric(12, 777 + k)
        a[i, j] = a[j, i] = v
        for b in (1, 3, 5, 12):
            want = port.factor(a, b)
            got = bbk.factor_host(a, b, mode="fp64_ordered")
            assert np.array_equal(np.triu(got.factors), np.triu(want.factors), equal_nan=True), (i, j, v, b)
            assert np.array_equal(got.perm, want.perm), (i, j, v, b)
            assert np.array_equal(got.pivot_types, want.pivot_types), (i, j, v, b)


@pytest.mark.parametrize("n,h,b", [(800, 600, 32), (1200, 960, 64), (3000, 2400, 128)])
def test_kkt_bitwise_ordered(cuda, bbk, port, n, h, b):
    # Saddle-point matrices: most candidate steps keep their pivot, so most
    # rows are computed ahead in the candidate phase; the ordered mode must
    # still be the reference bit for bit, and the reassociated mode must
    # take the same pivots.
    a = kkt_matrix(n, h, 5 + n)
    want = port.factor(a, b)
    got = bbk.factor_host(a, b, mode="fp64_ordered")
    assert np.array_equal(np.triu(got.factors), np.triu(want.factors))
    assert np.array_equal(got.perm, want.perm) and np.array_equal(got.pivot_types, want.pivot_types)
    assert np.array_equal(got.panel_end, want.panel_end)
    fast = bbk.factor_host(a, b, mode="fp64")
    assert np.array_equal(fast.pivot_types, want.pivot_types) and np.array_equal(fast.perm, want.perm)
    res = relative_error(reconstruct(fast.factors, fast.perm, fast.pivot_types), a)
    assert res < TOLERANCE, res


@pytest.mark.parametrize("n,b,seed", [(900, 24, 77), (1100, 40, 78)])
def test_boundary_shifts_bitwise_ordered(cuda, bbk, port, n, b, seed):
    # uniform matrices with many 2x2 pivots: boundary shifts after rows
    # computed ahead, candidates at p+2 / p+3, no-candidate steps after them
    a = uniform_symmetric(n, seed)
    want = port.factor(a, b)
    got = bbk.factor_host(a, b, mode="fp64_ordered")
    assert np.array_equal(np.triu(got.factors), np.triu(want.factors))
    assert np.array_equal(got.perm, want.perm) and np.array_equal(got.pivot_types, want.pivot_types)
    assert np.array_equal(got.panel_end, want.panel_end)
    assert any(e != min(n, (k + 1) * b) for k, e in enumerate(want.panel_end))  # shifts happen


@pytest.mark.parametrize("rows", [0, 7, 40])
def test_split_panel_rows_bitwise_ordered(cuda, bbk, port, monkeypatch, rows):
    # A slice too wide for shared memory keeps its first rows there and the
    # rest in global memory; BBK_PANEL_SMEM_ROWS forces that split at a small
    # size.  The ordered mode continues each sum across the split, so it must
    # stay the reference bit for bit; the reassociated mode must take the
    # same pivots.
    monkeypatch.setenv("BBK_PANEL_SMEM_ROWS", str(rows))
    for a, b in ((kkt_matrix(1200, 960, 1205), 64), (uniform_symmetric(1100, 78), 40)):
        want = port.factor(a, b)
        got = bbk.factor_host(a, b, mode="fp64_ordered")
        assert np.array_equal(np.triu(got.factors), np.triu(want.factors)), (rows, b)
        assert np.array_equal(got.perm, want.perm) and np.array_equal(got.pivot_types, want.pivot_types)
        assert np.array_equal(got.panel_end, want.panel_end)
        fast = bbk.factor_host(a, b, mode="fp64")
        assert np.array_equal(fast.pivot_types, want.pivot_types) and np.array_equal(fast.perm, want.perm)
        res = relative_error(reconstruct(fast.factors, fast.perm, fast.pivot_types), a)
        assert res < TOLERANCE, res


def test_scale_sweep(cuda, bbk, port):
    # tests/block_ldlt_decomposition_test.cc:40-99: value scales 1e-12 .. 1e12
    scales = [1e-12, 1e-9, 1e-6, 1e-3, 1.0, 1e3, 1e6, 1e9, 1e12]
    for n, b in ((50, 8), (100, 21), (200, 64)):
        for si, sc in enumerate(scales):
            a = port.random_symmetric(n, 910000 + 10000 * n + 100 * b + 10 * si, sc)
            want = port.factor(a, b)
            got = bbk.factor_host(a, b, mode="fp64")
            assert relative_error(reconstruct(got.factors, got.perm, got.pivot_types), a) < TOLERANCE
            assert np.array_equal(got.pivot_types, want.pivot_types), (n, b, sc)
            exact = bbk.factor_host(a, b, mode="fp64_ordered")
            assert np.array_equal(np.triu(exact.factors), np.triu(want.factors)), (n, b, sc)


@pytest.mark.parametrize("n", [500, 2000])
def test_uniform_fixture_bitwise_ordered(cuda, bbk, n):
    c = [c for c in load_large_cases() if c["n"] == n][0]
    a = uniform_symmetric(c["n"], c["seed"])
    r = bbk.factor_host(a, c["block_size"], mode="fp64_ordered")
    assert r.perm.tolist() == c["perm"]
    assert r.pivot_types.tolist() == c["pivot_types"]
    assert r.panel_end.tolist() == c["panel_end"]
    assert upper_hash(r.factors) == c["upper_sha256"]


def test_config1_tensor_core_parity(cuda, bbk):
    """n=2000, b=64, uniform[-1,1]: pivot sequence and residual vs the reference."""
    c = [c for c in load_large_cases() if c["n"] == 2000][0]
    a = uniform_symmetric(c["n"], c["seed"])
    r = bbk.factor_host(a, 64, mode="fp64")
    same_pt = r.pivot_types.tolist() == c["pivot_types"]
    same_perm = r.perm.tolist() == c["perm"]
    assert same_pt and same_perm, "pivot sequence diverged from the reference"
    res = relative_error(reconstruct(r.factors, r.perm, r.pivot_types), a)
    exact = bbk.factor_host(a, 64, mode="fp64_ordered")  # bitwise the reference's factors
    res_ref = relative_error(reconstruct(exact.factors, exact.perm, exact.pivot_types), a)
    assert res <= max(10 * res_ref, 1e-15) and res <= 2000 * EPS, (res, res_ref)


def test_device_api_matches_host_api(cuda, bbk):
    import torch
    a = uniform_symmetric(1500, 7)
    host = bbk.factor_host(a, 128)
    t = torch.from_numpy(a).to(cuda)
    perm, pt, pe = bbk.factor_device(t, 128)
    assert np.array_equal(perm.cpu().numpy(), host.perm)
    assert np.array_equal(pt.cpu().numpy(), host.pivot_types)
    assert np.array_equal(np.triu(t.cpu().numpy()), np.triu(host.factors))
    # async + caller workspace
    t2 = torch.from_numpy(a).to(cuda)
    ws = torch.empty(bbk.factor_workspace_size(1500, 128), dtype=torch.uint8, device=cuda)
    perm2, pt2, pe2, status = bbk.factor_device(t2, 128, workspace=ws, sync=False)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    assert torch.equal(t, t2) and torch.equal(perm, perm2)


def test_deterministic(cuda, bbk):
    a = uniform_symmetric(800, 11)
    r1 = bbk.factor_host(a, 64)
    r2 = bbk.factor_host(a, 64)
    assert np.array_equal(r1.factors, r2.factors) and np.array_equal(r1.perm, r2.perm)


def test_bounded_wait_times_out_and_context_survives(cuda, bbk):
    st = bbk.probe_bounded_wait(4, 50_000_000)  # 50 ms bound
    assert st == bbk.BBK_ERR_TIMEOUT
    d = bbk.BlockLdltDecomposition(GOLDEN_4x4, 2)
    d.factorize()
    assert d.pivot_types().tolist() == GOLDEN_4x4_PIVOTS


@pytest.mark.parametrize("n,b,seed", [(60, 4, 2), (333, 64, 4), (1200, 128, 5)])
def test_workspace_rows_and_log_bitwise_ordered(cuda, bbk, port, n, b, seed):
    # bbk_factor_device_ex in the ordered mode: the workspace rows (each
    # panel's W rows at its trailing columns) bitwise the oracle's, which
    # tests/test_oracle.py pins to the reference's Workspace(), and the
    # decision log equal to the oracle's (the same values were compared)
    import torch
    a = uniform_symmetric(n, seed)
    f = torch.from_numpy(a).to(cuda)
    w = torch.zeros(n, n, dtype=torch.float64, device=cuda)
    perm, pt, pe, log = bbk.factor_device_logged(f, b, mode="fp64_ordered", workspace_rows=w)
    want_f, want_log, want_w = port.factor_logged(a, b, workspace_rows=True)
    assert np.array_equal(w.cpu().numpy(), want_w)
    got_log = log.cpu().numpy()
    started = ~np.isnan(got_log[:, 0])
    assert np.array_equal(started, ~np.isnan(want_log[:, 0]))
    assert np.array_equal(got_log[started][:, :2], want_log[started][:, :2])
    assert np.array_equal(np.nan_to_num(got_log[started][:, 2:4], nan=-1.0),
                          np.nan_to_num(want_log[started][:, 3:5], nan=-1.0))
