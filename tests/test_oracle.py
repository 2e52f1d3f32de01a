"""CPU: the oracle against the reference's golden vectors and the reference.

The oracle is the checker for every GPU parity test, so it is pinned first:
bitwise against the reference's own golden compact factor, against fixtures
produced by the reference library (tests/golden/make_golden.py), and, where
the reference was compiled here, against the reference directly.
"""
import numpy as np
import pytest

from common import (FIXED, GOLDEN_4x4, GOLDEN_4x4_COMPACT, GOLDEN_4x4_PIVOTS, TOLERANCE,
                    load_large_cases, load_small_cases, reconstruct, relative_error, uniform_symmetric,
                    upper_hash)


def test_golden_compact_storage(port):
    # tests/block_ldlt_decomposition_test.cc:421-450
    f = port.factor(GOLDEN_4x4, 2)
    assert relative_error(np.triu(f.factors), GOLDEN_4x4_COMPACT) < TOLERANCE
    assert f.pivot_types.tolist() == GOLDEN_4x4_PIVOTS


def test_kernel_shapes(port):
    # tests/block_ldlt_decomposition_test.cc:367-385
    d0 = port.scale_one_by_one(2.0, [2.0, 4.0, 6.0])
    assert d0[0] == 1.0 and d0[2] == 3.0
    d1, d2 = port.scale_two_by_two(2.0, 1.0, 3.0, [1.0, 2.0], [3.0, 4.0])
    assert abs(d1[0]) < 1e-14 and abs(d2[0] - 1.0) < 1e-14


@pytest.mark.parametrize("ci", range(3))
@pytest.mark.parametrize("b", range(1, 5))
def test_fixed_factorizations(port, ci, b):
    # tests/block_ldlt_decomposition_test.cc:476-508
    a = FIXED[ci]
    f = port.factor(a, b)
    assert relative_error(port.reconstruct(f), a) < TOLERANCE
    assert relative_error(reconstruct(f.factors, f.perm, f.pivot_types), a) < TOLERANCE


def test_small_cases_bitwise_vs_fixtures(port):
    for c in load_small_cases():
        f = port.factor(c["a"], c["b"])
        assert np.array_equal(np.triu(f.factors), c["f"], equal_nan=True), c["name"]
        assert np.array_equal(f.perm, c["perm"]), c["name"]
        assert np.array_equal(f.pivot_types, c["pt"]), c["name"]
        assert np.array_equal(f.panel_end, c["ends"]), c["name"]


def test_large_case_bitwise_vs_fixture(port):
    c = [c for c in load_large_cases() if c["n"] == 500][0]
    f = port.factor(uniform_symmetric(c["n"], c["seed"]), c["block_size"])
    assert f.perm.tolist() == c["perm"]
    assert f.pivot_types.tolist() == c["pivot_types"]
    assert f.panel_end.tolist() == c["panel_end"]
    assert upper_hash(f.factors) == c["upper_sha256"]


def test_random_factorizations_vs_reference(port, reference):
    # tests/block_ldlt_decomposition_test.cc:510-522 (sizes 3..16, every block size)
    for n in range(3, 17):
        for b in range(1, n + 1):
            for s in range(2):
                a = port.random_symmetric(n, 10000 * n + 100 * b + s)
                fp, fr = port.factor(a, b), reference.factor(a, b)
                assert np.array_equal(np.triu(fp.factors), np.triu(fr.factors)), (n, b, s)
                assert np.array_equal(fp.perm, fr.perm) and np.array_equal(fp.pivot_types, fr.pivot_types)


def test_scale_sweep_vs_reference(port, reference):
    # tests/block_ldlt_decomposition_test.cc:40-99, 524-534 (a subset)
    scales = [1e-12, 1e-9, 1e-6, 1e-3, 1.0, 1e3, 1e6, 1e9, 1e12]
    for n in (5, 20, 50):
        for b in (1, 3, 8, 21):
            if b > n:
                continue
            for si, sc in enumerate(scales):
                a = port.random_symmetric(n, 910000 + 10000 * n + 100 * b + 10 * si, sc)
                fp, fr = port.factor(a, b), reference.factor(a, b)
                assert np.array_equal(np.triu(fp.factors), np.triu(fr.factors)), (n, b, sc)
                assert relative_error(port.reconstruct(fp), a) < TOLERANCE


def test_non_finite_entries_vs_reference(port, reference):
    # NaN / inf entries: pins the oracle's argmax (a NaN never wins) and its
    # NaN propagation to the reference itself
    for k, (i, j, v) in enumerate(((3, 7, np.nan), (0, 5, np.inf), (4, 4, np.nan), (1, 9, -np.inf))):
        a = port.random_symmetric(12, 777 + k)
        a[i, j] = a[j, i] = v
        for b in (1, 3, 5, 12):
            fp, fr = port.factor(a, b), reference.factor(a, b)
            assert np.array_equal(np.triu(fp.factors), np.triu(fr.factors), equal_nan=True), (i, j, v, b)
            assert np.array_equal(fp.perm, fr.perm) and np.array_equal(fp.pivot_types, fr.pivot_types)


def test_solve_restatement(port):
    a = uniform_symmetric(60, 3)
    f = port.factor(a, 8)
    rng = np.random.default_rng(0)
    b = rng.standard_normal((60, 3))
    x = port.solve(f, b)
    assert np.linalg.norm(a @ x - b) / np.linalg.norm(b) < 1e-10


def test_decision_log_describes_each_step(port):
    # bko_factor_logged: one record per pivot step at the position where its
    # pivot starts; a step that needed no candidate passed the first test
    # |W(p,p)| >= alpha omega (src/block_ldlt_decomposition.cc:90-92), one
    # that did failed it; the second row of a 2x2 pivot has no record
    from common import ALPHA
    a = uniform_symmetric(300, 31)
    f, log = port.factor_logged(a, 32)
    plain = port.factor(a, 32)
    assert np.array_equal(f.factors, plain.factors) and np.array_equal(f.perm, plain.perm)
    pt = f.pivot_types
    started = ~np.isnan(log[:, 0])
    assert np.array_equal(started, pt != -2)
    d, om, second, sg, arr = (log[started, k] for k in range(5))
    cand = ~np.isnan(sg)
    assert np.all((d >= ALPHA * om) | (om == 0.0) | cand)
    assert np.all(d[cand] < ALPHA * om[cand])
    assert np.all(second <= om)
    assert np.array_equal(cand, ~np.isnan(arr))


def test_oracle_reproduces_the_reference_kkt10000_fixture(port):
    # The C restatement against the reference's own factorization of the
    # full-size saddle-point workload (n=10000, block 128), stored by
    # tests/golden/make_golden.py --kkt: identical factor bits, permutation,
    # pivot types and panel ends (about a minute on one core).
    import os
    from common import GOLDEN, kkt_matrix_exact
    z = np.load(os.path.join(GOLDEN, "ref_kkt10000.npz"))
    a, sha = kkt_matrix_exact(int(z["n"]), int(z["h"]), int(z["seed"]))
    assert sha == str(z["input_sha256"])
    f = port.factor(a, int(z["block_size"]))
    assert upper_hash(f.factors) == str(z["upper_sha256"])
    assert np.array_equal(f.perm, z["perm"])
    assert np.array_equal(f.pivot_types, z["pivot_types"].astype(np.int32))
    assert np.array_equal(f.panel_end, z["panel_end"])


def test_sampled_residual_restatement(port):
    # SampledRelativeResidual (tests/block_ldlt_large_stress_test.cc:220-244)
    # on the reference's own sample set: its first four samples are fixed
    # (:207-210), and at a size where the full reconstruction fits it agrees
    # with the residual of those entries of P^T L D L^T P
    n, b = 300, 32
    a = uniform_symmetric(n, 77)
    f = port.factor(a, b)
    rows, cols = port.residual_samples(n, 3, 4096)
    assert list(zip(rows[:4], cols[:4])) == [(0, 0), (0, n - 1), (n // 2, n // 2), (n - 1, n - 1)]
    got = port.sampled_residual(a, f, rows, cols)
    rec = reconstruct(f.factors, f.perm, f.pivot_types)
    d = rec[rows, cols] - a[rows, cols]
    want = np.sqrt(np.sum(d * d)) / max(np.sqrt(np.sum(a[rows, cols] ** 2)), 1.0)
    assert got < 1e-12
    assert abs(got - want) <= 0.5 * want + 1e-16


@pytest.mark.parametrize("n,b", [(4, 2), (37, 5), (64, 16)])
def test_reference_full_mode_factors(reference, port, n, b):
    # the reference's own LFactor()/DFactor() (kFull mode) equal the dense
    # extraction of the compact factors that the GPU tests use
    # (ExtractRegularFactorsFromCompact, src/block_ldlt_decomposition.cc:746-763)
    a = uniform_symmetric(n, 900 + n)
    rec, lf, df = reference.factor_full(a, b)
    f = port.factor(a, b)
    two = np.where(f.pivot_types == 2)[0]
    lt = np.triu(f.factors, 1)
    lt[two, two + 1] = 0.0
    l = lt.T.copy()
    l[np.diag_indices(n)] = 1.0
    d = np.diag(np.diag(f.factors))
    d[two, two + 1] = f.factors[two, two + 1]
    d[two + 1, two] = f.factors[two, two + 1]
    assert np.array_equal(lf, l)
    assert np.array_equal(df, d)
    assert relative_error(rec, a) < TOLERANCE


@pytest.mark.parametrize("n,b,seed", [(40, 7, 1), (60, 4, 2), (200, 32, 3), (333, 64, 4)])
def test_workspace_rows_match_the_reference(reference, port, n, b, seed):
    # each panel's W rows at the columns its trailing update reads: exactly
    # the reference's Workspace() outside the diagonal blocks (the first two
    # cases include boundary shifts)
    a = uniform_symmetric(n, seed)
    f, _, w = port.factor_logged(a, b, workspace_rows=True)
    ws = reference.workspace(a, b)
    mask = np.zeros((n, n), bool)
    k0 = 0
    for e in f.panel_end:
        mask[k0:e, e:] = True
        k0 = e
    assert np.array_equal(w[mask], ws[mask])
    assert np.all(w[~mask] == 0.0)
