"""GPU: batched factor + solve (many small matrices, one persistent launch).

Every matrix of a batch must factor exactly as the reference factors it on
its own with the block size the plan chose: bit for bit in the ordered mode
(factors, permutation, pivot types), and with the same pivot sequence and a
residual within 10x of the reference's in the FP64 mode.  The solve and the
FP32-update + FP64-refinement mode are checked by backward error."""
import numpy as np
import pytest

from common import backward_error, kkt_matrix, reconstruct, relative_error, uniform_symmetric

pytestmark = pytest.mark.gpu
EPS = np.finfo(np.float64).eps


def _batch(sizes, seed):
    mats, rhs = [], []
    rng = np.random.default_rng(seed)
    for k, n in enumerate(sizes):
        if n >= 8 and k % 2 == 0:
            mats.append(kkt_matrix(n, max(1, (3 * n) // 4), seed + k))
        else:
            mats.append(uniform_symmetric(n, seed + k))
        rhs.append(rng.standard_normal(n))
    return mats, rhs


SIZES = [1, 2, 3, 5, 16, 17, 31, 32, 33, 48, 64, 65, 100, 127, 128, 129, 200, 255, 256, 257, 300, 384, 512]


def _run(bbk, sizes, seed, mode, block_sizes=None, **kw):
    plan = bbk.BatchedPlan(sizes, block_sizes=block_sizes)
    mats, rhs = _batch(sizes, seed)
    a, x = plan.pack(mats, rhs)
    a0 = a.clone()
    perm, pt, info = bbk.batched_factor_solve(plan, a, x, mode=mode,
                                              a_orig=a0 if kw.get("max_iter", 0) else None, **kw)
    return plan, mats, rhs, a.cpu().numpy(), x.cpu().numpy(), perm.cpu().numpy(), pt.cpu().numpy(), info


def test_batched_ordered_is_the_reference(cuda, bbk, port):
    plan, mats, rhs, a, x, perm, pt, info = _run(bbk, SIZES, 11, "fp64_ordered",
                                                 block_sizes=[8, 16, 32, 24, 16, 8])
    for k, m in enumerate(mats):
        want = port.factor(m, int(plan.block_sizes[k]))
        got = plan.matrix(a, k)
        assert np.array_equal(np.triu(got), np.triu(want.factors), equal_nan=True), (k, m.shape)
        assert np.array_equal(plan.vector(perm, k), want.perm), k
        assert np.array_equal(plan.vector(pt, k), want.pivot_types), k
        xs = plan.vector(x, k)
        assert backward_error(m, xs, rhs[k]) < 20 * m.shape[0] * EPS, k


def test_batched_fp64_same_pivots_and_residual(cuda, bbk, port):
    sizes = SIZES + [96, 160, 320, 448]
    plan, mats, rhs, a, x, perm, pt, info = _run(bbk, sizes, 23, "fp64")
    for k, m in enumerate(mats):
        b = int(plan.block_sizes[k])
        want = port.factor(m, b)
        assert np.array_equal(plan.vector(pt, k), want.pivot_types), k
        assert np.array_equal(plan.vector(perm, k), want.perm), k
        f = plan.matrix(a, k)
        res = relative_error(reconstruct(f, plan.vector(perm, k), plan.vector(pt, k)), m)
        res_ref = relative_error(reconstruct(want.upper(), want.perm, want.pivot_types), m)
        n = m.shape[0]
        assert res <= max(10 * res_ref, 1e-15) and res <= n * EPS * 8, (k, n, res, res_ref)
        assert backward_error(m, plan.vector(x, k), rhs[k]) < 20 * n * EPS, k


def test_batched_fp32_update_with_fp64_refinement(cuda, bbk):
    rng = np.random.default_rng(5)
    sizes = [int(v) for v in rng.integers(16, 513, size=64)]
    plan, mats, rhs, a, x, perm, pt, info = _run(bbk, sizes, 31, "fp32", tol=1e-12, max_iter=12)
    assert info["converged"].all(), info
    for k, m in enumerate(mats):
        be = backward_error(m, plan.vector(x, k), rhs[k])
        assert be <= 2e-12, (k, be, info[k])
        assert info["backward_error"][k] <= 1e-12


def test_batched_results_do_not_depend_on_the_batch(cuda, bbk):
    sizes = [300, 40, 7, 129]
    _, mats, rhs, a1, x1, p1, t1, _ = _run(bbk, sizes, 3, "fp64")
    plan2 = bbk.BatchedPlan([129, 7])
    a2, xx2 = plan2.pack([mats[3], mats[2]], [rhs[3], rhs[2]])
    perm2, pt2, _ = bbk.batched_factor_solve(plan2, a2, xx2, mode="fp64")
    plan1 = bbk.BatchedPlan(sizes)
    assert np.array_equal(plan1.matrix(a1, 3), plan2.matrix(a2.cpu().numpy(), 0))
    assert np.array_equal(plan1.vector(x1, 2), plan2.vector(xx2.cpu().numpy(), 1))


def test_batched_plan_validation_and_block_clamp(cuda, bbk):
    with pytest.raises(bbk.InvalidArgument):
        bbk.BatchedPlan([4, bbk.BATCH_MAX_N + 1])
    with pytest.raises(bbk.InvalidArgument):
        bbk.BatchedPlan([0])
    plan = bbk.BatchedPlan([512, 1024, 20, 33], block_sizes=[64, 64, 64, 64, 64, 64])
    assert plan.block_sizes[2] == 20  # never wider than the matrix
    assert 1 <= plan.block_sizes[1] < plan.block_sizes[0] <= 64  # shared memory bounds the panel width
