"""GPU: pivot-sequence parity with the reference at a benchmark size.

The saddle-point workload at full size (n=10000: H 8000 SPD, B Gaussian, a
zero (2,2) block; block size 128) against the reference's own factorization
of the same input, stored in tests/golden/ref_kkt10000.npz by
tests/golden/make_golden.py --kkt.  The input comes from
tests/common.py's kkt_matrix_exact, which every machine computes bit for bit;
its SHA-256 is checked first.

* BBK_UPDATE_FP64_ORDERED keeps the reference's arithmetic: the compact
  factor must be bitwise the reference's (SHA-256), with the same
  permutation, pivot types and panel ends.
* BBK_UPDATE_FP64 (tensor-core update, reassociated panel sums) may round
  differently, so its pivot sequence must equal the reference's except after
  a logged near-tie: the first position where the sequences differ must be a
  decision whose relative margin (in the GPU's decision log or in the
  reference's, recomputed by the C restatement) is below 64 n eps.  Its
  relative reconstruction residual ||P A P^T - L D L^T||_F / ||A||_F must be
  at most 10x the reference's and at most n eps.
"""
import hashlib
import os

import numpy as np
import pytest

from common import GOLDEN, kkt_matrix_exact

pytestmark = pytest.mark.gpu

EPS = np.finfo(np.float64).eps


@pytest.fixture(scope="module")
def case():
    z = np.load(os.path.join(GOLDEN, "ref_kkt10000.npz"))
    fx = {k: z[k] for k in z.files}
    n, h, seed = int(fx["n"]), int(fx["h"]), int(fx["seed"])
    a, sha = kkt_matrix_exact(n, h, seed)
    assert sha == str(fx["input_sha256"]), "the input generator no longer reproduces the fixture's input"
    fx["a"] = a
    return fx


def _first_divergence(perm, pt, want_perm, want_pt):
    bad = np.nonzero((perm != want_perm) | (pt != want_pt))[0]
    return int(bad[0]) if bad.size else None


def test_ordered_mode_is_bitwise_the_reference(case, cuda, bbk):
    import torch
    n, b = int(case["n"]), int(case["block_size"])
    f = torch.from_numpy(case["a"]).to(cuda)
    perm, pt, pe = bbk.factor_device(f, b, mode="fp64_ordered")
    assert np.array_equal(perm.cpu().numpy(), case["perm"])
    assert np.array_equal(pt.cpu().numpy(), case["pivot_types"].astype(np.int32))
    assert np.array_equal(pe.cpu().numpy(), case["panel_end"])
    up = torch.triu(f).cpu().numpy()
    assert hashlib.sha256(np.ascontiguousarray(up).tobytes()).hexdigest() == str(case["upper_sha256"])


def test_fp64_mode_pivots_match_except_logged_near_ties(case, cuda, bbk):
    import torch
    n, b = int(case["n"]), int(case["block_size"])
    a = torch.from_numpy(case["a"]).to(cuda)
    f = a.clone()
    perm, pt, pe, log = bbk.factor_device_logged(f, b, mode="fp64")
    perm_h, pt_h, log_h = perm.cpu().numpy(), pt.cpu().numpy(), log.cpu().numpy()
    want_perm, want_pt = case["perm"], case["pivot_types"].astype(np.int32)
    tol = 64 * n * EPS
    k = _first_divergence(perm_h, pt_h, want_perm, want_pt)
    if k is None:
        assert np.array_equal(pe.cpu().numpy(), case["panel_end"])
        # the two logs describe the same decisions: where a step started,
        # the GPU's |W(p,p)| and omega agree with the reference's to rounding
        started = ~np.isnan(log_h[:, 0])
        assert np.array_equal(started, ~np.isnan(case["log"][:, 0]))
        ref = case["log"][started][:, :2].astype(np.float64)
        got = log_h[started][:, :2]
        assert np.all(np.abs(got - ref) <= 1e-5 * np.maximum(np.abs(ref), 1e-300))
    else:
        # the step that decided position k started at k or, inside a 2x2, at k - 1
        p = k - 1 if k > 0 and want_pt[k] == -2 else k
        gpu_m = bbk.decision_margins(log_h)[p]
        ref_m = float(case["margin"][p])
        assert min(gpu_m, ref_m) < tol, (
            f"pivot sequences differ at position {k} without a near-tie "
            f"(margins: GPU {gpu_m:.3e}, reference {ref_m:.3e}, tolerance {tol:.3e})")
        print(f"logged near-tie at position {p}: margins GPU {gpu_m:.3e}, reference {ref_m:.3e}")
    rec = bbk.reconstruct_device(f, perm, pt)
    res = float(torch.linalg.norm(rec - a) / torch.linalg.norm(a))
    assert res <= 10.0 * float(case["residual"])
    assert res <= n * EPS
