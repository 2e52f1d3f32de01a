"""GPU: the reference stress test's sampled residual on the device.

bbk_sampled_residual_device restates SampledRelativeResidual
(tests/block_ldlt_large_stress_test.cc:160-244): each sampled entry of
P^T L D L^T P is summed over the pivots in the reference's order, so for the
same factors it must equal the oracle's restatement bit for bit.  The factors
come from the ordered mode (bitwise the reference's), the samples from the
reference's own generator (ResidualSamples, :204-218)."""
import numpy as np
import pytest

from common import kkt_matrix, uniform_symmetric

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,n,b", [("uniform", 2000, 64), ("kkt", 2400, 128), ("uniform", 333, 16)])
def test_sampled_residual_matches_oracle_bitwise(cuda, bbk, port, kind, n, b):
    import torch
    a = uniform_symmetric(n, n) if kind == "uniform" else kkt_matrix(n, int(0.8 * n), seed=n)
    a0 = torch.from_numpy(a).to(cuda)
    f = a0.clone()
    perm, pt, _ = bbk.factor_device(f, b, mode="fp64_ordered")
    rows, cols = port.residual_samples(n, 5, 4096)
    got = bbk.sampled_residual_device(a0, f, perm, pt, torch.from_numpy(rows).to(cuda),
                                      torch.from_numpy(cols).to(cuda))
    fac = port.factor(a, b)
    assert np.array_equal(np.triu(f.cpu().numpy()), np.triu(fac.factors))
    want = port.sampled_residual(a, fac, rows, cols)
    assert got == want
    assert got < 1e-8


def test_sampled_residual_out_of_range_sample_gives_nan(cuda, bbk):
    # samples outside the matrix make the result NaN instead of reading
    # outside the arrays
    import torch
    n = 64
    a0 = torch.eye(n, dtype=torch.float64, device=cuda)
    f = a0.clone()
    perm, pt, _ = bbk.factor_device(f, 16)
    rows = torch.tensor([0, n + 5], dtype=torch.int32, device=cuda)
    cols = torch.tensor([0, 1], dtype=torch.int32, device=cuda)
    assert np.isnan(bbk.sampled_residual_device(a0, f, perm, pt, rows, cols))
