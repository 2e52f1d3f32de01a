"""GPU: the kFull outputs on the device.

bbk_extract_ld_device restates ExtractRegularFactorsFromCompact
(src/block_ldlt_decomposition.cc:746-763) and must give exactly the L and D
that the test-side extraction (the same rule that tests/test_oracle.py pins to
the reference's own LFactor()/DFactor()) builds from the same factors.
bbk_reconstruct_device (ReconstructOriginal, :61-78) runs the product on the
FP64 tensor cores; it must reproduce the original matrix to the reference
tests' 1e-10 and agree with a test-side FP64 product of the same factors to
rounding.  Sizes cover the 64x64 and the 128x128 tile kernels (n >= ~3000
uses the latter)."""
import numpy as np
import pytest

from common import TOLERANCE, relative_error, uniform_symmetric

pytestmark = pytest.mark.gpu


def _ld(f, pt):
    n = f.shape[0]
    two = np.where(pt == 2)[0]
    lt = np.triu(f, 1)
    lt[two, two + 1] = 0.0
    l = lt.T.copy()
    l[np.diag_indices(n)] = 1.0
    d = np.diag(np.diag(f))
    d[two, two + 1] = f[two, two + 1]
    d[two + 1, two] = f[two, two + 1]
    return l, d


@pytest.mark.parametrize("n,b", [(5, 2), (100, 16), (333, 32), (1000, 64), (3200, 128)])
def test_extract_and_reconstruct(cuda, bbk, n, b):
    import torch
    a = uniform_symmetric(n, 5 * n + 1)
    f = torch.from_numpy(a).to(cuda)
    perm, pt, _ = bbk.factor_device(f, b, mode="fp64_ordered")
    fh, pth, permh = np.triu(f.cpu().numpy()), pt.cpu().numpy(), perm.cpu().numpy()
    l, d = bbk.extract_ld_device(f, pt)
    lw, dw = _ld(fh, pth)
    assert np.array_equal(l.cpu().numpy(), lw)
    assert np.array_equal(d.cpu().numpy(), dw)
    rec = bbk.reconstruct_device(f, perm, pt).cpu().numpy()
    assert relative_error(rec, a) < TOLERANCE
    m = lw @ dw @ lw.T
    want = np.empty_like(m)
    want[np.ix_(permh, permh)] = m
    assert np.max(np.abs(rec - want)) <= 1e-12 * max(1.0, np.max(np.abs(want)))
    assert np.array_equal(rec, rec.T)
