"""GPU: the BF16 trailing updates on the 5th-generation tensor cores
(tcgen05.mma with the accumulator in tensor memory).

Orders and block sizes cover one and several 128 x 128 tiles per CTA, k
chunks from 2 to 9 per tile and the boundary rows below the 64-aligned split
origin.  The factors of a BF16x3 update carry about FP32 accuracy, those of a
single-term BF16 update about BF16 accuracy; both must reconstruct the matrix
to that level, and the three-term factors must match the FP64 factorization's
pivots on these well-separated inputs."""
import numpy as np
import pytest

from common import relative_error, reconstruct, uniform_symmetric

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,b", [(300, 32), (1000, 64), (2000, 128), (6000, 256)])
@pytest.mark.parametrize("mode,bound", [("bf16x3", 5e-5), ("bf16", 0.3)])
def test_tensor_memory_bf16_update(cuda, bbk, n, b, mode, bound):
    import torch
    a = uniform_symmetric(n, 3 * n + b)
    f = torch.from_numpy(a).to(cuda)
    perm, pt, _ = bbk.factor_device(f, b, mode=mode)
    fh, ph, pth = f.cpu().numpy(), perm.cpu().numpy(), pt.cpu().numpy()
    assert np.all(np.isfinite(np.triu(fh)))
    res = relative_error(reconstruct(fh, ph, pth), a) if n <= 2000 else None
    if res is not None:
        assert res < bound, res
    if mode == "bf16x3" and n <= 1000:
        g = torch.from_numpy(a).to(cuda)
        perm64, pt64, _ = bbk.factor_device(g, b, mode="fp64")
        assert np.array_equal(pt64.cpu().numpy(), pth)
        assert np.array_equal(perm64.cpu().numpy(), ph)
        assert np.max(np.abs(np.triu(fh) - np.triu(g.cpu().numpy()))) < 1e-3 * np.max(np.abs(np.triu(fh)))
    if n > 2000:
        # large order: the backward error of a solve with these factors, to
        # the update's accuracy
        rhs = torch.from_numpy(np.random.default_rng(1).standard_normal((1, n))).to(cuda)
        x = bbk.solve_device(f, perm, pt, rhs.clone())
        a0 = torch.from_numpy(a).to(cuda)
        r = rhs - x @ a0
        be = float(r.abs().max() / (a0.abs().sum(1).max() * x.abs().max() + rhs.abs().max()))
        assert be < (1e-5 if mode == "bf16x3" else 0.1), be
