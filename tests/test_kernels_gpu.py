"""GPU: the kernels.h boundary (ScaleOneByOnePivot, ScaleTwoByTwoPivot,
UpdateTrailingBlock) through the C ABI against the oracle."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def test_scale_kernels_known_answers(cuda, bbk):
    import torch
    L = bbk.lib()
    src = torch.tensor([2.0, 4.0, 6.0], dtype=torch.float64, device=cuda)
    dst = torch.zeros(3, dtype=torch.float64, device=cuda)
    bbk.check(L.bbk_scale_one_by_one(3, 2.0, _p(src), 1, _p(dst), 1, None))
    torch.cuda.synchronize()
    assert dst.tolist() == [1.0, 2.0, 3.0]
    s1 = torch.tensor([1.0, 2.0], dtype=torch.float64, device=cuda)
    s2 = torch.tensor([3.0, 4.0], dtype=torch.float64, device=cuda)
    d1 = torch.zeros(2, dtype=torch.float64, device=cuda)
    d2 = torch.zeros(2, dtype=torch.float64, device=cuda)
    bbk.check(L.bbk_scale_two_by_two(2, 2.0, 1.0, 3.0, _p(s1), 1, _p(s2), 1, _p(d1), 1, _p(d2), 1, None))
    torch.cuda.synchronize()
    assert abs(d1[0].item()) < 1e-14 and abs(d2[0].item() - 1.0) < 1e-14
    # zero pivot / zero determinant give zeros (src/kernels.cc:17-22, 47-53)
    bbk.check(L.bbk_scale_one_by_one(3, 0.0, _p(src), 1, _p(dst), 1, None))
    bbk.check(L.bbk_scale_two_by_two(2, 1.0, 1.0, 1.0, _p(s1), 1, _p(s2), 1, _p(d1), 1, _p(d2), 1, None))
    torch.cuda.synchronize()
    assert dst.abs().sum().item() == 0.0 and d1.abs().sum().item() == 0.0


@pytest.mark.parametrize("rows,cols,inner", [(5, 7, 3), (64, 64, 64), (130, 70, 33), (200, 300, 129)])
def test_update_trailing_block(cuda, bbk, port, rows, cols, inner):
    import torch
    rng = np.random.default_rng(rows * cols)
    left = rng.standard_normal((inner, rows))
    ws = rng.standard_normal((inner, cols))
    tgt = rng.standard_normal((rows, cols))
    want = port.update_trailing_block(left, ws, tgt)
    L = bbk.lib()
    for mode, tol in ((bbk.UPDATE_FP64_ORDERED, 0.0), (bbk.UPDATE_FP64, 1e-13), (bbk.UPDATE_FP32, 1e-5)):
        tl, tw = torch.from_numpy(left).to(cuda), torch.from_numpy(ws).to(cuda)
        tt = torch.from_numpy(tgt).to(cuda)
        bbk.check(L.bbk_update_trailing_block(rows, cols, inner, _p(tl), rows, _p(tw), cols, _p(tt), cols,
                                              mode, None))
        torch.cuda.synchronize()
        got = tt.cpu().numpy()
        err = np.max(np.abs(got - want)) / max(1.0, np.max(np.abs(want)))
        assert err <= tol, (mode, err)
