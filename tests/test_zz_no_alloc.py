"""GPU: the solve entry point that allocates nothing.

bbk_solve_device_noalloc serves callers that cannot allocate device memory
(a framework's caching allocator owns the device memory, a fixed pool, or a
loop that cannot afford cudaMalloc's device-wide synchronisation); its
scratch is one fixed array inside the library.  Its results must match the
allocating entry point bbk_solve_device on two calls in a row (the second
call reuses the array the first one left behind).  This file is collected
last so that a failure here comes after every other test has run.
"""
import ctypes

import numpy as np
import pytest

from common import uniform_symmetric

pytestmark = pytest.mark.gpu


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _solve_existing(bbk, f, perm, pt, b):
    x = b.clone()
    bbk.solve_device(f, perm, pt, x)
    return x


def _solve_noalloc(bbk, f, perm, pt, b):
    import torch
    x = b.clone()
    n = f.shape[0]
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    bbk.check(bbk.lib().bbk_solve_device_noalloc(n, _p(f), f.stride(0), _p(perm), _p(pt), x.shape[0],
                                                 _p(x), x.stride(0), stream))
    torch.cuda.synchronize()
    return x


def test_noalloc_matches_existing_solve_twice(cuda, bbk):
    # Both entry points run the same kernels on the same data, so the
    # results must be identical bit for bit (a stale or overlapping scratch
    # would show as a difference).
    import torch
    n, blk = 1500, 64
    f = torch.from_numpy(uniform_symmetric(n, 99)).to(cuda)
    perm, pt, _ = bbk.factor_device(f, blk)
    rng = np.random.default_rng(3)
    for nrhs in (3, 1):  # two calls in a row; the second reuses the array
        b = torch.from_numpy(rng.standard_normal((nrhs, n))).to(cuda)
        want = _solve_existing(bbk, f, perm, pt, b).cpu().numpy()
        got = _solve_noalloc(bbk, f, perm, pt, b).cpu().numpy()
        assert np.array_equal(got, want)


def test_noalloc_at_its_size_limit_and_with_strided_rhs(cuda, bbk):
    # n * nrhs exactly at the limit puts the block flags and the status word
    # at the end of the array; a leading dimension above n checks that only
    # the first n entries of each right-hand side are read and written.
    import torch
    n, blk = 4096, 128
    nrhs = bbk.SOLVE_NOALLOC_MAX_ELEMENTS // n
    assert n * nrhs == bbk.SOLVE_NOALLOC_MAX_ELEMENTS
    f = torch.from_numpy(uniform_symmetric(n, 4097)).to(cuda)
    perm, pt, _ = bbk.factor_device(f, blk)
    rng = np.random.default_rng(11)
    b = torch.from_numpy(rng.standard_normal((nrhs, n))).to(cuda)
    assert np.array_equal(_solve_noalloc(bbk, f, perm, pt, b).cpu().numpy(),
                          _solve_existing(bbk, f, perm, pt, b).cpu().numpy())
    ldb = n + 5
    wide = torch.from_numpy(rng.standard_normal((3, ldb))).to(cuda)
    got = _solve_noalloc(bbk, f, perm, pt, wide).cpu().numpy()
    want = _solve_existing(bbk, f, perm, pt, wide).cpu().numpy()
    assert np.array_equal(got, want)
    assert np.array_equal(got[:, n:], wide[:, n:].cpu().numpy())  # padding untouched


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda, bbk):
    import torch
    n = 1024
    nrhs = bbk.SOLVE_NOALLOC_MAX_ELEMENTS // n + 1
    f = torch.eye(n, dtype=torch.float64, device=cuda)
    perm = torch.arange(n, dtype=torch.int32, device=cuda)
    pt = torch.ones(n, dtype=torch.int32, device=cuda)
    b = torch.zeros((nrhs, n), dtype=torch.float64, device=cuda)
    with pytest.raises(bbk.InvalidArgument):
        _solve_noalloc(bbk, f, perm, pt, b)
