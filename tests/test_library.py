"""CPU: the C-ABI library loads, exports every declared symbol and rejects bad
arguments before touching a device (no compute call needs a GPU here)."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "bbk_ldlt.h")).read()
    return sorted(set(re.findall(r"\b(bbk_[a-z0-9_]+)\s*\(", src)))


def test_header_matches_python_exports(bbk):
    assert declared_symbols() == sorted(bbk.EXPORTS)


def test_library_exports_every_declared_symbol(bbk):
    lib = ctypes.CDLL(bbk.LIB_PATH)
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_abi_version_and_status_strings(bbk):
    L = bbk.lib()
    assert L.bbk_abi_version() == 1
    assert L.bbk_status_string(bbk.BBK_ERR_TIMEOUT) == b"device-side wait timed out"


def test_invalid_arguments_rejected_without_device(bbk):
    a = np.zeros((4, 4))
    with pytest.raises(bbk.InvalidArgument):
        bbk.factor_host(a, 0)          # block size must be positive
    with pytest.raises(bbk.InvalidArgument):
        bbk.factor_host(np.zeros((0, 0)), 2)
    with pytest.raises(bbk.InvalidArgument):
        bbk.factor_host(a, 2, mode=7)
    with pytest.raises(bbk.InvalidArgument):
        bbk.BlockLdltDecomposition(np.zeros((3, 4)), 2)


def test_workspace_sizes_positive(bbk):
    assert bbk.factor_workspace_size(10000, 128) > 10000 * 128 * 8
    assert bbk.solve_workspace_size(100, 4) == 2 * 100 * 4 * 8
    assert bbk.factor_workspace_size(0, 4) == 0


def test_compute_without_gpu_fails_loudly(bbk):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    with pytest.raises(bbk.BbkError) as e:
        bbk.factor_host(np.eye(4), 2)
    assert e.value.status in (bbk.BBK_ERR_NO_DEVICE, bbk.BBK_ERR_CUDA)


def test_reconstruct_requires_full_mode(bbk):
    d = bbk.BlockLdltDecomposition(np.eye(3), 2, full=False)
    with pytest.raises(bbk.LogicError):
        d.reconstruct_original()
