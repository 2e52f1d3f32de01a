"""B200-native blocked Bunch-Kaufman LDL^T.

Python access to ``libbbk_b200.so`` (CUDA kernels for sm_100a behind the C ABI
of ``include/bbk_ldlt.h``).  There is no CPU fallback: importing works without
a GPU (so the library can be inspected), but every compute call needs the
built library and an sm_100 device and raises otherwise.

The class :class:`BlockLdltDecomposition` mirrors the reference's
``naive_block_ldlt::BlockLdltDecomposition`` (include/block_ldlt_decomposition.h:
11-31 in wentianshu/BlockedBunchKaufmanLDLT): construct from a symmetric
matrix and a block size, ``factorize()``, then read the compact factors,
permutation and pivot types, or ``reconstruct_original()`` in full mode.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbbk_b200.so")

BBK_OK = 0
BBK_ERR_INVALID_ARGUMENT = 1
BBK_ERR_OUT_OF_RANGE = 2
BBK_ERR_LOGIC = 3
BBK_ERR_ALLOC = 4
BBK_ERR_CUDA = 5
BBK_ERR_TIMEOUT = 6
BBK_ERR_NO_DEVICE = 7
BBK_ERR_WORKSPACE = 8

UPDATE_FP64 = 0
UPDATE_FP64_ORDERED = 1
UPDATE_FP32 = 2
UPDATE_BF16 = 3
UPDATE_BF16X3 = 4
UPDATE_MODES = {"fp64": UPDATE_FP64, "fp64_ordered": UPDATE_FP64_ORDERED, "fp32": UPDATE_FP32,
                "bf16": UPDATE_BF16, "bf16x3": UPDATE_BF16X3}
REFINE_CLASSICAL = 0
REFINE_GMRES = 1

# Every symbol include/bbk_ldlt.h declares.
EXPORTS = (
    "bbk_abi_version", "bbk_last_error", "bbk_status_string", "bbk_kernel_launch_count",
    "bbk_set_wait_timeout_ns", "bbk_probe_bounded_wait", "bbk_probe_exchange_ns", "bbk_factor_workspace_size",
    "bbk_factor_device", "bbk_factor_device_async", "bbk_factor_device_ex", "bbk_factor_host",
    "bbk_solve_workspace_size", "bbk_solve_device", "bbk_solve_host", "bbk_factor_solve_host",
    "bbk_reconstruct_device", "bbk_extract_ld_device", "bbk_sampled_residual_device", "bbk_scale_one_by_one", "bbk_scale_two_by_two",
    "bbk_update_trailing_block", "bbk_profile_begin", "bbk_profile_end", "bbk_panel_stats", "bbk_panel_stats_raw", "bbk_solve_device_noalloc",
    "bbk_solve_refined_workspace_size", "bbk_solve_refined_device",
    "bbk_batched_workspace_size", "bbk_batched_plan", "bbk_batched_factor_solve",
)


class RefineInfo(ctypes.Structure):
    """bbk_refine_info"""
    _fields_ = [("iterations", ctypes.c_int), ("inner_iterations", ctypes.c_int),
                ("converged", ctypes.c_int), ("reserved", ctypes.c_int),
                ("initial_backward_error", ctypes.c_double), ("backward_error", ctypes.c_double)]
SOLVE_NOALLOC_MAX_ELEMENTS = 524288  # n * nrhs limit of bbk_solve_device_noalloc
BATCH_MAX_N = 1024                  # largest order of a batched item
BATCH_BUCKETS = 6                   # block-size buckets: n <= 32, 64, 128, 256, 512, 1024


class BatchItem(ctypes.Structure):
    """bbk_batch_item"""
    _fields_ = [("n", ctypes.c_int), ("lda", ctypes.c_int), ("a", ctypes.c_longlong),
                ("rhs", ctypes.c_longlong), ("piv", ctypes.c_longlong)]


class BatchInfo(ctypes.Structure):
    """bbk_batch_info"""
    _fields_ = [("iterations", ctypes.c_int), ("converged", ctypes.c_int), ("backward_error", ctypes.c_double)]
PROFILE_CLASSES = ("init", "panel", "finalize", "update", "solve")


class BbkError(RuntimeError):
    """A libbbk_b200 call failed; ``status`` is the bbk_status code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status


class InvalidArgument(BbkError, ValueError):
    """The reference's std::invalid_argument."""


class OutOfRange(BbkError, IndexError):
    """The reference's std::out_of_range."""


class LogicError(BbkError):
    """The reference's std::logic_error."""


_EXC = {BBK_ERR_INVALID_ARGUMENT: InvalidArgument, BBK_ERR_OUT_OF_RANGE: OutOfRange,
        BBK_ERR_LOGIC: LogicError}

_c_int, _c_ll, _c_dbl, _c_sz, _vp = ctypes.c_int, ctypes.c_longlong, ctypes.c_double, ctypes.c_size_t, ctypes.c_void_p
_lib = None


def build(verbose: bool = False) -> str:
    from . import buildlib as _b
    return _b.build(verbose=verbose)


def lib() -> ctypes.CDLL:
    """Load libbbk_b200.so (raises if it was never built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with "
                           "`python -c 'import __graft_entry__ as g; g.build()'`")
    L = ctypes.CDLL(LIB_PATH)
    sig = {
        "bbk_abi_version": ([], _c_int),
        "bbk_last_error": ([], ctypes.c_char_p),
        "bbk_status_string": ([_c_int], ctypes.c_char_p),
        "bbk_kernel_launch_count": ([], ctypes.c_ulonglong),
        "bbk_set_wait_timeout_ns": ([ctypes.c_ulonglong], _c_int),
        "bbk_profile_begin": ([], _c_int),
        "bbk_profile_end": ([_vp, _vp], _c_int),
        "bbk_panel_stats": ([_c_int, _vp], _c_int),
        "bbk_panel_stats_raw": ([_vp, _c_sz], _c_int),
        "bbk_probe_bounded_wait": ([_c_int, ctypes.c_ulonglong, _vp], _c_int),
        "bbk_probe_exchange_ns": ([_c_int, _c_int, _vp, _vp], _c_int),
        "bbk_factor_workspace_size": ([_c_int, _c_int], _c_sz),
        "bbk_factor_device": ([_c_int, _c_int, _vp, _c_ll, _vp, _vp, _vp, _c_int, _vp, _c_sz, _vp], _c_int),
        "bbk_factor_device_async": ([_c_int, _c_int, _vp, _c_ll, _vp, _vp, _vp, _c_int, _vp, _c_sz,
                                     _vp, _vp], _c_int),
        "bbk_factor_device_ex": ([_c_int, _c_int, _vp, _c_ll, _vp, _vp, _vp, _c_int, _vp, _vp, _c_sz,
                                  _vp, _vp], _c_int),
        "bbk_factor_host": ([_c_int, _c_int, _vp, _c_ll, _vp, _vp, _vp, _c_int], _c_int),
        "bbk_solve_workspace_size": ([_c_int, _c_int], _c_sz),
        "bbk_solve_device": ([_c_int, _vp, _c_ll, _vp, _vp, _c_int, _vp, _c_ll, _vp, _c_sz, _vp], _c_int),
        "bbk_solve_host": ([_c_int, _vp, _c_ll, _vp, _vp, _c_int, _vp, _c_ll], _c_int),
        "bbk_solve_device_noalloc": ([_c_int, _vp, _c_ll, _vp, _vp, _c_int, _vp, _c_ll, _vp], _c_int),
        "bbk_solve_refined_workspace_size": ([_c_int, _c_int, _c_int], _c_sz),
        "bbk_batched_workspace_size": ([_c_int, _c_int], _c_sz),
        "bbk_batched_plan": ([_c_int, _vp, _vp, _vp, _vp, _c_sz, _vp], _c_int),
        "bbk_batched_factor_solve": ([_c_int, _vp, _vp, _vp, _vp, _vp, _c_int, ctypes.c_double, _c_int, _vp,
                                      _vp, _c_sz, _vp], _c_int),
        "bbk_solve_refined_device": ([_c_int, _vp, _c_ll, _vp, _c_ll, _vp, _vp, _c_int, _vp, _c_ll, _vp,
                                      _c_ll, ctypes.c_double, _c_int, _c_int, _c_int, _vp, _vp, _c_sz,
                                      _vp], _c_int),
        "bbk_factor_solve_host": ([_c_int, _c_int, _vp, _c_ll, _vp, _vp, _vp, _c_int, _vp, _c_ll,
                                   _c_int], _c_int),
        "bbk_reconstruct_device": ([_c_int, _vp, _c_ll, _vp, _vp, _vp, _c_ll, _vp], _c_int),
        "bbk_extract_ld_device": ([_c_int, _vp, _c_ll, _vp, _vp, _c_ll, _vp, _c_ll, _vp], _c_int),
        "bbk_sampled_residual_device": ([_c_int, _vp, _c_ll, _vp, _c_ll, _vp, _vp, _c_int, _vp, _vp, _vp, _vp],
                                        _c_int),
        "bbk_scale_one_by_one": ([_c_int, _c_dbl, _vp, _c_int, _vp, _c_int, _vp], _c_int),
        "bbk_scale_two_by_two": ([_c_int, _c_dbl, _c_dbl, _c_dbl, _vp, _c_int, _vp, _c_int, _vp,
                                  _c_int, _vp, _c_int, _vp], _c_int),
        "bbk_update_trailing_block": ([_c_int, _c_int, _c_int, _vp, _c_int, _vp, _c_int, _vp,
                                       _c_int, _c_int, _vp], _c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def check(status: int) -> None:
    if status != BBK_OK:
        msg = lib().bbk_last_error().decode(errors="replace")
        raise _EXC.get(status, BbkError)(status, msg)


def kernel_launch_count() -> int:
    return int(lib().bbk_kernel_launch_count())


def profile_begin() -> None:
    check(lib().bbk_profile_begin())


def profile_end() -> dict:
    """Per-class device milliseconds and launch counts since profile_begin()."""
    ms = (ctypes.c_double * 5)()
    cnt = (ctypes.c_longlong * 5)()
    check(lib().bbk_profile_end(ctypes.cast(ms, ctypes.c_void_p), ctypes.cast(cnt, ctypes.c_void_p)))
    return {k: {"ms": ms[i], "launches": cnt[i]} for i, k in enumerate(PROFILE_CLASSES)}


PANEL_PHASES = ("row_update", "exchange_1", "candidate", "exchange_2", "swap_scale")


def panel_stats(enable: bool):
    """Arm (True) or read and disarm (False) the panel phase timers."""
    out = (ctypes.c_ulonglong * 10)()
    check(lib().bbk_panel_stats(1 if enable else 0, ctypes.cast(out, ctypes.c_void_p)))
    if enable:
        return None
    d = {k: out[i] / 1e6 for i, k in enumerate(PANEL_PHASES)}  # ms
    d["pivots"] = int(out[5])
    d["candidates"] = int(out[6])
    d["exchange_ms"] = out[7] / 1e6  # CTA 0: from its arrival to the records read, all exchanges
    d["rows_ahead"] = int(out[9])  # steps whose row the previous candidate phase computed
    return d


def set_wait_timeout_ns(ns: int) -> None:
    check(lib().bbk_set_wait_timeout_ns(int(ns)))


def _np_ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _mode(mode) -> int:
    if isinstance(mode, str):
        return UPDATE_MODES[mode]
    return int(mode)


# ---------------------------------------------------------------------------
# Device (torch CUDA tensor) entry points
# ---------------------------------------------------------------------------
def _stream_ptr(stream):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def factor_device(a, block_size: int, mode="fp64", stream=None, workspace=None,
                  sync: bool = True):
    """Factor the upper triangle of the CUDA float64 tensor ``a`` (n x lda,
    row-major, modified in place into compact factors).  Returns device int32
    tensors (perm, pivot_types, panel_end)."""
    import torch
    if a.dtype != torch.float64 or not a.is_cuda or a.dim() != 2 or a.stride(1) != 1:
        raise InvalidArgument(BBK_ERR_INVALID_ARGUMENT, "need a row-major CUDA float64 matrix")
    n = a.shape[0]
    nb = (n + block_size - 1) // block_size if block_size > 0 else 0
    perm = torch.empty(n, dtype=torch.int32, device=a.device)
    pt = torch.empty(n, dtype=torch.int32, device=a.device)
    pe = torch.empty(max(nb, 1), dtype=torch.int32, device=a.device)
    ws_ptr, ws_bytes = (None, 0)
    if workspace is not None:
        ws_ptr, ws_bytes = ctypes.c_void_p(workspace.data_ptr()), workspace.numel() * workspace.element_size()
    if sync:
        check(lib().bbk_factor_device(n, block_size, ctypes.c_void_p(a.data_ptr()), a.stride(0),
                                      ctypes.c_void_p(perm.data_ptr()), ctypes.c_void_p(pt.data_ptr()),
                                      ctypes.c_void_p(pe.data_ptr()), _mode(mode), ws_ptr, ws_bytes,
                                      _stream_ptr(stream)))
    else:
        status = torch.zeros(1, dtype=torch.int32, device=a.device)
        check(lib().bbk_factor_device_async(n, block_size, ctypes.c_void_p(a.data_ptr()), a.stride(0),
                                            ctypes.c_void_p(perm.data_ptr()),
                                            ctypes.c_void_p(pt.data_ptr()),
                                            ctypes.c_void_p(pe.data_ptr()), _mode(mode), ws_ptr,
                                            ws_bytes, ctypes.c_void_p(status.data_ptr()),
                                            _stream_ptr(stream)))
        return perm, pt, pe, status
    return perm, pt, pe


PIVOT_LOG_WORDS = 4  # |W(p,p)|, omega, sigma, |W(r,r)| per factored position
ALPHA = 0.6403882032022076  # the Bunch-Kaufman threshold (1 + sqrt 17) / 8


class FactorExtras(ctypes.Structure):
    """bbk_factor_extras"""
    _fields_ = [("pivot_log", ctypes.c_void_p), ("workspace_rows", ctypes.c_void_p),
                ("workspace_ld", ctypes.c_longlong)]


def factor_device_logged(a, block_size: int, mode="fp64", stream=None, workspace_rows=None):
    """factor_device plus the optional outputs of bbk_factor_device_ex:
    returns (perm, pivot_types, panel_end, log) with log an n x 4 float64
    device tensor (|W(p,p)|, omega, sigma, |W(r,r)| at each position where a
    pivot step started; NaN elsewhere and where no candidate was needed).
    ``workspace_rows`` (CUDA float64, n x ld, optional) receives each panel's
    W rows at its trailing columns."""
    import torch
    if a.dtype != torch.float64 or not a.is_cuda or a.dim() != 2 or a.stride(1) != 1:
        raise InvalidArgument(BBK_ERR_INVALID_ARGUMENT, "need a row-major CUDA float64 matrix")
    n = a.shape[0]
    nb = (n + block_size - 1) // block_size if block_size > 0 else 0
    perm = torch.empty(n, dtype=torch.int32, device=a.device)
    pt = torch.empty(n, dtype=torch.int32, device=a.device)
    pe = torch.empty(max(nb, 1), dtype=torch.int32, device=a.device)
    log = torch.empty(n, PIVOT_LOG_WORDS, dtype=torch.float64, device=a.device)
    status = torch.zeros(1, dtype=torch.int32, device=a.device)
    ex = FactorExtras(log.data_ptr(), workspace_rows.data_ptr() if workspace_rows is not None else None,
                      workspace_rows.stride(0) if workspace_rows is not None else 0)
    check(lib().bbk_factor_device_ex(n, block_size, ctypes.c_void_p(a.data_ptr()), a.stride(0),
                                     ctypes.c_void_p(perm.data_ptr()), ctypes.c_void_p(pt.data_ptr()),
                                     ctypes.c_void_p(pe.data_ptr()), _mode(mode), ctypes.byref(ex), None, 0,
                                     ctypes.c_void_p(status.data_ptr()), _stream_ptr(stream)))
    torch.cuda.current_stream().synchronize() if stream is None else stream.synchronize()
    st = int(status.item())
    if st != BBK_OK:
        raise _EXC.get(st, BbkError)(st, "factorization aborted on the device")
    return perm, pt, pe, log


def decision_margins(log: np.ndarray) -> np.ndarray:
    """Relative margin of the decision recorded at each position of a pivot
    log (n x 4: |W(p,p)|, omega, sigma, |W(r,r)|): the smallest, over the
    comparisons the step actually made, of |lhs - rhs| / max(|lhs|, |rhs|)
    for |W(p,p)| >= alpha omega (src/block_ldlt_decomposition.cc:90-92) and,
    after a candidate, |W(p,p)| sigma >= alpha omega^2 and |W(r,r)| >= alpha
    sigma (SelectPivot, :369-390).  NaN where no step started.  A decision
    whose margin is within rounding of zero could flip under another
    summation order: a near-tie."""
    d, om, sg, arr = (log[:, k] for k in range(4))
    with np.errstate(invalid="ignore", divide="ignore"):
        def rel(x, y):
            den = np.maximum(np.abs(x), np.abs(y))
            return np.where(den > 0, np.abs(x - y) / np.where(den > 0, den, 1.0), np.inf)
        m = rel(d, ALPHA * om)
        m = np.where(om == 0.0, np.inf, m)
        cand = ~np.isnan(sg)
        m2 = rel(d * sg, ALPHA * om * om)
        m3 = rel(arr, ALPHA * sg)
        m = np.where(cand, np.minimum(m, np.minimum(m2, m3)), m)
        return np.where(np.isnan(d), np.nan, m)


def factor_workspace_size(n: int, block_size: int) -> int:
    return int(lib().bbk_factor_workspace_size(n, block_size))


def solve_workspace_size(n: int, nrhs: int) -> int:
    return int(lib().bbk_solve_workspace_size(n, nrhs))


def solve_device(f, perm, pivot_types, b, stream=None, workspace=None):
    """Solve with compact factors on the device.  ``b`` is a CUDA float64
    tensor of shape (nrhs, n) (each row one right-hand side), overwritten."""
    n = f.shape[0]
    nrhs = b.shape[0] if b.dim() == 2 else 1
    ldb = b.stride(0) if b.dim() == 2 else n
    ws_ptr, ws_bytes = (None, 0)
    if workspace is not None:
        ws_ptr, ws_bytes = ctypes.c_void_p(workspace.data_ptr()), workspace.numel() * workspace.element_size()
    check(lib().bbk_solve_device(n, ctypes.c_void_p(f.data_ptr()), f.stride(0),
                                 ctypes.c_void_p(perm.data_ptr()), ctypes.c_void_p(pivot_types.data_ptr()),
                                 nrhs, ctypes.c_void_p(b.data_ptr()), ldb, ws_ptr, ws_bytes,
                                 _stream_ptr(stream)))
    return b


def solve_refined_device(a, f, perm, pivot_types, b, tol=1e-12, max_iter=30, method="gmres",
                         restart=20, stream=None, workspace=None):
    """FP64-refined solve on the device.  ``a`` is the original matrix (upper
    triangle used), ``f`` the compact factors, ``b`` (nrhs, n) right-hand
    sides.  Returns (x, RefineInfo)."""
    import torch
    n = f.shape[0]
    bb = b if b.dim() == 2 else b.reshape(1, n)
    x = torch.empty_like(bb)
    info = RefineInfo()
    meth = {"classical": REFINE_CLASSICAL, "gmres": REFINE_GMRES}[method] if isinstance(method, str) else method
    ws_ptr, ws_bytes = (None, 0)
    if workspace is not None:
        ws_ptr, ws_bytes = ctypes.c_void_p(workspace.data_ptr()), workspace.numel() * workspace.element_size()
    check(lib().bbk_solve_refined_device(n, ctypes.c_void_p(a.data_ptr()), a.stride(0),
                                         ctypes.c_void_p(f.data_ptr()), f.stride(0),
                                         ctypes.c_void_p(perm.data_ptr()), ctypes.c_void_p(pivot_types.data_ptr()),
                                         bb.shape[0], ctypes.c_void_p(bb.data_ptr()), bb.stride(0),
                                         ctypes.c_void_p(x.data_ptr()), x.stride(0), tol, max_iter, meth,
                                         restart, ctypes.byref(info), ws_ptr, ws_bytes, _stream_ptr(stream)))
    return (x if b.dim() == 2 else x.reshape(n)), info


def sampled_residual_device(a, f, perm, pivot_types, rows, cols, stream=None) -> float:
    """The reference stress test's sampled relative residual of the compact
    factors ``f`` against the original ``a`` (CUDA float64, upper triangles),
    at the sampled entries (rows[k], cols[k]) (CUDA int32 tensors)."""
    n = f.shape[0]
    out = ctypes.c_double(0.0)
    check(lib().bbk_sampled_residual_device(n, ctypes.c_void_p(a.data_ptr()), a.stride(0),
                                            ctypes.c_void_p(f.data_ptr()), f.stride(0),
                                            ctypes.c_void_p(perm.data_ptr()),
                                            ctypes.c_void_p(pivot_types.data_ptr()), rows.numel(),
                                            ctypes.c_void_p(rows.data_ptr()), ctypes.c_void_p(cols.data_ptr()),
                                            ctypes.byref(out), _stream_ptr(stream)))
    return out.value


def extract_ld_device(f, pivot_types, stream=None):
    """Dense (L, D) of the compact factors ``f`` (CUDA float64, n x ldf) on
    the device: the reference's LFactor() / DFactor()."""
    import torch
    n = f.shape[0]
    l = torch.empty(n, n, dtype=torch.float64, device=f.device)
    d = torch.empty(n, n, dtype=torch.float64, device=f.device)
    check(lib().bbk_extract_ld_device(n, ctypes.c_void_p(f.data_ptr()), f.stride(0),
                                      ctypes.c_void_p(pivot_types.data_ptr()), ctypes.c_void_p(l.data_ptr()), n,
                                      ctypes.c_void_p(d.data_ptr()), n, _stream_ptr(stream)))
    return l, d


def reconstruct_device(f, perm, pivot_types, stream=None):
    import torch
    n = f.shape[0]
    out = torch.empty((n, n), dtype=torch.float64, device=f.device)
    check(lib().bbk_reconstruct_device(n, ctypes.c_void_p(f.data_ptr()), f.stride(0),
                                       ctypes.c_void_p(perm.data_ptr()),
                                       ctypes.c_void_p(pivot_types.data_ptr()),
                                       ctypes.c_void_p(out.data_ptr()), n, _stream_ptr(stream)))
    return out


def probe_bounded_wait(ctas: int, timeout_ns: int, stream=None) -> int:
    """Run the bounded-wait probe; returns the bbk_status (BBK_ERR_TIMEOUT
    when the device-side wait bound works)."""
    return int(lib().bbk_probe_bounded_wait(ctas, timeout_ns, _stream_ptr(stream)))


def probe_exchange_ns(ctas: int, iters: int = 2000, stream=None) -> float:
    """Mean device nanoseconds of one grid exchange on `ctas` blocks."""
    out = ctypes.c_double(0.0)
    check(lib().bbk_probe_exchange_ns(ctas, iters, ctypes.byref(out), _stream_ptr(stream)))
    return out.value


# ---------------------------------------------------------------------------
# Host (numpy) entry points
# ---------------------------------------------------------------------------
@dataclass
class HostFactors:
    factors: np.ndarray
    perm: np.ndarray
    pivot_types: np.ndarray
    panel_end: np.ndarray


def factor_host(a: np.ndarray, block_size: int, mode="fp64") -> HostFactors:
    """Factor on the GPU from host memory; ``a`` is not modified."""
    f = np.array(a, dtype=np.float64, order="C", copy=True)
    n = f.shape[0]
    nb = (n + block_size - 1) // block_size if block_size > 0 else 1
    perm = np.zeros(n, np.int32)
    pt = np.zeros(n, np.int32)
    pe = np.zeros(max(nb, 1), np.int32)
    check(lib().bbk_factor_host(n, block_size, _np_ptr(f), f.shape[1], _np_ptr(perm), _np_ptr(pt),
                                _np_ptr(pe), _mode(mode)))
    return HostFactors(f, perm, pt, pe)


def factor_solve_host(a: np.ndarray, block_size: int, b: np.ndarray, mode="fp64"):
    """One call: factor ``a`` and solve for the columns of ``b`` (n or n x nrhs)."""
    f = np.array(a, dtype=np.float64, order="C", copy=True)
    n = f.shape[0]
    bb = np.array(b, dtype=np.float64, copy=True)
    one = bb.ndim == 1
    bt = np.ascontiguousarray(bb.reshape(n, -1).T)  # (nrhs, n): each row one rhs
    nb = (n + block_size - 1) // block_size if block_size > 0 else 1
    perm = np.zeros(n, np.int32)
    pt = np.zeros(n, np.int32)
    pe = np.zeros(max(nb, 1), np.int32)
    check(lib().bbk_factor_solve_host(n, block_size, _np_ptr(f), f.shape[1], _np_ptr(perm),
                                      _np_ptr(pt), _np_ptr(pe), bt.shape[0], _np_ptr(bt), n,
                                      _mode(mode)))
    x = bt.T.copy()
    return HostFactors(f, perm, pt, pe), (x[:, 0] if one else x)


def solve_host(fac: HostFactors, b: np.ndarray) -> np.ndarray:
    n = fac.factors.shape[0]
    bb = np.array(b, dtype=np.float64, copy=True)
    one = bb.ndim == 1
    bt = np.ascontiguousarray(bb.reshape(n, -1).T)
    ff = np.ascontiguousarray(fac.factors)
    check(lib().bbk_solve_host(n, _np_ptr(ff), ff.shape[1], _np_ptr(fac.perm),
                               _np_ptr(fac.pivot_types), bt.shape[0], _np_ptr(bt), n))
    x = bt.T.copy()
    return x[:, 0] if one else x


# ---------------------------------------------------------------------------
# Mirror of the reference's BlockLdltDecomposition
# ---------------------------------------------------------------------------
class BlockLdltDecomposition:
    """Python mirror of naive_block_ldlt::BlockLdltDecomposition.

    ``matrix`` is a dense symmetric matrix (only the upper triangle is read,
    like BlockMatrix(RegularMatrix, block_size, MatrixTriangle::kUpper)) and
    ``block_size`` the BlockMatrix block size.  ``full=True`` is kFull mode
    (L/D factors and reconstruct_original available), ``full=False`` is
    kCompactOnly.  The factorization runs on the GPU; nothing runs on the CPU.
    """

    def __init__(self, matrix: np.ndarray, block_size: int, full: bool = True,
                 mode="fp64", lower: bool = False):
        m = np.asarray(matrix, dtype=np.float64)
        if m.ndim != 2 or m.shape[0] != m.shape[1]:
            raise InvalidArgument(BBK_ERR_INVALID_ARGUMENT, "block matrix input must be square")
        if m.shape[0] <= 0:
            raise InvalidArgument(BBK_ERR_INVALID_ARGUMENT, "matrix size must be positive")
        if block_size <= 0:
            raise InvalidArgument(BBK_ERR_INVALID_ARGUMENT, "block size must be positive")
        self._input = np.ascontiguousarray(m.T if lower else m)
        self.block_size = block_size
        self.full = full
        self.mode = mode
        self._fac: HostFactors | None = None

    def factorize(self) -> None:
        self._fac = factor_host(self._input, self.block_size, self.mode)

    def _need(self) -> HostFactors:
        if self._fac is None:
            raise LogicError(BBK_ERR_LOGIC, "Factorize() must be called first")
        return self._fac

    def compact_factors(self) -> np.ndarray:
        """Upper triangle of the compact factor (lower triangle zero)."""
        return np.triu(self._need().factors)

    def permutation(self) -> np.ndarray:
        return self._need().perm

    def pivot_types(self) -> np.ndarray:
        return self._need().pivot_types

    def panel_end(self) -> np.ndarray:
        return self._need().panel_end

    def reconstruct_original(self) -> np.ndarray:
        if not self.full:
            raise LogicError(BBK_ERR_LOGIC, "ReconstructOriginal() requires full factor storage")
        fac = self._need()
        import torch
        dev = torch.device("cuda")
        f = torch.from_numpy(np.ascontiguousarray(fac.factors)).to(dev)
        perm = torch.from_numpy(fac.perm).to(dev)
        pt = torch.from_numpy(fac.pivot_types).to(dev)
        return reconstruct_device(f, perm, pt).cpu().numpy()

    def solve(self, b: np.ndarray) -> np.ndarray:
        return solve_host(self._need(), b)


# ---------------------------------------------------------------------------
# Batched factor + solve
# ---------------------------------------------------------------------------
class BatchedPlan:
    """A planned batch: packed layout of `sizes` (matrix k is n_k x n_k at
    element offset a_offsets[k], its right-hand side at rhs_offsets[k], its
    perm / pivot types at piv_offsets[k]), the block size chosen per item
    and the device workspace holding the schedule."""

    def __init__(self, sizes, block_sizes=None, device=None, stream=None):
        import torch
        sizes = [int(n) for n in sizes]
        if not sizes:
            raise InvalidArgument(BBK_ERR_INVALID_ARGUMENT, "empty batch")
        self.sizes = np.asarray(sizes, dtype=np.int64)
        self.count = len(sizes)
        self.a_offsets = np.concatenate([[0], np.cumsum(self.sizes * self.sizes)[:-1]]).astype(np.int64)
        self.rhs_offsets = np.concatenate([[0], np.cumsum(self.sizes)[:-1]]).astype(np.int64)
        self.piv_offsets = self.rhs_offsets.copy()
        self.a_elements = int((self.sizes * self.sizes).sum())
        self.vec_elements = int(self.sizes.sum())
        items = (BatchItem * self.count)()
        for k, n in enumerate(sizes):
            items[k].n = n
            items[k].lda = n
            items[k].a = int(self.a_offsets[k])
            items[k].rhs = int(self.rhs_offsets[k])
            items[k].piv = int(self.piv_offsets[k])
        self.device = device if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.bytes = lib().bbk_batched_workspace_size(self.count, max(sizes))
        if self.bytes == 0:
            raise InvalidArgument(BBK_ERR_INVALID_ARGUMENT, "batched sizes outside 1..%d" % BATCH_MAX_N)
        self.workspace = torch.empty(self.bytes, dtype=torch.uint8, device=self.device)
        chosen = np.zeros(self.count, dtype=np.int32)
        table = None
        if block_sizes is not None:
            bs = np.zeros(BATCH_BUCKETS, dtype=np.int32)
            bs[:len(block_sizes)] = np.asarray(block_sizes, dtype=np.int32)
            table = bs
        check(lib().bbk_batched_plan(self.count, ctypes.cast(items, ctypes.c_void_p),
                                     _np_ptr(table) if table is not None else None, _np_ptr(chosen),
                                     ctypes.c_void_p(self.workspace.data_ptr()), self.bytes, _stream_ptr(stream)))
        self.block_sizes = chosen

    def pack(self, mats, vecs=None):
        """Host lists of square matrices / vectors -> packed CUDA tensors."""
        import torch
        a = np.empty(self.a_elements)
        for k, m in enumerate(mats):
            o = int(self.a_offsets[k])
            a[o:o + m.size] = np.ascontiguousarray(m, dtype=np.float64).ravel()
        out = [torch.from_numpy(a).to(self.device)]
        if vecs is not None:
            x = np.empty(self.vec_elements)
            for k, v in enumerate(vecs):
                o = int(self.rhs_offsets[k])
                x[o:o + v.size] = np.asarray(v, dtype=np.float64).ravel()
            out.append(torch.from_numpy(x).to(self.device))
        return out

    def matrix(self, a, k):
        n = int(self.sizes[k])
        o = int(self.a_offsets[k])
        return a[o:o + n * n].reshape(n, n)

    def vector(self, x, k):
        o = int(self.rhs_offsets[k])
        return x[o:o + int(self.sizes[k])]


def batched_factor_solve(plan: BatchedPlan, a, x, mode="fp64", a_orig=None, tol: float = 1e-12,
                         max_iter: int = 0, stream=None, sync: bool = True):
    """Factor every matrix of the packed CUDA float64 tensor ``a`` in place and
    solve into ``x`` (overwritten).  Returns (perm, pivot_types, info) device
    tensors; info is a structured numpy array when ``sync``."""
    import torch
    perm = torch.empty(plan.vec_elements, dtype=torch.int32, device=plan.device)
    pt = torch.empty(plan.vec_elements, dtype=torch.int32, device=plan.device)
    info = torch.zeros(plan.count * ctypes.sizeof(BatchInfo), dtype=torch.uint8, device=plan.device)
    check(lib().bbk_batched_factor_solve(
        plan.count, ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(a_orig.data_ptr()) if a_orig is not None else None,
        ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(perm.data_ptr()), ctypes.c_void_p(pt.data_ptr()),
        _mode(mode), float(tol), int(max_iter), ctypes.c_void_p(info.data_ptr()),
        ctypes.c_void_p(plan.workspace.data_ptr()), plan.bytes, _stream_ptr(stream)))
    if not sync:
        return perm, pt, info
    torch.cuda.synchronize(plan.device)
    raw = info.cpu().numpy().tobytes()
    rec = np.frombuffer(raw, dtype=np.dtype([("iterations", "<i4"), ("converged", "<i4"),
                                             ("backward_error", "<f8")]))
    return perm, pt, rec
