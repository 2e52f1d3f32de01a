"""TEST INFRASTRUCTURE ONLY -- Python access to the CPU oracle.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU baseline
use this module, and only as the checker / the timed CPU baseline.  The product
(``blockedbunchkaufmanldlt_b200``) never imports it.

Two oracles live here:

* ``Port``: ``libbk_oracle.so``, the plain-C restatement of the reference's
  blocked Bunch-Kaufman algorithm (``bk_oracle.c``) plus the reference tests'
  libstdc++ input generators (``testgen.cc``).
* ``Reference``: ``_ref/libbbk_ref.so``, the reference library itself
  (its ``src/*.cc`` compiled by ``Makefile``) behind a small C shim.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "libbk_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libbbk_ref.so")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def build() -> None:
    """Compile the oracle (and the reference, where its sources exist)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _ptr(arr, kind=_dp):
    return arr.ctypes.data_as(kind) if arr is not None else None


@dataclass
class Factorization:
    factors: np.ndarray      # n x n row-major; upper triangle meaningful
    perm: np.ndarray         # int32[n]
    pivot_types: np.ndarray  # int32[n]
    panel_end: np.ndarray | None = None
    shifted: np.ndarray | None = None
    geometry: np.ndarray | None = None
    seconds: float | None = None

    def upper(self) -> np.ndarray:
        return np.triu(self.factors)


class Port:
    """The C restatement of the reference algorithm."""

    def __init__(self, path: str = PORT_SO):
        if not os.path.exists(path):
            build()
        lib = ctypes.CDLL(path)
        lib.bko_factor.argtypes = [ctypes.c_int, ctypes.c_int, _dp, ctypes.c_longlong,
                                   _ip, _ip, _ip, _ip]
        lib.bko_factor.restype = ctypes.c_int
        lib.bko_factor_panels.argtypes = [ctypes.c_int, ctypes.c_int, _dp,
                                          ctypes.c_longlong, _ip, _ip, _ip, _ip,
                                          ctypes.c_int]
        lib.bko_factor_panels.restype = ctypes.c_int
        lib.bko_factor_logged.argtypes = [ctypes.c_int, ctypes.c_int, _dp, ctypes.c_longlong,
                                          _ip, _ip, _ip, _ip, _dp, _dp]
        lib.bko_factor_logged.restype = ctypes.c_int
        lib.bko_sampled_residual.argtypes = [ctypes.c_int, _dp, ctypes.c_longlong, _dp, ctypes.c_longlong,
                                             _ip, _ip, ctypes.c_int, _ip, _ip]
        lib.bko_sampled_residual.restype = ctypes.c_double
        lib.bko_solve.argtypes = [ctypes.c_int, _dp, ctypes.c_longlong, _ip, _ip,
                                  ctypes.c_int, _dp, ctypes.c_longlong]
        lib.bko_reconstruct.argtypes = [ctypes.c_int, _dp, ctypes.c_longlong, _ip, _ip, _dp]
        lib.bko_ref_random_symmetric.argtypes = [ctypes.c_int, ctypes.c_int,
                                                 ctypes.c_double, _dp]
        lib.bko_ref_random_block_fill.argtypes = [ctypes.c_int, ctypes.c_int,
                                                  ctypes.c_int, ctypes.c_double, _dp]
        lib.bko_ref_residual_samples.argtypes = [ctypes.c_int, ctypes.c_int,
                                                 ctypes.c_int, _ip, _ip]
        lib.bko_scale_one_by_one.argtypes = [ctypes.c_int, ctypes.c_double, _dp,
                                             ctypes.c_int, _dp, ctypes.c_int]
        lib.bko_scale_two_by_two.argtypes = [ctypes.c_int, ctypes.c_double,
                                             ctypes.c_double, ctypes.c_double,
                                             _dp, ctypes.c_int, _dp, ctypes.c_int,
                                             _dp, ctypes.c_int, _dp, ctypes.c_int]
        lib.bko_update_trailing_block.argtypes = [ctypes.c_int, ctypes.c_int,
                                                  ctypes.c_int, _dp, ctypes.c_int,
                                                  _dp, ctypes.c_int, _dp, ctypes.c_int]
        self.lib = lib

    def factor(self, a: np.ndarray, block_size: int, max_panels: int | None = None
               ) -> Factorization:
        n = a.shape[0]
        f = np.ascontiguousarray(a, dtype=np.float64).copy()
        perm = np.zeros(n, np.int32)
        pt = np.zeros(n, np.int32)
        nb = (n + block_size - 1) // block_size
        pe = np.zeros(nb, np.int32)
        sh = np.zeros(nb, np.int32)
        if max_panels is None:
            rc = self.lib.bko_factor(n, block_size, _ptr(f), n, _ptr(perm, _ip),
                                     _ptr(pt, _ip), _ptr(pe, _ip), _ptr(sh, _ip))
        else:
            rc = self.lib.bko_factor_panels(n, block_size, _ptr(f), n, _ptr(perm, _ip),
                                            _ptr(pt, _ip), _ptr(pe, _ip), _ptr(sh, _ip),
                                            max_panels)
            rc = 0 if rc >= 0 else rc
        if rc != 0:
            raise ValueError("oracle factorization rejected its arguments")
        return Factorization(f, perm, pt, pe, sh)

    LOG_WORDS = 5  # BKO_LOG_WORDS

    def factor_logged(self, a: np.ndarray, block_size: int, workspace_rows: bool = False):
        """factor() plus the decision log of bko_factor_logged: an n x 5
        array (|W(p,p)|, omega, runner-up of the row argmax, sigma, |W(r,r)|)
        at every position where a pivot step started, NaN elsewhere.  With
        workspace_rows, returns (factorization, log, W) where W (n x n, zero
        elsewhere) holds each panel's W rows at its trailing columns."""
        n = a.shape[0]
        f = np.ascontiguousarray(a, dtype=np.float64).copy()
        perm = np.zeros(n, np.int32)
        pt = np.zeros(n, np.int32)
        nb = (n + block_size - 1) // block_size
        pe = np.zeros(nb, np.int32)
        sh = np.zeros(nb, np.int32)
        log = np.zeros((n, self.LOG_WORDS))
        w = np.zeros((n, n)) if workspace_rows else None
        rc = self.lib.bko_factor_logged(n, block_size, _ptr(f), n, _ptr(perm, _ip), _ptr(pt, _ip),
                                        _ptr(pe, _ip), _ptr(sh, _ip), _ptr(log), _ptr(w))
        if rc != 0:
            raise ValueError("oracle factorization rejected its arguments")
        if workspace_rows:
            return Factorization(f, perm, pt, pe, sh), log, w
        return Factorization(f, perm, pt, pe, sh), log

    def solve(self, f: Factorization, b: np.ndarray) -> np.ndarray:
        n = f.factors.shape[0]
        bb = np.array(b, dtype=np.float64, order="F", copy=True)
        if bb.ndim == 1:
            bb = bb.reshape(n, 1, order="F")
        ff = np.ascontiguousarray(f.factors)
        self.lib.bko_solve(n, _ptr(ff), n, _ptr(f.perm, _ip), _ptr(f.pivot_types, _ip),
                           bb.shape[1], bb.ctypes.data_as(_dp), n)
        return bb if np.ndim(b) == 2 else bb[:, 0]

    def reconstruct(self, f: Factorization) -> np.ndarray:
        n = f.factors.shape[0]
        out = np.zeros((n, n))
        ff = np.ascontiguousarray(f.factors)
        self.lib.bko_reconstruct(n, _ptr(ff), n, _ptr(f.perm, _ip),
                                 _ptr(f.pivot_types, _ip), _ptr(out))
        return out

    # -- the reference tests' input generators ---------------------------
    def random_symmetric(self, n: int, seed: int, scale: float = 1.0) -> np.ndarray:
        out = np.zeros((n, n))
        self.lib.bko_ref_random_symmetric(n, seed, scale, _ptr(out))
        return out

    def random_block_fill(self, n: int, block_size: int, seed: int,
                          scale: float = 1.0) -> np.ndarray:
        out = np.zeros((n, n))
        self.lib.bko_ref_random_block_fill(n, block_size, seed, scale, _ptr(out))
        return out

    def sampled_residual(self, a: np.ndarray, f: Factorization, rows, cols) -> float:
        """The reference stress test's SampledRelativeResidual on compact factors."""
        n = a.shape[0]
        aa = np.ascontiguousarray(a, np.float64)
        ff = np.ascontiguousarray(f.factors, np.float64)
        r = np.ascontiguousarray(rows, np.int32)
        c = np.ascontiguousarray(cols, np.int32)
        return float(self.lib.bko_sampled_residual(n, _ptr(aa), n, _ptr(ff), n, _ptr(f.perm, _ip),
                                                   _ptr(f.pivot_types, _ip), len(r), _ptr(r, _ip),
                                                   _ptr(c, _ip)))

    def residual_samples(self, n: int, seed: int, count: int = 4096):
        rows = np.zeros(count, np.int32)
        cols = np.zeros(count, np.int32)
        self.lib.bko_ref_residual_samples(n, seed, count, _ptr(rows, _ip), _ptr(cols, _ip))
        return rows, cols

    # -- kernels.h restatements ------------------------------------------
    def scale_one_by_one(self, pivot, src):
        src = np.ascontiguousarray(src, np.float64)
        dst = np.zeros_like(src)
        self.lib.bko_scale_one_by_one(len(src), pivot, _ptr(src), 1, _ptr(dst), 1)
        return dst

    def scale_two_by_two(self, a, b, c, s1, s2):
        s1 = np.ascontiguousarray(s1, np.float64)
        s2 = np.ascontiguousarray(s2, np.float64)
        d1 = np.zeros_like(s1)
        d2 = np.zeros_like(s2)
        self.lib.bko_scale_two_by_two(len(s1), a, b, c, _ptr(s1), 1, _ptr(s2), 1,
                                      _ptr(d1), 1, _ptr(d2), 1)
        return d1, d2

    def update_trailing_block(self, left, ws, target):
        left = np.ascontiguousarray(left, np.float64)
        ws = np.ascontiguousarray(ws, np.float64)
        out = np.array(target, dtype=np.float64, copy=True)
        inner, rows = left.shape
        cols = ws.shape[1]
        self.lib.bko_update_trailing_block(rows, cols, inner, _ptr(left), rows,
                                           _ptr(ws), cols, _ptr(out), cols)
        return out


class Reference:
    """The reference library itself (oracle/_ref/libbbk_ref.so)."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        lib = ctypes.CDLL(path)
        lib.ref_factor.argtypes = [ctypes.c_int, ctypes.c_int, _dp, ctypes.c_longlong,
                                   _dp, ctypes.c_longlong, _ip, _ip, _ip, _dp]
        lib.ref_factor.restype = ctypes.c_int
        lib.ref_factor_workspace.argtypes = [ctypes.c_int, ctypes.c_int, _dp, ctypes.c_longlong, _dp,
                                             ctypes.c_longlong]
        lib.ref_factor_workspace.restype = ctypes.c_int
        lib.ref_factor_full.argtypes = [ctypes.c_int, ctypes.c_int, _dp,
                                        ctypes.c_longlong, _dp, _dp, _dp]
        lib.ref_factor_full.restype = ctypes.c_int
        lib.ref_openmp_threads.restype = ctypes.c_int
        lib.ref_scale_one_by_one.argtypes = [ctypes.c_int, ctypes.c_double, _dp,
                                             ctypes.c_int, _dp, ctypes.c_int]
        lib.ref_scale_two_by_two.argtypes = [ctypes.c_int, ctypes.c_double,
                                             ctypes.c_double, ctypes.c_double,
                                             _dp, ctypes.c_int, _dp, ctypes.c_int,
                                             _dp, ctypes.c_int, _dp, ctypes.c_int]
        lib.ref_update_trailing_block.argtypes = [ctypes.c_int, ctypes.c_int,
                                                  ctypes.c_int, _dp, ctypes.c_int,
                                                  _dp, ctypes.c_int, _dp, ctypes.c_int]
        self.lib = lib

    @staticmethod
    def available(path: str = REF_SO) -> bool:
        return os.path.exists(path)

    def threads(self) -> int:
        return self.lib.ref_openmp_threads()

    def factor(self, a: np.ndarray, block_size: int) -> Factorization:
        n = a.shape[0]
        src = np.ascontiguousarray(a, dtype=np.float64)
        out = np.zeros((n, n))
        perm = np.zeros(n, np.int32)
        pt = np.zeros(n, np.int32)
        nb = (n + block_size - 1) // block_size
        geo = np.zeros((nb * (nb + 1) // 2, 4), np.int32)
        secs = ctypes.c_double(0.0)
        rc = self.lib.ref_factor(n, block_size, _ptr(src), n, _ptr(out), n,
                                 _ptr(perm, _ip), _ptr(pt, _ip), _ptr(geo, _ip),
                                 ctypes.byref(secs))
        if rc != 0:
            raise RuntimeError("reference factorization threw")
        return Factorization(out, perm, pt, geometry=geo, seconds=secs.value)

    def workspace(self, a: np.ndarray, block_size: int) -> np.ndarray:
        """The reference's Workspace() after Factorize() (compact-only mode),
        as a dense upper triangle (n x n, zero below the diagonal)."""
        n = a.shape[0]
        src = np.ascontiguousarray(a, dtype=np.float64)
        out = np.zeros((n, n))
        if self.lib.ref_factor_workspace(n, block_size, _ptr(src), n, _ptr(out), n) != 0:
            raise RuntimeError("reference factorization threw")
        return out

    def factor_full(self, a: np.ndarray, block_size: int):
        n = a.shape[0]
        src = np.ascontiguousarray(a, dtype=np.float64)
        rec = np.zeros((n, n))
        lf = np.zeros((n, n))
        df = np.zeros((n, n))
        rc = self.lib.ref_factor_full(n, block_size, _ptr(src), n, _ptr(rec),
                                      _ptr(lf), _ptr(df))
        if rc != 0:
            raise RuntimeError("reference factorization threw")
        return rec, lf, df

    def scale_one_by_one(self, pivot, src):
        src = np.ascontiguousarray(src, np.float64)
        dst = np.zeros_like(src)
        self.lib.ref_scale_one_by_one(len(src), pivot, _ptr(src), 1, _ptr(dst), 1)
        return dst

    def scale_two_by_two(self, a, b, c, s1, s2):
        s1 = np.ascontiguousarray(s1, np.float64)
        s2 = np.ascontiguousarray(s2, np.float64)
        d1 = np.zeros_like(s1)
        d2 = np.zeros_like(s2)
        self.lib.ref_scale_two_by_two(len(s1), a, b, c, _ptr(s1), 1, _ptr(s2), 1,
                                      _ptr(d1), 1, _ptr(d2), 1)
        return d1, d2

    def update_trailing_block(self, left, ws, target):
        left = np.ascontiguousarray(left, np.float64)
        ws = np.ascontiguousarray(ws, np.float64)
        out = np.array(target, dtype=np.float64, copy=True)
        inner, rows = left.shape
        cols = ws.shape[1]
        self.lib.ref_update_trailing_block(rows, cols, inner, _ptr(left), rows,
                                           _ptr(ws), cols, _ptr(out), cols)
        return out


def relative_error(actual: np.ndarray, expected: np.ndarray) -> float:
    """The reference tests' metric (tests/block_ldlt_decomposition_test.cc:131-135):
    ||actual - expected||_F / max(||expected||_F, 1)."""
    return float(np.linalg.norm(actual - expected) / max(np.linalg.norm(expected), 1.0))
