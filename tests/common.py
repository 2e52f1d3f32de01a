"""Shared helpers for the tests (inputs and fixtures, no product code)."""
import hashlib
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# tests/block_ldlt_decomposition_test.cc:421-450 of the reference: the golden
# 4x4 input, its expected compact upper factor and pivot types.
GOLDEN_4x4 = np.array([[6.0, 12.0, 3.0, -6.0], [12.0, -8.0, -13.0, 4.0],
                       [3.0, -13.0, -1.0, 1.0], [-6.0, 4.0, 1.0, 6.0]])
GOLDEN_4x4_COMPACT = np.array([[6.0, 12.0, -0.6875, 0.0],
                               [0.0, -8.0, 0.59375, -0.5],
                               [0.0, 0.0, 8.78125, -0.6263345195729537],
                               [0.0, 0.0, 0.0, 4.555160142348754]])
GOLDEN_4x4_PIVOTS = [2, -2, 1, 1]
# tests/block_ldlt_decomposition_test.cc:476-499: the fixed matrices
FIXED = [GOLDEN_4x4,
         np.array([[0, 1, 0, 0], [1, 0, 0, 0], [0, 0, 0, 1], [0, 0, 1, 0]], float),
         np.diag([2.0, -3.0, 0.0, 5.0])]
TOLERANCE = 1e-10  # tests/block_ldlt_decomposition_test.cc:31


def uniform_symmetric(n: int, seed: int) -> np.ndarray:
    """Entries i.i.d. uniform[-1, 1] from numpy PCG64, upper triangle mirrored."""
    rng = np.random.default_rng(seed)
    u = rng.uniform(-1.0, 1.0, size=(n, n))
    return np.triu(u) + np.triu(u, 1).T


def relative_error(actual, expected) -> float:
    """||actual - expected||_F / max(||expected||_F, 1), the reference's metric."""
    return float(np.linalg.norm(actual - expected) / max(np.linalg.norm(expected), 1.0))


def upper_hash(f: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(np.triu(f)).tobytes()).hexdigest()


def load_small_cases():
    z = np.load(os.path.join(GOLDEN, "ref_cases.npz"))
    out = []
    for name in z["names"]:
        name = str(name)
        out.append(dict(name=name, a=z[f"{name}__a"], f=z[f"{name}__f"], perm=z[f"{name}__perm"],
                        pt=z[f"{name}__pt"], ends=z[f"{name}__ends"], b=int(z[f"{name}__b"][0])))
    return out


def load_large_cases():
    with open(os.path.join(GOLDEN, "ref_large.json")) as fh:
        return json.load(fh)


def reconstruct(f: np.ndarray, perm: np.ndarray, pt: np.ndarray) -> np.ndarray:
    """P^T L D L^T P in numpy from compact factors (test-side checker)."""
    n = f.shape[0]
    L = np.eye(n)
    D = np.zeros((n, n))
    for k in range(n):
        D[k, k] = f[k, k]
        for i in range(k + 1, n):
            if pt[k] == 2 and i == k + 1:
                D[k, k + 1] = D[k + 1, k] = f[k, k + 1]
            else:
                L[i, k] = f[k, i]
    m = L @ D @ L.T
    out = np.zeros_like(m)
    out[np.ix_(perm, perm)] = m
    return out


def kkt_matrix(n: int, h: int, seed: int, ridge: float = 1e-2) -> np.ndarray:
    """Saddle-point [[H, B^T], [B, 0]]: H = G G^T / h + ridge I (G Gaussian
    h x h), B Gaussian (n-h) x h, zero (2,2) block."""
    rng = np.random.default_rng(seed)
    g = rng.standard_normal((h, h))
    hm = g @ g.T / h + ridge * np.eye(h)
    bm = rng.standard_normal((n - h, h))
    a = np.zeros((n, n))
    a[:h, :h] = hm
    a[h:, :h] = bm
    a[:h, h:] = bm.T
    return a


def kkt_matrix_exact(n: int, h: int, seed: int, ridge: float = 1e-2):
    """The saddle-point structure of kkt_matrix with an input that every
    machine computes bit for bit: G's Gaussian entries are rounded to
    multiples of 2^-10, so every product and partial sum of G G^T is an
    integer multiple of 2^-20 below 2^39 in magnitude, exact in FP64 whatever
    the BLAS's summation order, blocking or FMA use; the division by h and
    the ridge are single IEEE roundings.  Returns (matrix, SHA-256 of its
    bytes)."""
    rng = np.random.default_rng(seed)
    g = np.round(rng.standard_normal((h, h)) * 1024.0) / 1024.0
    hm = g @ g.T
    del g
    hm /= h
    hm[np.diag_indices(h)] += ridge
    bm = rng.standard_normal((n - h, h))
    a = np.zeros((n, n))
    a[:h, :h] = hm
    del hm
    a[h:, :h] = bm
    a[:h, h:] = bm.T
    return a, hashlib.sha256(a.tobytes()).hexdigest()


def relative_residual(a: np.ndarray, f: np.ndarray, perm: np.ndarray, pt: np.ndarray) -> float:
    """||A - P^T L D L^T P||_F / ||A||_F from compact factors, vectorised
    (L(i,k) = F(k,i) below the diagonal except inside a 2x2 pivot, D from
    the diagonal and the (k,k+1) entries of 2x2 pivots)."""
    n = f.shape[0]
    two = np.where(np.asarray(pt) == 2)[0]
    lt = np.triu(f, 1)
    lt[two, two + 1] = 0.0
    lt = lt.T.copy()
    lt[np.diag_indices(n)] = 1.0
    ld = lt * np.diag(f)[None, :]
    ld[:, two] += lt[:, two + 1] * f[two, two + 1][None, :]
    ld[:, two + 1] += lt[:, two] * f[two, two + 1][None, :]
    m = ld @ lt.T
    del ld, lt
    rec = np.empty_like(m)
    rec[np.ix_(perm, perm)] = m
    del m
    return float(np.linalg.norm(a - rec) / np.linalg.norm(a))


ALPHA = 0.6403882032022076  # src/block_ldlt_decomposition.cc:14


def reference_margins(log: np.ndarray) -> np.ndarray:
    """Relative margins of the comparisons each pivot step of the reference
    made, from the C restatement's decision log (oracle bko_factor_logged:
    |W(p,p)|, omega, runner-up of the row argmax, sigma, |W(r,r)| per
    position): the smallest |lhs - rhs| / max(|lhs|, |rhs|) over
    |W(p,p)| >= alpha omega (:90-92), omega against its runner-up (the row
    argmax, :164-182) and, after a candidate, the two SelectPivot tests
    (:369-390).  NaN where no step started."""
    d, om, second, sg, arr = (np.asarray(log[:, k], np.float64) for k in range(5))

    def rel(x, y):
        den = np.maximum(np.abs(x), np.abs(y))
        with np.errstate(invalid="ignore", divide="ignore"):
            return np.where(den > 0, np.abs(x - y) / np.where(den > 0, den, 1.0), np.inf)
    with np.errstate(invalid="ignore"):
        m = np.where(om == 0.0, np.inf, rel(d, ALPHA * om))
        m = np.minimum(m, rel(om, second))
        cand = ~np.isnan(sg)
        m = np.where(cand, np.minimum(m, np.minimum(rel(d * sg, ALPHA * om * om), rel(arr, ALPHA * sg))), m)
    return np.where(np.isnan(d), np.nan, m)


def spectral_matrix(n: int, seed: int, lo: float = 1e-4, hi: float = 1e4) -> np.ndarray:
    """A = Q diag(lam) Q^T with Q from the QR of a Gaussian matrix, |lam|
    log-uniform in [lo, hi] and half of the signs negative (condition number
    about hi/lo): the structure of the mixed-precision workload."""
    rng = np.random.default_rng(seed)
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    mag = np.exp(rng.uniform(np.log(lo), np.log(hi), n))
    sign = np.ones(n)
    sign[rng.permutation(n)[: n // 2]] = -1.0
    a = (q * (sign * mag)) @ q.T
    return (a + a.T) / 2


def backward_error(a: np.ndarray, x: np.ndarray, b: np.ndarray) -> float:
    """max over columns of ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf)."""
    x = x.reshape(a.shape[0], -1)
    b = b.reshape(a.shape[0], -1)
    r = b - a @ x
    an = np.abs(a).sum(1).max()
    return float(np.max(np.abs(r).max(0) / (an * np.abs(x).max(0) + np.abs(b).max(0))))
