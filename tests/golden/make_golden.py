"""Regenerate the golden fixtures in this folder from the reference itself.

Runs in the build container only (it needs oracle/_ref/libbbk_ref.so, compiled
from the reference's own sources by oracle/Makefile).  Each case stores the
reference's outputs for an input that the tests can regenerate exactly:

* ``ref_cases.npz``: small cases (the reference tests' libstdc++ generator,
  the golden 4x4, the fixed matrices): full compact upper factor, perm, pivot
  types, panel ends;
* ``ref_large.json``: larger cases (seeded uniform[-1,1] inputs from numpy's
  PCG64): perm and pivot types in full, plus a SHA-256 of the compact upper
  factor's bytes so a bitwise match can be checked without storing it.
* ``ref_geometry.txt``: cases with several boundary shifts (the reference
  tests' generator, so C++ can regenerate the input): the reference's block
  geometry after factorization (row0, rows, col0, cols per block id), its
  permutation, pivot types, compact upper factor and the upper triangle of
  its Workspace() (%.17g), read by tests/cpp/test_cpp_surface.cc.

* ``ref_kkt10000.npz`` (``--kkt``, a few minutes): the saddle-point
  workload at full size (n=10000, H 8000, block 128) from
  tests/common.py's kkt_matrix_exact, whose input every machine computes bit
  for bit (its SHA-256 is stored and checked).  The reference's permutation,
  pivot types, panel ends, a SHA-256 of its compact upper factor and its
  relative reconstruction residual; the C restatement's per-step decision
  log (oracle/bk_oracle.h, bko_factor_logged; float32) and the relative
  margin of every decision computed from it in float64
  (tests/common.py reference_margins), after checking that the restatement
  reproduces the reference bit for bit on this input.

Usage: python tests/golden/make_golden.py [--kkt]
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle.oracle import Port, Reference  # noqa: E402

GOLDEN_4x4 = [[6.0, 12.0, 3.0, -6.0], [12.0, -8.0, -13.0, 4.0],
              [3.0, -13.0, -1.0, 1.0], [-6.0, 4.0, 1.0, 6.0]]
FIXED = [GOLDEN_4x4,
         [[0, 1, 0, 0], [1, 0, 0, 0], [0, 0, 0, 1], [0, 0, 1, 0]],
         [[2, 0, 0, 0], [0, -3, 0, 0], [0, 0, 0, 0], [0, 0, 0, 5]]]


def uniform_symmetric(n: int, seed: int) -> np.ndarray:
    """Entries i.i.d. uniform[-1, 1], upper triangle read and mirrored."""
    rng = np.random.default_rng(seed)
    u = rng.uniform(-1.0, 1.0, size=(n, n))
    return np.triu(u) + np.triu(u, 1).T


def upper_hash(f: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(np.triu(f)).tobytes()).hexdigest()


def small_cases(port: Port):
    cases = []
    for ci, m in enumerate(FIXED):
        for b in range(1, 5):
            cases.append((f"fixed{ci}_b{b}", np.array(m, float), b))
    for n in (5, 8, 13, 16):
        for b in sorted({1, 2, 3, n // 2, n}):
            seed = 10000 * n + 100 * b
            cases.append((f"rand_n{n}_b{b}", port.random_symmetric(n, seed), b))
    for n, b, scale in ((33, 8, 1e-6), (33, 5, 1e6), (64, 16, 1.0), (64, 21, 1e-12)):
        seed = 910000 + 10000 * n + 100 * b
        cases.append((f"stress_n{n}_b{b}_s{scale:g}", port.random_symmetric(n, seed, scale), b))
    for n, b in ((40, 7), (48, 16)):
        cases.append((f"uniform_n{n}_b{b}", uniform_symmetric(n, 1000 + n), b))
    return cases


KKT_CASE = {"n": 10000, "h": 8000, "block_size": 128, "seed": 20240}


def kkt_parity_fixture():
    sys.path.insert(0, os.path.dirname(HERE))
    from common import kkt_matrix_exact, reference_margins, relative_residual
    port, ref = Port(), Reference()
    n, h, b, seed = (KKT_CASE[k] for k in ("n", "h", "block_size", "seed"))
    a, a_sha = kkt_matrix_exact(n, h, seed)
    r = ref.factor(a, b)
    f, log = port.factor_logged(a, b)
    assert upper_hash(f.factors) == upper_hash(r.factors), "restatement differs from the reference"
    assert np.array_equal(f.perm, r.perm) and np.array_equal(f.pivot_types, r.pivot_types)
    nbk = (n + b - 1) // b
    ends = np.array([g[0] + g[1] for g in (r.geometry[bc + bc * (bc + 1) // 2] for bc in range(nbk))],
                    np.int32)
    assert np.array_equal(ends, f.panel_end)
    res = relative_residual(a, r.factors, r.perm, r.pivot_types)
    np.savez_compressed(os.path.join(HERE, "ref_kkt10000.npz"),
                        n=n, h=h, block_size=b, seed=seed, input_sha256=a_sha,
                        perm=r.perm, pivot_types=r.pivot_types.astype(np.int8), panel_end=ends,
                        upper_sha256=upper_hash(r.factors), residual=res,
                        reference_seconds=r.seconds, log=log.astype(np.float32),
                        margin=reference_margins(log))
    print(f"kkt n={n}: reference {r.seconds:.1f} s, residual {res:.3e}, "
          f"{int((r.pivot_types == 1).sum())} 1x1 + {int((r.pivot_types == 2).sum())} 2x2 pivots")


def main():
    if "--kkt" in sys.argv:
        kkt_parity_fixture()
        return
    port, ref = Port(), Reference()
    out = {}
    names = []
    for name, a, b in small_cases(port):
        r = ref.factor(a, b)
        n = a.shape[0]
        ends = np.array([g[0] + g[1] for g in
                         (r.geometry[bc + bc * (bc + 1) // 2] for bc in range((n + b - 1) // b))],
                        np.int32)
        out[f"{name}__a"] = a
        out[f"{name}__f"] = np.triu(r.factors)
        out[f"{name}__perm"] = r.perm
        out[f"{name}__pt"] = r.pivot_types
        out[f"{name}__ends"] = ends
        out[f"{name}__b"] = np.array([b], np.int32)
        names.append(name)
    out["names"] = np.array(names)
    np.savez_compressed(os.path.join(HERE, "ref_cases.npz"), **out)

    large = []
    for n, b, seed in ((500, 64, 500), (2000, 64, 12345)):
        a = uniform_symmetric(n, seed)
        r = ref.factor(a, b)
        nbk = (n + b - 1) // b
        ends = [int(g[0] + g[1]) for g in (r.geometry[bc + bc * (bc + 1) // 2] for bc in range(nbk))]
        large.append({"n": n, "block_size": b, "seed": seed, "generator": "numpy-pcg64-uniform[-1,1]",
                      "perm": r.perm.tolist(), "pivot_types": r.pivot_types.tolist(),
                      "panel_end": ends, "upper_sha256": upper_hash(r.factors),
                      "upper_sum": float(np.triu(r.factors).sum())})
    with open(os.path.join(HERE, "ref_large.json"), "w") as fh:
        json.dump(large, fh)

    geo_cases = [(40, 7, 777000 + 100 * 40 + 10 * 7 + 1), (60, 4, 777000 + 100 * 60 + 10 * 4)]
    with open(os.path.join(HERE, "ref_geometry.txt"), "w") as fh:
        fh.write(f"{len(geo_cases)}\n")
        for n, b, seed in geo_cases:
            a = port.random_symmetric(n, seed)
            r = ref.factor(a, b)
            nbk = (n + b - 1) // b
            fh.write(f"{n} {b} {seed} {nbk * (nbk + 1) // 2}\n")
            for g in r.geometry:
                fh.write(" ".join(str(int(x)) for x in g) + "\n")
            fh.write(" ".join(str(int(x)) for x in r.perm) + "\n")
            fh.write(" ".join(str(int(x)) for x in r.pivot_types) + "\n")
            up = np.triu(r.factors)
            for i in range(n):
                fh.write(" ".join(f"{x:.17g}" for x in up[i]) + "\n")
            ws = ref.workspace(a, b)
            for i in range(n):
                fh.write(" ".join(f"{x:.17g}" for x in ws[i]) + "\n")
    print(f"wrote {len(names)} small cases, {len(large)} large cases, {len(geo_cases)} geometry cases")


if __name__ == "__main__":
    main()
