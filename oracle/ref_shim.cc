// TEST INFRASTRUCTURE ONLY -- a C-ABI shim around the reference library
// itself, so tests and the CPU baseline can drive the unmodified reference
// from Python.  oracle/Makefile compiles this file together with the
// reference's own src/*.cc (read where they lie, never copied) into
// oracle/_ref/libbbk_ref.so.  Nothing in the product links it.
#include <chrono>
#include <cstring>
#include <exception>
#include <vector>

#include "block.h"
#include "block_ldlt_decomposition.h"
#include "block_matrix.h"
#include "kernels.h"
#include "regular_matrix.h"

#if defined(_OPENMP)
#include <omp.h>
#endif

using naive_block_ldlt::Block;
using naive_block_ldlt::BlockLdltDecomposition;
using naive_block_ldlt::BlockMatrix;
using naive_block_ldlt::RegularMatrix;

namespace {

// Block-wise fill of the upper triangle, the way
// tests/block_ldlt_large_stress_test.cc:116-136 builds large inputs (the
// RegularMatrix constructor's element accessor is O(#blocks) per entry).
BlockMatrix FillFromDense(int n, int b, const double* a, long long lda) {
  BlockMatrix m(n, b);
  for (int bc = 0; bc < m.num_blocks(); ++bc) {
    for (int br = 0; br <= bc; ++br) {
      Block& blk = m.GetBlock(br, bc);
      for (int r = 0; r < blk.rows(); ++r) {
        const int gi = blk.row0() + r;
        for (int c = 0; c < blk.cols(); ++c) {
          const int gj = blk.col0() + c;
          if (gi > gj) continue;
          blk(r, c) = a[static_cast<long long>(gi) * lda + gj];
        }
      }
    }
  }
  return m;
}

void ExtractUpper(const BlockMatrix& m, double* out, long long ldo) {
  const int n = m.Rows();
  for (int bc = 0; bc < m.num_blocks(); ++bc) {
    for (int br = 0; br <= bc; ++br) {
      const Block& blk = m.GetBlock(br, bc);
      for (int r = 0; r < blk.rows(); ++r) {
        const int gi = blk.row0() + r;
        for (int c = 0; c < blk.cols(); ++c) {
          const int gj = blk.col0() + c;
          if (gi < 0 || gj < 0 || gi >= n || gj >= n || gi > gj) continue;
          out[static_cast<long long>(gi) * ldo + gj] = blk(r, c);
        }
      }
    }
  }
}

}  // namespace

extern "C" {

// Factor the upper triangle of `a` (n x n row-major, lda) with the reference
// in compact-only mode.  Outputs the compact upper factor, permutation, pivot
// types and, per block id (br + bc(bc+1)/2), each block's geometry after
// factorization.  `seconds` receives the wall time of constructor +
// Factorize().  Returns 0 on success, 1 on a C++ exception.
int ref_factor(int n, int b, const double* a, long long lda, double* out,
               long long ldo, int* perm, int* pivot_types, int* geometry,
               double* seconds) {
  try {
    BlockMatrix input = FillFromDense(n, b, a, lda);
    const auto t0 = std::chrono::steady_clock::now();
    BlockLdltDecomposition dec(input,
                               BlockLdltDecomposition::FactorizationMode::kCompactOnly);
    dec.Factorize();
    const auto t1 = std::chrono::steady_clock::now();
    if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
    if (out) ExtractUpper(dec.CompactFactors(), out, ldo);
    for (int i = 0; i < n; ++i) {
      if (perm) perm[i] = dec.Permutation()[i];
      if (pivot_types) pivot_types[i] = dec.PivotTypes()[i];
    }
    if (geometry) {
      const BlockMatrix& f = dec.CompactFactors();
      for (int bc = 0; bc < f.num_blocks(); ++bc) {
        for (int br = 0; br <= bc; ++br) {
          const Block& blk = f.GetBlock(br, bc);
          int* g = geometry + 4 * f.BlockId(br, bc);
          g[0] = blk.row0();
          g[1] = blk.rows();
          g[2] = blk.col0();
          g[3] = blk.cols();
        }
      }
    }
    return 0;
  } catch (const std::exception&) {
    return 1;
  }
}

// Compact-only factorization; `out` (ldo) receives the upper triangle of
// Workspace() in its final geometry.
int ref_factor_workspace(int n, int b, const double* a, long long lda, double* out, long long ldo) {
  try {
    BlockMatrix input = FillFromDense(n, b, a, lda);
    BlockLdltDecomposition dec(input, BlockLdltDecomposition::FactorizationMode::kCompactOnly);
    dec.Factorize();
    ExtractUpper(dec.Workspace(), out, ldo);
    return 0;
  } catch (const std::exception&) {
    return 1;
  }
}

// Full mode: ReconstructOriginal() (n x n row-major) plus LFactor/DFactor.
int ref_factor_full(int n, int b, const double* a, long long lda,
                    double* reconstructed, double* l_out, double* d_out) {
  try {
    BlockMatrix input = FillFromDense(n, b, a, lda);
    BlockLdltDecomposition dec(input);
    dec.Factorize();
    const RegularMatrix rec = dec.ReconstructOriginal();
    for (int i = 0; i < n; ++i) {
      for (int j = 0; j < n; ++j) {
        const long long k = static_cast<long long>(i) * n + j;
        if (reconstructed) reconstructed[k] = rec(i, j);
        if (l_out) l_out[k] = dec.LFactor()(i, j);
        if (d_out) d_out[k] = dec.DFactor()(i, j);
      }
    }
    return 0;
  } catch (const std::exception&) {
    return 1;
  }
}

void ref_scale_one_by_one(int count, double pivot, const double* source,
                          int source_stride, double* destination,
                          int destination_stride) {
  naive_block_ldlt::kernels::ScaleOneByOnePivot(count, pivot, source, source_stride,
                                                destination, destination_stride);
}

void ref_scale_two_by_two(int count, double a, double b, double c,
                          const double* s1, int s1s, const double* s2, int s2s,
                          double* d1, int d1s, double* d2, int d2s) {
  naive_block_ldlt::kernels::ScaleTwoByTwoPivot(count, a, b, c, s1, s1s, s2, s2s,
                                                d1, d1s, d2, d2s);
}

void ref_update_trailing_block(int rows, int cols, int inner, const double* left,
                               int left_stride, const double* ws, int ws_stride,
                               double* target, int target_stride) {
  naive_block_ldlt::kernels::UpdateTrailingBlock(rows, cols, inner, left, left_stride,
                                                 ws, ws_stride, target, target_stride);
}

int ref_openmp_threads(void) {
#if defined(_OPENMP)
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
