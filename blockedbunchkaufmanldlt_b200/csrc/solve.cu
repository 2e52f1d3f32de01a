// Solve A X = B with compact Bunch-Kaufman factors, and the dense
// reconstruction P^T L D L^T P.
//
// The reference has no solve; L and D are read exactly as its stress test
// reads them (tests/block_ldlt_large_stress_test.cc:160-194 in
// wentianshu/BlockedBunchKaufmanLDLT): L(i,k) = F(k,i) for k < i, except
// L(k+1,k) = 0 when a 2x2 pivot starts at k; D(k,k) = F(k,k) and
// D(k,k+1) = F(k,k+1) for that 2x2.  With (P A P^T)(i,j) = A(perm[i], perm[j]):
//   y = B[perm]; L z = y; D w = z; L^T v = w; X[perm] = v.
// The triangular sweeps are memory-bound: one launch per 64-row block, each
// CTA solves the block's small triangle redundantly in a warp (one warp per
// right-hand side, values exchanged by shuffles) and then applies the block's
// contribution to its own rows, reading every factor entry once per sweep.
#include <algorithm>

#include "bbk_internal.cuh"

namespace bbk {
namespace {

constexpr int kSB = 64;           // solve block
constexpr int kSolveThreads = 256;
constexpr int kRowsPerCta = 256;  // forward: rows updated per CTA (one per thread)
constexpr int kRowsBack = 64;     // backward: rows updated per CTA (warp per row)
constexpr int kMaxRhsChunk = 8;   // right-hand sides per pass
constexpr int kKChunk = 16;       // coefficient loads kept in flight per thread

__global__ void gather_kernel(int n, int nrhs, const double* b, long long ldb, const int* perm,
                              double* y) {
  const long long total = static_cast<long long>(n) * nrhs;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int c = static_cast<int>(t / n), i = static_cast<int>(t % n);
    y[t] = b[c * ldb + perm[i]];
  }
}

__global__ void scatter_kernel(int n, int nrhs, double* b, long long ldb, const int* perm,
                               const double* y) {
  const long long total = static_cast<long long>(n) * nrhs;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int c = static_cast<int>(t / n), i = static_cast<int>(t % n);
    b[c * ldb + perm[i]] = y[t];
  }
}

// D w = z for all right-hand sides.
__global__ void dsolve_kernel(int n, int nrhs, const double* f, long long ldf, const int* pt,
                              double* y) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    if (pt[k] == -2) continue;  // handled with its partner
    if (pt[k] == 2 && k + 1 < n) {
      const double d11 = f[k * ldf + k], d21 = f[k * ldf + k + 1], d22 = f[(k + 1) * ldf + k + 1];
      const double det = d11 * d22 - d21 * d21;
      const double i11 = d22 / det, i22 = d11 / det, i21 = -d21 / det;
      for (int c = 0; c < nrhs; ++c) {
        double* yc = y + static_cast<long long>(c) * n;
        const double x = yc[k], z = yc[k + 1];
        yc[k] = i11 * x + i21 * z;
        yc[k + 1] = i21 * x + i22 * z;
      }
    } else {
      const double d = f[k * ldf + k];
      for (int c = 0; c < nrhs; ++c) {
        double* yc = y + static_cast<long long>(c) * n;
        yc[k] = d == 0.0 ? 0.0 : yc[k] / d;
      }
    }
  }
}

// One block [k0, k1) of the forward (kForward) or backward sweep.  The block's
// right-hand sides are final in `y` (every earlier block already subtracted
// its contribution); the solved block goes to `out` (written by CTA 0 only)
// so no CTA of the launch can read a half-solved block.
//   forward:  solve L_blk z_blk = y_blk, then y_i -= sum_k F(k,i) z_k for i >= k1
//   backward: solve L_blk^T v_blk = w_blk, then w_i -= sum_k F(i,k) v_k for i < k0
template <bool kForward>
__global__ void __launch_bounds__(kSolveThreads) sweep_kernel(int n, int nrhs, const double* f,
                                                             long long ldf, const int* pt,
                                                             double* y, double* out, int k0,
                                                             int k1) {
  __shared__ double fs[kSB][kSB + 1];      // fs[r][c] = F(k0 + r, k0 + c), r < c
  __shared__ double ys[kMaxRhsChunk][kSB];  // solved block values
  __shared__ int pts[kSB];
  const int bs = k1 - k0;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  {
    double v[kSB * kSB / kSolveThreads];
#pragma unroll
    for (int it = 0; it < kSB * kSB / kSolveThreads; ++it) {
      const int idx = t + it * kSolveThreads, r = idx / kSB, c = idx % kSB;
      v[it] = (r < c && c < bs) ? f[static_cast<long long>(k0 + r) * ldf + k0 + c] : 0.0;
    }
#pragma unroll
    for (int it = 0; it < kSB * kSB / kSolveThreads; ++it) {
      const int idx = t + it * kSolveThreads;
      fs[idx / kSB][idx % kSB] = v[it];
    }
  }
  for (int r = t; r < kSB; r += kSolveThreads) pts[r] = r < bs ? pt[k0 + r] : 1;
  // the 2x2 coupling can straddle the block edge: pivot k0-1 with k0
  const int pt_before = (k0 > 0) ? pt[k0 - 1] : 1;
  __syncthreads();

  for (int c0 = 0; c0 < nrhs; c0 += kMaxRhsChunk) {
    const int nc = min(kMaxRhsChunk, nrhs - c0);
    // ---- block triangle: one warp per right-hand side
    for (int cc = warp; cc < nc; cc += kSolveThreads / 32) {
      const double* yc = y + static_cast<long long>(c0 + cc) * n;
      double v0 = lane < bs ? yc[k0 + lane] : 0.0;
      double v1 = lane + 32 < bs ? yc[k0 + lane + 32] : 0.0;
      if (kForward) {
        for (int k = 0; k < bs; ++k) {
          const double yk = __shfl_sync(0xffffffffu, k < 32 ? v0 : v1, k & 31);
          const bool skip_next = pts[k] == 2;
          const int i0 = lane, i1 = lane + 32;
          if (i0 > k && i0 < bs && !(skip_next && i0 == k + 1)) v0 -= fs[k][i0] * yk;
          if (i1 > k && i1 < bs && !(skip_next && i1 == k + 1)) v1 -= fs[k][i1] * yk;
        }
      } else {
        for (int k = bs - 1; k >= 0; --k) {
          const double yk = __shfl_sync(0xffffffffu, k < 32 ? v0 : v1, k & 31);
          const int i0 = lane, i1 = lane + 32;
          // L(k, i) = F(i, k) for i < k, except i == k-1 opening a 2x2
          if (i0 < k && !(i0 == k - 1 && pts[i0] == 2)) v0 -= fs[i0][k] * yk;
          if (i1 < k && !(i1 == k - 1 && pts[i1] == 2)) v1 -= fs[i1][k] * yk;
        }
      }
      if (lane < bs) ys[cc][lane] = v0;
      if (lane + 32 < bs) ys[cc][lane + 32] = v1;
    }
    __syncthreads();
    if (blockIdx.x == 0) {
      for (int idx = t; idx < nc * bs; idx += kSolveThreads) {
        const int cc = idx / bs, r = idx % bs;
        out[static_cast<long long>(c0 + cc) * n + k0 + r] = ys[cc][r];
      }
    }
    // ---- contribution of the block to the other rows
    if (kForward) {
      const int i = k1 + blockIdx.x * kRowsPerCta + t;
      if (i < n) {
        double acc[kMaxRhsChunk];
#pragma unroll
        for (int cc = 0; cc < kMaxRhsChunk; ++cc) acc[cc] = 0.0;
        for (int kc = 0; kc < bs; kc += kKChunk) {
          double l[kKChunk];
#pragma unroll
          for (int kk = 0; kk < kKChunk; ++kk) {
            const int k = kc + kk;
            const bool ok = k < bs && !(i == k0 + k + 1 && pts[k] == 2);
            l[kk] = ok ? f[static_cast<long long>(k0 + k) * ldf + i] : 0.0;
          }
#pragma unroll
          for (int kk = 0; kk < kKChunk; ++kk)
#pragma unroll
            for (int cc = 0; cc < kMaxRhsChunk; ++cc)
              if (cc < nc && kc + kk < bs) acc[cc] += l[kk] * ys[cc][kc + kk];
        }
        for (int cc = 0; cc < nc; ++cc) y[static_cast<long long>(c0 + cc) * n + i] -= acc[cc];
      }
    } else {
      // rows i < k0, F(i, k0..k1) contiguous: one warp per row, four rows per
      // pass so every lane keeps eight loads in flight
      const int rows_lo = blockIdx.x * kRowsBack;
      const int rows_hi = min(k0, rows_lo + kRowsBack);
      constexpr int kR = 4;
      for (int i0 = rows_lo + warp * kR; i0 < rows_hi; i0 += kR * (kSolveThreads / 32)) {
        double l[kR][2];
#pragma unroll
        for (int rr = 0; rr < kR; ++rr) {
          const int i = i0 + rr;
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int k = lane + 32 * h;
            const bool ok = i < rows_hi && k < bs && !(k == 0 && i == k0 - 1 && pt_before == 2);
            l[rr][h] = ok ? f[static_cast<long long>(i) * ldf + k0 + k] : 0.0;
          }
        }
        for (int cc = 0; cc < nc; ++cc) {
          const double y0 = lane < bs ? ys[cc][lane] : 0.0;
          const double y1 = lane + 32 < bs ? ys[cc][lane + 32] : 0.0;
#pragma unroll
          for (int rr = 0; rr < kR; ++rr) {
            double v = l[rr][0] * y0 + l[rr][1] * y1;
            for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
            if (lane == 0 && i0 + rr < rows_hi) y[static_cast<long long>(c0 + cc) * n + i0 + rr] -= v;
          }
        }
      }
    }
    __syncthreads();
  }
}

// M = L D (row-major n x n), M(i,k) for k <= i+1.
__global__ void ld_kernel(int n, const double* f, long long ldf, const int* pt, double* m) {
  const long long total = static_cast<long long>(n) * n;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(t / n), k = static_cast<int>(t % n);
    auto lval = [&](int row, int col) -> double {
      if (row == col) return 1.0;
      if (row < col) return 0.0;
      if (pt[col] == 2 && row == col + 1) return 0.0;
      return f[static_cast<long long>(col) * ldf + row];
    };
    double v;
    if (pt[k] == 2 && k + 1 < n) {
      v = lval(i, k) * f[k * ldf + k] + lval(i, k + 1) * f[k * ldf + k + 1];
    } else if (pt[k] == -2 && k > 0) {
      v = lval(i, k - 1) * f[(k - 1) * ldf + k] + lval(i, k) * f[k * ldf + k];
    } else {
      v = lval(i, k) * f[k * ldf + k];
    }
    m[t] = v;
  }
}

// out(perm[i], perm[j]) = sum_k M(i,k) L(j,k)
__global__ void rec_kernel(int n, const double* f, long long ldf, const int* pt, const int* perm,
                           const double* m, double* out, long long ldo) {
  const int i = blockIdx.y * 16 + threadIdx.y;
  const int j = blockIdx.x * 16 + threadIdx.x;
  if (i >= n || j >= n) return;
  const int kmax = min(n - 1, min(i + 1, j));
  double s = 0.0;
  for (int k = 0; k <= kmax; ++k) {
    double l;
    if (j == k) {
      l = 1.0;
    } else if (j < k || (pt[k] == 2 && j == k + 1)) {
      l = 0.0;
    } else {
      l = f[static_cast<long long>(k) * ldf + j];
    }
    s += m[static_cast<long long>(i) * n + k] * l;
  }
  out[static_cast<long long>(perm[i]) * ldo + perm[j]] = s;
}

int grid_for(long long work, int threads) {
  const long long g = (work + threads - 1) / threads;
  return static_cast<int>(std::max(1LL, std::min(g, 4096LL)));
}

}  // namespace

size_t solve_work_doubles(int n, int nrhs) { return 2 * static_cast<size_t>(n) * nrhs; }

// work: 2 n nrhs doubles (two ping-pong copies of the right-hand sides)
int solve_enqueue(int n, const double* f, long long ldf, const int* perm, const int* pivot_types,
                  int nrhs, double* b, long long ldb, double* work, cudaStream_t s) {
  double* y = work;
  double* z = work + static_cast<size_t>(n) * nrhs;
  const long long total = static_cast<long long>(n) * nrhs;
  gather_kernel<<<grid_for(total, 256), 256, 0, s>>>(n, nrhs, b, ldb, perm, y);
  BBK_CUDA_TRY(cudaGetLastError());
  count_launch();
  for (int k0 = 0; k0 < n; k0 += kSB) {
    const int k1 = std::min(n, k0 + kSB);
    const int rows = n - k1;
    const int grid = std::max(1, (rows + kRowsPerCta - 1) / kRowsPerCta);
    sweep_kernel<true><<<grid, kSolveThreads, 0, s>>>(n, nrhs, f, ldf, pivot_types, y, z, k0, k1);
    BBK_CUDA_TRY(cudaGetLastError());
    count_launch();
  }
  dsolve_kernel<<<grid_for(n, 256), 256, 0, s>>>(n, nrhs, f, ldf, pivot_types, z);
  BBK_CUDA_TRY(cudaGetLastError());
  count_launch();
  const int nblk = (n + kSB - 1) / kSB;
  for (int bi = nblk - 1; bi >= 0; --bi) {
    const int k0 = bi * kSB, k1 = std::min(n, k0 + kSB);
    const int grid = std::max(1, (k0 + kRowsBack - 1) / kRowsBack);
    sweep_kernel<false><<<grid, kSolveThreads, 0, s>>>(n, nrhs, f, ldf, pivot_types, z, y, k0, k1);
    BBK_CUDA_TRY(cudaGetLastError());
    count_launch();
  }
  scatter_kernel<<<grid_for(total, 256), 256, 0, s>>>(n, nrhs, b, ldb, perm, y);
  BBK_CUDA_TRY(cudaGetLastError());
  count_launch();
  return BBK_OK;
}

int reconstruct_enqueue(int n, const double* f, long long ldf, const int* perm,
                        const int* pivot_types, double* out, long long ldo, double* m,
                        cudaStream_t s) {
  const long long total = static_cast<long long>(n) * n;
  ld_kernel<<<grid_for(total, 256), 256, 0, s>>>(n, f, ldf, pivot_types, m);
  BBK_CUDA_TRY(cudaGetLastError());
  count_launch();
  dim3 blk(16, 16), grd((n + 15) / 16, (n + 15) / 16);
  rec_kernel<<<grd, blk, 0, s>>>(n, f, ldf, pivot_types, perm, m, out, ldo);
  BBK_CUDA_TRY(cudaGetLastError());
  count_launch();
  return BBK_OK;
}

}  // namespace bbk
