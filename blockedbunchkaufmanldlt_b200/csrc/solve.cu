// Solve A X = B with compact Bunch-Kaufman factors, and the dense
// reconstruction P^T L D L^T P.
//
// The reference has no solve; L and D are read exactly as its stress test
// reads them (tests/block_ldlt_large_stress_test.cc:160-194 in
// wentianshu/BlockedBunchKaufmanLDLT): L(i,k) = F(k,i) for k < i, except
// L(k+1,k) = 0 when a 2x2 pivot starts at k; D(k,k) = F(k,k) and
// D(k,k+1) = F(k,k+1) for that 2x2.  With (P A P^T)(i,j) = A(perm[i], perm[j]):
//   y = B[perm]; L z = y; D w = z; L^T v = w; X[perm] = v.
// Each triangular sweep is a persistent cooperative launch over 64-row
// blocks in sweep order: CTA c owns blocks c, c+G, ...; a solved block is
// published with a release flag.  Two forms:
//  * pull (up to 32 right-hand sides, 8 per launch): the owner of a block
//    gathers the contributions of all earlier blocks into it, the old ones
//    while the blocks just before it are still being solved elsewhere, then
//    solves its triangle.  The critical path per block is one flag, one fold
//    and the triangle.
//  * streaming (more right-hand sides): every solved block is pushed into
//    each later block of every CTA, all right-hand sides at once, so the
//    factor is read once per sweep.
#include <algorithm>
#include <mutex>

#include "bbk_internal.cuh"

namespace bbk {
namespace {

constexpr int kSB = 64;           // solve block
constexpr int kSolveThreads = 256;
constexpr int kMaxRhsChunk = 8;   // right-hand sides per pass
constexpr int kAhead = 4;         // pull sweep: factor blocks prefetched into L2 ahead of the fold

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

struct SweepArgs {
  int n;
  int nrhs;
  const double* f;
  long long ldf;
  const int* pt;
  double* y;       // n x nrhs (ld n), solved in place
  int* flags;      // per block: == mark once the block is solved in this sweep
  int* status;     // nonzero: a wait ran out; every CTA returns
  int mark;
  unsigned long long timeout_ns;
};

__device__ __forceinline__ int ld_acquire_s32(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Waits (thread 0, bounded) until block k is solved; all threads learn
// whether to go on.
__device__ bool wait_block(const SweepArgs& A, int k, int* s_ok) {
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned long long t0 = globaltimer_ns();
    for (unsigned it = 1; ld_acquire_s32(A.flags + k) != A.mark; ++it) {
      if ((it & 31u) == 0) {
        if (ld_relaxed_s32(A.status) != 0) {
          ok = 0;
          break;
        }
        if (globaltimer_ns() - t0 > A.timeout_ns) {
          atomicCAS(A.status, 0, BBK_ERR_TIMEOUT);
          ok = 0;
          break;
        }
      }
    }
    *s_ok = ok;
  }
  __syncthreads();
  return *s_ok != 0;
}

__device__ __forceinline__ void cp_async_8z(double* smem_dst, const double* gsrc, bool valid) {
  const unsigned saddr = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(saddr), "l"(gsrc), "r"(valid ? 8 : 0)
               : "memory");
}

constexpr int kTriPitch = kSB + 1;
constexpr size_t kSweepSmem = (kSB * kTriPitch + 4 * kMaxRhsChunk * kSB + kMaxRhsChunk * kSB) * sizeof(double);

template <bool kForward>
__global__ void __launch_bounds__(kSolveThreads) psweep_kernel(SweepArgs A) {
  extern __shared__ double psm[];
  double* tri = psm;                               // [kSB][kTriPitch]: F(k0+r, k0+c), r < c
  double (*red)[kMaxRhsChunk][kSB] =
      reinterpret_cast<double (*)[kMaxRhsChunk][kSB]>(psm + kSB * kTriPitch);  // 4 quarters
  double (*zs)[kSB] = reinterpret_cast<double (*)[kSB]>(psm + kSB * kTriPitch + 4 * kMaxRhsChunk * kSB);
  __shared__ int pts[kSB];
  __shared__ int s_ok;
  const int n = A.n, nrhs = A.nrhs;
  const long long ldf = A.ldf;
  const int nblk = (n + kSB - 1) / kSB;
  const int G = gridDim.x, c = blockIdx.x;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int row = t & (kSB - 1), quarter = t >> 6;  // 64 rows x 4 quarters of the k range
  const int dir = kForward ? 1 : -1;
  // this CTA's blocks in wavefront order: first .. last, stride G
  const int my_first = kForward ? c : (nblk - 1) - ((nblk - 1 - c) % G);
  if (kForward ? my_first >= nblk : my_first < 0) return;
  const int my_last = kForward ? c + ((nblk - 1 - c) / G) * G : c;
  // the diagonal triangle of an own block, streamed into shared memory ahead of time
  auto prefetch_tri = [&](int b) {
    const int b0 = b * kSB, bsz = min(n, b0 + kSB) - b0;
    for (int idx = t; idx < kSB * kSB; idx += kSolveThreads) {
      const int r = idx / kSB, cc = idx % kSB;
      const bool ok = r < cc && cc < bsz;
      cp_async_8z(&tri[r * kTriPitch + cc], ok ? A.f + static_cast<long long>(b0 + r) * ldf + b0 + cc : A.f, ok);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  // factor entries that fold block k into own block b (this thread's 16)
  auto load_fold = [&](int k, int b, double (&l)[kSB / 4]) {
    const int k0 = k * kSB, bs = min(n, k0 + kSB) - k0;
    const int i = b * kSB + row;
    const int pt_edge = kForward ? A.pt[k0 + bs - 1] : (k0 > 0 ? A.pt[k0 - 1] : 1);
#pragma unroll
    for (int u = 0; u < kSB / 4; ++u) {
      const int kk = quarter * (kSB / 4) + u;
      const int kg = k0 + kk;
      bool ok = i < n && kk < bs;
      double v = 0.0;
      if (kForward) {
        // L(i, kg) = F(kg, i); the (kg+1, kg) entry of a 2x2 is zero
        ok = ok && !(i == kg + 1 && kk == bs - 1 && pt_edge == 2);
        if (ok) v = A.f[static_cast<long long>(kg) * ldf + i];
      } else {
        // L(kg, i) = F(i, kg); the (i+1, i) entry of a 2x2 is zero
        ok = ok && !(kg == i + 1 && kk == 0 && pt_edge == 2);
        if (ok) v = A.f[static_cast<long long>(i) * ldf + kg];
      }
      l[u] = v;
    }
  };
  prefetch_tri(my_first);
  for (int step = 0; step < nblk; ++step) {
    const int k = kForward ? step : nblk - 1 - step;
    if (kForward ? k > my_last : k < my_last) break;
    const int k0 = k * kSB, k1 = min(n, k0 + kSB), bs = k1 - k0;
    const bool mine = k % G == c;
    // the nearest own block after k receives k's contribution first (critical path)
    // (the first b beyond k in wavefront order with b % G == c)
    const int gap = kForward ? (((c - k) % G) + G) % G : (((k - c) % G) + G) % G;
    const int near = mine ? k + dir * G : k + dir * gap;
    const bool has_near = kForward ? near <= my_last : near >= my_last;
    double lnear[kSB / 4];
    if (has_near) load_fold(k, near, lnear);
    if (mine) {
      // ---- own block: every earlier block's contribution is in; solve the triangle
      for (int r = t; r < kSB; r += kSolveThreads) pts[r] = r < bs ? A.pt[k0 + r] : 1;
      asm volatile("cp.async.wait_all;" ::: "memory");
      __syncthreads();
      for (int rc = warp; rc < nrhs; rc += kSolveThreads / 32) {
        double* yc = A.y + static_cast<long long>(rc) * n;
        double v0 = lane < bs ? yc[k0 + lane] : 0.0;
        double v1 = lane + 32 < bs ? yc[k0 + lane + 32] : 0.0;
        if (kForward) {
          for (int kk = 0; kk < bs; ++kk) {
            const double yk = __shfl_sync(0xffffffffu, kk < 32 ? v0 : v1, kk & 31);
            const bool skip_next = pts[kk] == 2;
            const int i0 = lane, i1 = lane + 32;
            if (i0 > kk && i0 < bs && !(skip_next && i0 == kk + 1)) v0 -= tri[kk * kTriPitch + i0] * yk;
            if (i1 > kk && i1 < bs && !(skip_next && i1 == kk + 1)) v1 -= tri[kk * kTriPitch + i1] * yk;
          }
        } else {
          for (int kk = bs - 1; kk >= 0; --kk) {
            const double yk = __shfl_sync(0xffffffffu, kk < 32 ? v0 : v1, kk & 31);
            const int i0 = lane, i1 = lane + 32;
            // L(kk, i) = F(i, kk) for i < kk, except i == kk-1 opening a 2x2
            if (i0 < kk && !(i0 == kk - 1 && pts[i0] == 2)) v0 -= tri[i0 * kTriPitch + kk] * yk;
            if (i1 < kk && !(i1 == kk - 1 && pts[i1] == 2)) v1 -= tri[i1 * kTriPitch + kk] * yk;
          }
        }
        if (lane < bs) yc[k0 + lane] = v0;
        if (lane + 32 < bs) yc[k0 + lane + 32] = v1;
      }
      __syncthreads();
      if (t == 0) {
        fence_acq_rel_gpu();
        asm volatile("st.relaxed.gpu.global.b32 [%0], %1;" ::"l"(A.flags + k), "r"(A.mark) : "memory");
      }
      if (has_near) prefetch_tri(near);  // the triangle buffer is free again
    } else {
      if (!wait_block(A, k, &s_ok)) return;
    }
    // ---- fold block k into this CTA's later blocks
    for (int c0 = 0; c0 < nrhs; c0 += kMaxRhsChunk) {
      const int nc = min(kMaxRhsChunk, nrhs - c0);
      __syncthreads();
      for (int idx = t; idx < nc * kSB; idx += kSolveThreads) {
        const int cc = idx / kSB, r = idx % kSB;
        zs[cc][r] = r < bs ? __ldcg(A.y + static_cast<long long>(c0 + cc) * n + k0 + r) : 0.0;
      }
      __syncthreads();
      for (int b = near; has_near && (kForward ? b <= my_last : b >= my_last); b += dir * G) {
        double lo[kSB / 4];
        if (b == near) {
#pragma unroll
          for (int u = 0; u < kSB / 4; ++u) lo[u] = lnear[u];
        } else {
          load_fold(k, b, lo);
        }
        const int b0 = b * kSB;
        double acc[kMaxRhsChunk];
#pragma unroll
        for (int cc = 0; cc < kMaxRhsChunk; ++cc) acc[cc] = 0.0;
#pragma unroll
        for (int u = 0; u < kSB / 4; ++u)
#pragma unroll
          for (int cc = 0; cc < kMaxRhsChunk; ++cc)
            if (cc < nc) acc[cc] += lo[u] * zs[cc][quarter * (kSB / 4) + u];
#pragma unroll
        for (int cc = 0; cc < kMaxRhsChunk; ++cc)
          if (cc < nc) red[quarter][cc][row] = acc[cc];
        __syncthreads();
        for (int idx = t; idx < nc * kSB; idx += kSolveThreads) {
          const int cc = idx / kSB, r = idx % kSB;
          const int ii = b0 + r;
          if (ii < n) {
            const double s4 = (red[0][cc][r] + red[1][cc][r]) + (red[2][cc][r] + red[3][cc][r]);
            A.y[static_cast<long long>(c0 + cc) * n + ii] -= s4;
          }
        }
        __syncthreads();
      }
    }
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
}

// Pull sweep (at most kMaxRhsChunk right-hand sides per launch).  CTA c owns
// blocks c, c+G, ... in sweep order and handles one at a time: it folds in
// the contribution of every earlier block (in sweep order) as soon as that
// block is solved, then solves the block's own triangle and raises its
// flag.  Contributions of blocks solved long ago stream in while the blocks
// just before this one are still being solved elsewhere, so the critical
// path per block is one flag, one load of the newest solved block, its fold,
// the reduction and the triangle.
//   forward: thread (row, quarter) accumulates L(i, kg) y(kg) over its
//     quarter of each earlier block (warp loads of F rows are contiguous in
//     i); the four quarters are added at the end.
//   backward: warp w owns rows i = 8w..8w+7 and lane l the columns kg = l,
//     l + 32 of each later block (F rows are contiguous in kg); the lanes
//     are added by a butterfly at the end.
// Each warp learns which blocks are solved on its own (one relaxed scan of
// up to 32 flags, one acquire load of the newest set one, or a bounded wait
// on the next), so no CTA barrier is taken per block.
// The triangle is staged so that step kk of the substitution reads row kk
// of the staged array in both directions (backward: transposed).
__device__ __forceinline__ int ld_relaxed_flag(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Makes block k (and every block before it in sweep order) visible to this
// warp; returns the newest block in sweep order known to be solved (>= k in
// sweep order), or `fail` when the wait ran out or another CTA gave up.
template <bool kForward>
__device__ int warp_wait_solved(const SweepArgs& A, int k, int k_end, int fail) {
  const int lane = threadIdx.x & 31;
  const int dir = kForward ? 1 : -1;
  const int idx = k + dir * lane;
  const bool valid = kForward ? idx <= k_end : idx >= k_end;
  const bool set = valid && ld_relaxed_flag(A.flags + idx) == A.mark;
  const unsigned run = __ballot_sync(0xffffffffu, set);
  const int m = run == 0xffffffffu ? 32 : __ffs(~run) - 1;  // solved blocks from k on, in order
  int top = fail;
  if (lane == 0) {
    if (m > 0) {
      top = k + dir * (m - 1);
      (void)ld_acquire_s32(A.flags + top);
    } else {
      // the bound is checked after every unsuccessful poll (a poll is an L2
      // round trip), the other CTAs' status every 32 polls
      const unsigned long long t0 = globaltimer_ns();
      for (unsigned it = 1;; ++it) {
        if (ld_acquire_s32(A.flags + k) == A.mark) {
          top = k;
          break;
        }
        if (globaltimer_ns() - t0 > A.timeout_ns) {
          atomicCAS(A.status, 0, BBK_ERR_TIMEOUT);
          break;
        }
        if ((it & 31u) == 0 && ld_relaxed_s32(A.status) != 0) break;
      }
    }
  }
  top = __shfl_sync(0xffffffffu, top, 0);
  __syncwarp();
  return top;
}

template <bool kForward>
__global__ void __launch_bounds__(kSolveThreads, 1) psweep_pull_kernel(SweepArgs A) {
  extern __shared__ double psm[];
  double* tri = psm;                            // [kSB][kTriPitch], row kk = step kk's operands
  double* red = psm + kSB * kTriPitch;          // [4][kMaxRhsChunk][kSB] partial sums
  double* ys = red + 4 * kMaxRhsChunk * kSB;    // [kMaxRhsChunk][kSB]: the block being solved
  __shared__ int pts[kSB];
  __shared__ int s_fail;
  const int n = A.n, nc = A.nrhs;
  const long long ldf = A.ldf;
  const int nblk = (n + kSB - 1) / kSB;
  const int G = gridDim.x, c = blockIdx.x;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int dir = kForward ? 1 : -1;
  const int my_first = kForward ? c : (nblk - 1) - ((nblk - 1 - c) % G);
  if (kForward ? my_first >= nblk : my_first < 0) return;
  const int my_last = kForward ? c + ((nblk - 1 - c) / G) * G : c;
  const int kNone = kForward ? -1 : nblk;  // "no block" in sweep order
  const int kFail = kForward ? -2 : nblk + 1;
  auto stage_tri = [&](int b) {
    const int b0 = b * kSB, bsz = min(n, b0 + kSB) - b0;
    for (int idx = t; idx < kSB * kSB; idx += kSolveThreads) {
      const int r = idx / kSB, cc = idx % kSB;  // F(b0 + r, b0 + cc), r < cc
      const bool ok = r < cc && cc < bsz;
      double* dst = kForward ? &tri[r * kTriPitch + cc] : &tri[cc * kTriPitch + r];
      cp_async_8z(dst, ok ? A.f + static_cast<long long>(b0 + r) * ldf + b0 + cc : A.f, ok);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  if (t == 0) s_fail = 0;
  __syncthreads();
  int known = kNone;  // per warp: newest block (sweep order) known to be solved
  stage_tri(my_first);
  for (int b = my_first; kForward ? b <= my_last : b >= my_last; b += dir * G) {
    const int b0 = b * kSB, bsz = min(n, b0 + kSB) - b0;
    for (int r = t; r < kSB; r += kSolveThreads) pts[r] = r < bsz ? A.pt[b0 + r] : 1;
    // this block's right-hand sides, for the threads that finish them
    double yin[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int idx = t + h * kSolveThreads, cc = idx / kSB, r = idx % kSB;
      yin[h] = cc < nc && r < bsz ? A.y[static_cast<long long>(cc) * n + b0 + r] : 0.0;
    }
    // the 32 KB of the factor that fold k reads, into L2 (one 128-byte line
    // per thread: 64 rows of 4 lines; a row's lines may straddle a fifth)
    auto prefetch_f = [&](int k) {
      const int a = t >> 2, seg = (t & 3) * 16;
      const int x = kForward ? k * kSB + a : b0 + a;    // factor row
      const int y0 = kForward ? b0 + seg : k * kSB + seg;  // first column
      if (x < n && y0 < n) {
        const double* p = A.f + static_cast<long long>(x) * ldf + y0;
        asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
        asm volatile("prefetch.global.L2 [%0];" ::"l"(p + min(15, n - 1 - y0)));
      }
    };
    const int k_first = kForward ? 0 : nblk - 1;
    const int k_end = b - dir;  // the last block folded into b (sweep order)
    const bool any = kForward ? b > 0 : b < nblk - 1;
    bool fail = false;
    if (kForward) {
      const int row = t & (kSB - 1), quarter = t >> 6;
      const int i = b0 + row;
      double acc[kMaxRhsChunk];
#pragma unroll
      for (int cc = 0; cc < kMaxRhsChunk; ++cc) acc[cc] = 0.0;
      auto load_f = [&](int k, double (&l)[kSB / 4]) {
        const int k0 = k * kSB, bs = min(n, k0 + kSB) - k0;
        const bool edge = k == b - 1 && A.pt[k0 + bs - 1] == 2;  // 2x2 across the boundary
#pragma unroll
        for (int u = 0; u < kSB / 4; ++u) {
          const int kk = quarter * (kSB / 4) + u, kg = k0 + kk;
          const bool ok = i < n && kk < bs && !(edge && i == kg + 1);
          l[u] = ok ? A.f[static_cast<long long>(kg) * ldf + i] : 0.0;
        }
      };
      // lane l: entries l, l + 32, ... of (cc, u) = (e / 16, e % 16) of
      // this quarter's solved values of block k
      auto load_y = [&](int k, double (&yv)[kMaxRhsChunk / 2]) {
        const int kq = k * kSB + quarter * (kSB / 4);
#pragma unroll
        for (int e2 = 0; e2 < kMaxRhsChunk / 2; ++e2) {
          const int e = lane + 32 * e2, cc = e >> 4, u = e & 15;
          yv[e2] = cc < nc && kq + u < n ? __ldcg(A.y + static_cast<long long>(cc) * n + kq + u) : 0.0;
        }
      };
      double fc[kSB / 4], fn[kSB / 4];
      for (int k = k_first; any && k < k_first + kAhead && k <= k_end; ++k) prefetch_f(k);
      if (any) load_f(k_first, fc);
      for (int k = k_first; any && k <= k_end; ++k) {
        if (k + kAhead <= k_end) prefetch_f(k + kAhead);
        if (k < k_end) load_f(k + 1, fn);
        if (k > known) {
          known = warp_wait_solved<true>(A, k, k_end, kFail);
          if (known == kFail) {
            fail = true;
            known = k_end;
          }
        }
        // this quarter's 16 x nc solved values, all loaded at once and each
        // broadcast to the warp by a shuffle
        double yl[kMaxRhsChunk / 2];
        load_y(k, yl);
#pragma unroll
        for (int u = 0; u < kSB / 4; ++u)
#pragma unroll
          for (int cc = 0; cc < kMaxRhsChunk; ++cc)
            if (cc < nc) {
              const double yv = __shfl_sync(0xffffffffu, yl[(cc * 16 + u) >> 5], (cc * 16 + u) & 31);
              acc[cc] = __fma_rn(fc[u], yv, acc[cc]);
            }
#pragma unroll
        for (int u = 0; u < kSB / 4; ++u) fc[u] = fn[u];
      }
#pragma unroll
      for (int cc = 0; cc < kMaxRhsChunk; ++cc)
        if (cc < nc) red[(quarter * kMaxRhsChunk + cc) * kSB + row] = acc[cc];
    } else {
      // rows 8 warp .. 8 warp + 7 of the block, columns lane and lane + 32 of block k
      double acc[8][kMaxRhsChunk];
#pragma unroll
      for (int j = 0; j < 8; ++j)
#pragma unroll
        for (int cc = 0; cc < kMaxRhsChunk; ++cc) acc[j][cc] = 0.0;
      auto load_f = [&](int k, double (&l)[16]) {
        const int k0 = k * kSB;
        const bool edge = k == b + 1 && b0 + kSB - 1 < n && A.pt[b0 + kSB - 1] == 2;
#pragma unroll
        for (int j = 0; j < 8; ++j)
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int ii = b0 + warp * 8 + j, kg = k0 + lane + 32 * h;
            const bool ok = ii < n && kg < n && !(edge && kg == ii + 1);
            l[j * 2 + h] = ok ? A.f[static_cast<long long>(ii) * ldf + kg] : 0.0;
          }
      };
      double fc[16], fn[16];
      for (int k = k_first; any && k > k_first - kAhead && k >= k_end; --k) prefetch_f(k);
      if (any) load_f(k_first, fc);
      for (int k = k_first; any && k >= k_end; --k) {
        if (k - kAhead >= k_end) prefetch_f(k - kAhead);
        if (k > k_end) load_f(k - 1, fn);
        if (k < known) {
          known = warp_wait_solved<false>(A, k, k_end, kFail);
          if (known == kFail) {
            fail = true;
            known = k_end;
          }
        }
        double yv[2][kMaxRhsChunk];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int kg = k * kSB + lane + 32 * h;
#pragma unroll
          for (int cc = 0; cc < kMaxRhsChunk; ++cc)
            yv[h][cc] = cc < nc && kg < n ? __ldcg(A.y + static_cast<long long>(cc) * n + kg) : 0.0;
        }
#pragma unroll
        for (int j = 0; j < 8; ++j)
#pragma unroll
          for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int cc = 0; cc < kMaxRhsChunk; ++cc)
              if (cc < nc) acc[j][cc] = __fma_rn(fc[j * 2 + h], yv[h][cc], acc[j][cc]);
#pragma unroll
        for (int u = 0; u < 16; ++u) fc[u] = fn[u];
      }
      // add the 64 sums of (j, cc) over the lanes by recursive halving: at
      // offset o each lane keeps one half of its values and adds the
      // partner's copy of that half; after five levels lane l holds the
      // totals of entries 2l and 2l + 1 (62 shuffles, depth 5)
      static_assert(8 * kMaxRhsChunk == 64, "the halving below assumes 64 sums per lane");
      double v[64];
#pragma unroll
      for (int j = 0; j < 8; ++j)
#pragma unroll
        for (int cc = 0; cc < kMaxRhsChunk; ++cc) v[j * kMaxRhsChunk + cc] = acc[j][cc];
#pragma unroll
      for (int o = 16, m = 64; o > 0; o >>= 1, m >>= 1) {
        const bool up = (lane & o) != 0;
#pragma unroll
        for (int e = 0; e < m / 2; ++e) {
          const double send = up ? v[e] : v[e + m / 2];
          const double keep = up ? v[e + m / 2] : v[e];
          v[e] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
      }
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int e = 2 * lane + h, j = e / kMaxRhsChunk, cc = e % kMaxRhsChunk;
        if (cc < nc) red[cc * kSB + warp * 8 + j] = v[h];
      }
    }
    if (fail) s_fail = 1;
    __syncthreads();
    if (s_fail) return;  // uniform: the status word already says why
    // ---- this block's right-hand sides less the folded sums
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int idx = t + h * kSolveThreads, cc = idx / kSB, r = idx % kSB;
      if (cc < nc) {
        double sum;
        if (kForward)
          sum = (red[(0 * kMaxRhsChunk + cc) * kSB + r] + red[(1 * kMaxRhsChunk + cc) * kSB + r]) +
                (red[(2 * kMaxRhsChunk + cc) * kSB + r] + red[(3 * kMaxRhsChunk + cc) * kSB + r]);
        else
          sum = red[cc * kSB + r];
        ys[cc * kSB + r] = any ? yin[h] - sum : yin[h];
      }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
    // ---- the block's triangle: one warp per right-hand side
    for (int rc = warp; rc < nc; rc += kSolveThreads / 32) {
      double* yb = ys + rc * kSB;
      double v0 = lane < bsz ? yb[lane] : 0.0;
      double v1 = lane + 32 < bsz ? yb[lane + 32] : 0.0;
      const int i0 = lane, i1 = lane + 32;
      // (the backward loop is unrolled over the block so the staged operands
      // load ahead of the chain; steps past a short last block change
      // nothing.  Unrolling the forward loop made it slower.)
      if (kForward) {
        for (int kk = 0; kk < bsz; ++kk) {
          const double yk = __shfl_sync(0xffffffffu, kk < 32 ? v0 : v1, kk & 31);
          const bool skip_next = pts[kk] == 2;
          if (i0 > kk && i0 < bsz && !(skip_next && i0 == kk + 1)) v0 -= tri[kk * kTriPitch + i0] * yk;
          if (i1 > kk && i1 < bsz && !(skip_next && i1 == kk + 1)) v1 -= tri[kk * kTriPitch + i1] * yk;
        }
      } else {        const bool open0 = pts[i0] == 2, open1 = pts[i1] == 2;
#pragma unroll
        for (int kk = kSB - 1; kk >= 0; --kk) {
          const double yk = __shfl_sync(0xffffffffu, kk < 32 ? v0 : v1, kk & 31);
          // L(kk, i) = F(i, kk) for i < kk < bsz, except i == kk-1 opening a 2x2
          if (kk < bsz && i0 < kk && !(i0 == kk - 1 && open0)) v0 -= tri[kk * kTriPitch + i0] * yk;
          if (kk < bsz && i1 < kk && !(i1 == kk - 1 && open1)) v1 -= tri[kk * kTriPitch + i1] * yk;
        }
      }
      double* yc = A.y + static_cast<long long>(rc) * n;
      if (lane < bsz) yc[b0 + lane] = v0;
      if (lane + 32 < bsz) yc[b0 + lane + 32] = v1;
    }
    __syncthreads();
    if (t == 0) {
      fence_acq_rel_gpu();
      asm volatile("st.relaxed.gpu.global.b32 [%0], %1;" ::"l"(A.flags + b), "r"(A.mark) : "memory");
    }
    const int nb = b + dir * G;
    if (kForward ? nb <= my_last : nb >= my_last) stage_tri(nb);  // the buffers are free again
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
}

__global__ void reset_flags_kernel(int* flags, int count) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) flags[i] = 0;
}

// L(row, col) of the compact factors: unit diagonal, F(col, row) below it
// except the coupling entry of a 2x2 pivot (ExtractRegularFactorsFromCompact,
// src/block_ldlt_decomposition.cc:746-763).
__device__ __forceinline__ double l_entry(const double* f, long long ldf, const int* pt, int row, int col) {
  if (row == col) return 1.0;
  if (row < col) return 0.0;
  if (pt[col] == 2 && row == col + 1) return 0.0;
  return f[static_cast<long long>(col) * ldf + row];
}

// M = L D and U = L^T (both ld x ld, zero outside the order n): the two
// operands of the reconstruction product.
__global__ void ld_lt_kernel(int n, const double* f, long long ldf, const int* pt, long long ld, double* m,
                             double* u) {
  const long long total = ld * ld;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(t / ld), k = static_cast<int>(t % ld);
    double mv = 0.0, uv = 0.0;
    if (i < n && k < n) {
      if (pt[k] == 2 && k + 1 < n) {
        mv = l_entry(f, ldf, pt, i, k) * f[k * ldf + k] + l_entry(f, ldf, pt, i, k + 1) * f[k * ldf + k + 1];
      } else if (pt[k] == -2 && k > 0) {
        mv = l_entry(f, ldf, pt, i, k - 1) * f[(k - 1) * ldf + k] + l_entry(f, ldf, pt, i, k) * f[k * ldf + k];
      } else {
        mv = l_entry(f, ldf, pt, i, k) * f[k * ldf + k];
      }
      uv = l_entry(f, ldf, pt, k, i);  // U(i, k) = L(k, i)
    }
    m[t] = mv;
    u[t] = uv;
  }
}

// out(perm[i], perm[j]) = (L D L^T)(i, j) = -C(min(i,j), max(i,j)).
__global__ void rec_scatter_kernel(int n, const double* c, long long ld, const int* perm, double* out,
                                   long long ldo) {
  const long long total = static_cast<long long>(n) * n;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(t / n), j = static_cast<int>(t % n);
    const int lo = min(i, j), hi = max(i, j);
    out[static_cast<long long>(perm[i]) * ldo + perm[j]] = -c[static_cast<long long>(lo) * ld + hi];
  }
}

// Dense L (unit lower) and D (block diagonal) from the compact factors.
__global__ void extract_ld_kernel(int n, const double* f, long long ldf, const int* pt, double* l, long long ldl,
                                  double* d, long long ldd) {
  const long long total = static_cast<long long>(n) * n;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(t / n), k = static_cast<int>(t % n);
    if (l) l[static_cast<long long>(i) * ldl + k] = l_entry(f, ldf, pt, i, k);
    if (d) {
      double v = 0.0;
      if (i == k) {
        v = f[static_cast<long long>(i) * ldf + i];
      } else if (k == i + 1 && pt[i] == 2) {
        v = f[static_cast<long long>(i) * ldf + k];
      } else if (i == k + 1 && pt[k] == 2) {
        v = f[static_cast<long long>(k) * ldf + i];
      }
      d[static_cast<long long>(i) * ldd + k] = v;
    }
  }
}

constexpr int kMaxAttrDevices = 64;
std::once_flag g_sweep_attr[kMaxAttrDevices];
// right-hand sides up to which the pull sweep is used (in launches of
// kMaxRhsChunk); more go through the streaming sweep, which reads the
// factor once for all of them
constexpr int kPullMaxRhs = 4 * kMaxRhsChunk;

int grid_for(long long work, int threads) {
  const long long g = (work + threads - 1) / threads;
  return static_cast<int>(std::max(1LL, std::min(g, 4096LL)));
}

}  // namespace

size_t solve_work_doubles(int n, int nrhs) { return 2 * static_cast<size_t>(n) * nrhs; }

int* solve_status_word(double* work, int n, int nrhs) {
  const int nblk = (n + kSB - 1) / kSB;
  return reinterpret_cast<int*>(work + static_cast<long long>(n) * nrhs) + nblk;
}

int solve_status(double* work, int n, int nrhs, cudaStream_t s) {
  int h = BBK_OK;
  BBK_CUDA_TRY(cudaMemcpyAsync(&h, solve_status_word(work, n, nrhs), sizeof(int), cudaMemcpyDeviceToHost, s));
  BBK_CUDA_TRY(cudaStreamSynchronize(s));
  if (h != BBK_OK) return set_error(h, "solve aborted on the device: %s", bbk_status_string(h));
  return BBK_OK;
}

// work: 2 n nrhs doubles: the right-hand sides being solved in place, then
// the block flags and the status word.
int solve_enqueue(int n, const double* f, long long ldf, const int* perm, const int* pivot_types,
                  int nrhs, double* b, long long ldb, double* work, cudaStream_t s) {
  double* y = work;
  const long long total = static_cast<long long>(n) * nrhs;
  const int nblk = (n + kSB - 1) / kSB;
  int* flags = reinterpret_cast<int*>(work + total);
  int* status = solve_status_word(work, n, nrhs);
  reset_flags_kernel<<<std::max(1, std::min(64, (nblk + 256) / 256)), 256, 0, s>>>(flags, nblk + 1);
  BBK_CUDA_TRY(cudaGetLastError());
  count_launch();
  gather_kernel<<<grid_for(total, 256), 256, 0, s>>>(n, nrhs, b, ldb, perm, y);
  BBK_CUDA_TRY(cudaGetLastError());
  count_launch();
  SweepArgs A{n, nrhs, f, ldf, pivot_types, y, flags, status, 1, wait_timeout_ns()};
  // both sweeps need more than the default 48 KB of dynamic shared memory;
  // the attributes are set per device, each under its own once-flag
  // (callers may be on several host threads)
  int dev = 0;
  BBK_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxAttrDevices) return set_error(BBK_ERR_NO_DEVICE, "device %d out of range", dev);
  cudaError_t attr_err = cudaSuccess;
  std::call_once(g_sweep_attr[dev], [&] {
    const void* fns[4] = {reinterpret_cast<const void*>(psweep_kernel<true>),
                          reinterpret_cast<const void*>(psweep_kernel<false>),
                          reinterpret_cast<const void*>(psweep_pull_kernel<true>),
                          reinterpret_cast<const void*>(psweep_pull_kernel<false>)};
    for (int i = 0; i < 4 && attr_err == cudaSuccess; ++i)
      attr_err = cudaFuncSetAttribute(fns[i], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(kSweepSmem));
  });
  BBK_CUDA_TRY(attr_err);
  const int grid = std::max(1, std::min(nblk, device_sm_count()));
  auto sweep = [&](const void* fn, SweepArgs& args) -> int {
    void* kargs[] = {&args};
    BBK_CUDA_TRY(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kSolveThreads), kargs, kSweepSmem, s));
    count_launch();
    return BBK_OK;
  };
  const bool pull = nrhs <= kPullMaxRhs;
  // every sweep launch waits for its own flag value
  int mark = 0;
  auto sweeps = [&](bool forward) -> int {
    const void* fn = pull ? (forward ? reinterpret_cast<const void*>(psweep_pull_kernel<true>)
                                     : reinterpret_cast<const void*>(psweep_pull_kernel<false>))
                          : (forward ? reinterpret_cast<const void*>(psweep_kernel<true>)
                                     : reinterpret_cast<const void*>(psweep_kernel<false>));
    const int chunk = pull ? kMaxRhsChunk : nrhs;
    for (int c0 = 0; c0 < nrhs; c0 += chunk) {
      SweepArgs a = A;
      a.y = y + static_cast<long long>(c0) * n;
      a.nrhs = std::min(chunk, nrhs - c0);
      a.mark = ++mark;
      const int rc = sweep(fn, a);
      if (rc) return rc;
    }
    return BBK_OK;
  };
  int rc = sweeps(true);
  if (rc) return rc;
  dsolve_kernel<<<grid_for(n, 256), 256, 0, s>>>(n, nrhs, f, ldf, pivot_types, y);
  BBK_CUDA_TRY(cudaGetLastError());
  count_launch();
  rc = sweeps(false);
  if (rc) return rc;
  scatter_kernel<<<grid_for(total, 256), 256, 0, s>>>(n, nrhs, b, ldb, perm, y);
  BBK_CUDA_TRY(cudaGetLastError());
  count_launch();
  return BBK_OK;
}

size_t reconstruct_work_doubles(int n) {
  const size_t ld = align_up(static_cast<size_t>(n), 128);
  return 3 * ld * ld;
}

// P^T L D L^T P: M = L D and U = L^T formed on the device, the upper tiles
// of M U on the FP64 tensor cores (the trailing-update tile kernels with
// C = 0), then mirrored and permuted.  work: reconstruct_work_doubles(n).
int reconstruct_enqueue(int n, const double* f, long long ldf, const int* perm,
                        const int* pivot_types, double* out, long long ldo, double* work,
                        cudaStream_t s) {
  const long long ld = static_cast<long long>(align_up(static_cast<size_t>(n), 128));
  double* m = work;
  double* u = m + ld * ld;
  double* c = u + ld * ld;
  BBK_CUDA_TRY(cudaMemsetAsync(c, 0, static_cast<size_t>(ld * ld) * sizeof(double), s));
  ld_lt_kernel<<<grid_for(ld * ld, 256), 256, 0, s>>>(n, f, ldf, pivot_types, ld, m, u);
  BBK_CUDA_TRY(cudaGetLastError());
  count_launch();
  int rc = launch_upper_product(n, m, u, ld, c, s);
  if (rc) return rc;
  rec_scatter_kernel<<<grid_for(static_cast<long long>(n) * n, 256), 256, 0, s>>>(n, c, ld, perm, out, ldo);
  BBK_CUDA_TRY(cudaGetLastError());
  count_launch();
  return BBK_OK;
}

int extract_ld_enqueue(int n, const double* f, long long ldf, const int* pivot_types, double* l, long long ldl,
                       double* d, long long ldd, cudaStream_t s) {
  extract_ld_kernel<<<grid_for(static_cast<long long>(n) * n, 256), 256, 0, s>>>(n, f, ldf, pivot_types, l, ldl,
                                                                                 d, ldd);
  BBK_CUDA_TRY(cudaGetLastError());
  count_launch();
  return BBK_OK;
}

}  // namespace bbk
