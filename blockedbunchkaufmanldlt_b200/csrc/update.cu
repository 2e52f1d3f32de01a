// Trailing update A22 -= U^T W of the blocked Bunch-Kaufman LDL^T
// (UpdateTrailingBlocks + kernels::UpdateTrailingBlock,
// src/block_ldlt_decomposition.cc:706-744 and src/kernels.cc:67-91 in
// wentianshu/BlockedBunchKaufmanLDLT), plus the standalone kernels.h entry
// points (ScaleOneByOnePivot / ScaleTwoByTwoPivot / UpdateTrailingBlock).
//
// C(i,j) -= sum_k A(i,k) B(k,j) with A(i,k) = U[k, i] and B(k,j) = W[k, j].
// Arithmetics:
//   FP64          FP64 tensor cores: mma.sync.m16n8k8.f64 from shared-memory
//                 tiles staged with cp.async (double-buffered); 64x64 C tile
//                 per CTA, 32x32 per warp.
//   FP64_ORDERED  SIMT, every product and sum rounded separately with k
//                 ascending and one final subtraction: bitwise the
//                 reference's arithmetic.
//   FP32          operands rounded to FP32, FP32 FMA accumulation, the result
//                 subtracted in FP64.
//   BF16, BF16X3  operands scaled by per-64-block powers of two and split
//                 into one or three BF16 terms, mma.sync m16n8k16 BF16 with
//                 FP32 accumulation, the result unscaled and subtracted in FP64.
// In the factorization the C tiles cover the upper triangle of the trailing
// matrix only (the reference also fills the unused lower halves of its
// diagonal blocks; nothing ever reads them).
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <type_traits>

#include "bbk_internal.cuh"

namespace bbk {
namespace {

constexpr int kBM = 64, kBN = 64, kBK = 32;
constexpr int kThreadsMma = 128;
constexpr int kPadA = 4, kPadB = 4;  // leading dims = 4 (mod 16) doubles: conflict-free fragments

struct UpdArgs {
  // A(i,k) = a[i*a_si + k*a_sk], B(k,j) = b[k*b_sk + j], C(i,j) = c[i*ldc + j]
  const double* a;
  long long a_si, a_sk;
  const double* b;
  long long b_sk;
  double* c;
  long long ldc;
  int i_lo, i_hi, j_lo, j_hi, inner;
  int upper_only;  // only write i <= j
  int tile_i0, tile_j0;  // origin of the tile grid (tile rows/cols start here)
  int tiles_m, tiles_n;  // tile grid extent (rectangular mode)
  int triangular;        // enumerate tiles (I <= J) of a square grid of tiles_m
  // panel mode: read the range from the device state
  const DeviceState* st;
  int panel;
  int n;
  // BF16 mode: per 64-block power-of-two scales of A rows and B columns
  const double* a_scale;
  const double* b_scale;
};

__device__ __forceinline__ void cp_async_8(double* smem_dst, const double* gsrc, bool valid) {
  const unsigned saddr = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  const int src_bytes = valid ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(saddr), "l"(gsrc),
               "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_16(double* smem_dst, const double* gsrc, int src_bytes) {
  const unsigned saddr = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(saddr), "l"(gsrc),
               "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Resolve the panel-mode range from the device state.
__device__ __forceinline__ bool resolve_range(UpdArgs& U) {
  if (U.st == nullptr) return true;
  if (ld_relaxed_s32(&U.st->abort)) return false;
  const int k0 = ldcg(&U.st->kstart[U.panel & 1]);
  const int e = ldcg(&U.st->kstart[(U.panel + 1) & 1]);
  U.inner = e - k0;
  U.i_lo = U.j_lo = e;
  U.i_hi = U.j_hi = U.n;
  U.tile_i0 = U.tile_j0 = (e / kBM) * kBM;
  U.tiles_m = U.tiles_n = (U.n - U.tile_i0 + kBM - 1) / kBM;
  // Ucm/W hold rows q relative to the panel start.
  return U.inner > 0 && e < U.n;
}

__device__ __forceinline__ int tile_count(const UpdArgs& U) {
  return U.triangular ? U.tiles_m * (U.tiles_m + 1) / 2 : U.tiles_m * U.tiles_n;
}

__device__ __forceinline__ void tile_coords(const UpdArgs& U, int t, int& I, int& J) {
  if (!U.triangular) {
    I = t % U.tiles_m;
    J = t / U.tiles_m;
    return;
  }
  // column-major over the upper triangle: J(J+1)/2 <= t < (J+1)(J+2)/2
  int j = static_cast<int>((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
  while (j * (j + 1) / 2 > t) --j;
  while ((j + 1) * (j + 2) / 2 <= t) ++j;
  J = j;
  I = t - j * (j + 1) / 2;
}

// ---------------------------------------------------------------------------
// FP64 tensor-core tile
// ---------------------------------------------------------------------------
template <bool kAK>  // true: A contiguous along k (a_sk == 1); false: along i
struct MmaSmem {
  static constexpr int kAStride = kAK ? (kBK + kPadA) : (kBM + kPadA);
  static constexpr int kASize = kAK ? kBM * kAStride : kBK * kAStride;
  static constexpr int kBStride = kBN + kPadB;
  static constexpr int kBSize = kBK * kBStride;
  static constexpr int kStage = kASize + kBSize;
  static constexpr size_t kBytes = 2 * kStage * sizeof(double);
  __device__ static double& a_at(double* as, int i, int k) {
    return kAK ? as[i * kAStride + k] : as[k * kAStride + i];
  }
};

template <bool kAK, bool kVec>
__device__ __forceinline__ void load_stage(const UpdArgs& U, double* as, double* bs, int i0, int j0,
                                           int k0) {
  using Sm = MmaSmem<kAK>;
  const int t = threadIdx.x;
  if (kVec) {
    // A: 64 rows x 32 k, contiguous along k, 16-byte chunks (2 doubles)
    for (int c = t; c < kBM * (kBK / 2); c += kThreadsMma) {
      const int ii = c / (kBK / 2), kk = (c % (kBK / 2)) * 2;
      const int k = k0 + kk;
      const int nvalid = max(0, min(2, U.inner - k));
      const double* src = U.a + static_cast<long long>(i0 + ii) * U.a_si + (nvalid ? k : 0);
      cp_async_16(&as[ii * Sm::kAStride + kk], src, nvalid * 8);
    }
    // B: 32 k x 64 j
    for (int c = t; c < kBK * (kBN / 2); c += kThreadsMma) {
      const int kk = c / (kBN / 2), jj = (c % (kBN / 2)) * 2;
      const int k = k0 + kk;
      const bool ok = k < U.inner;
      const double* src = U.b + static_cast<long long>(ok ? k : 0) * U.b_sk + j0 + jj;
      cp_async_16(&bs[kk * Sm::kBStride + jj], src, ok ? 16 : 0);
    }
  } else {
    for (int c = t; c < kBM * kBK; c += kThreadsMma) {
      int ii, kk;
      if (kAK) {
        ii = c / kBK;
        kk = c % kBK;
      } else {
        kk = c / kBM;
        ii = c % kBM;
      }
      const int i = i0 + ii, k = k0 + kk;
      const bool ok = k < U.inner && i >= U.i_lo && i < U.i_hi;
      const double* src = ok ? U.a + static_cast<long long>(i) * U.a_si + static_cast<long long>(k) * U.a_sk : U.a;
      cp_async_8(&Sm::a_at(as, ii, kk), src, ok);
    }
    for (int c = t; c < kBK * kBN; c += kThreadsMma) {
      const int kk = c / kBN, jj = c % kBN;
      const int j = j0 + jj, k = k0 + kk;
      const bool ok = k < U.inner && j >= U.j_lo && j < U.j_hi;
      const double* src = ok ? U.b + static_cast<long long>(k) * U.b_sk + j : U.b;
      cp_async_8(&bs[kk * Sm::kBStride + jj], src, ok);
    }
  }
  cp_async_commit();
}

__device__ __forceinline__ void mma_16x8x8(double (&c)[4], const double (&a)[4], const double (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

__device__ __forceinline__ void mma_16x8x16(double (&c)[4], const double (&a)[8], const double (&b)[4]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
      "{%4,%5,%6,%7,%8,%9,%10,%11}, {%12,%13,%14,%15}, {%0,%1,%2,%3};"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]),
        "d"(b[0]), "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

constexpr int kCPitch = kBM + 4;  // C tile staged in a free stage buffer
static_assert(kBM * kCPitch <= MmaSmem<true>::kStage, "C tile must fit in one stage buffer");

// C tile (rows i0.., cols j0..) -> shared memory, 16-byte cp.async chunks;
// entries outside the trailing region are zero-filled and never written back.
__device__ __forceinline__ void load_c_tile(const UpdArgs& U, double* cs, int i0, int j0) {
  for (int c = threadIdx.x; c < kBM * (kBN / 2); c += kThreadsMma) {
    const int ii = c / (kBN / 2), jj = (c % (kBN / 2)) * 2;
    const int i = i0 + ii, j = j0 + jj;
    const bool ok = i >= U.i_lo && i < U.i_hi && j + 1 < U.j_hi && j >= U.j_lo;
    const double* src = ok ? U.c + static_cast<long long>(i) * U.ldc + j : U.c;
    cp_async_16(&cs[ii * kCPitch + jj], src, ok ? 16 : 0);
  }
}


__device__ __forceinline__ void mma_bf16_16x8x16(float (&c)[4], const unsigned (&a)[4], const unsigned (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Split of a (scaled) double into BF16 terms: x ~ t0 + t1 + t2, each term
// the BF16 rounding of what the previous terms left over (kTerms = 1 is the
// plain rounding).
template <int kTerms>
__device__ __forceinline__ void split_bf16(double x, float (&t)[3]) {
  float rest = static_cast<float>(x);
#pragma unroll
  for (int k = 0; k < kTerms; ++k) {
    t[k] = __bfloat162float(__float2bfloat16_rn(rest));
    rest -= t[k];
  }
}

__device__ __forceinline__ unsigned pack2(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);  // exact: both are BF16 values
  return *reinterpret_cast<const unsigned*>(&v);
}

// BF16 chunk: FP64 tile in shared memory, operands scaled by sa / sb and
// split into kTerms BF16 terms while building fragments, FP32 accumulation.
// With three terms the products t_i(a) t_j(b), i + j <= 2, are kept (six
// MMAs per fragment pair), which carries about FP32 accuracy.
//   A frag (16x16): a0,a1 (g, 2t..2t+1); a2,a3 (g+8, 2t..); a4,a5 (g, 2t+8..);
//   a6,a7 (g+8, 2t+8..).  B frag (16x8): b0,b1 (2t..2t+1, g); b2,b3 (2t+8.., g).
template <bool kAK, int kTerms>
__device__ __forceinline__ void bf16_chunk(double* as, double* bs, float (&acc)[2][4][4], int wm, int wn,
                                           int g, int tq, double sa, double sb) {
  using Sm = MmaSmem<kAK>;
#pragma unroll
  for (int ks = 0; ks < kBK; ks += 16) {
    unsigned af[kTerms][2][4], bf[kTerms][4][2];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
      const int r = wm + mt * 16 + g;
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int rr = r + 8 * (u & 1), kk = ks + 2 * tq + 8 * (u >> 1);
        float x0[3], x1[3];
        split_bf16<kTerms>(Sm::a_at(as, rr, kk) * sa, x0);
        split_bf16<kTerms>(Sm::a_at(as, rr, kk + 1) * sa, x1);
#pragma unroll
        for (int k = 0; k < kTerms; ++k) af[k][mt][u] = pack2(x0[k], x1[k]);
      }
    }
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      const int col = wn + nt * 8 + g;
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int kk = ks + 2 * tq + 8 * u;
        float y0[3], y1[3];
        split_bf16<kTerms>(bs[kk * Sm::kBStride + col] * sb, y0);
        split_bf16<kTerms>(bs[(kk + 1) * Sm::kBStride + col] * sb, y1);
#pragma unroll
        for (int k = 0; k < kTerms; ++k) bf[k][nt][u] = pack2(y0[k], y1[k]);
      }
    }
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        // smallest products first
#pragma unroll
        for (int ia = kTerms - 1; ia >= 0; --ia)
#pragma unroll
          for (int ib = kTerms - 1; ib >= 0; --ib)
            if (ia + ib <= kTerms - 1) mma_bf16_16x8x16(acc[mt][nt], af[ia][mt], bf[ib][nt]);
      }
  }
}

template <bool kAK, bool K16>
__device__ __forceinline__ void mma_chunk(double* as, double* bs, double (&acc)[2][4][4], int wm, int wn,
                                          int g, int tq) {
  using Sm = MmaSmem<kAK>;
  if (K16) {
    // m16n8k16 fragments: a_i at (g + 8(i%2), tq + 4(i/2)), b_i at (tq + 4i, g)
#pragma unroll
    for (int ks = 0; ks < kBK; ks += 16) {
      double af[2][8], bf[4][4];
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        const int r = wm + mt * 16 + g;
#pragma unroll
        for (int u = 0; u < 8; ++u) af[mt][u] = Sm::a_at(as, r + 8 * (u & 1), ks + tq + 4 * (u >> 1));
      }
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const int col = wn + nt * 8 + g;
#pragma unroll
        for (int u = 0; u < 4; ++u) bf[nt][u] = bs[(ks + tq + 4 * u) * Sm::kBStride + col];
      }
#pragma unroll
      for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) mma_16x8x16(acc[mt][nt], af[mt], bf[nt]);
    }
  } else {
#pragma unroll
    for (int ks = 0; ks < kBK; ks += 8) {
      double af[2][4], bf[4][2];
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        const int r = wm + mt * 16 + g;
        af[mt][0] = Sm::a_at(as, r, ks + tq);
        af[mt][1] = Sm::a_at(as, r + 8, ks + tq);
        af[mt][2] = Sm::a_at(as, r, ks + tq + 4);
        af[mt][3] = Sm::a_at(as, r + 8, ks + tq + 4);
      }
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const int col = wn + nt * 8 + g;
        bf[nt][0] = bs[(ks + tq) * Sm::kBStride + col];
        bf[nt][1] = bs[(ks + tq + 4) * Sm::kBStride + col];
      }
#pragma unroll
      for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) mma_16x8x8(acc[mt][nt], af[mt], bf[nt]);
    }
  }
}

// Persistent over tiles, double-buffered over K chunks.  At a tile's last
// chunk the idle buffer receives the C tile (vector path), and right after
// the last chunk's MMAs the buffer just freed receives the next tile's first
// chunk, so neither latency sits on the critical path.
template <bool kAK, bool kVec, bool K16, int kBf16Terms = 0>
__global__ void __launch_bounds__(kThreadsMma) mma_update_kernel(UpdArgs U) {
  using Sm = MmaSmem<kAK>;
  constexpr bool kBf16 = kBf16Terms > 0;
  using Acc = typename std::conditional<kBf16, float, double>::type;
  extern __shared__ double smem[];
  if (!resolve_range(U)) return;
  const int ntiles = tile_count(U);
  int t = blockIdx.x;
  if (t >= ntiles) return;
  const int nchunks = (U.inner + kBK - 1) / kBK;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, tq = lane & 3;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  double* stage[2] = {smem, smem + Sm::kStage};

  int I, J;
  tile_coords(U, t, I, J);
  int i0 = U.tile_i0 + I * kBM, j0 = U.tile_j0 + J * kBN;
  load_stage<kAK, kVec>(U, stage[0], stage[0] + Sm::kASize, i0, j0, 0);
  cp_async_commit();
  int cur = 0;
  for (;;) {
    Acc acc[2][4][4];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[a][b][c] = Acc(0);
    double sa = 1.0, sb = 1.0;
    if (kBf16) {
      sa = U.a_scale[(i0 - U.tile_i0) / kBM];
      sb = U.b_scale[(j0 - U.tile_j0) / kBN];
    }
    for (int ch = 0; ch < nchunks; ++ch) {
      const int nxt = cur ^ 1;
      if (ch + 1 < nchunks) {
        load_stage<kAK, kVec>(U, stage[nxt], stage[nxt] + Sm::kASize, i0, j0, (ch + 1) * kBK);
        cp_async_commit();
        cp_async_wait<1>();
      } else if (kVec) {
        load_c_tile(U, stage[nxt], i0, j0);
        cp_async_commit();
        cp_async_wait<1>();
      } else {
        cp_async_wait<0>();
      }
      __syncthreads();  // chunk ch is in stage[cur]
      if constexpr (kBf16)
        bf16_chunk<kAK, (kBf16Terms > 0 ? kBf16Terms : 1)>(stage[cur], stage[cur] + Sm::kASize, acc, wm,
                                                          wn, g, tq, sa, sb);
      else
        mma_chunk<kAK, K16>(stage[cur], stage[cur] + Sm::kASize, acc, wm, wn, g, tq);
      __syncthreads();  // every warp is done with stage[cur]
      if (ch + 1 < nchunks) cur = nxt;
    }
    // stage[cur] is free; stage[cur ^ 1] holds the C tile (vector path)
    const int tn = t + static_cast<int>(gridDim.x);
    int ni0 = 0, nj0 = 0;
    if (tn < ntiles) {
      int nI, nJ;
      tile_coords(U, tn, nI, nJ);
      ni0 = U.tile_i0 + nI * kBM;
      nj0 = U.tile_j0 + nJ * kBN;
      load_stage<kAK, kVec>(U, stage[cur], stage[cur] + Sm::kASize, ni0, nj0, 0);
      cp_async_commit();
      if (kVec) cp_async_wait<1>();
    } else if (kVec) {
      cp_async_wait<0>();
    }
    if (kVec) __syncthreads();  // C tile visible
    const double* cs = stage[cur ^ 1];
    // C -= acc on the valid part of the tile
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int ii = wm + mt * 16 + g + h * 8;
        const int i = i0 + ii;
        if (i < U.i_lo || i >= U.i_hi) continue;
        double* crow = U.c + static_cast<long long>(i) * U.ldc;
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
          const int jj = wn + nt * 8 + tq * 2;
          const int j = j0 + jj;
          const double unscale = kBf16 ? 1.0 / (sa * sb) : 1.0;
          const double v0 = static_cast<double>(acc[mt][nt][h * 2]) * unscale;
          const double v1 = static_cast<double>(acc[mt][nt][h * 2 + 1]) * unscale;
          const bool ok0 = j >= U.j_lo && j < U.j_hi && (!U.upper_only || i <= j);
          const bool ok1 = j + 1 >= U.j_lo && j + 1 < U.j_hi && (!U.upper_only || i <= j + 1);
          if (kVec && ok0 && ok1) {
            double2 cv = *reinterpret_cast<const double2*>(cs + ii * kCPitch + jj);
            cv.x -= v0;
            cv.y -= v1;
            *reinterpret_cast<double2*>(crow + j) = cv;
          } else {
            if (ok0) crow[j] -= v0;
            if (ok1) crow[j + 1] -= v1;
          }
        }
      }
    }
    if (tn >= ntiles) break;
    __syncthreads();  // the C buffer becomes the next tile's second chunk buffer
    t = tn;
    i0 = ni0;
    j0 = nj0;
  }
  cp_async_wait<0>();
}

// ---------------------------------------------------------------------------
// FP64 tensor-core update with wide C tiles (the large trailing matrices):
// BM x BN tiles (BN a multiple of BM), warps of WM x WN, k chunks of 32 in a
// Stages-deep cp.async ring that runs across tile boundaries (the next
// tile's first chunks load while this tile finishes).  Each C tile is
// prefetched into L2 when its first chunk is consumed and updated straight
// from registers (C -= acc) at its end.  Every A/B element staged feeds BN
// (resp. BM) outputs instead of 64, which cuts the operand traffic from L2
// per flop; the C traffic per flop is the same as with 64 x 64 tiles.
// Tiles cover the upper triangle of the trailing matrix: column block J
// (BN wide) holds row blocks I <= (J + 1) R - 1, R = BN / BM, so the first
// R J(J+1)/2 tiles are the column blocks before J.
// ---------------------------------------------------------------------------
template <int BM, int BN, int WM, int WN, int Stages, int BK = kBK, int MinBlocks = 1>
struct Wide {
  static constexpr int kWarps = (BM / WM) * (BN / WN);
  static constexpr int kThreads = kWarps * 32;
  static constexpr int kMinBlocks = MinBlocks;
  static constexpr int kR = BN / BM;
  static constexpr int kAPitch = BK + kPadA;  // A stage [BM][BK + 4]: k contiguous
  static constexpr int kBPitch = BN + kPadB;  // B stage [BK][BN + 4]: j contiguous
  static constexpr int kAStage = BM * kAPitch;
  static constexpr int kStage = kAStage + BK * kBPitch;
  static constexpr size_t kBytes = static_cast<size_t>(Stages) * kStage * sizeof(double);
  static constexpr int kMT = WM / 16, kNT = WN / 8;  // m16n8k8 tiles per warp
  static_assert(BN % BM == 0, "column blocks must cover whole row blocks");
  static_assert(kBytes <= 227 * 1024, "stages must fit the shared memory of one CTA");
  static_assert((BM * BK / 2) % kThreads == 0 && (BK * BN / 2) % kThreads == 0, "even copy split");

  __device__ static int tiles(int tn) { return kR * tn * (tn + 1) / 2; }
  __device__ static void origin(const UpdArgs& U, int t, int& i0, int& j0) {
    int j = static_cast<int>((sqrt(8.0 * t / kR + 1.0) - 1.0) * 0.5);
    while (j > 0 && kR * j * (j + 1) / 2 > t) --j;
    while (kR * (j + 1) * (j + 2) / 2 <= t) ++j;
    i0 = U.tile_i0 + (t - kR * j * (j + 1) / 2) * BM;
    j0 = U.tile_i0 + j * BN;
  }
  // chunk at k0 of tile (i0, j0) into stage st (k >= inner zero-filled)
  __device__ static void load(const UpdArgs& U, double* st, int i0, int j0, int k0) {
    double* as = st;
    double* bs = st + kAStage;
    const int t = threadIdx.x;
#pragma unroll
    for (int u = 0; u < (BM * BK / 2) / kThreads; ++u) {
      const int c = t + u * kThreads;
      const int ii = c / (BK / 2), kk = (c % (BK / 2)) * 2;
      const int k = k0 + kk;
      const int nvalid = max(0, min(2, U.inner - k));
      const double* src = U.a + static_cast<long long>(i0 + ii) * U.a_si + (nvalid ? k : 0);
      cp_async_16(&as[ii * kAPitch + kk], src, nvalid * 8);
    }
#pragma unroll
    for (int u = 0; u < (BK * BN / 2) / kThreads; ++u) {
      const int c = t + u * kThreads;
      const int kk = c / (BN / 2), jj = (c % (BN / 2)) * 2;
      const int k = k0 + kk;
      const bool ok = k < U.inner;
      const double* src = U.b + static_cast<long long>(ok ? k : 0) * U.b_sk + j0 + jj;
      cp_async_16(&bs[kk * kBPitch + jj], src, ok ? 16 : 0);
    }
  }
};

template <int BM, int BN, int WM, int WN, int Stages, int BK = kBK, int MinBlocks = 1>
__global__ void __launch_bounds__(Wide<BM, BN, WM, WN, Stages, BK, MinBlocks>::kThreads, MinBlocks)
    mma_update_wide_kernel(UpdArgs U) {
  using W = Wide<BM, BN, WM, WN, Stages, BK, MinBlocks>;
  extern __shared__ double smem[];
  if (U.st != nullptr) {
    // panel mode: range from the device state, tiles from the BN-aligned
    // row at or below the trailing matrix's first row
    if (ld_relaxed_s32(&U.st->abort)) return;
    const int k0 = ldcg(&U.st->kstart[U.panel & 1]);
    const int e = ldcg(&U.st->kstart[(U.panel + 1) & 1]);
    U.inner = e - k0;
    U.i_lo = U.j_lo = e;
    U.i_hi = U.j_hi = U.n;
    U.tile_i0 = U.tile_j0 = (e / BN) * BN;
    if (U.inner <= 0 || e >= U.n) return;
  }
  const int tn = (U.n - U.tile_i0 + BN - 1) / BN;
  const int ntiles = W::tiles(tn);
  if (static_cast<int>(blockIdx.x) >= ntiles) return;
  const int nchunks = (U.inner + BK - 1) / BK;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, tq = lane & 3;
  const int wm = (warp / (BN / WN)) * WM, wn = (warp % (BN / WN)) * WN;
  // (tile, chunk) items of this CTA, in order: tiles blockIdx.x + m * gridDim.x
  const int my_tiles = (ntiles - static_cast<int>(blockIdx.x) + static_cast<int>(gridDim.x) - 1) /
                       static_cast<int>(gridDim.x);
  const long long items = static_cast<long long>(my_tiles) * nchunks;
  long long ld_item = 0;  // loader cursor: item ld_item = tile ld_m, chunk ld_ch
  int ld_ch = 0, ld_m = 0, ld_i0 = 0, ld_j0 = 0;
  W::origin(U, blockIdx.x, ld_i0, ld_j0);
  auto issue = [&]() {
    if (ld_item < items) {
      W::load(U, smem + static_cast<size_t>(ld_item % Stages) * W::kStage, ld_i0, ld_j0, ld_ch * BK);
      ++ld_item;
      if (++ld_ch == nchunks) {
        ld_ch = 0;
        ++ld_m;
        if (ld_m < my_tiles)
          W::origin(U, static_cast<int>(blockIdx.x) + ld_m * static_cast<int>(gridDim.x), ld_i0, ld_j0);
      }
    }
    cp_async_commit();  // one group per item slot, empty past the end
  };
#pragma unroll
  for (int s = 0; s < Stages - 1; ++s) issue();

  long long item = 0;
  for (int m = 0; m < my_tiles; ++m) {
    int i0, j0;
    W::origin(U, static_cast<int>(blockIdx.x) + m * static_cast<int>(gridDim.x), i0, j0);
    // the C tile's rows go to L2 now; the epilogue reads them after the k loop
    for (int r = threadIdx.x / (BN / 16); r < BM; r += W::kThreads / (BN / 16)) {
      const int i = i0 + r;
      const int jc = j0 + (threadIdx.x % (BN / 16)) * 16;
      if (i >= U.i_lo && i < U.i_hi && jc < U.j_hi && i <= jc + 15)
        asm volatile("prefetch.global.L2 [%0];" ::"l"(U.c + static_cast<long long>(i) * U.ldc + jc));
    }
    double acc[W::kMT][W::kNT][4];
#pragma unroll
    for (int a = 0; a < W::kMT; ++a)
#pragma unroll
      for (int b = 0; b < W::kNT; ++b)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.0;
    for (int ch = 0; ch < nchunks; ++ch, ++item) {
      cp_async_wait<Stages - 2>();
      __syncthreads();  // item's stage has landed; every warp is done with the stage refilled next
      issue();
      const double* as = smem + static_cast<size_t>(item % Stages) * W::kStage;
      const double* bs = as + W::kAStage;
#pragma unroll
      for (int ks = 0; ks < BK; ks += 8) {
        double af[W::kMT][4], bf[W::kNT][2];
#pragma unroll
        for (int mt = 0; mt < W::kMT; ++mt) {
          const int r = wm + mt * 16 + g;
          af[mt][0] = as[r * W::kAPitch + ks + tq];
          af[mt][1] = as[(r + 8) * W::kAPitch + ks + tq];
          af[mt][2] = as[r * W::kAPitch + ks + tq + 4];
          af[mt][3] = as[(r + 8) * W::kAPitch + ks + tq + 4];
        }
#pragma unroll
        for (int nt = 0; nt < W::kNT; ++nt) {
          const int col = wn + nt * 8 + g;
          bf[nt][0] = bs[(ks + tq) * W::kBPitch + col];
          bf[nt][1] = bs[(ks + tq + 4) * W::kBPitch + col];
        }
#pragma unroll
        for (int mt = 0; mt < W::kMT; ++mt)
#pragma unroll
          for (int nt = 0; nt < W::kNT; ++nt) mma_16x8x8(acc[mt][nt], af[mt], bf[nt]);
      }
    }
    // C -= acc on the tile's valid part (upper triangle of the trailing matrix)
#pragma unroll
    for (int mt = 0; mt < W::kMT; ++mt) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int i = i0 + wm + mt * 16 + g + h * 8;
        if (i < U.i_lo || i >= U.i_hi) continue;
        double* crow = U.c + static_cast<long long>(i) * U.ldc;
#pragma unroll
        for (int nt = 0; nt < W::kNT; ++nt) {
          const int j = j0 + wn + nt * 8 + tq * 2;
          const double v0 = acc[mt][nt][h * 2], v1 = acc[mt][nt][h * 2 + 1];
          const bool ok0 = j >= U.j_lo && j < U.j_hi && (!U.upper_only || i <= j);
          const bool ok1 = j + 1 >= U.j_lo && j + 1 < U.j_hi && (!U.upper_only || i <= j + 1);
          if (ok0 && ok1) {
            double2 cv = *reinterpret_cast<const double2*>(crow + j);
            cv.x -= v0;
            cv.y -= v1;
            *reinterpret_cast<double2*>(crow + j) = cv;
          } else {
            if (ok0) crow[j] -= v0;
            if (ok1) crow[j + 1] -= v1;
          }
        }
      }
    }
  }
  cp_async_wait<0>();
}

// The wide-tile configurations: 128 x 128 (8 warps of 64 x 32, 3 stages,
// one CTA per SM) and 64 x 128 (4 warps of 32 x 64, 2 stages, two CTAs per
// SM so one CTA's barrier waits and epilogue overlap the other's MMAs).
using WideSquare = Wide<128, 128, 64, 32, 3>;
using WideHalf = Wide<64, 128, 32, 64, 2>;
// 64 x 64 tiles, 4 warps of 32 x 32, k chunks of 16 in a 3-stage ring
// (56.8 KB of shared memory: four CTAs, 16 warps, per SM) or of 8 in a
// 4-stage ring (42 KB, 94 registers: five CTAs, 20 warps, per SM)
using WideS3 = Wide<64, 64, 32, 32, 3, 16, 4>;
using WideS4 = Wide<64, 64, 32, 32, 4, 8, 5>;

// ---------------------------------------------------------------------------
// SIMT tiles: reference-ordered FP64 and FP32.  256 threads, 4x4 per thread.
// ---------------------------------------------------------------------------
constexpr int kThreadsSimt = 256;
constexpr int kSK = 16;  // k chunk

template <typename T, bool kOrdered>
__device__ void simt_tile(const UpdArgs& U, T* as, T* bs, int I, int J) {
  // as[kSK][kBM], bs[kSK][kBN]
  const int i0 = U.tile_i0 + I * kBM, j0 = U.tile_j0 + J * kBN;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  T acc[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[r][c] = T(0);
  for (int k0 = 0; k0 < U.inner; k0 += kSK) {
    for (int c = threadIdx.x; c < kSK * kBM; c += kThreadsSimt) {
      const int kk = c / kBM, ii = c % kBM;
      const int i = i0 + ii, k = k0 + kk;
      const bool ok = k < U.inner && i >= U.i_lo && i < U.i_hi;
      as[kk * kBM + ii] =
          ok ? T(U.a[static_cast<long long>(i) * U.a_si + static_cast<long long>(k) * U.a_sk]) : T(0);
    }
    for (int c = threadIdx.x; c < kSK * kBN; c += kThreadsSimt) {
      const int kk = c / kBN, jj = c % kBN;
      const int j = j0 + jj, k = k0 + kk;
      const bool ok = k < U.inner && j >= U.j_lo && j < U.j_hi;
      bs[kk * kBN + jj] = ok ? T(U.b[static_cast<long long>(k) * U.b_sk + j]) : T(0);
    }
    __syncthreads();
    const int kmax = min(kSK, U.inner - k0);
    for (int kk = 0; kk < kmax; ++kk) {
      T av[4], bv[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) av[r] = as[kk * kBM + ty + 16 * r];
#pragma unroll
      for (int c = 0; c < 4; ++c) bv[c] = bs[kk * kBN + tx + 16 * c];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          if (kOrdered) {
            acc[r][c] = xadd(acc[r][c], xmul(av[r], bv[c]));
          } else {
            acc[r][c] = fmaf(av[r], bv[c], acc[r][c]);
          }
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int i = i0 + ty + 16 * r;
    if (i < U.i_lo || i >= U.i_hi) continue;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int j = j0 + tx + 16 * c;
      if (j < U.j_lo || j >= U.j_hi || (U.upper_only && i > j)) continue;
      double* p = U.c + static_cast<long long>(i) * U.ldc + j;
      if (kOrdered) {
        *p = xsub(*p, acc[r][c]);
      } else {
        *p = *p - static_cast<double>(acc[r][c]);
      }
    }
  }
}

template <typename T, bool kOrdered>
__global__ void __launch_bounds__(kThreadsSimt) simt_update_kernel(UpdArgs U) {
  __shared__ T as[kSK * kBM];
  __shared__ T bs[kSK * kBN];
  if (!resolve_range(U)) return;
  const int ntiles = tile_count(U);
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    int I, J;
    tile_coords(U, t, I, J);
    simt_tile<T, kOrdered>(U, as, bs, I, J);
  }
}

// MMA shape of the tensor-core update: m16n8k8 by default; BBK_UPDATE_K16=1
// selects m16n8k16 (tuning; the same speed on this part).
bool use_k16() {
  static const bool v = [] {
    const char* e = getenv("BBK_UPDATE_K16");
    return e ? atoi(e) != 0 : false;
  }();
  return v;
}

// Tile shape of the FP64 tensor-core update for large trailing matrices:
// by default 64 x 64 tiles in the 4-stage ring of k chunks of 8 (five CTAs
// per SM; n=40000: 27.9 TFLOP/s, against 26.9 for the 3-stage ring of 16
// and 25.7 for the two-stage 64 x 64 kernel).  BBK_UPDATE_TILE (tuning) =
// 64 (the two-stage 64 x 64 kernel everywhere), 128 (128 x 128), 64x128,
// 64s3 or 64s4 (the default).
int wide_tile_choice() {
  static const int v = [] {
    const char* e = getenv("BBK_UPDATE_TILE");
    if (!e) return 4;
    if (std::strcmp(e, "64") == 0) return 0;
    if (std::strcmp(e, "128") == 0) return 1;
    if (std::strcmp(e, "64x128") == 0) return 2;
    if (std::strcmp(e, "64s3") == 0) return 3;
    return 4;
  }();
  return v;
}

// Launches the wide-tile kernel `choice` (1: 128 x 128, 2: 64 x 128) for U
// when its upper triangle has at least two tiles per resident CTA; returns
// false (nothing launched) otherwise.
int launch_wide(const UpdArgs& U, int choice, long long order, bool* launched, cudaStream_t s) {
  *launched = false;
  const int sms = device_sm_count();
  const long long tn = choice >= 3 ? (order + 63) / 64 : (order + 127) / 128;
  const int per_sm = choice == 1 ? 1 : choice == 3 ? 4 : choice == 4 ? 5 : 2;
  const long long tiles = (choice == 2 ? 2 : 1) * tn * (tn + 1) / 2;
  if (choice == 0 || tiles < 2LL * per_sm * sms) return BBK_OK;
  static std::once_flag attr_once[4][64];
  int dev = 0;
  BBK_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return set_error(BBK_ERR_NO_DEVICE, "device %d out of range", dev);
  cudaError_t attr_err = cudaSuccess;
  const int grid = static_cast<int>(std::min<long long>(tiles, static_cast<long long>(per_sm) * sms));
  if (choice == 1) {
    auto fn = mma_update_wide_kernel<128, 128, 64, 32, 3>;
    std::call_once(attr_once[0][dev], [&] {
      attr_err = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(WideSquare::kBytes));
    });
    BBK_CUDA_TRY(attr_err);
    fn<<<grid, WideSquare::kThreads, WideSquare::kBytes, s>>>(U);
  } else if (choice == 2) {
    auto fn = mma_update_wide_kernel<64, 128, 32, 64, 2>;
    std::call_once(attr_once[1][dev], [&] {
      attr_err = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(WideHalf::kBytes));
    });
    BBK_CUDA_TRY(attr_err);
    fn<<<grid, WideHalf::kThreads, WideHalf::kBytes, s>>>(U);
  } else if (choice == 4) {
    auto fn = mma_update_wide_kernel<64, 64, 32, 32, 4, 8, 5>;
    std::call_once(attr_once[3][dev], [&] {
      attr_err = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(WideS4::kBytes));
    });
    BBK_CUDA_TRY(attr_err);
    fn<<<grid, WideS4::kThreads, WideS4::kBytes, s>>>(U);
  } else {
    auto fn = mma_update_wide_kernel<64, 64, 32, 32, 3, 16, 4>;
    std::call_once(attr_once[2][dev], [&] {
      attr_err = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(WideS3::kBytes));
    });
    BBK_CUDA_TRY(attr_err);
    fn<<<grid, WideS3::kThreads, WideS3::kBytes, s>>>(U);
  }
  BBK_CUDA_TRY(cudaGetLastError());
  count_launch();
  *launched = true;
  return BBK_OK;
}

template <bool kAK, bool kVec>
int launch_mma(const UpdArgs& U, int grid, cudaStream_t s) {
  const size_t bytes = MmaSmem<kAK>::kBytes;
  auto fn = use_k16() ? mma_update_kernel<kAK, kVec, true> : mma_update_kernel<kAK, kVec, false>;
  BBK_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(bytes)));
  fn<<<grid, kThreadsMma, bytes, s>>>(U);
  BBK_CUDA_TRY(cudaGetLastError());
  count_launch();
  return BBK_OK;
}

__global__ void block_scale_kernel(UpdArgs U, double* a_scale, double* b_scale);

// ---------------------------------------------------------------------------
// BF16 update of the factorization, split once per panel.  split_kernel
// writes the panel's operands, scaled by the 64-block powers of two, as
// kTerms BF16 terms in global memory, k contiguous and zero-padded to kpad:
//   ah[t][(i - tile_i0) * kpad + k]  = term t of a_scale(i) * U(i, k)
//   bh[t][(j - tile_i0) * kpad + k]  = term t of b_scale(j) * W(k, j)
// (rows outside [i_lo, n) and k >= inner are zero), so the tile kernel only
// loads BF16 and issues MMAs: converting in its inner loop put an FP64
// multiply and an FP64 -> FP32 conversion per operand per warp on the FP64
// pipe, which then limited the tensor cores.
// ---------------------------------------------------------------------------
constexpr int kSplitTile = 32;

template <int kTerms>
__global__ void __launch_bounds__(256) split_kernel(UpdArgs U, __nv_bfloat16* ah, __nv_bfloat16* bh, int kpad,
                                                    size_t term_stride) {
  __shared__ double tile[kSplitTile][kSplitTile + 1];
  if (!resolve_range(U)) return;
  const int rows = U.n - U.tile_i0;
  const int rt = (rows + kSplitTile - 1) / kSplitTile, kt = kpad / kSplitTile;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
  for (int blk = blockIdx.x; blk < 2 * rt * kt; blk += gridDim.x) {
    const bool is_a = blk < rt * kt;
    const int b2 = is_a ? blk : blk - rt * kt;
    const int r0 = (b2 / kt) * kSplitTile, k0 = (b2 % kt) * kSplitTile;
    // load the 32 x 32 block (rows r0.., k k0..) scaled; A reads along k, B along the rows
    for (int yy = ty; yy < kSplitTile; yy += 8) {
      int r, k;
      if (is_a) {
        r = r0 + yy;
        k = k0 + tx;
      } else {
        r = r0 + tx;
        k = k0 + yy;
      }
      const int c = U.tile_i0 + r;
      double v = 0.0;
      if (r < rows && c >= U.i_lo && k < U.inner) {
        const double sc = (is_a ? U.a_scale : U.b_scale)[r / kBM];
        v = sc * (is_a ? U.a[static_cast<long long>(c) * U.a_si + k] : U.b[static_cast<long long>(k) * U.b_sk + c]);
      }
      if (is_a)
        tile[yy][tx] = v;  // [row][k]
      else
        tile[tx][yy] = v;  // [row][k]
    }
    __syncthreads();
    __nv_bfloat16* dst = is_a ? ah : bh;
    for (int yy = ty; yy < kSplitTile; yy += 8) {
      const int r = r0 + yy, k = k0 + tx;
      if (r < rows) {
        float rest = static_cast<float>(tile[yy][tx]);
#pragma unroll
        for (int t = 0; t < kTerms; ++t) {
          const __nv_bfloat16 h = __float2bfloat16_rn(rest);
          dst[t * term_stride + static_cast<size_t>(r) * kpad + k] = h;
          rest -= __bfloat162float(h);
        }
      }
    }
    __syncthreads();
  }
}

constexpr int kHPitch = kBK + 8;  // BF16 per smem row: 20 words, conflict-free fragment loads

template <int kTerms>
struct HSmem {
  static constexpr int kOp = kTerms * kBM * kHPitch;  // one operand of one stage
  static constexpr int kStage = 2 * kOp;
  static constexpr size_t kBytes = 2 * kStage * sizeof(__nv_bfloat16);
};

__device__ __forceinline__ void cp_async_16h(__nv_bfloat16* smem_dst, const __nv_bfloat16* gsrc, bool valid) {
  const unsigned saddr = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(saddr), "l"(gsrc), "r"(valid ? 16 : 0)
               : "memory");
}

template <int kTerms>
__device__ __forceinline__ void load_stage_h(const UpdArgs& U, const __nv_bfloat16* ah, const __nv_bfloat16* bh,
                                             int kpad, size_t term_stride, __nv_bfloat16* st, int i0, int j0,
                                             int k0) {
  using Hs = HSmem<kTerms>;
  const int rows = U.n - U.tile_i0;
  constexpr int kChunks = kBM * (kBK / 8);  // 16-byte chunks per operand per term
  for (int c = threadIdx.x; c < 2 * kTerms * kChunks; c += kThreadsMma) {
    const int op = c / (kTerms * kChunks);
    const int rem = c - op * (kTerms * kChunks);
    const int t = rem / kChunks, q = rem - t * kChunks;
    const int rr = q / (kBK / 8), kk = (q % (kBK / 8)) * 8;
    const int r = (op == 0 ? i0 : j0) - U.tile_i0 + rr;
    const bool ok = r < rows;
    const __nv_bfloat16* src = (op == 0 ? ah : bh) + t * term_stride +
                               static_cast<size_t>(ok ? r : 0) * kpad + k0 + kk;
    cp_async_16h(st + op * Hs::kOp + (t * kBM + rr) * kHPitch + kk, src, ok);
  }
}

template <int kTerms>
__global__ void __launch_bounds__(kThreadsMma) bf16s_update_kernel(UpdArgs U, const __nv_bfloat16* ah,
                                                                   const __nv_bfloat16* bh, int kpad,
                                                                   size_t term_stride, int vec) {
  using Hs = HSmem<kTerms>;
  extern __shared__ __align__(16) __nv_bfloat16 hsm[];
  if (!resolve_range(U)) return;
  const int ntiles = tile_count(U);
  int t = blockIdx.x;
  if (t >= ntiles) return;
  const int nchunks = (U.inner + kBK - 1) / kBK;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, tq = lane & 3;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  __nv_bfloat16* stage[2] = {hsm, hsm + Hs::kStage};
  int I, J;
  tile_coords(U, t, I, J);
  int i0 = U.tile_i0 + I * kBM, j0 = U.tile_j0 + J * kBN;
  load_stage_h<kTerms>(U, ah, bh, kpad, term_stride, stage[0], i0, j0, 0);
  cp_async_commit();
  int cur = 0;
  for (;;) {
    float acc[2][4][4];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.0f;
    for (int ch = 0; ch < nchunks; ++ch) {
      const int nxt = cur ^ 1;
      if (ch + 1 < nchunks) {
        load_stage_h<kTerms>(U, ah, bh, kpad, term_stride, stage[nxt], i0, j0, (ch + 1) * kBK);
        cp_async_commit();
        cp_async_wait<1>();
      } else {
        cp_async_wait<0>();
      }
      __syncthreads();  // chunk ch is in stage[cur]
      const __nv_bfloat16* as = stage[cur];
      const __nv_bfloat16* bs = stage[cur] + Hs::kOp;
#pragma unroll
      for (int ks = 0; ks < kBK; ks += 16) {
        unsigned af[kTerms][2][4], bf[kTerms][4][2];
#pragma unroll
        for (int tt = 0; tt < kTerms; ++tt) {
#pragma unroll
          for (int mt = 0; mt < 2; ++mt)
#pragma unroll
            for (int u = 0; u < 4; ++u) {
              const int rr = wm + mt * 16 + g + 8 * (u & 1), kk = ks + 2 * tq + 8 * (u >> 1);
              af[tt][mt][u] = *reinterpret_cast<const unsigned*>(as + (tt * kBM + rr) * kHPitch + kk);
            }
#pragma unroll
          for (int nt = 0; nt < 4; ++nt)
#pragma unroll
            for (int u = 0; u < 2; ++u) {
              const int cc = wn + nt * 8 + g, kk = ks + 2 * tq + 8 * u;
              bf[tt][nt][u] = *reinterpret_cast<const unsigned*>(bs + (tt * kBM + cc) * kHPitch + kk);
            }
        }
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
          for (int nt = 0; nt < 4; ++nt) {
            // smallest products first
#pragma unroll
            for (int ia = kTerms - 1; ia >= 0; --ia)
#pragma unroll
              for (int ib = kTerms - 1; ib >= 0; --ib)
                if (ia + ib <= kTerms - 1) mma_bf16_16x8x16(acc[mt][nt], af[ia][mt], bf[ib][nt]);
          }
      }
      __syncthreads();  // every warp is done with stage[cur]
      if (ch + 1 < nchunks) cur = nxt;
    }
    // prefetch the next tile's first chunk while this tile's C is updated
    const int tn = t + static_cast<int>(gridDim.x);
    int ni0 = 0, nj0 = 0;
    if (tn < ntiles) {
      int nI, nJ;
      tile_coords(U, tn, nI, nJ);
      ni0 = U.tile_i0 + nI * kBM;
      nj0 = U.tile_j0 + nJ * kBN;
      load_stage_h<kTerms>(U, ah, bh, kpad, term_stride, stage[cur ^ 1], ni0, nj0, 0);
      cp_async_commit();
    }
    const double unscale = 1.0 / (U.a_scale[(i0 - U.tile_i0) / kBM] * U.b_scale[(j0 - U.tile_j0) / kBN]);
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int i = i0 + wm + mt * 16 + g + h * 8;
        if (i < U.i_lo || i >= U.i_hi) continue;
        double* crow = U.c + static_cast<long long>(i) * U.ldc;
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
          const int j = j0 + wn + nt * 8 + tq * 2;
          const double v0 = static_cast<double>(acc[mt][nt][h * 2]) * unscale;
          const double v1 = static_cast<double>(acc[mt][nt][h * 2 + 1]) * unscale;
          const bool ok0 = j >= U.j_lo && j < U.j_hi && (!U.upper_only || i <= j);
          const bool ok1 = j + 1 >= U.j_lo && j + 1 < U.j_hi && (!U.upper_only || i <= j + 1);
          if (vec && ok0 && ok1) {
            double2 cv = *reinterpret_cast<const double2*>(crow + j);
            cv.x -= v0;
            cv.y -= v1;
            *reinterpret_cast<double2*>(crow + j) = cv;
          } else {
            if (ok0) crow[j] -= v0;
            if (ok1) crow[j + 1] -= v1;
          }
        }
      }
    }
    if (tn >= ntiles) break;
    cur ^= 1;
    t = tn;
    i0 = ni0;
    j0 = nj0;
  }
  cp_async_wait<0>();
}

// The split operands in the tensor core's shared-memory order, for the
// tcgen05 update: rows relative to t_i0 (the 128-aligned row at or below the
// trailing matrix), in blocks of 128 rows x 16 k (2048 BF16 = 4 KB each,
// block (rb, kc) at (rb * kpad / 16 + kc) * 2048), and inside a block the
// K-major core-matrix layout the UMMA descriptors describe: element (r, k)
// at (r / 8) * 128 + (k / 8) * 64 + (r % 8) * 8 + k % 8.  One bulk copy moves
// a block into shared memory.  Rows outside [e, n) and k >= inner are zero.
constexpr int kBlkRows = 128, kBlkK = 16, kBlkElems = kBlkRows * kBlkK;

__device__ __forceinline__ size_t blocked_offset(int r, int k, int nkc) {
  return static_cast<size_t>((r / kBlkRows) * nkc + k / kBlkK) * kBlkElems +
         ((r % kBlkRows) / 8) * 128 + ((k % kBlkK) / 8) * 64 + (r % 8) * 8 + (k % 8);
}

template <int kTerms>
__global__ void __launch_bounds__(256) split_blocked_kernel(UpdArgs U, __nv_bfloat16* ah, __nv_bfloat16* bh,
                                                            int kpad, size_t term_stride) {
  __shared__ double tile[kSplitTile][kSplitTile + 1];
  if (!resolve_range(U)) return;  // U.tile_i0: the 64-aligned origin of the scales
  const int t_i0 = (U.i_lo / kBlkRows) * kBlkRows;
  const int rows = ((U.n - t_i0 + kBlkRows - 1) / kBlkRows) * kBlkRows;  // whole 128-row blocks
  const int rt = rows / kSplitTile, kt = kpad / kSplitTile, nkc = kpad / kBlkK;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
  for (int blk = blockIdx.x; blk < 2 * rt * kt; blk += gridDim.x) {
    const bool is_a = blk < rt * kt;
    const int b2 = is_a ? blk : blk - rt * kt;
    const int r0 = (b2 / kt) * kSplitTile, k0 = (b2 % kt) * kSplitTile;
    // the 32 x 32 block (rows r0.., k k0..), scaled; A read along k, B along the rows
    for (int yy = ty; yy < kSplitTile; yy += 8) {
      int r, k;
      if (is_a) {
        r = r0 + yy;
        k = k0 + tx;
      } else {
        r = r0 + tx;
        k = k0 + yy;
      }
      const int c = t_i0 + r;
      double v = 0.0;
      if (c >= U.i_lo && c < U.n && k < U.inner) {
        const double sc = (is_a ? U.a_scale : U.b_scale)[(c - U.tile_i0) / kBM];
        v = sc * (is_a ? U.a[static_cast<long long>(c) * U.a_si + k] : U.b[static_cast<long long>(k) * U.b_sk + c]);
      }
      if (is_a)
        tile[yy][tx] = v;  // [row][k]
      else
        tile[tx][yy] = v;
    }
    __syncthreads();
    __nv_bfloat16* dst = is_a ? ah : bh;
    for (int yy = ty; yy < kSplitTile; yy += 8) {
      const int r = r0 + yy, k = k0 + tx;
      float rest = static_cast<float>(tile[yy][tx]);
      const size_t off = blocked_offset(r, k, nkc);
#pragma unroll
      for (int t = 0; t < kTerms; ++t) {
        const __nv_bfloat16 h = __float2bfloat16_rn(rest);
        dst[t * term_stride + off] = h;
        rest -= __bfloat162float(h);
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// BF16 update on the 5th-generation tensor cores (tcgen05 / UMMA).
//
// The split operands (split_blocked_kernel: kTerms scaled BF16 terms per
// operand, stored in 4 KB blocks already in the shared-memory order of the
// UMMA descriptors: no-swizzle K-major core matrices of 8 rows x 16 bytes,
// 128 bytes apart along k and 256 bytes apart along the rows) are moved into
// shared memory by bulk asynchronous copies, one per block, and one thread
// issues tcgen05.mma.kind::f16 (M = N = 128, K = 16) for every product
// t_a(A) t_b(B), a + b < kTerms, smallest first, into an FP32 accumulator in
// tensor memory (128 lanes x 128 columns).  Completion is tracked by
// mbarriers (transaction bytes for the copies, tcgen05.commit for the MMAs);
// every wait is bounded and a wait that runs out aborts the factorization
// with BBK_ERR_TIMEOUT.  The epilogue reads an accumulator with tcgen05.ld
// (warp w: lanes 32w.., one C row per thread), unscales it and subtracts it
// from the FP64 trailing matrix, while the other accumulator takes the next
// tile's MMAs.  Two CTAs per SM.
// ---------------------------------------------------------------------------
constexpr int kUM = 128, kUN = 128;  // C tile


// Per term count: the k chunk (BF16 elements) and the stages, sized so that
// two CTAs fit one SM with the same bytes in flight (three terms: more,
// shorter stages, so a stage is refilled soon after its MMAs finish).
template <int kTerms>
struct USmem {
  static constexpr int kK = kBlkK;
  static constexpr int kOpBytes = kUM * kK * 2;  // one term of one operand per stage: one 4 KB block
  static constexpr int kRowGroup = (kK / 8) * 128;  // bytes between 8-row core-matrix groups
  static constexpr int kStageBytes = 2 * kTerms * kOpBytes;
  static constexpr int kStages = kTerms == 3 ? 4 : 8;
  // stages, then the barriers (2 x kStages + 4) and the accumulator address
  static constexpr size_t kBytes = static_cast<size_t>(kStages) * kStageBytes + 256;
  static_assert((2 * kStages + 4) * 8 + 4 <= 256, "barrier area");
};
static_assert(2 * USmem<3>::kBytes + 2048 <= 228 * 1024, "two CTAs per SM");

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor, SWIZZLE_NONE K-major: start address,
// leading (k-direction, 128 B) and stride (row-direction) byte offsets,
// version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t sbo) {
  constexpr uint64_t kLbo = 128 >> 4;
  return (static_cast<uint64_t>((saddr >> 4) & 0x3FFF)) | (kLbo << 16) |
         (static_cast<uint64_t>(sbo >> 4) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulate, BF16 A and B, both
// K-major, N = 128, M = 128.
constexpr uint32_t kUIdesc = (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(kUN >> 3) << 17) |
                             (static_cast<uint32_t>(kUM >> 4) << 24);

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(kUIdesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void umma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t mbar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(done)
      : "r"(mbar), "r"(parity)
      : "memory");
  return done != 0;
}

// Bounded wait for phase `parity` of mbarrier `mbar`: false when it ran out
// (or another kernel of the factorization aborted).
__device__ bool mbar_wait(uint32_t mbar, uint32_t parity, const DeviceState* st, unsigned long long timeout_ns) {
  unsigned long long t0 = 0;
  for (unsigned it = 1;; ++it) {
    if (mbar_try(mbar, parity)) return true;
    if ((it & 63u) == 0) {
      const unsigned long long now = globaltimer_ns();
      if (t0 == 0) t0 = now;
      if (now - t0 > timeout_ns || ld_relaxed_s32(&st->abort)) return false;
    }
  }
}

// Roles (warp-specialized, no CTA barrier inside the main loop):
//   warps 0-3   epilogue: wait until an accumulator is full, read it with
//               tcgen05.ld (warp w: lanes 32w..32w+31, one C row per
//               thread), C -= unscale * acc, then mark the accumulator empty;
//   warp 4      lane 0 moves the next chunk into a free stage with bulk
//               asynchronous copies (one 4 KB block per operand and term,
//               split_blocked_kernel's layout) that complete the stage's
//               "full" barrier;
//   warp 5      lane 0 issues the MMAs of each full stage, commits them to
//               the stage's "empty" barrier and, after a tile's last chunk,
//               to the accumulator's "full" barrier.
// Two accumulators (2 x 128 TMEM columns) let the epilogue of one tile run
// while the next tile's MMAs execute.
constexpr int kUEpi = 4, kUProd = 1;
constexpr int kUWarps = kUEpi + kUProd + 1;
constexpr int kUBlock = kUWarps * 32;

__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
}

template <int kTerms>
__global__ void __launch_bounds__(kUBlock, 2) umma_bf16s_update_kernel(UpdArgs U, const __nv_bfloat16* ah,
                                                                       const __nv_bfloat16* bh, int kpad,
                                                                       size_t term_stride,
                                                                       unsigned long long timeout_ns) {
  using S = USmem<kTerms>;
  constexpr int kUK = S::kK;
  constexpr int kUOpBytes = S::kOpBytes;
  extern __shared__ __align__(1024) unsigned char usm[];
  uint64_t* full = reinterpret_cast<uint64_t*>(usm + S::kStages * S::kStageBytes);
  uint64_t* empty = full + S::kStages;
  uint64_t* accfull = empty + S::kStages;  // 2
  uint64_t* accempty = accfull + 2;        // 2
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(accempty + 2);
  // the panel's range (the split operands start at split_i0, the 64-aligned
  // row at or below the trailing matrix; tiles here are 128-aligned)
  if (ld_relaxed_s32(&U.st->abort)) return;
  const int k0p = ldcg(&U.st->kstart[U.panel & 1]);
  const int e = ldcg(&U.st->kstart[(U.panel + 1) & 1]);
  const int inner = e - k0p;
  if (inner <= 0 || e >= U.n) return;
  const int split_i0 = (e / kBM) * kBM;
  const int t_i0 = (e / kUM) * kUM;
  const int tm = (U.n - t_i0 + kUM - 1) / kUM;
  const int ntiles = tm * (tm + 1) / 2;
  if (static_cast<int>(blockIdx.x) >= ntiles) return;
  const int nchunks = (inner + kUK - 1) / kUK;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int my_tiles = (ntiles - static_cast<int>(blockIdx.x) + static_cast<int>(gridDim.x) - 1) /
                       static_cast<int>(gridDim.x);

  if (warp == kUWarps - 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(2 * kUN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    if (lane == 0) {
      for (int st = 0; st < S::kStages; ++st) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&full[st])) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&empty[st])) : "memory");
      }
      for (int b = 0; b < 2; ++b) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&accfull[b])) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&accempty[b])), "r"(kUEpi)
                     : "memory");
      }
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  auto tile_of = [&](int t, int& i0, int& j0) {
    int j = static_cast<int>((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
    while (j > 0 && j * (j + 1) / 2 > t) --j;
    while ((j + 1) * (j + 2) / 2 <= t) ++j;
    i0 = t_i0 + (t - j * (j + 1) / 2) * kUM;
    j0 = t_i0 + j * kUN;
  };
  bool ok = true;

  if (warp == kUEpi) {
    // ---- producer: one thread moves each stage's 2 x kTerms blocks with
    // bulk asynchronous copies that complete the stage's "full" barrier
    if (lane == 0) {
      const int nkc = kpad / kBlkK;
      long long item = 0;
      for (int m = 0; m < my_tiles && ok; ++m) {
        int i0, j0;
        tile_of(static_cast<int>(blockIdx.x) + m * static_cast<int>(gridDim.x), i0, j0);
        const int rba = (i0 - t_i0) / kBlkRows, rbb = (j0 - t_i0) / kBlkRows;
        for (int ch = 0; ch < nchunks; ++ch, ++item) {
          const int st = static_cast<int>(item % S::kStages);
          const long long use = item / S::kStages;
          if (use >= 1 &&
              !mbar_wait(smem_u32(&empty[st]), static_cast<uint32_t>((use - 1) & 1), U.st, timeout_ns)) {
            ok = false;
            break;
          }
          const uint32_t fb = smem_u32(&full[st]);
          asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(fb), "r"(S::kStageBytes)
                       : "memory");
          const uint32_t base = smem_u32(usm + st * S::kStageBytes);
          for (int blk = 0; blk < 2 * kTerms; ++blk) {
            const int op = blk / kTerms, term = blk - op * kTerms;
            const __nv_bfloat16* src = (op == 0 ? ah : bh) + term * term_stride +
                                       static_cast<size_t>((op == 0 ? rba : rbb) * nkc + ch) * kBlkElems;
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    base + blk * kUOpBytes),
                "l"(src), "r"(kUOpBytes), "r"(fb)
                : "memory");
          }
        }
      }
    }
  } else if (warp == kUWarps - 1) {
    // ---- MMA issue (one thread)
    if (lane == 0) {
      long long item = 0;
      long long committed = -1;  // last stage commit
      int acc_commits = 0;       // accumulator commits issued
      for (int m = 0; m < my_tiles && ok; ++m) {
        const int b = m & 1, v = m >> 1;
        if (v >= 1 && !mbar_wait(smem_u32(&accempty[b]), static_cast<uint32_t>((v - 1) & 1), U.st, timeout_ns)) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t acc = tmem + static_cast<uint32_t>(b * kUN);
        for (int ch = 0; ch < nchunks; ++ch, ++item) {
          const int st = static_cast<int>(item % S::kStages);
          if (!mbar_wait(smem_u32(&full[st]), static_cast<uint32_t>((item / S::kStages) & 1), U.st, timeout_ns)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t sb = smem_u32(usm + st * S::kStageBytes);
          for (int ia = kTerms - 1; ia >= 0; --ia)
            for (int ib = kTerms - 1 - ia; ib >= 0; --ib) {
              const uint32_t a0 = sb + ia * kUOpBytes, b0 = sb + (kTerms + ib) * kUOpBytes;
#pragma unroll
              for (int ks = 0; ks < kUK / 16; ++ks) {
                const bool first = ch == 0 && ks == 0 && ia == kTerms - 1 && ib == kTerms - 1 - ia;
                umma_bf16(acc, umma_desc(a0 + ks * 256, S::kRowGroup), umma_desc(b0 + ks * 256, S::kRowGroup),
                          first ? 0u : 1u);
              }
            }
          umma_commit(smem_u32(&empty[st]));
          committed = item;
        }
        if (!ok) break;
        umma_commit(smem_u32(&accfull[b]));
        ++acc_commits;
      }
      if (!ok && committed >= 0) {
        // let the MMAs already issued finish before the accumulators are released
        const uint32_t mb = smem_u32(&empty[committed % S::kStages]);
        const uint32_t par = static_cast<uint32_t>((committed / S::kStages) & 1);
        const unsigned long long t0 = globaltimer_ns();
        while (!mbar_try(mb, par) && globaltimer_ns() - t0 < timeout_ns) {
        }
      }
      (void)acc_commits;
    }
  } else {
    // ---- epilogue
    for (int m = 0; m < my_tiles && ok; ++m) {
      const int b = m & 1, v = m >> 1;
      int i0, j0;
      tile_of(static_cast<int>(blockIdx.x) + m * static_cast<int>(gridDim.x), i0, j0);
      const int i = i0 + warp * 32 + lane;  // this thread's row of the tile
      const bool row_ok = i >= e && i < U.n;
      if (row_ok) {
        const double* row = U.c + static_cast<long long>(i) * U.ldc;
        for (int jc = max(j0, i) & ~15; jc < min(j0 + kUN, U.n); jc += 16)
          asm volatile("prefetch.global.L2 [%0];" ::"l"(row + jc));
      }
      if (!mbar_wait(smem_u32(&accfull[b]), static_cast<uint32_t>(v & 1), U.st, timeout_ns)) {
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int is = min(max(i, split_i0), U.n - 1);  // scale block of a row inside the matrix
      const double sa = U.a_scale[(is - split_i0) / kBM];
      double* crow = U.c + static_cast<long long>(is) * U.ldc;
      // C values of the 8-column group at c0 (entries this thread does not
      // update read as 0); the next group's load is in flight while a group
      // is updated
      auto load_c = [&](int c0, double (&cv)[8]) {
#pragma unroll
        for (int u = 0; u < 8; u += 2) {
          const int j = j0 + c0 + u;
          const bool ok0 = row_ok && j >= e && j < U.n && i <= j;
          const bool ok1 = row_ok && j + 1 >= e && j + 1 < U.n && i <= j + 1;
          if (ok0 && ok1) {
            const double2 t = *reinterpret_cast<const double2*>(crow + j);
            cv[u] = t.x;
            cv[u + 1] = t.y;
          } else {
            cv[u] = ok0 ? crow[j] : 0.0;
            cv[u + 1] = ok1 ? crow[j + 1] : 0.0;
          }
        }
      };
      double cur[8], nxt[8];
      load_c(0, cur);
      const uint32_t tacc = tmem + static_cast<uint32_t>(b * kUN) + (static_cast<uint32_t>(warp * 32) << 16);
#pragma unroll 1
      for (int c0 = 0; c0 < kUN; c0 += 8) {
        uint32_t r[8];
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                     : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                       "=r"(r[7])
                     : "r"(tacc + static_cast<uint32_t>(c0)));
        if (c0 + 8 < kUN) load_c(c0 + 8, nxt);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        const int jb = j0 + c0;
        const int js = min(max(jb, split_i0), U.n - 1);
        const double unscale = 1.0 / (sa * U.b_scale[(js - split_i0) / kBM]);
        if (row_ok) {
#pragma unroll
          for (int u = 0; u < 8; u += 2) {
            const int j = jb + u;
            const double v0 = cur[u] - static_cast<double>(__uint_as_float(r[u])) * unscale;
            const double v1 = cur[u + 1] - static_cast<double>(__uint_as_float(r[u + 1])) * unscale;
            const bool ok0 = j >= e && j < U.n && i <= j;
            const bool ok1 = j + 1 >= e && j + 1 < U.n && i <= j + 1;
            if (ok0 && ok1) {
              *reinterpret_cast<double2*>(crow + j) = make_double2(v0, v1);
            } else {
              if (ok0) crow[j] = v0;
              if (ok1) crow[j + 1] = v1;
            }
          }
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) cur[u] = nxt[u];
      }
      // this warp is done reading the accumulator
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&accempty[b]));
    }
  }
  if (!ok) {
    atomicCAS(const_cast<int*>(&U.st->status), 0, BBK_ERR_TIMEOUT);
    atomicExch(const_cast<int*>(&U.st->abort), 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == kUWarps - 1)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * kUN) : "memory");
}

template <int kTerms>
int launch_umma_bf16(const UpdArgs& U, const __nv_bfloat16* ah, const __nv_bfloat16* bh, int kpad,
                     size_t term_stride, long long order, cudaStream_t s) {
  using S = USmem<kTerms>;
  static std::once_flag attr_once[64];
  int dev = 0;
  BBK_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return set_error(BBK_ERR_NO_DEVICE, "device %d out of range", dev);
  cudaError_t attr_err = cudaSuccess;
  std::call_once(attr_once[dev], [&] {
    attr_err = cudaFuncSetAttribute(umma_bf16s_update_kernel<kTerms>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(S::kBytes));
  });
  BBK_CUDA_TRY(attr_err);
  const long long tm = (order + kUM - 1) / kUM + 1;
  const long long tiles = tm * (tm + 1) / 2;
  const int grid = static_cast<int>(std::max(1LL, std::min<long long>(tiles, 2LL * device_sm_count())));
  umma_bf16s_update_kernel<kTerms><<<grid, kUBlock, S::kBytes, s>>>(U, ah, bh, kpad, term_stride,
                                                                    wait_timeout_ns());
  BBK_CUDA_TRY(cudaGetLastError());
  count_launch();
  return BBK_OK;
}

// BF16 updates on tcgen05 (default) or the warp-level MMA kernel
// (BBK_BF16_UMMA=0: comparison).
bool use_umma_bf16() {
  static const bool v = [] {
    const char* e = getenv("BBK_BF16_UMMA");
    return e ? atoi(e) != 0 : true;
  }();
  return v;
}

template <int kTerms>
int launch_bf16_split(const UpdArgs& U, __nv_bfloat16* buf, int kpad, size_t term_stride, int grid_mma, bool vec,
                      long long order, cudaStream_t s) {
  const int sms = device_sm_count();
  __nv_bfloat16* ah = buf;
  __nv_bfloat16* bh = buf + static_cast<size_t>(kTerms) * term_stride;
  if (vec && use_umma_bf16() && kpad % kBlkK == 0) {
    split_blocked_kernel<kTerms><<<4 * sms, 256, 0, s>>>(U, ah, bh, kpad, term_stride);
    BBK_CUDA_TRY(cudaGetLastError());
    count_launch();
    return launch_umma_bf16<kTerms>(U, ah, bh, kpad, term_stride, order, s);
  }
  split_kernel<kTerms><<<4 * sms, 256, 0, s>>>(U, ah, bh, kpad, term_stride);
  BBK_CUDA_TRY(cudaGetLastError());
  count_launch();
  const size_t bytes = HSmem<kTerms>::kBytes;
  static std::once_flag attr_once[64];
  int dev = 0;
  BBK_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return set_error(BBK_ERR_NO_DEVICE, "device %d out of range", dev);
  cudaError_t attr_err = cudaSuccess;
  std::call_once(attr_once[dev], [&] {
    attr_err = cudaFuncSetAttribute(bf16s_update_kernel<kTerms>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(bytes));
  });
  BBK_CUDA_TRY(attr_err);
  bf16s_update_kernel<kTerms><<<grid_mma, kThreadsMma, bytes, s>>>(U, ah, bh, kpad, term_stride, vec ? 1 : 0);
  BBK_CUDA_TRY(cudaGetLastError());
  count_launch();
  return BBK_OK;
}

int launch_by_mode(const UpdArgs& U, int mode, bool ak, bool vec, int grid_mma, int grid_simt,
                   cudaStream_t s) {
  switch (mode) {
    case BBK_UPDATE_FP64:
      if (ak && vec) return launch_mma<true, true>(U, grid_mma, s);
      if (ak) return launch_mma<true, false>(U, grid_mma, s);
      return launch_mma<false, false>(U, grid_mma, s);
    case BBK_UPDATE_FP64_ORDERED:
      simt_update_kernel<double, true><<<grid_simt, kThreadsSimt, 0, s>>>(U);
      break;
    case BBK_UPDATE_FP32:
      simt_update_kernel<float, false><<<grid_simt, kThreadsSimt, 0, s>>>(U);
      break;
    case BBK_UPDATE_BF16:
    case BBK_UPDATE_BF16X3: {
      if (!(ak && vec) || U.a_scale == nullptr)
        return set_error(BBK_ERR_INVALID_ARGUMENT, "BF16 update needs the factorization layout");
      const int sms = device_sm_count();
      block_scale_kernel<<<2 * sms, 256, 0, s>>>(U, const_cast<double*>(U.a_scale),
                                                  const_cast<double*>(U.b_scale));
      BBK_CUDA_TRY(cudaGetLastError());
      count_launch();
      const size_t bytes = MmaSmem<true>::kBytes;
      auto fn = mode == BBK_UPDATE_BF16 ? mma_update_kernel<true, true, false, 1>
                                        : mma_update_kernel<true, true, false, 3>;
      BBK_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(bytes)));
      fn<<<grid_mma, kThreadsMma, bytes, s>>>(U);
      break;
    }
    default:
      return set_error(BBK_ERR_INVALID_ARGUMENT, "unknown update mode %d", mode);
  }
  BBK_CUDA_TRY(cudaGetLastError());
  count_launch();
  return BBK_OK;
}

// Power-of-two scales for the BF16 update: for every 64-block of trailing
// columns, 2^-e with 2^e >= max |entry| over the panel's U rows (a_scale) and
// W rows (b_scale), so the scaled operands have magnitude <= 1.
__global__ void block_scale_kernel(UpdArgs U, double* a_scale, double* b_scale) {
  if (!resolve_range(U)) return;
  const int nblk = U.tiles_m;
  for (int blk = blockIdx.x; blk < 2 * nblk; blk += gridDim.x) {
    const bool is_a = blk < nblk;
    const int bi = is_a ? blk : blk - nblk;
    const int c0 = U.tile_i0 + bi * kBM;
    // consecutive threads walk the operand's contiguous direction (k for
    // the row-major A block, the column for B), four loads in flight each;
    // the maximum does not depend on the order
    double m = 0.0;
    const int total = kBM * U.inner;
    for (int base = threadIdx.x; base < total; base += 4 * blockDim.x) {
      double v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int idx = base + u * blockDim.x;
        v[u] = 0.0;
        if (idx < total) {
          const int cc = c0 + (is_a ? idx / U.inner : idx % kBM);
          const int k = is_a ? idx % U.inner : idx / kBM;
          if (cc >= U.i_lo && cc < U.n)
            v[u] = is_a ? U.a[static_cast<long long>(cc) * U.a_si + k] : U.b[static_cast<long long>(k) * U.b_sk + cc];
        }
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) m = fmax(m, fabs(v[u]));
    }
    for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, off));
    __shared__ double red[8];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int w = 1; w < static_cast<int>(blockDim.x >> 5); ++w) m = fmax(m, red[w]);
      m = fmax(m, red[0]);
      int e = 0;
      frexp(m, &e);  // m = f * 2^e, 0.5 <= f < 1
      const double sc = (m > 0.0 && isfinite(m)) ? ldexp(1.0, -e) : 1.0;
      (is_a ? a_scale : b_scale)[bi] = sc;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// kernels::ScaleOneByOnePivot / ScaleTwoByTwoPivot (src/kernels.cc:11-65)
// ---------------------------------------------------------------------------
__global__ void scale_1x1_kernel(int count, double pivot, const double* src, int ss, double* dst,
                                 int ds) {
  const bool zero = fabs(pivot) == 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    dst[static_cast<long long>(i) * ds] =
        zero ? 0.0 : xdiv(src[static_cast<long long>(i) * ss], pivot);
  }
}

__global__ void scale_2x2_kernel(int count, double a, double b, double c, const double* s1,
                                 int s1s, const double* s2, int s2s, double* d1, int d1s,
                                 double* d2, int d2s) {
  const double det = xsub(xmul(a, c), xmul(b, b));
  const bool zero = fabs(det) == 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const double x = s1[static_cast<long long>(i) * s1s];
    const double y = s2[static_cast<long long>(i) * s2s];
    // (x*c - y*b)/det and (-x*b + y*a)/det, as src/kernels.cc:57-63
    d1[static_cast<long long>(i) * d1s] = zero ? 0.0 : xdiv(xsub(xmul(x, c), xmul(y, b)), det);
    d2[static_cast<long long>(i) * d2s] = zero ? 0.0 : xdiv(xadd(xmul(-x, b), xmul(y, a)), det);
  }
}

}  // namespace

int launch_update(const FactorPlan& plan, int panel, cudaStream_t s) {
  if (panel + 1 >= plan.nb) return BBK_OK;  // nothing trails the last panel
  UpdArgs U{};
  U.a = plan.ucm;
  U.a_si = plan.ldu;
  U.a_sk = 1;
  U.b = plan.w;
  U.b_sk = plan.ldw;
  U.c = plan.a;
  U.ldc = plan.lda;
  U.upper_only = 1;
  U.triangular = 1;
  U.st = plan.state;
  U.panel = panel;
  U.n = plan.n;
  U.a_scale = plan.scales;
  U.b_scale = plan.scales ? plan.scales + (plan.n / kBM + 2) : nullptr;
  const int sms = device_sm_count();
  // tiles of the first trailing panel bound the work; persistent grid
  const long long nominal_e = std::max(0LL, static_cast<long long>(panel + 1) * plan.b - 1);
  const long long tm = (plan.n - (nominal_e / kBM) * kBM + kBM - 1) / kBM;
  const long long tiles = tm * (tm + 1) / 2;
  const int grid_mma = static_cast<int>(std::max(1LL, std::min<long long>(tiles, 3LL * sms)));
  const int grid_simt = static_cast<int>(std::max(1LL, std::min<long long>(tiles, 4LL * sms)));
  // vector path needs 16-byte aligned rows: ldu, ldw, lda even and a/c 16-byte aligned
  const bool vec = (plan.ldu % 2 == 0) && (plan.ldw % 2 == 0) && (plan.lda % 2 == 0) &&
                   (reinterpret_cast<uintptr_t>(plan.a) % 16 == 0);
  // BF16 modes: operands split once per panel (16-byte copies need the split
  // buffer 16-byte aligned; a caller's unaligned workspace keeps the
  // in-loop split)
  if ((plan.mode == BBK_UPDATE_BF16 || plan.mode == BBK_UPDATE_BF16X3) && plan.hsplit != nullptr &&
      reinterpret_cast<uintptr_t>(plan.hsplit) % 16 == 0 && vec) {
    if (U.a_scale == nullptr) return set_error(BBK_ERR_LOGIC, "BF16 update without its scales");
    block_scale_kernel<<<2 * sms, 256, 0, s>>>(U, const_cast<double*>(U.a_scale), const_cast<double*>(U.b_scale));
    BBK_CUDA_TRY(cudaGetLastError());
    count_launch();
    auto* buf = static_cast<__nv_bfloat16*>(plan.hsplit);
    return plan.mode == BBK_UPDATE_BF16
               ? launch_bf16_split<1>(U, buf, plan.kpad, plan.hstride, grid_mma, vec, plan.n - nominal_e, s)
               : launch_bf16_split<3>(U, buf, plan.kpad, plan.hstride, grid_mma, vec, plan.n - nominal_e, s);
  }
  if (plan.mode == BBK_UPDATE_FP64 && vec) {
    bool launched = false;
    const int rc = launch_wide(U, wide_tile_choice(), plan.n - nominal_e, &launched, s);
    if (rc || launched) return rc;
  }
  return launch_by_mode(U, plan.mode, true, vec, grid_mma, grid_simt, s);
}

// C(i, j) -= sum_k M(i, k) U(k, j) on the upper tiles (i <= j) of an n x n
// product, all three row-major with leading dimension ld (even, >= the
// order rounded up to 128, rows up to that bound readable): the
// reconstruction P^T L D L^T P runs this with M = L D, U = L^T and C = 0.
int launch_upper_product(int n, const double* m, const double* u, long long ld, double* c, cudaStream_t s) {
  UpdArgs U{};
  U.a = m;
  U.a_si = ld;
  U.a_sk = 1;
  U.b = u;
  U.b_sk = ld;
  U.c = c;
  U.ldc = ld;
  U.i_lo = U.j_lo = 0;
  U.i_hi = U.j_hi = n;
  U.inner = n;
  U.upper_only = 1;
  U.triangular = 1;
  U.tile_i0 = U.tile_j0 = 0;
  U.n = n;
  const int sms = device_sm_count();
  bool launched = false;
  const int rc = launch_wide(U, wide_tile_choice(), n, &launched, s);
  if (rc || launched) return rc;
  U.tiles_m = U.tiles_n = (n + kBM - 1) / kBM;
  const long long tiles = static_cast<long long>(U.tiles_m) * (U.tiles_m + 1) / 2;
  return launch_mma<true, true>(U, static_cast<int>(std::max(1LL, std::min<long long>(tiles, 3LL * sms))), s);
}

int launch_update_block(int rows, int cols, int inner, const double* left, int ls,
                        const double* ws, int wss, double* target, int ts, int mode,
                        cudaStream_t s) {
  if (rows <= 0 || cols <= 0 || inner <= 0) return BBK_OK;
  UpdArgs U{};
  U.a = left;
  U.a_si = 1;
  U.a_sk = ls;
  U.b = ws;
  U.b_sk = wss;
  U.c = target;
  U.ldc = ts;
  U.i_lo = 0;
  U.i_hi = rows;
  U.j_lo = 0;
  U.j_hi = cols;
  U.inner = inner;
  U.upper_only = 0;
  U.triangular = 0;
  U.tile_i0 = 0;
  U.tile_j0 = 0;
  U.tiles_m = (rows + kBM - 1) / kBM;
  U.tiles_n = (cols + kBN - 1) / kBN;
  const int sms = device_sm_count();
  const long long tiles = static_cast<long long>(U.tiles_m) * U.tiles_n;
  const int grid = static_cast<int>(std::max(1LL, std::min<long long>(tiles, 4LL * sms)));
  return launch_by_mode(U, mode, false, false, grid, grid, s);
}

int launch_scale_1x1(int count, double pivot, const double* src, int ss, double* dst, int ds,
                     cudaStream_t s) {
  if (count <= 0) return BBK_OK;
  const int grid = std::min(1024, (count + 255) / 256);
  scale_1x1_kernel<<<grid, 256, 0, s>>>(count, pivot, src, ss, dst, ds);
  BBK_CUDA_TRY(cudaGetLastError());
  count_launch();
  return BBK_OK;
}

int launch_scale_2x2(int count, double a, double b, double c, const double* s1, int s1s,
                     const double* s2, int s2s, double* d1, int d1s, double* d2, int d2s,
                     cudaStream_t s) {
  if (count <= 0) return BBK_OK;
  const int grid = std::min(1024, (count + 255) / 256);
  scale_2x2_kernel<<<grid, 256, 0, s>>>(count, a, b, c, s1, s1s, s2, s2s, d1, d1s, d2, d2s);
  BBK_CUDA_TRY(cudaGetLastError());
  count_launch();
  return BBK_OK;
}

}  // namespace bbk
