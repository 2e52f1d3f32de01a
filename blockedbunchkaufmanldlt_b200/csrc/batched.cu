// Batched factor + solve: thousands of independent small symmetric matrices
// (order <= BBK_BATCH_MAX_N) in one persistent launch.  Each CTA takes the
// next matrix from a largest-first queue and runs the whole blocked
// Bunch-Kaufman factorization of BlockLdltDecomposition::Factorize
// (src/block_ldlt_decomposition.cc:28-78 in wentianshu/BlockedBunchKaufmanLDLT,
// panels per FactorPanel :80-704, trailing updates per UpdateTrailingBlocks
// :706-744) and then the one-right-hand-side solve (and, for FP32 updates,
// FP64 iterative refinement) with no other CTA involved.
//
// Per panel, the CTA keeps in shared memory, by column slot as the
// multi-CTA panel kernel does: the panel's rows of A (staged once, each
// becoming the workspace row W when its pivot row is updated), the U
// columns of every slot, the candidate column and the slot maps.  An
// interchange only swaps two slots in the maps; at the end of the panel the
// moved rows and columns of A are gathered into per-CTA scratch and written
// back, the compact factor rows are written, and the trailing upper triangle
// is updated from the shared-memory W and U with register-tiled FMAs.  A
// itself stays in global memory (L2-resident while the CTA works on it).
//
// Arithmetic modes: FP64_ORDERED reproduces the reference bit for bit
// (ordered dot products and trailing sums, every product and sum rounded
// separately); FP64 reassociates them into FMA chains; FP32 runs the
// trailing update in FP32 and refines the solution in FP64.
#include <algorithm>
#include <climits>
#include <map>
#include <mutex>
#include <vector>

#include "bbk_internal.cuh"

namespace bbk {
namespace {

constexpr int kBT = 256;              // threads per CTA
constexpr int kBWarps = kBT / 32;
constexpr int kBC = (BBK_BATCH_MAX_N + kBT - 1) / kBT;  // slots per thread
constexpr int kMaxB = 64;             // largest block size
constexpr int kCap = 2 * kMaxB + 4;   // moved indices per panel
constexpr int kWU = kMaxB + 2;        // a panel has at most b + 1 pivot rows
constexpr size_t kBatchSmem = 220 * 1024;
constexpr int kSolveBlk = 32;

struct BatchItemDev {
  int n, lda, b, orig;
  long long a, rhs, piv;
};

struct BatchArgs {
  int count;
  const BatchItemDev* items;
  double* a;
  const double* a_orig;
  double* x;
  int* perm;
  int* ptype;
  int mode;
  double tol;
  int max_iter;
  bbk_batch_info* info;
  int* counter;
  double* scratch;        // per CTA: gbuf (kCap x max_n), gbuf2 (max_n x kCap), vectors
  long long scratch_stride;
  int max_n;
};

// Shared-memory carve-up for one item.
struct Smem {
  double* wsm;   // (b+2) x nw: staged panel rows -> workspace rows, by slot
  double* usm;   // n x ldu: U by slot
  double* wcs;   // n: candidate column by slot (also the solve vector)
  double* dlog;  // 2 (b+2)
  double* red_v; // 2 x kBWarps (alternating reductions)
  int* win;      // b+2
  int* mypos;    // n: index held by slot
  int* srcmap;   // n: slot of index
  int* moved;    // kCap
  int* red_i;    // 2 x kBWarps
  int* red_s;    // 2 x kBWarps
  int* misc;     // 8
  double* tile;  // kSolveBlk x (kSolveBlk + 1): a diagonal block of the factor (solve)
  int* tpt;      // kSolveBlk: that block's pivot types
  int ldu;
  int nw;
};

// U and W leading dimensions = 4 (mod 16) doubles: the tensor-core fragment
// loads of the trailing update are then free of bank conflicts.
__host__ __device__ inline int batch_ldu(int b) { return (b + 2 + 11) / 16 * 16 + 4; }
__host__ __device__ inline int batch_nw(int n) { return (n + 11) / 16 * 16 + 4; }

__host__ __device__ inline size_t batch_smem_bytes(int n, int b) {
  const size_t nd = static_cast<size_t>(b + 2) * batch_nw(n) + static_cast<size_t>(n) * batch_ldu(b) + n +
                    2 * static_cast<size_t>(b + 2) + 2 * kBWarps + kSolveBlk * (kSolveBlk + 1);
  const size_t ni = static_cast<size_t>(b + 2) + 2 * static_cast<size_t>(n) + kCap + 4 * kBWarps + 8 + kSolveBlk;
  return nd * sizeof(double) + ni * sizeof(int);
}

__device__ Smem carve(double* base, int n, int b) {
  Smem S;
  S.ldu = batch_ldu(b);
  S.nw = batch_nw(n);
  S.wsm = base;
  S.usm = S.wsm + static_cast<size_t>(b + 2) * S.nw;
  S.wcs = S.usm + static_cast<size_t>(n) * S.ldu;
  S.dlog = S.wcs + n;
  S.red_v = S.dlog + 2 * (b + 2);
  S.tile = S.red_v + 2 * kBWarps;
  int* ib = reinterpret_cast<int*>(S.tile + kSolveBlk * (kSolveBlk + 1));
  S.win = ib;
  S.mypos = S.win + (b + 2);
  S.srcmap = S.mypos + n;
  S.moved = S.srcmap + n;
  S.red_i = S.moved + kCap;
  S.red_s = S.red_i + 2 * kBWarps;
  S.misc = S.red_s + 2 * kBWarps;
  S.tpt = S.misc + 8;
  return S;
}

__device__ __forceinline__ void argmax_join3(double& v, int& i, int& s, double v2, int i2, int s2) {
  if (v2 > v || (v2 == v && i2 < i)) {
    v = v2;
    i = i2;
    s = s2;
  }
}

// CTA argmax (value, index, slot) with the reference's tie rule; every
// thread gets the result.  Consecutive reductions alternate between two
// scratch sets (`parity`), so one barrier suffices: a set is written again
// only after the barrier of the reduction in between.
__device__ void block_argmax(const Smem& S, int& parity, double& v, int& i, int& s) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int off = 16; off > 0; off >>= 1) {
    const double v2 = __shfl_down_sync(0xffffffffu, v, off);
    const int i2 = __shfl_down_sync(0xffffffffu, i, off);
    const int s2 = __shfl_down_sync(0xffffffffu, s, off);
    argmax_join3(v, i, s, v2, i2, s2);
  }
  const int base = parity * kBWarps;
  parity ^= 1;
  if (lane == 0) {
    S.red_v[base + warp] = v;
    S.red_i[base + warp] = i;
    S.red_s[base + warp] = s;
  }
  __syncthreads();
  v = S.red_v[base];
  i = S.red_i[base];
  s = S.red_s[base];
  for (int k = 1; k < kBWarps; ++k)
    argmax_join3(v, i, s, S.red_v[base + k], S.red_i[base + k], S.red_s[base + k]);
}

__device__ __forceinline__ void cp_async_8(double* smem_dst, const double* gsrc) {
  const unsigned saddr = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(saddr), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// for idx in [0, total): st(idx, ld(idx)), each thread keeping kDepth loads
// in flight (the loads do not wait on the stores)
template <int kDepth, typename Ld, typename St>
__device__ __forceinline__ void pipelined_copy(int total, Ld&& ld, St&& st) {
  for (int base = threadIdx.x; base < total; base += kBT * kDepth) {
    double v[kDepth];
#pragma unroll
    for (int u = 0; u < kDepth; ++u) {
      const int idx = base + u * kBT;
      v[u] = idx < total ? ld(idx) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kDepth; ++u) {
      const int idx = base + u * kBT;
      if (idx < total) st(idx, v[u]);
    }
  }
}

__device__ __forceinline__ double asym(const double* A, int lda, int x, int z) {
  return x <= z ? A[static_cast<long long>(x) * lda + z] : A[static_cast<long long>(z) * lda + x];
}

// ---------------------------------------------------------------------------
// Trailing update A[i, j] -= sum_q U[q, i] W[q, j] over the upper triangle
// i <= j of [e, n), with U and W in shared memory in index order
// (usm[i * ldu + q], wsm[q * nw + j]).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mma_f64_16x8x8(double (&c)[4], const double (&a)[4], const double (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

// FP64 tensor cores: each warp owns 32 x 32 tiles of the upper tile
// triangle (2 x 4 fragments of m16n8k8).
__device__ void trailing_dmma(const Smem& S, double* A, int lda, int n, int e, int kb) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, tq = lane & 3;
  const int m = n - e;
  const int tiles = (m + 31) / 32;
  const int ntile = tiles * (tiles + 1) / 2;
  const double* U = S.usm;
  const double* W = S.wsm;
  const int ldu = S.ldu, nw = S.nw;
  for (int tid = warp; tid < ntile; tid += kBWarps) {
    int J = static_cast<int>((sqrtf(8.0f * tid + 1.0f) - 1.0f) * 0.5f);
    while (J * (J + 1) / 2 > tid) --J;
    while ((J + 1) * (J + 2) / 2 <= tid) ++J;
    const int I = tid - J * (J + 1) / 2;
    const int i0 = e + 32 * I, j0 = e + 32 * J;
    double acc[2][4][4] = {};
    for (int ks = 0; ks < kb; ks += 8) {
      const int k0 = ks + tq, k1 = ks + tq + 4;
      double af[2][4], bf[4][2];
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        const int r0 = i0 + mt * 16 + g, r1 = r0 + 8;
        af[mt][0] = (r0 < n && k0 < kb) ? U[static_cast<size_t>(r0) * ldu + k0] : 0.0;
        af[mt][1] = (r1 < n && k0 < kb) ? U[static_cast<size_t>(r1) * ldu + k0] : 0.0;
        af[mt][2] = (r0 < n && k1 < kb) ? U[static_cast<size_t>(r0) * ldu + k1] : 0.0;
        af[mt][3] = (r1 < n && k1 < kb) ? U[static_cast<size_t>(r1) * ldu + k1] : 0.0;
      }
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const int col = j0 + nt * 8 + g;
        bf[nt][0] = (col < n && k0 < kb) ? W[k0 * nw + col] : 0.0;
        bf[nt][1] = (col < n && k1 < kb) ? W[k1 * nw + col] : 0.0;
      }
#pragma unroll
      for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) mma_f64_16x8x8(acc[mt][nt], af[mt], bf[nt]);
    }
    // C -= acc: every load of the tile first, then every store
    double cv[2][4][4];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
          for (int u = 0; u < 2; ++u) {
            const int i = i0 + mt * 16 + g + 8 * h, j = j0 + nt * 8 + tq * 2 + u;
            cv[mt][nt][2 * h + u] = (i < n && j < n && i <= j) ? A[static_cast<long long>(i) * lda + j] : 0.0;
          }
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
          for (int u = 0; u < 2; ++u) {
            const int i = i0 + mt * 16 + g + 8 * h, j = j0 + nt * 8 + tq * 2 + u;
            if (i < n && j < n && i <= j)
              A[static_cast<long long>(i) * lda + j] = cv[mt][nt][2 * h + u] - acc[mt][nt][2 * h + u];
          }
  }
}

// SIMT 4 x 4 register tiles: the reference's order (FP64_ORDERED: every
// product and sum rounded, one final subtraction) or FP32 products and sums.
template <int kMode>
__device__ void trailing_simt(const Smem& S, double* A, int lda, int n, int e, int kb) {
  constexpr bool kOrdered = kMode == BBK_UPDATE_FP64_ORDERED;
  const int m = n - e;
  const int tiles = (m + 3) / 4;
  const int ntile = tiles * (tiles + 1) / 2;
  for (int tid = threadIdx.x; tid < ntile; tid += kBT) {
    int J = static_cast<int>((sqrtf(8.0f * tid + 1.0f) - 1.0f) * 0.5f);
    while (J * (J + 1) / 2 > tid) --J;
    while ((J + 1) * (J + 2) / 2 <= tid) ++J;
    const int I = tid - J * (J + 1) / 2;
    const int i0 = e + 4 * I, j0 = e + 4 * J;
    int ri[4], cj[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      ri[u] = min(i0 + u, n - 1);
      cj[u] = min(j0 + u, n - 1);
    }
    double cval[4][4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const int i = i0 + u, j = j0 + v;
        cval[u][v] = (i < n && j < n && i <= j) ? A[static_cast<long long>(i) * lda + j] : 0.0;
      }
    if (kMode == BBK_UPDATE_FP32) {
      float acc[4][4] = {};
      for (int q = 0; q < kb; ++q) {
        float uv[4], wv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          uv[u] = static_cast<float>(S.usm[static_cast<size_t>(ri[u]) * S.ldu + q]);
          wv[u] = static_cast<float>(S.wsm[q * S.nw + cj[u]]);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int v = 0; v < 4; ++v) acc[u][v] = fmaf(uv[u], wv[v], acc[u][v]);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          const int i = i0 + u, j = j0 + v;
          if (i < n && j < n && i <= j)
            A[static_cast<long long>(i) * lda + j] = cval[u][v] - static_cast<double>(acc[u][v]);
        }
    } else {
      double acc[4][4] = {};
      for (int q = 0; q < kb; ++q) {
        double uv[4], wv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          uv[u] = S.usm[static_cast<size_t>(ri[u]) * S.ldu + q];
          wv[u] = S.wsm[q * S.nw + cj[u]];
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int v = 0; v < 4; ++v)
            acc[u][v] = kOrdered ? xadd(acc[u][v], xmul(uv[u], wv[v])) : __fma_rn(uv[u], wv[v], acc[u][v]);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          const int i = i0 + u, j = j0 + v;
          if (i < n && j < n && i <= j) A[static_cast<long long>(i) * lda + j] = xsub(cval[u][v], acc[u][v]);
        }
    }
  }
}

// ---------------------------------------------------------------------------
// Factorization of one matrix by one CTA
// ---------------------------------------------------------------------------
template <int kMode>  // BBK_UPDATE_FP64_ORDERED, BBK_UPDATE_FP64 or BBK_UPDATE_FP32
__device__ void factor_one(const Smem& S, double* A, int n, int lda, int b, int* perm, int* pt,
                           double* gbuf, double* gbuf2, int* permbuf, double* wutmp) {
  constexpr bool kOrdered = kMode == BBK_UPDATE_FP64_ORDERED;
  const int t = threadIdx.x;
  const int nb = (n + b - 1) / b;
  const int nw = S.nw;
  int red_parity = 0;
  for (int i = t; i < n; i += kBT) {
    perm[i] = i;
    pt[i] = 0;
  }
  int k0 = 0;
  for (int panel = 0; panel < nb && k0 < n; ++panel) {
    const int nominal_end = min((panel + 1) * b, n);
    const bool can_shift = panel + 1 < nb;
    const int nwin = min(b + 2, n - k0);
    // ---- stage the panel rows; identity maps
    for (int m = t; m < nwin; m += kBT) S.win[m] = k0 + m;
    for (int z = k0 + t; z < n; z += kBT) S.mypos[z] = z;
    for (int idx = t; idx < nwin * (n - k0); idx += kBT) {
      const int m = idx / (n - k0), z = k0 + idx % (n - k0);
      const int x = k0 + m;
      cp_async_8(&S.wsm[m * nw + z], x <= z ? A + static_cast<long long>(x) * lda + z
                                           : A + static_cast<long long>(z) * lda + x);
    }
    cp_async_wait_all();
    if (t == 0) S.misc[0] = 0;
    __syncthreads();

    int p = k0;
    while (p < nominal_end) {
      const int lp = p - k0;
      const int sp = S.win[lp];
      const bool staged = sp - k0 == lp;
      const double* ucol = S.usm + static_cast<size_t>(sp) * S.ldu;
      // ---- row update W[p, j] = A[p, j] - sum_q U[q, p] W[q, j]  (:122-182)
      double best = 0.0;
      int best_j = INT_MAX, best_z = -1;
#pragma unroll
      for (int k = 0; k < kBC; ++k) {
        const int z = k0 + t + k * kBT;
        if (z < n && S.mypos[z] >= p) {
          const double av = staged ? S.wsm[lp * nw + z] : asym(A, lda, sp, z);
          // coefficients U[q, p]: the slot's U column (all q < lp are in
          // shared memory, the newest written by the previous step)
          const double acc = kOrdered ? ordered_dot(ucol, lp, [&](int q) { return S.wsm[q * nw + z]; })
                                      : split_dot(ucol, lp, [&](int q) { return S.wsm[q * nw + z]; });
          const double wv = xsub(av, acc);
          S.wsm[lp * nw + z] = wv;
          const int j = S.mypos[z];
          if (j > p) {
            const double v = fabs(wv);
            if (v > best || (v == best && j < best_j)) {
              best = v;
              best_j = j;
              best_z = z;
            }
          }
        }
      }
      block_argmax(S, red_parity, best, best_j, best_z);  // barrier inside: row lp is visible
      const double omega = best;
      const int r = best_j, rs = best_z;
      const double dpp = S.wsm[lp * nw + sp];
      const int s1 = lp + 1 < nwin ? S.win[lp + 1] : -1;

      int kind = 1;
      bool cand = false;
      double wc_r = 0.0, wc_p = 0.0;
      if (!(fabs(dpp) >= xmul(kAlpha, omega) || omega == 0.0)) {  // :90-92
        cand = true;
        // ---- candidate column W(i, r) = A(i, r) - sum_q U[q, r] W[q, i]  (:184-367)
        const double* rcol = S.usm + static_cast<size_t>(rs) * S.ldu;
        double sig = 0.0;
#pragma unroll
        for (int k = 0; k < kBC; ++k) {
          const int z = k0 + t + k * kBT;
          if (z < n && S.mypos[z] >= p) {
            const double cv = asym(A, lda, z, rs);
            const double acc = kOrdered ? ordered_dot(rcol, lp, [&](int q) { return S.wsm[q * nw + z]; })
                                        : split_dot(rcol, lp, [&](int q) { return S.wsm[q * nw + z]; });
            const double v = xsub(cv, acc);
            S.wcs[z] = v;
            if (S.mypos[z] != r) {
              const double a2 = fabs(v);
              sig = (sig < a2) ? a2 : sig;
            }
          }
        }
        int di = 0, ds = 0;
        block_argmax(S, red_parity, sig, di, ds);
        const double sigma = sig;
        wc_r = S.wcs[rs];
        wc_p = S.wcs[sp];
        if (xsub(xmul(fabs(dpp), sigma), xmul(xmul(kAlpha, omega), omega)) >= 0.0) {  // :369-390
          kind = 1;
        } else if (xsub(fabs(wc_r), xmul(kAlpha, sigma)) >= 0.0) {
          kind = -1;
        } else {
          kind = 2;
        }
        if (kind == 2 && p == nominal_end - 1 && can_shift) {  // :104-108
          __syncthreads();
          break;
        }
      }
      __syncthreads();  // everyone has read the reduction scratch and the pivot values

      if (kind == 1) {  // ScaleOneByOnePivot :633-656
        const double d = dpp, den = safe_denominator(d);
#pragma unroll
        for (int k = 0; k < kBC; ++k) {
          const int z = k0 + t + k * kBT;
          if (z < n && S.mypos[z] > p) {
            double wv = S.wsm[lp * nw + z];
            if (cand && S.mypos[z] == r) {
              wv = wc_p;
              S.wsm[lp * nw + z] = wv;
            }
            S.usm[static_cast<size_t>(z) * S.ldu + lp] = div_or_zero(wv, den);
          }
        }
        if (t == 0) {
          S.dlog[2 * lp] = d;
          pt[p] = 1;
        }
        p += 1;
      } else if (kind == -1) {  // SwapOneByOnePivot + ScaleOneByOnePivot
        const double d = wc_r, den = safe_denominator(d);
        if (t == 0) {
          S.win[lp] = rs;
          if (r - k0 < nwin) S.win[r - k0] = sp;
          S.mypos[sp] = r;
          S.mypos[rs] = p;
          S.dlog[2 * lp] = d;
          pt[p] = 1;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kBC; ++k) {
          const int z = k0 + t + k * kBT;
          if (z < n && S.mypos[z] > p) {
            const double wv = S.wcs[z];
            S.wsm[lp * nw + z] = wv;
            S.usm[static_cast<size_t>(z) * S.ldu + lp] = div_or_zero(wv, den);
          }
        }
        p += 1;
      } else {  // SwapTwoByTwoPivot + ScaleTwoByTwoPivot :403-412, :500-587, :658-704
        const int ls = lp + 1;
        const double d11 = dpp, d21 = wc_p, d22 = wc_r;
        const double det = xsub(xmul(d11, d22), xmul(d21, d21));
        const double i11 = xdiv(d22, det), i22 = xdiv(d11, det), i21 = xdiv(-d21, det);
        if (t == 0) {
          if (r != p + 1) {
            S.win[ls] = rs;
            if (r - k0 < nwin) S.win[r - k0] = s1;
            S.mypos[s1] = r;
            S.mypos[rs] = p + 1;
          }
          S.dlog[2 * lp] = d11;
          S.dlog[2 * lp + 1] = d21;
          S.dlog[2 * ls] = d22;
          pt[p] = 2;
          pt[p + 1] = -2;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kBC; ++k) {
          const int z = k0 + t + k * kBT;
          if (z < n && S.mypos[z] > p + 1) {
            const double xv = S.wsm[lp * nw + z], yv = S.wcs[z];
            S.wsm[ls * nw + z] = yv;
            S.usm[static_cast<size_t>(z) * S.ldu + lp] = xadd(xmul(i11, xv), xmul(i21, yv));
            S.usm[static_cast<size_t>(z) * S.ldu + ls] = xadd(xmul(i21, xv), xmul(i22, yv));
          }
        }
        p += 2;
      }
      __syncthreads();
    }
    const int e = p, kb = e - k0;

    // ---- interchanges: slot of every index and the moved list
    for (int z = k0 + t; z < n; z += kBT) {
      const int x = S.mypos[z];
      S.srcmap[x] = z;
      if (x != z) S.moved[atomicAdd(&S.misc[0], 1)] = x;
    }
    __syncthreads();
    const int cnt = S.misc[0];
    const int m = n - k0;
    // gather: rows of the moved indices, factored rows at the moved
    // columns, permutation entries, and the moved W columns / U rows
    pipelined_copy<8>(
        cnt * m,
        [&](int idx) {
          const int ix = idx / m, y = k0 + idx % m;
          return asym(A, lda, S.srcmap[S.moved[ix]], S.srcmap[y]);
        },
        [&](int idx, double v) { gbuf[static_cast<long long>(idx / m) * n + k0 + idx % m] = v; });
    pipelined_copy<8>(
        k0 * cnt,
        [&](int idx) { return A[static_cast<long long>(idx / cnt) * lda + S.srcmap[S.moved[idx % cnt]]]; },
        [&](int idx, double v) { gbuf2[static_cast<long long>(idx / cnt) * kCap + idx % cnt] = v; });
    for (int ix = t; ix < cnt; ix += kBT) permbuf[ix] = perm[S.srcmap[S.moved[ix]]];
    for (int idx = t; idx < cnt * kb; idx += kBT) {
      const int ix = idx / kb, q = idx % kb;
      const int z = S.srcmap[S.moved[ix]];
      wutmp[(2 * ix) * kWU + q] = S.wsm[q * nw + z];
      wutmp[(2 * ix + 1) * kWU + q] = S.usm[static_cast<size_t>(z) * S.ldu + q];
    }
    __syncthreads();
    // write back: A in the interchanged order, the permutation, and W / U in
    // index order (from here on index = slot)
    const int mt0 = n - e;
    pipelined_copy<8>(
        cnt * mt0, [&](int idx) { return gbuf[static_cast<long long>(idx / mt0) * n + e + idx % mt0]; },
        [&](int idx, double v) {
          const int x = S.moved[idx / mt0], y = e + idx % mt0;
          if (x < e) return;
          if (x <= y)
            A[static_cast<long long>(x) * lda + y] = v;
          else
            A[static_cast<long long>(y) * lda + x] = v;
        });
    pipelined_copy<8>(
        k0 * cnt, [&](int idx) { return gbuf2[static_cast<long long>(idx / cnt) * kCap + idx % cnt]; },
        [&](int idx, double v) { A[static_cast<long long>(idx / cnt) * lda + S.moved[idx % cnt]] = v; });
    for (int ix = t; ix < cnt; ix += kBT) perm[S.moved[ix]] = permbuf[ix];
    for (int idx = t; idx < cnt * kb; idx += kBT) {
      const int ix = idx / kb, q = idx % kb;
      const int x = S.moved[ix];
      S.wsm[q * nw + x] = wutmp[(2 * ix) * kWU + q];
      S.usm[static_cast<size_t>(x) * S.ldu + q] = wutmp[(2 * ix + 1) * kWU + q];
    }
    __syncthreads();
    // ---- compact factor rows [k0, e)
    for (int idx = t; idx < kb * (n - k0); idx += kBT) {
      const int q = idx / (n - k0), j = k0 + idx % (n - k0);
      if (j < k0 + q) continue;
      const int lj = j - k0;
      double v;
      if (j < e && q == lj)
        v = S.dlog[2 * lj];
      else if (j < e && q == lj - 1 && pt[j] == -2)
        v = S.dlog[2 * q + 1];
      else
        v = S.usm[static_cast<size_t>(j) * S.ldu + q];
      A[static_cast<long long>(k0 + q) * lda + j] = v;
    }

    // ---- trailing update of the upper triangle [e, n): A -= U^T W  (:706-744)
    const int mt = n - e;
    if (mt > 0 && kb > 0) {
      if (kMode == BBK_UPDATE_FP64)
        trailing_dmma(S, A, lda, n, e, kb);
      else
        trailing_simt<kMode>(S, A, lda, n, e, kb);
    }
    __syncthreads();
    k0 = e;
  }
}

// ---------------------------------------------------------------------------
// Solve with the compact factors (one right-hand side) by one CTA.  y holds
// b on entry (shared memory) and the solution on exit; reads follow the
// multi-matrix solve (csrc/solve.cu).
// ---------------------------------------------------------------------------
__device__ void solve_one(const Smem& S, const double* F, int n, int lda, const int* perm, const int* pt,
                          double* y, double* tmp) {
  const int t = threadIdx.x, lane = t & 31;
  constexpr int kT = kSolveBlk + 1;
  // y <- P b (tmp as staging)
  for (int i = t; i < n; i += kBT) tmp[i] = y[perm[i]];
  __syncthreads();
  for (int i = t; i < n; i += kBT) y[i] = tmp[i];
  // stage the diagonal block [c0, c1) of the factor's strict upper triangle
  auto stage = [&](int c0, int bs) {
    for (int idx = t; idx < bs * bs; idx += kBT) {
      const int r = idx / bs, c = idx % bs;
      S.tile[r * kT + c] = r < c ? F[static_cast<long long>(c0 + r) * lda + c0 + c] : 0.0;
    }
    for (int r = t; r < bs; r += kBT) S.tpt[r] = pt[c0 + r];
  };
  // forward: L z = y with L(i,k) = F(k,i), k < i, except the (k+1,k) entry of a 2x2
  for (int c0 = 0; c0 < n; c0 += kSolveBlk) {
    const int c1 = min(n, c0 + kSolveBlk), bs = c1 - c0;
    __syncthreads();
    stage(c0, bs);
    __syncthreads();
    if (t < 32) {
      double v = lane < bs ? y[c0 + lane] : 0.0;
      for (int k = 0; k < bs; ++k) {
        const double yk = __shfl_sync(0xffffffffu, v, k);
        if (lane > k && lane < bs && !(S.tpt[k] == 2 && lane == k + 1)) v -= S.tile[k * kT + lane] * yk;
      }
      if (lane < bs) y[c0 + lane] = v;
    }
    __syncthreads();
    const bool coupled = S.tpt[bs - 1] == 2;  // 2x2 from c1-1 into row c1
    for (int i = c1 + t; i < n; i += kBT) {
      double f[kSolveBlk];
#pragma unroll
      for (int k = 0; k < kSolveBlk; ++k) f[k] = k < bs ? F[static_cast<long long>(c0 + k) * lda + i] : 0.0;
      const int skip = (coupled && i == c1) ? bs - 1 : -1;
      double acc = 0.0;
#pragma unroll
      for (int k = 0; k < kSolveBlk; ++k) acc += (k < bs && k != skip) ? f[k] * y[c0 + k] : 0.0;
      y[i] -= acc;
    }
  }
  __syncthreads();
  // D w = z
  for (int k = t; k < n; k += kBT) {
    if (pt[k] == -2) continue;
    if (pt[k] == 2 && k + 1 < n) {
      const double d11 = F[static_cast<long long>(k) * lda + k], d21 = F[static_cast<long long>(k) * lda + k + 1];
      const double d22 = F[static_cast<long long>(k + 1) * lda + k + 1];
      const double det = d11 * d22 - d21 * d21;
      const double i11 = d22 / det, i22 = d11 / det, i21 = -d21 / det;
      const double xv = y[k], zv = y[k + 1];
      y[k] = i11 * xv + i21 * zv;
      y[k + 1] = i21 * xv + i22 * zv;
    } else {
      const double d = F[static_cast<long long>(k) * lda + k];
      y[k] = d == 0.0 ? 0.0 : y[k] / d;
    }
  }
  // backward: L^T v = w
  for (int c1 = n; c1 > 0; c1 -= kSolveBlk) {
    const int c0 = max(0, c1 - kSolveBlk), bs = c1 - c0;
    __syncthreads();
    stage(c0, bs);
    __syncthreads();
    if (t < 32) {
      double v = lane < bs ? y[c0 + lane] : 0.0;
      for (int k = bs - 1; k >= 0; --k) {
        const double vk = __shfl_sync(0xffffffffu, v, k);
        if (lane < k && !(S.tpt[lane] == 2 && k == lane + 1)) v -= S.tile[lane * kT + k] * vk;
      }
      if (lane < bs) y[c0 + lane] = v;
    }
    __syncthreads();
    const bool coupled = c0 > 0 && pt[c0 - 1] == 2;  // 2x2 from c0-1 into column c0
    for (int i = t; i < c0; i += kBT) {
      double f[kSolveBlk];
#pragma unroll
      for (int k = 0; k < kSolveBlk; ++k) f[k] = k < bs ? F[static_cast<long long>(i) * lda + c0 + k] : 0.0;
      if (coupled && i == c0 - 1) f[0] = 0.0;
      double acc = 0.0;
#pragma unroll
      for (int k = 0; k < kSolveBlk; ++k) acc += k < bs ? f[k] * y[c0 + k] : 0.0;
      y[i] -= acc;
    }
  }
  __syncthreads();
  // X[perm] = v
  for (int i = t; i < n; i += kBT) tmp[perm[i]] = y[i];
  __syncthreads();
  for (int i = t; i < n; i += kBT) y[i] = tmp[i];
  __syncthreads();
}

// r = b - A x with A symmetric from its upper triangle; returns (on every
// thread) the backward error max|r| / (||A||_inf ||x||_inf + ||b||_inf).
__device__ double residual_one(const double* A, int n, int lda, const double* bvec, const double* xv,
                               double* r, double* red) {
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  double rmax = 0.0, xmax = 0.0, bmax = 0.0, amax = 0.0;
  for (int i = warp; i < n; i += kBWarps) {
    double s = 0.0, sa = 0.0;
    for (int j = lane; j < n; j += 32) {
      const double aij = asym(A, lda, i, j);
      s = __fma_rn(aij, xv[j], s);
      sa += fabs(aij);
    }
    for (int off = 16; off > 0; off >>= 1) {
      s += __shfl_down_sync(0xffffffffu, s, off);
      sa += __shfl_down_sync(0xffffffffu, sa, off);
    }
    if (lane == 0) {
      const double ri = bvec[i] - s;
      r[i] = ri;
      rmax = fmax(rmax, fabs(ri));
      amax = fmax(amax, sa);
      xmax = fmax(xmax, fabs(xv[i]));
      bmax = fmax(bmax, fabs(bvec[i]));
    }
  }
  if (lane == 0) {
    red[4 * warp + 0] = rmax;
    red[4 * warp + 1] = amax;
    red[4 * warp + 2] = xmax;
    red[4 * warp + 3] = bmax;
  }
  __syncthreads();
  double m[4] = {0.0, 0.0, 0.0, 0.0};
  for (int w = 0; w < kBWarps; ++w)
    for (int k = 0; k < 4; ++k) m[k] = fmax(m[k], red[4 * w + k]);
  __syncthreads();
  const double den = m[1] * m[2] + m[3];
  return den > 0.0 ? m[0] / den : (m[0] > 0.0 ? INFINITY : 0.0);
}

template <int kMode>
__global__ void __launch_bounds__(kBT, 1) batched_kernel(BatchArgs B) {
  extern __shared__ double bsm[];
  __shared__ int s_item;
  double* gbuf = B.scratch + static_cast<long long>(blockIdx.x) * B.scratch_stride;
  double* gbuf2 = gbuf + static_cast<long long>(kCap) * B.max_n;
  double* vb = gbuf2 + static_cast<long long>(B.max_n) * kCap;  // right-hand side copy
  double* vr = vb + B.max_n;                                        // residual
  double* vt = vr + B.max_n;                                        // staging
  double* wutmp = vt + B.max_n;                                     // 2 kCap x kWU
  int* permbuf = reinterpret_cast<int*>(wutmp + 2 * kCap * kWU);
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(B.counter, 1);
    __syncthreads();
    const int it = s_item;
    __syncthreads();
    if (it >= B.count) break;
    const BatchItemDev I = B.items[it];
    const int n = I.n, lda = I.lda;
    double* A = B.a + I.a;
    double* X = B.x + I.rhs;
    int* perm = B.perm + I.piv;
    int* pt = B.ptype + I.piv;
    Smem S = carve(bsm, n, I.b);
    factor_one<kMode>(S, A, n, lda, I.b, perm, pt, gbuf, gbuf2, permbuf, wutmp);
    // solve (the candidate-column buffer holds the vector)
    double* y = S.wcs;
    for (int i = threadIdx.x; i < n; i += kBT) {
      y[i] = X[i];
      vb[i] = X[i];
    }
    __syncthreads();
    solve_one(S, A, n, lda, perm, pt, y, vt);
    int iters = 0, conv = 1;
    double berr = 0.0;
    const bool refine = kMode == BBK_UPDATE_FP32 && B.a_orig != nullptr && B.max_iter > 0;
    if (refine) {
      const double* A0 = B.a_orig + I.a;
      conv = 0;
      // the solution stays in X (global) while y carries the correction
      for (int i = threadIdx.x; i < n; i += kBT) X[i] = y[i];
      __syncthreads();
      for (;;) {
        berr = residual_one(A0, n, lda, vb, X, vr, S.usm);
        if (berr <= B.tol) {
          conv = 1;
          break;
        }
        if (iters >= B.max_iter || !isfinite(berr)) break;
        for (int i = threadIdx.x; i < n; i += kBT) y[i] = vr[i];
        __syncthreads();
        solve_one(S, A, n, lda, perm, pt, y, vt);
        for (int i = threadIdx.x; i < n; i += kBT) X[i] += y[i];
        __syncthreads();
        ++iters;
      }
    } else {
      for (int i = threadIdx.x; i < n; i += kBT) X[i] = y[i];
    }
    if (B.info && threadIdx.x == 0) {
      bbk_batch_info inf;
      inf.iterations = iters;
      inf.converged = conv;
      inf.backward_error = berr;
      B.info[I.orig] = inf;
    }
    __syncthreads();
  }
}

constexpr size_t kHeaderBytes = 256;

// Host-side record of planned workspaces (workspace -> count, largest order),
// so a launch needs no device read.
std::mutex g_plan_mu;
std::map<const void*, std::pair<int, int>> g_plans;

void batch_plan_record(const void* ws, int count, int max_n) {
  std::lock_guard<std::mutex> lk(g_plan_mu);
  g_plans[ws] = {count, max_n};
}

bool batch_plan_lookup(const void* ws, int count, int* max_n) {
  std::lock_guard<std::mutex> lk(g_plan_mu);
  auto it = g_plans.find(ws);
  if (it == g_plans.end() || it->second.first != count) return false;
  *max_n = it->second.second;
  return true;
}

size_t scratch_doubles(int max_n) {
  // gbuf + gbuf2 + three vectors + the W/U staging + the permutation staging
  return 2 * static_cast<size_t>(kCap) * max_n + 3 * static_cast<size_t>(max_n) +
         2 * static_cast<size_t>(kCap) * kWU + kCap;
}

int default_block(int bucket) {
  static const int kDefault[BBK_BATCH_BUCKETS] = {32, 32, 32, 32, 24, 12};
  return kDefault[bucket];
}

int bucket_of(int n) {
  int bkt = 0;
  for (int lim = 32; lim < n && bkt < BBK_BATCH_BUCKETS - 1; lim *= 2) ++bkt;
  return bkt;
}

// Layout of the workspace: header (counter, count, max_n, grid), the
// sorted item table, then the per-CTA scratch.
struct BatchLayout {
  int* header;
  BatchItemDev* items;
  double* scratch;
  long long scratch_stride;
  size_t bytes;
};

BatchLayout batch_layout(void* base, int count, int max_n, int grid) {
  BatchLayout L{};
  char* p = static_cast<char*>(base);
  size_t off = 0;
  L.header = reinterpret_cast<int*>(p ? p + off : nullptr);
  off += kHeaderBytes;
  L.items = reinterpret_cast<BatchItemDev*>(p ? p + off : nullptr);
  off = align_up(off + static_cast<size_t>(count) * sizeof(BatchItemDev), 256);
  L.scratch_stride = static_cast<long long>(align_up(scratch_doubles(max_n), 32));
  L.scratch = reinterpret_cast<double*>(p ? p + off : nullptr);
  off += static_cast<size_t>(grid) * L.scratch_stride * sizeof(double);
  L.bytes = off;
  return L;
}

}  // namespace
}  // namespace bbk

using namespace bbk;

extern "C" size_t bbk_batched_workspace_size(int count, int max_n) {
  if (count <= 0 || max_n <= 0 || max_n > BBK_BATCH_MAX_N) return 0;
  return batch_layout(nullptr, count, max_n, device_sm_count()).bytes;
}

extern "C" int bbk_batched_plan(int count, const bbk_batch_item* items, const int* block_sizes,
                                int* chosen_blocks, void* workspace, size_t workspace_bytes, void* stream) {
  if (count <= 0) return set_error(BBK_ERR_INVALID_ARGUMENT, "batch count must be positive");
  if (!items || !workspace) return set_error(BBK_ERR_INVALID_ARGUMENT, "null items or workspace");
  std::vector<BatchItemDev> v(count);
  int max_n = 0;
  for (int k = 0; k < count; ++k) {
    const bbk_batch_item& it = items[k];
    if (it.n <= 0 || it.n > BBK_BATCH_MAX_N)
      return set_error(BBK_ERR_INVALID_ARGUMENT, "item %d: order %d outside 1..%d", k, it.n, BBK_BATCH_MAX_N);
    if (it.lda < it.n) return set_error(BBK_ERR_INVALID_ARGUMENT, "item %d: lda < n", k);
    if (it.a < 0 || it.rhs < 0 || it.piv < 0)
      return set_error(BBK_ERR_INVALID_ARGUMENT, "item %d: negative offset", k);
    const int bkt = bucket_of(it.n);
    int b = (block_sizes && block_sizes[bkt] > 0) ? block_sizes[bkt] : default_block(bkt);
    b = std::min(std::min(b, kMaxB), it.n);
    while (b > 1 && batch_smem_bytes(it.n, b) > kBatchSmem) --b;
    if (batch_smem_bytes(it.n, b) > kBatchSmem)
      return set_error(BBK_ERR_INVALID_ARGUMENT, "item %d: order %d does not fit shared memory", k, it.n);
    v[k] = BatchItemDev{it.n, it.lda, b, k, it.a, it.rhs, it.piv};
    if (chosen_blocks) chosen_blocks[k] = b;
    max_n = std::max(max_n, it.n);
  }
  // largest first; ties keep the caller's order
  std::stable_sort(v.begin(), v.end(), [](const BatchItemDev& x, const BatchItemDev& y) { return x.n > y.n; });
  int rc = check_device();
  if (rc) return rc;
  const int grid = device_sm_count();
  BatchLayout L = batch_layout(workspace, count, max_n, grid);
  if (workspace_bytes < L.bytes)
    return set_error(BBK_ERR_WORKSPACE, "batched workspace of %zu bytes, %zu needed", workspace_bytes, L.bytes);
  int header[4] = {0, count, max_n, grid};
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  BBK_CUDA_TRY(cudaMemcpyAsync(L.header, header, sizeof(header), cudaMemcpyHostToDevice, s));
  BBK_CUDA_TRY(cudaMemcpyAsync(L.items, v.data(), v.size() * sizeof(BatchItemDev), cudaMemcpyHostToDevice, s));
  BBK_CUDA_TRY(cudaStreamSynchronize(s));
  // the launch reads these back without a device round trip
  batch_plan_record(workspace, count, max_n);
  return BBK_OK;
}

extern "C" int bbk_batched_factor_solve(int count, double* a, const double* a_orig, double* x, int* perm,
                                        int* pivot_types, int update_mode, double tol, int max_iter,
                                        bbk_batch_info* info, void* workspace, size_t workspace_bytes,
                                        void* stream) {
  if (count <= 0) return set_error(BBK_ERR_INVALID_ARGUMENT, "batch count must be positive");
  if (!a || !x || !perm || !pivot_types || !workspace)
    return set_error(BBK_ERR_INVALID_ARGUMENT, "null buffer");
  if (update_mode != BBK_UPDATE_FP64 && update_mode != BBK_UPDATE_FP64_ORDERED && update_mode != BBK_UPDATE_FP32)
    return set_error(BBK_ERR_INVALID_ARGUMENT, "batched update mode must be FP64, FP64_ORDERED or FP32");
  int max_n = 0;
  if (!batch_plan_lookup(workspace, count, &max_n))
    return set_error(BBK_ERR_LOGIC, "workspace was not planned for %d items (call bbk_batched_plan)", count);
  int rc = check_device();
  if (rc) return rc;
  const int grid = device_sm_count();
  BatchLayout L = batch_layout(workspace, count, max_n, grid);
  if (workspace_bytes < L.bytes)
    return set_error(BBK_ERR_WORKSPACE, "batched workspace of %zu bytes, %zu needed", workspace_bytes, L.bytes);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  BatchArgs B{};
  B.count = count;
  B.items = L.items;
  B.a = a;
  B.a_orig = a_orig;
  B.x = x;
  B.perm = perm;
  B.ptype = pivot_types;
  B.mode = update_mode;
  B.tol = tol;
  B.max_iter = max_iter;
  B.info = info;
  B.counter = L.header;
  B.scratch = L.scratch;
  B.scratch_stride = L.scratch_stride;
  B.max_n = max_n;
  BBK_CUDA_TRY(cudaMemsetAsync(L.header, 0, sizeof(int), s));
  const void* fn = update_mode == BBK_UPDATE_FP64_ORDERED
                       ? reinterpret_cast<const void*>(batched_kernel<BBK_UPDATE_FP64_ORDERED>)
                       : update_mode == BBK_UPDATE_FP64 ? reinterpret_cast<const void*>(batched_kernel<BBK_UPDATE_FP64>)
                                                        : reinterpret_cast<const void*>(batched_kernel<BBK_UPDATE_FP32>);
  {
    // once per device and mode, so a later call can run under stream capture
    static std::mutex mu;
    static bool done[3][64] = {};
    int dev = 0;
    BBK_CUDA_TRY(cudaGetDevice(&dev));
    const int mi = update_mode == BBK_UPDATE_FP64_ORDERED ? 0 : update_mode == BBK_UPDATE_FP64 ? 1 : 2;
    std::lock_guard<std::mutex> lk(mu);
    if (dev < 0 || dev >= 64 || !done[mi][dev]) {
      BBK_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kBatchSmem)));
      if (dev >= 0 && dev < 64) done[mi][dev] = true;
    }
  }
  void* kargs[] = {&B};
  BBK_CUDA_TRY(cudaLaunchKernel(fn, dim3(grid), dim3(kBT), kargs, kBatchSmem, s));
  count_launch();
  return BBK_OK;
}
