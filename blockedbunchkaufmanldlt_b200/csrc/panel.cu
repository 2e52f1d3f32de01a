// Panel factorization of the blocked Bunch-Kaufman LDL^T: one persistent
// cooperative launch per panel runs the panel's sequential pivot chain with
// all CTAs, each owning a contiguous slice of the active columns [k0, n).
//
// Follows BlockLdltDecomposition::FactorPanel and its helpers
// (src/block_ldlt_decomposition.cc:80-704 in wentianshu/BlockedBunchKaufmanLDLT)
// in the reference's own operation order, so the panel's arithmetic is
// bitwise identical to the reference (every product and sum separately
// rounded; this file is also compiled with --fmad=false).
//
// Data during a panel whose first row is k0 (lp = p - k0 is the local pivot):
//   A    n x lda row-major upper: rows >= p are the partially updated matrix;
//        the panel's own rows stay frozen until finalize_kernel writes the
//        compact factor rows into them.
//   W    row lp holds the workspace row W[p, j] (j >= p) of pivot p.
//   Ucm  column-major U: Ucm[j*ldu + lp] = U[p, j].  Column j belongs to the
//        CTA that owns column j, so U[., r] is one contiguous read.
//   Uout the final compact column of each pivot column of the panel
//        (rows < lp from Ucm after the last interchange touching it, then D).
//   wc   the candidate column W(i, r), i >= p.
//
// Per pivot step the grid meets once (no candidate) or twice (candidate
// column needed).  Between one step's interchange/scaling phase and the next
// step's row update there is no grid barrier: every write of the scaling phase
// goes to a column its writer owns, except three kinds of value that the
// next row update needs from other columns -- the next coefficients U[p, p']
// (recomputed redundantly by every CTA from published scalars), the single
// moved entry A[p', r] (read from the frozen row p instead), and a swapped
// Ucm column (read from its pre-swap location).  Everything else is read
// only after the next exchange.
#include <climits>
#include <cstdio>
#include <cstdlib>

#include "bbk_internal.cuh"

#ifndef BBK_PANEL_THREADS
#define BBK_PANEL_THREADS 128
#endif

namespace bbk {
namespace {

constexpr int kThreads = BBK_PANEL_THREADS;
constexpr int kWarps = kThreads / 32;
constexpr int kCols = 4;  // columns per thread: S <= kCols * kThreads
constexpr int kMaxPollPerLane = 8;  // exchange records polled per lane (grid <= 256)

struct PanelArgs {
  int n;
  int panel;
  int nominal_end;  // min((panel+1)*b, n)
  int can_shift;    // another panel follows
  double* a;
  long long lda;
  double* w;
  long long ldw;
  double* ucm;
  int ldu;
  double* uout;
  double* wc;
  double* wstage;    // 2 x coef_cap: W columns p and p+1 for an interchange
  int* perm;
  int* ptype;
  int* panel_end;
  unsigned long long* slots;
  DeviceState* st;
  int nslots;        // records each exchange waits for (gridDim.x normally)
  int slot_stride;   // records per parity in `slots` (>= nslots)
  unsigned tag_base;
  unsigned long long timeout_ns;
  int coef_cap;      // doubles reserved for the coefficient column
  int w_smem;        // keep this CTA's workspace slice in shared memory
  int smem_cols;     // slice width the shared-memory allocation holds
  unsigned long long* stats;  // optional per-phase nanoseconds (CTA 0)
  unsigned long long* pub_ts; // with stats: each CTA's publish timestamp
  unsigned poll_ns;           // pause between polls of the exchange records
};

struct ExchangeOut {
  double val;
  int idx;
  int ok;
  double pub[kMaxPub];
};

__device__ __forceinline__ void fail(DeviceState* st, int code) {
  atomicCAS(&st->status, 0, code);
  atomicExch(&st->abort, 1);
}

__device__ __forceinline__ double join_hi_lo(unsigned long long hi, unsigned long long lo) {
  const unsigned long long bits = ((hi & 0xffffffffull) << 32) | (lo & 0xffffffffull);
  return __longlong_as_double(static_cast<long long>(bits));
}

// Argmax combine with the reference's tie rule (src/block_ldlt_decomposition.cc:
// 164-182 scans ascending columns with a strict '>'): larger value wins, equal
// values keep the lower index.  NaN never enters (callers skip it).
__device__ __forceinline__ void argmax_join(double& v, int& i, double v2, int i2) {
  if (v2 > v || (v2 == v && i2 < i)) {
    v = v2;
    i = i2;
  }
}

// CTA-collective: reduce (my_val, my_idx) over the CTA, publish the CTA's
// record (reduction + its kMaxPub scalars in pub_in), wait for the records of
// all `nslots` CTAs, and return the grid-wide argmax plus pub[k] taken from
// the record of CTA pub_owner[k].  Must be called by every thread.
__device__ void exchange(const PanelArgs& P, unsigned tag, double my_val, int my_idx,
                         const double* pub_in, const int* pub_owner, int npub,
                         double* s_red_v, int* s_red_i, ExchangeOut* out) {
  const int t = threadIdx.x;
  const int lane = t & 31, warp = t >> 5;
  for (int off = 16; off > 0; off >>= 1) {
    const double v2 = __shfl_down_sync(0xffffffffu, my_val, off);
    const int i2 = __shfl_down_sync(0xffffffffu, my_idx, off);
    argmax_join(my_val, my_idx, v2, i2);
  }
  if (lane == 0) {
    s_red_v[warp] = my_val;
    s_red_i[warp] = my_idx;
  }
  __syncthreads();  // also orders this CTA's global writes before the fences
  // Structure-of-arrays records: word w of CTA c lives at
  // slots[((tag & 1) * kSlotWords + w) * slot_stride + c], so one warp load
  // polls word w of 32 consecutive CTAs in two cache lines.
  unsigned long long* par_base =
      P.slots + static_cast<size_t>(tag & 1u) * kSlotWords * P.slot_stride;
  if (warp == 0) {
    double v = s_red_v[0];
    int i = s_red_i[0];
    for (int k = 1; k < kWarps; ++k) argmax_join(v, i, s_red_v[k], s_red_i[k]);
    // one record word per lane: (tag | idx), (tag | hi v), (tag | lo v), pubs
    if (lane < 3 + 2 * npub) {
      unsigned word;
      if (lane == 0) {
        word = static_cast<unsigned>(i);
      } else {
        const double x = lane < 3 ? v : pub_in[(lane - 3) >> 1];
        const unsigned long long bits = static_cast<unsigned long long>(__double_as_longlong(x));
        const bool high = lane < 3 ? lane == 1 : ((lane - 3) & 1) == 0;
        word = high ? static_cast<unsigned>(bits >> 32) : static_cast<unsigned>(bits);
      }
      if (P.pub_ts && lane == 0) P.pub_ts[blockIdx.x] = globaltimer_ns();
      fence_acq_rel_gpu();  // release everything this CTA wrote so far
      st_relaxed_u64(par_base + static_cast<size_t>(lane) * P.slot_stride + blockIdx.x,
                     tag_word(tag, word));
    }
  }
  if (warp == 0) {
    // Every lane polls all of its records (CTAs lane, lane+32, ...) and its
    // published word pair at once, so the exchange completes one L2 round trip
    // after the last record lands.
    const size_t st = P.slot_stride;
    const unsigned long long* src[kMaxPollPerLane];
    unsigned long long wv[kMaxPollPerLane][3];
    int nmine = 0;
    for (int sidx = lane; sidx < P.nslots && nmine < kMaxPollPerLane; sidx += 32)
      src[nmine++] = par_base + sidx;
    const bool has_pub = lane < npub;
    const unsigned long long* psrc =
        has_pub ? par_base + static_cast<size_t>(3 + 2 * lane) * st + pub_owner[lane] : par_base;
    unsigned pending = (1u << nmine) - 1u;
    bool pub_pending = has_pub;
    unsigned long long pw0 = 0, pw1 = 0;
    const unsigned long long t0 = globaltimer_ns();
    bool ok = true;
    for (unsigned iter = 1; pending || pub_pending; ++iter) {
#pragma unroll
      for (int k = 0; k < kMaxPollPerLane; ++k) {
        if (pending & (1u << k)) {
          wv[k][0] = ld_relaxed_u64(src[k]);
          wv[k][1] = ld_relaxed_u64(src[k] + st);
          wv[k][2] = ld_relaxed_u64(src[k] + 2 * st);
        }
      }
      if (pub_pending) {
        pw0 = ld_relaxed_u64(psrc);
        pw1 = ld_relaxed_u64(psrc + st);
      }
#pragma unroll
      for (int k = 0; k < kMaxPollPerLane; ++k) {
        if ((pending & (1u << k)) && static_cast<unsigned>(wv[k][0] >> 32) == tag &&
            static_cast<unsigned>(wv[k][1] >> 32) == tag && static_cast<unsigned>(wv[k][2] >> 32) == tag)
          pending &= ~(1u << k);
      }
      if (pub_pending && static_cast<unsigned>(pw0 >> 32) == tag && static_cast<unsigned>(pw1 >> 32) == tag)
        pub_pending = false;
      if (P.poll_ns && (pending || pub_pending)) __nanosleep(P.poll_ns);
      if ((iter & 31u) == 0 && (pending || pub_pending)) {
        if (ld_relaxed_s32(&P.st->abort)) {
          ok = false;
          break;
        }
        if (globaltimer_ns() - t0 > P.timeout_ns) {
          fail(P.st, BBK_ERR_TIMEOUT);
          ok = false;
          break;
        }
      }
    }
    fence_acq_rel_gpu();  // acquire what the other CTAs released
    double v = 0.0;
    int i = INT_MAX;
    if (ok) {
      for (int k = 0; k < nmine; ++k)
        argmax_join(v, i, join_hi_lo(wv[k][1], wv[k][2]), static_cast<int>(wv[k][0] & 0xffffffffu));
    }
    for (int off = 16; off > 0; off >>= 1) {
      const double v2 = __shfl_down_sync(0xffffffffu, v, off);
      const int i2 = __shfl_down_sync(0xffffffffu, i, off);
      argmax_join(v, i, v2, i2);
    }
    const int all_ok = __all_sync(0xffffffffu, ok);
    if (P.pub_ts && blockIdx.x == 0 && all_ok) {
      // diagnostics: (last publish - own publish) and (done - last publish)
      const unsigned long long done = globaltimer_ns();
      unsigned long long last = 0;
      int who = 0;
      for (int sidx = lane; sidx < P.nslots; sidx += 32) {
        const unsigned long long v = __ldcg(P.pub_ts + sidx);
        if (v > last) {
          last = v;
          who = sidx;
        }
      }
      for (int off = 16; off > 0; off >>= 1) {
        const unsigned long long l2 = __shfl_down_sync(0xffffffffu, last, off);
        const int w2 = __shfl_down_sync(0xffffffffu, who, off);
        if (l2 > last) {
          last = l2;
          who = w2;
        }
      }
      if (lane == 0) {
        const unsigned long long mine = __ldcg(P.pub_ts);
        atomicAdd(P.stats + 7, last > mine ? last - mine : 0ull);
        atomicAdd(P.stats + 8, done > last ? done - last : 0ull);
        atomicAdd(P.stats + 16 + 1024 + who, 1ull);
      }
    }
    if (has_pub) out->pub[lane] = join_hi_lo(pw0, pw1);
    if (lane == 0) {
      out->val = v;
      out->idx = i;
      out->ok = all_ok;
    }
  }
  __syncthreads();
}

__device__ __forceinline__ double safe_denominator(double d) {
  // src/block_ldlt_decomposition.cc:21-26 (absolute threshold)
  return fabs(d) <= kDblEpsilon ? 0.0 : d;
}

__device__ __forceinline__ double div_or_zero(double x, double den) {
  return den == 0.0 ? 0.0 : xdiv(x, den);
}

// sum_{q < count} c[q] * w(q) in ascending q, every product and sum rounded
// separately (the reference's order).  The products do not depend on the
// running sum, so they are issued eight at a time ahead of the serial adds.
template <typename WGet>
__device__ __forceinline__ double ordered_dot(const double* c, int count, WGet&& w) {
  double acc = 0.0;
  int q = 0;
  for (; q + 8 <= count; q += 8) {
    double m[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) m[u] = xmul(c[q + u], w(q + u));
#pragma unroll
    for (int u = 0; u < 8; ++u) acc = xadd(acc, m[u]);
  }
  for (; q < count; ++q) acc = xadd(acc, xmul(c[q], w(q)));
  return acc;
}

__global__ void __launch_bounds__(kThreads) panel_kernel(PanelArgs P) {
  extern __shared__ double dsm[];
  __shared__ double s_red_v[kWarps];
  __shared__ int s_red_i[kWarps];
  __shared__ double s_pub[kMaxPub];
  __shared__ ExchangeOut s_x;

  if (ld_relaxed_s32(&P.st->abort)) return;
  const int G = gridDim.x;
  const int c = blockIdx.x;
  const int t = threadIdx.x;
  const int n = P.n;
  const int kstart = ldcg(&P.st->kstart[P.panel & 1]);
  const int S = (n - kstart + G - 1) / G;  // columns per CTA
  const int lo = kstart + c * S;
  const int hi = min(n, lo + S);
  const long long lda = P.lda, ldw = P.ldw;
  const int ldu = P.ldu;
  auto owner = [&](int j) -> int { return (j - kstart) / S; };
  // shared memory: coefficient column, then (when it fits) this CTA's slice
  // of the panel's workspace rows, wsm[q*S + (j - lo)] = W[q, j].
  // Stores other CTAs do not need right away stay out of global memory: the
  // slice of W (flushed at the end of the panel) and the candidate column.
  double* coef = dsm;
  double* wcs = dsm + P.coef_cap;  // candidate values of this CTA's columns
  double* wsm = (P.w_smem && S <= P.smem_cols) ? wcs + P.smem_cols : nullptr;
  auto wget = [&](int q, int j) -> double {
    return wsm ? wsm[q * S + (j - lo)] : ldcg(P.w + q * ldw + j);
  };
  auto wput = [&](int q, int j, double v) {
    if (wsm)
      wsm[q * S + (j - lo)] = v;
    else
      P.w[q * ldw + j] = v;
  };
  const bool timing = P.stats != nullptr && t == 0;
  unsigned long long tm[6] = {0, 0, 0, 0, 0, 0};
  unsigned long long tmark = timing ? globaltimer_ns() : 0;
  auto lap = [&](int k) {
    if (timing) {
      const unsigned long long now = globaltimer_ns();
      tm[k] += now - tmark;
      tmark = now;
    }
  };

  unsigned tag = P.tag_base;
  int p = kstart;
  // coefficients U[q, p] of the current row: rows q < n_old from Ucm column
  // coef_src, then lp - n_old (<= 2) values computed by every CTA.
  int coef_src = p, n_old = 0;
  double extra0 = 0.0, extra1 = 0.0;
  int fix_col = -1;          // A[p][fix_col] must be read from fix_src
  long long fix_src = 0;
  int ncand = 0;

  // Next-row prefetch: the row update of pivot p issues the loads of row p+1
  // (each thread keeps its own columns, j = lo + t + k*kThreads), so their
  // HBM latency hides behind the rest of the step.  A prefetched entry can
  // be stale only in a column that an interchange rewrote meanwhile: the
  // last step's swap column (fix_col, read from the frozen row instead) and
  // the swap column of the step before it (prev_swap, re-read once its
  // write is visible).
  double nav[kCols];
  int nav_row = -1;
  // the next row's coefficient column (rows q < n_old), loaded during the
  // interchange phase when it has at most 2 * kThreads rows
  double cpre[2] = {0.0, 0.0};
  bool coef_pre = false;
  int prev_swap = -1, last_swap = -1;

  while (p < P.nominal_end) {
    const int lp = p - kstart;
    // ---- row update: W[p, j] = A[p, j] - sum_q U[q, p] W[q, j]
    // (CopyCurrentRowToWorkspace + UpdateCurrentRowInWorkspace, :122-162)
    double av[kCols];
    const bool use_nav = nav_row == p;
#pragma unroll
    for (int k = 0; k < kCols; ++k) {
      const int j = lo + t + k * kThreads;
      double v = 0.0;
      if (j < hi && j >= p) {
        if (j == fix_col)
          v = ldcg(P.a + fix_src);
        else if (use_nav && j != prev_swap)
          v = nav[k];
        else
          v = ldcg(P.a + p * lda + j);
      }
      av[k] = v;
    }
#pragma unroll
    for (int k = 0; k < kCols; ++k) {
      const int j = lo + t + k * kThreads;
      nav[k] = (j < hi && j > p) ? ldcg(P.a + (p + 1) * lda + j) : 0.0;
    }
    nav_row = p + 1;
    prev_swap = last_swap;
    last_swap = -1;
    {
      const double* ucol = P.ucm + static_cast<size_t>(coef_src) * ldu;
      if (coef_pre) {
        if (t < n_old) coef[t] = cpre[0];
        if (t + kThreads < n_old) coef[t + kThreads] = cpre[1];
      } else {
        for (int q = t; q < n_old; q += kThreads) coef[q] = ldcg(ucol + q);
      }
      if (t == 0) {
        coef[n_old] = extra0;
        coef[n_old + 1] = extra1;
      }
      if (t < kMaxPub) s_pub[t] = 0.0;
    }
    __syncthreads();
    double best = 0.0;
    int best_j = INT_MAX;
#pragma unroll
    for (int k = 0; k < kCols; ++k) {
      const int j = lo + t + k * kThreads;
      if (j < hi && j >= p) {
        const double acc = ordered_dot(coef, lp, [&](int q) { return wget(q, j); });
        const double wv = xsub(av[k], acc);
        wput(lp, j, wv);
        if (j > p) {
          const double v = fabs(wv);
          if (v > best) {  // FindCurrentRowMax, :164-182
            best = v;
            best_j = j;
          }
        } else {
          s_pub[0] = wv;  // W[p, p]
        }
        if (j == p + 1) s_pub[1] = wv;
        if (j == p + 2) s_pub[2] = wv;
      }
    }
    fix_col = -1;
    lap(0);
    int owners[kMaxPub];
    owners[0] = owner(p);
    owners[1] = p + 1 < n ? owner(p + 1) : 0;
    owners[2] = p + 2 < n ? owner(p + 2) : 0;
    exchange(P, tag++, best, best_j, s_pub, owners, 3, s_red_v, s_red_i, &s_x);
    if (!s_x.ok) return;
    const double omega = s_x.val;
    const int r = s_x.idx;
    const double dpp = s_x.pub[0];
    const double w_p1 = s_x.pub[1];  // W[p, p+1] (current-row version)
    const double w_p2 = s_x.pub[2];  // W[p, p+2]
    __syncthreads();
    lap(1);

    int kind = 1;  // 1: 1x1 at p; -1: 1x1 after p<->r; 2: 2x2 with p+1<->r
    bool cand = false;
    double wc_r = 0.0, wc_p = 0.0, wc_p1 = 0.0, wc_p2 = 0.0;
    // FactorPanel's test, :90-92
    if (!(fabs(dpp) >= xmul(kAlpha, omega) || omega == 0.0)) {
      cand = true;
      ++ncand;
      // ---- candidate column W(i, r) = A(i, r) - sum_q U[q, r] W[q, i]
      // (CopyCandidateToWorkspace + UpdateCandidateInWorkspace, :184-352)
      double cv[kCols];
#pragma unroll
      for (int k = 0; k < kCols; ++k) {
        const int i = lo + t + k * kThreads;
        cv[k] = (i < hi && i >= p) ? (i <= r ? ldcg(P.a + i * lda + r) : ldcg(P.a + r * lda + i)) : 0.0;
      }
      {
        const double* ucol = P.ucm + static_cast<size_t>(r) * ldu;
        for (int q = t; q < lp; q += kThreads) coef[q] = ldcg(ucol + q);
        if (t < kMaxPub) s_pub[t] = 0.0;
      }
      __syncthreads();
      double sig = 0.0;
#pragma unroll
      for (int k = 0; k < kCols; ++k) {
        const int i = lo + t + k * kThreads;
        if (i < hi && i >= p) {
          const double acc = ordered_dot(coef, lp, [&](int q) { return wget(q, i); });
          const double v = xsub(cv[k], acc);
          wcs[i - lo] = v;
          if (i != r) {
            const double av2 = fabs(v);
            sig = (sig < av2) ? av2 : sig;  // std::max, FindCandidateColumnMax :354-367
          } else {
            s_pub[0] = v;
          }
          if (i == p) s_pub[1] = v;
          if (i == p + 1) s_pub[2] = v;
          if (i == p + 2) s_pub[3] = v;
        }
      }
      // stage W[q, p] and W[q, p+1] (q < lp) for the owner of r: the
      // interchange moves one of these columns into column r
      if (p >= lo && p < hi)
        for (int q = t; q < lp; q += kThreads) P.wstage[q] = wget(q, p);
      if (p + 1 >= lo && p + 1 < hi)
        for (int q = t; q < lp; q += kThreads) P.wstage[P.coef_cap + q] = wget(q, p + 1);
      lap(2);
      owners[0] = owner(r);
      owners[1] = owner(p);
      owners[2] = p + 1 < n ? owner(p + 1) : 0;
      owners[3] = p + 2 < n ? owner(p + 2) : 0;
      exchange(P, tag++, sig, 0, s_pub, owners, 4, s_red_v, s_red_i, &s_x);
      if (!s_x.ok) return;
      const double sigma = s_x.val;
      wc_r = s_x.pub[0];
      wc_p = s_x.pub[1];
      wc_p1 = s_x.pub[2];
      wc_p2 = s_x.pub[3];
      __syncthreads();
      lap(3);
      // SelectPivot, :369-390
      if (xsub(xmul(fabs(dpp), sigma), xmul(xmul(kAlpha, omega), omega)) >= 0.0) {
        kind = 1;
      } else if (xsub(fabs(wc_r), xmul(kAlpha, sigma)) >= 0.0) {
        kind = -1;
      } else {
        kind = 2;
      }
      // :104-108: a 2x2 pivot starting at the panel's last column moves that
      // column into the next panel (ShiftBoundaryColumnToNextBlock).
      if (kind == 2 && p == P.nominal_end - 1 && P.can_shift) break;
    }

    if (kind == 1) {
      // ScaleOneByOnePivot (:633-656); after a candidate evaluation the
      // reference's W(p, r) holds the column version of that entry.
      const double d = dpp;
      const double den = safe_denominator(d);
      for (int j = max(lo, p + 1) + t; j < hi; j += kThreads) {
        double wv;
        if (cand && j == r) {
          wv = wc_p;
          wput(lp, j, wv);
        } else {
          wv = wget(lp, j);
        }
        P.ucm[static_cast<size_t>(j) * ldu + lp] = div_or_zero(wv, den);
      }
      if (c == owner(p)) {
        for (int q = t; q < lp; q += kThreads)
          P.uout[static_cast<size_t>(lp) * ldu + q] = ldcg(P.ucm + static_cast<size_t>(p) * ldu + q);
        if (t == 0) {
          P.uout[static_cast<size_t>(lp) * ldu + lp] = d;
          P.ptype[p] = 1;
        }
      }
      // next row's coefficients: U[q, p+1] for q < p, then U[p, p+1]
      coef_src = p + 1;
      n_old = lp;
      extra0 = div_or_zero((cand && r == p + 1) ? wc_p : w_p1, den);
      p += 1;
    } else if (kind == -1) {
      // SwapOneByOnePivot (:392-401, :414-498) + ScaleOneByOnePivot.
      const double d = wc_r;
      const double den = safe_denominator(d);
      for (int j = max(lo, p) + t; j < hi; j += kThreads) {
        if (j == p) {
          wput(lp, j, d);
          continue;
        }
        const double wv = (j == r) ? wc_p : wcs[j - lo];
        wput(lp, j, wv);
        P.ucm[static_cast<size_t>(j) * ldu + lp] = div_or_zero(wv, den);
        // old row p moves to row r (j > r) / column r (j < r); row p itself
        // stays frozen so other CTAs may still read it.
        const double old_apj = ldcg(P.a + p * lda + j);
        if (j > r) {
          P.a[r * lda + j] = old_apj;
        } else if (j < r) {
          P.a[j * lda + r] = old_apj;
        } else {
          P.a[r * lda + r] = ldcg(P.a + p * lda + p);
        }
      }
      if (c == owner(r)) {
        for (int q = t; q < lp; q += kThreads) {
          const double ur = ldcg(P.ucm + static_cast<size_t>(r) * ldu + q);
          P.uout[static_cast<size_t>(lp) * ldu + q] = ur;  // final column p
          P.ucm[static_cast<size_t>(r) * ldu + q] = ldcg(P.ucm + static_cast<size_t>(p) * ldu + q);
          wput(q, r, ldcg(P.wstage + q));
        }
      }
      // previously factored rows: columns p and r exchange (:472-491)
      for (int i = c * kThreads + t; i < kstart; i += G * kThreads) {
        double* x = P.a + i * lda + p;
        double* y = P.a + i * lda + r;
        const double tx = *x;
        *x = *y;
        *y = tx;
      }
      if (c == 0 && t == 0) {
        P.uout[static_cast<size_t>(lp) * ldu + lp] = d;
        P.ptype[p] = 1;
        const int tp = P.perm[p];
        P.perm[p] = P.perm[r];
        P.perm[r] = tp;
      }
      coef_src = (r == p + 1) ? p : p + 1;
      n_old = lp;
      extra0 = div_or_zero((r == p + 1) ? wc_p : wc_p1, den);
      if (p + 1 < r) {
        fix_col = r;
        fix_src = p * lda + (p + 1);  // new A[p+1, r] = old A[p, p+1]
      } else {
        // r == p+1: the next row is the old row p (its diagonal is old A[p, p])
#pragma unroll
        for (int k = 0; k < kCols; ++k) {
          const int j = lo + t + k * kThreads;
          nav[k] = (j < hi && j > p + 1) ? av[k] : ((j == p + 1 && j < hi) ? ldcg(P.a + p * lda + p) : 0.0);
        }
      }
      last_swap = r;
      p += 1;
    } else {
      // SwapTwoByTwoPivot (:403-412, :500-587) + ScaleTwoByTwoPivot (:658-704)
      const int s = p + 1, ls = lp + 1;
      const double d11 = dpp, d21 = wc_p, d22 = wc_r;
      const double det = xsub(xmul(d11, d22), xmul(d21, d21));
      const double i11 = xdiv(d22, det);
      const double i22 = xdiv(d11, det);
      const double i21 = xdiv(-d21, det);
      for (int j = max(lo, p + 2) + t; j < hi; j += kThreads) {
        double x;
        if (j == r) {
          x = w_p1;  // W(p, s) and W(p, r) exchange
          wput(lp, j, x);
        } else {
          x = wget(lp, j);
        }
        const double y = (j == r) ? wc_p1 : wcs[j - lo];
        wput(ls, j, y);
        P.ucm[static_cast<size_t>(j) * ldu + lp] = xadd(xmul(i11, x), xmul(i21, y));
        P.ucm[static_cast<size_t>(j) * ldu + ls] = xadd(xmul(i21, x), xmul(i22, y));
        if (r != s) {
          const double old_asj = ldcg(P.a + s * lda + j);
          if (j > r) {
            P.a[r * lda + j] = old_asj;
          } else if (j < r) {
            P.a[j * lda + r] = old_asj;
          } else {
            P.a[r * lda + r] = ldcg(P.a + s * lda + s);
          }
        }
      }
      if (c == owner(p)) {
        for (int q = t; q < lp; q += kThreads)
          P.uout[static_cast<size_t>(lp) * ldu + q] = ldcg(P.ucm + static_cast<size_t>(p) * ldu + q);
      }
      if (c == owner(r)) {
        for (int q = t; q < lp; q += kThreads) {
          const double ur = ldcg(P.ucm + static_cast<size_t>(r) * ldu + q);
          P.uout[static_cast<size_t>(ls) * ldu + q] = ur;  // final column s
          if (r != s) {
            P.ucm[static_cast<size_t>(r) * ldu + q] = ldcg(P.ucm + static_cast<size_t>(s) * ldu + q);
            wput(q, r, ldcg(P.wstage + P.coef_cap + q));
          }
        }
      }
      if (r != s) {
        for (int i = c * kThreads + t; i < kstart; i += G * kThreads) {
          double* x = P.a + i * lda + s;
          double* y = P.a + i * lda + r;
          const double tx = *x;
          *x = *y;
          *y = tx;
        }
      }
      if (c == 0 && t == 0) {
        P.uout[static_cast<size_t>(lp) * ldu + lp] = d11;
        P.uout[static_cast<size_t>(ls) * ldu + lp] = d21;
        P.uout[static_cast<size_t>(ls) * ldu + ls] = d22;
        P.ptype[p] = 2;
        P.ptype[s] = -2;
        const int tp = P.perm[s];
        P.perm[s] = P.perm[r];
        P.perm[r] = tp;
      }
      // next row p+2: coefficients U[q, p+2], q < p, then U[p, p+2], U[s, p+2]
      const double x = (r == p + 2) ? w_p1 : w_p2;
      const double y = (r == p + 2) ? wc_p1 : wc_p2;
      coef_src = (r == p + 2) ? s : p + 2;
      n_old = lp;
      extra0 = xadd(xmul(i11, x), xmul(i21, y));
      extra1 = xadd(xmul(i21, x), xmul(i22, y));
      if (p + 2 < r) {
        fix_col = r;
        fix_src = s * lda + (p + 2);  // new A[p+2, r] = old A[s, p+2]
      }
      if (r != s) last_swap = r;
      p += 2;
    }
    coef_pre = n_old <= 2 * kThreads;
    if (coef_pre) {
      const double* ucol = P.ucm + static_cast<size_t>(coef_src) * ldu;
      cpre[0] = t < n_old ? ldcg(ucol + t) : 0.0;
      cpre[1] = t + kThreads < n_old ? ldcg(ucol + t + kThreads) : 0.0;
    }
    __syncthreads();
    lap(4);
  }

  if (P.stats && t == 0)
    for (int k = 0; k < 5; ++k) atomicAdd(P.stats + 16 + 2048 + c * 5 + k, tm[k]);
  // the trailing update reads W from global memory
  if (wsm) {
    const int kb = p - kstart;
    for (int q = 0; q < kb; ++q)
      for (int j = lo + t; j < hi; j += kThreads) P.w[q * ldw + j] = wsm[q * S + (j - lo)];
  }
  if (c == 0 && t == 0) {
    // panel range [kstart, p); the next panel starts at p.
    P.st->kstart[(P.panel + 1) & 1] = p;
    if (P.panel_end) P.panel_end[P.panel] = p;
    if (P.stats) {
      for (int k = 0; k < 5; ++k) atomicAdd(P.stats + k, tm[k]);
      atomicAdd(P.stats + 5, static_cast<unsigned long long>(p - kstart));
      atomicAdd(P.stats + 6, static_cast<unsigned long long>(ncand));
    }
  }
}

// Writes the panel's compact factor rows [k0, e) into A:
// A[q, j] = Uout (pivot columns j < e) or Ucm (trailing columns j >= e).
constexpr int kFinTile = 32;
__global__ void __launch_bounds__(256) finalize_kernel(double* a, long long lda, const double* ucm,
                                                       int ldu, const double* uout, int n,
                                                       DeviceState* st, int panel) {
  __shared__ double tile[kFinTile][kFinTile + 1];
  if (ld_relaxed_s32(&st->abort)) return;
  const int k0 = ldcg(&st->kstart[panel & 1]);
  const int e = ldcg(&st->kstart[(panel + 1) & 1]);
  const int kb = e - k0;
  if (kb <= 0) return;
  // tiles over (q in [0, kb), j in [k0, n))
  const int qt = (kb + kFinTile - 1) / kFinTile;
  const int jt = (n - k0 + kFinTile - 1) / kFinTile;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
  for (int tileid = blockIdx.x; tileid < qt * jt; tileid += gridDim.x) {
    const int q0 = (tileid % qt) * kFinTile;
    const int j0 = k0 + (tileid / qt) * kFinTile;
    // load: rows of the tile are columns j (contiguous in q)
    for (int jj = ty; jj < kFinTile; jj += 8) {
      const int j = j0 + jj, q = q0 + tx;
      double v = 0.0;
      if (j < n && q < kb) {
        v = (j < e) ? uout[static_cast<size_t>(j - k0) * ldu + q]
                    : ucm[static_cast<size_t>(j) * ldu + q];
      }
      tile[jj][tx] = v;
    }
    __syncthreads();
    for (int qq = ty; qq < kFinTile; qq += 8) {
      const int q = q0 + qq, j = j0 + tx;
      if (q < kb && j < n && j >= k0 + q) a[static_cast<size_t>(k0 + q) * lda + j] = tile[tx][qq];
    }
    __syncthreads();
  }
}

__global__ void init_kernel(int n, int* perm, int* pivot_types, DeviceState* st,
                            unsigned long long* slots, size_t slot_words) {
  const size_t i0 = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
  for (size_t i = i0; i < static_cast<size_t>(n); i += stride) {
    perm[i] = static_cast<int>(i);
    pivot_types[i] = 0;
  }
  for (size_t i = i0; i < slot_words; i += stride) slots[i] = 0ull;
  if (i0 == 0) {
    st->kstart[0] = 0;
    st->kstart[1] = 0;
    st->abort = 0;
    st->status = 0;
  }
}

__global__ void status_copy_kernel(const DeviceState* st, int* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *out = st->status;
}

// Exchange probe.  With nslots == gridDim.x + 1 the single exchange also
// waits for a record nobody writes, so it must end by timeout (the
// bounded-wait test).  With nslots == gridDim.x it runs `iters` exchanges
// back to back and CTA 0 stores the elapsed nanoseconds in stats[0] (the
// exchange-latency measurement).
__global__ void __launch_bounds__(kThreads) probe_kernel(PanelArgs P) {
  __shared__ double s_red_v[kWarps];
  __shared__ int s_red_i[kWarps];
  __shared__ double s_pub[kMaxPub];
  __shared__ ExchangeOut s_x;
  if (threadIdx.x < kMaxPub) s_pub[threadIdx.x] = 0.0;
  int owners[kMaxPub] = {0, 0, 0, 0, 0, 0};
  __syncthreads();
  const unsigned long long t0 = globaltimer_ns();
  for (int it = 0; it < P.n; ++it) {
    exchange(P, P.tag_base + it, static_cast<double>(blockIdx.x), blockIdx.x, s_pub, owners, 3,
             s_red_v, s_red_i, &s_x);
    if (!s_x.ok) return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && P.stats) P.stats[0] = globaltimer_ns() - t0;
}

}  // namespace

static int cooperative_launch(const void* fn, int grid, PanelArgs* args, cudaStream_t s) {
  void* kargs[] = {args};
  cudaError_t err = cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kThreads), kargs, 0, s);
  if (err != cudaSuccess) return cuda_error(err, "cudaLaunchCooperativeKernel(panel)");
  count_launch();
  return BBK_OK;
}

int panel_grid_size(int n) {
  // enough CTAs that each owns <= 64 columns where possible, at most one per
  // SM, and never more than kCols columns per thread.  BBK_PANEL_COLS
  // overrides the target columns per CTA (tuning).
  const int sms = device_sm_count();
  static const int cols = [] {
    const char* e = getenv("BBK_PANEL_COLS");
    const int v = e ? atoi(e) : 0;
    return v > 0 ? v : 64;
  }();
  int g = (n + cols - 1) / cols;
  if (g > sms) g = sms;
  const int need = (n + kCols * kThreads - 1) / (kCols * kThreads);
  if (g < need) g = need;
  if (g < 1) g = 1;
  return g;
}

int panel_max_n() { return device_sm_count() * kCols * kThreads; }

int launch_init(int n, int* perm, int* pivot_types, DeviceState* st, unsigned long long* slots,
                size_t slot_words, cudaStream_t s) {
  init_kernel<<<256, 256, 0, s>>>(n, perm, pivot_types, st, slots, slot_words);
  BBK_CUDA_TRY(cudaGetLastError());
  count_launch();
  return BBK_OK;
}

int launch_panel(const FactorPlan& plan, int panel, cudaStream_t s) {
  PanelArgs P{};
  P.n = plan.n;
  P.panel = panel;
  const long long nominal = static_cast<long long>(panel + 1) * plan.b;
  P.nominal_end = nominal < plan.n ? static_cast<int>(nominal) : plan.n;
  P.can_shift = panel + 1 < plan.nb;
  P.a = plan.a;
  P.lda = plan.lda;
  P.w = plan.w;
  P.ldw = plan.ldw;
  P.ucm = plan.ucm;
  P.ldu = plan.ldu;
  P.uout = plan.uout;
  P.wc = plan.wc;
  P.wstage = plan.wc + align_up(static_cast<size_t>(plan.n), 64);
  P.perm = plan.perm;
  P.ptype = plan.pivot_types;
  P.panel_end = plan.panel_end;
  P.slots = plan.slots;
  P.st = plan.state;
  P.nslots = plan.grid;
  P.slot_stride = plan.grid;
  // tags: distinct for every exchange of the call (slots are zeroed per call)
  P.tag_base = 1u + static_cast<unsigned>(panel) * (2u * static_cast<unsigned>(plan.b) + 8u);
  P.timeout_ns = plan.timeout_ns;
  P.stats = plan.stats;
  P.pub_ts = plan.stats ? plan.stats + 16 : nullptr;
  static const unsigned poll_ns = [] {
    const char* e = getenv("BBK_POLL_NS");
    return e ? static_cast<unsigned>(atoi(e)) : 0u;
  }();
  P.poll_ns = poll_ns;
  if (plan.grid > 32 * kMaxPollPerLane)
    return set_error(BBK_ERR_INVALID_ARGUMENT, "panel grid %d exceeds %d", plan.grid, 32 * kMaxPollPerLane);
  // shared memory: coefficient column + (if it fits) the CTA's W slice
  const int smax = (plan.n + plan.grid - 1) / plan.grid;
  P.coef_cap = static_cast<int>(align_up(static_cast<size_t>(plan.b) + 4, 2));
  size_t bytes = (static_cast<size_t>(P.coef_cap) + smax) * sizeof(double);
  const size_t wbytes = static_cast<size_t>(plan.b + 2) * smax * sizeof(double);
  const size_t limit = 220 * 1024;
  P.w_smem = bytes + wbytes <= limit;
  P.smem_cols = smax;
  if (P.w_smem) bytes += wbytes;
  BBK_CUDA_TRY(cudaFuncSetAttribute(panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(bytes)));
  void* kargs[] = {&P};
  cudaError_t err = cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(panel_kernel),
                                                dim3(plan.grid), dim3(kThreads), kargs, bytes, s);
  if (err != cudaSuccess) return cuda_error(err, "cudaLaunchCooperativeKernel(panel)");
  count_launch();
  return BBK_OK;
}

int launch_finalize(const FactorPlan& plan, int panel, cudaStream_t s) {
  const int sms = device_sm_count();
  finalize_kernel<<<2 * sms, 256, 0, s>>>(plan.a, plan.lda, plan.ucm, plan.ldu, plan.uout,
                                          plan.n, plan.state, panel);
  BBK_CUDA_TRY(cudaGetLastError());
  count_launch();
  return BBK_OK;
}

int launch_status_copy(const DeviceState* st, int* status_out, cudaStream_t s) {
  status_copy_kernel<<<1, 32, 0, s>>>(st, status_out);
  BBK_CUDA_TRY(cudaGetLastError());
  count_launch();
  return BBK_OK;
}

int launch_probe_wait(int ctas, int nslots, int iters, unsigned long long timeout_ns,
                      DeviceState* st, unsigned long long* slots, unsigned long long* stats,
                      cudaStream_t s) {
  PanelArgs P{};
  P.slots = slots;
  P.st = st;
  P.nslots = nslots;
  P.slot_stride = ctas + 1;
  P.tag_base = 7u;
  P.timeout_ns = timeout_ns;
  P.n = iters;
  P.stats = stats;
  return cooperative_launch(reinterpret_cast<const void*>(probe_kernel), ctas, &P, s);
}

}  // namespace bbk
