// Panel factorization of the blocked Bunch-Kaufman LDL^T: one persistent
// cooperative launch per panel runs the panel's sequential pivot chain with
// all CTAs, each owning a contiguous range of column slots.
//
// Follows BlockLdltDecomposition::FactorPanel and its helpers
// (src/block_ldlt_decomposition.cc:80-704 in wentianshu/BlockedBunchKaufmanLDLT)
// in the reference's own operation order, so the panel's arithmetic is
// bitwise identical to the reference (every product and sum separately
// rounded; this file is also compiled with --fmad=false).
//
// Slots.  Every active index x >= k0 (k0 = the panel's first row) owns a
// slot: the physical row/column of A that holds its data, plus that slot's
// workspace column W[., slot], U column Uslot[slot, .] and candidate value.
// A symmetric interchange p <-> r (SwapOneByOnePivot / SwapTwoByTwoPivot,
// :392-587) only exchanges the slots of p and r in two small maps that every
// CTA updates identically: the window map (slot of each of the panel's rows)
// and the CTA's own slot -> index map.  No data moves while the panel runs,
// A is never written by this kernel, and the only values other CTAs read
// from global memory are U columns written at least one exchange earlier.
//
// Data during a panel:
//   shared   the CTA's slice of the panel rows: row m starts as
//            A[k0 + m, slot] (loaded once) and becomes W[k0 + m, slot] when
//            pivot row m is updated; the candidate column; the row computed
//            ahead; two coefficient columns; the maps.
//   Uslot    U[q, x] at Uslot[slot(x) * ldu + q].
//   dlog     D of every pivot; ptype.
// At the end the CTAs write W and U in final column order, publish the slot
// of every index, and gather the rows of the moved indices (and the
// factored rows' entries at the moved columns) into staging buffers.
// finalize_kernel then writes the interchanged entries back, the
// permutation, and the panel's compact factor rows.
//
// Per pivot step the grid meets in an exchange (arrival counter + one record
// per CTA) that is also the argmax reduction: once for the row, and once more
// when a candidate column is needed.  A candidate step also computes the next
// row as keeping its pivot would leave it and reduces that row's argmax in
// the same exchange, so when the pivot is kept (most steps of saddle-point
// matrices) the next step starts without a row exchange.
#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstdlib>

#include "bbk_internal.cuh"

#ifndef BBK_PANEL_THREADS
#define BBK_PANEL_THREADS 192
#endif

namespace bbk {
namespace {

constexpr int kThreads = BBK_PANEL_THREADS;
constexpr int kWarps = kThreads / 32;  // compute warps
constexpr int kCommWarp = kWarps;       // the communication warp
constexpr int kBlock = kThreads + 32;   // compute warps + the communication warp
constexpr int kCols = 3;  // slots per thread: S <= kCols * kThreads
constexpr int kPairSlots = 96;  // slots per CTA up to which the warps split the candidate sums by rows
constexpr int kAllWarps = kBlock / 32;
constexpr int kMaxGrid = kBlock;  // CTAs of a panel launch: every thread reads one record
constexpr int kRecA = 4;  // argmax words of a record: idx, value hi, value lo, slot
constexpr int kRecB = 6;  // second argmax: idx, value hi, value lo, slot, payload hi, payload lo
static_assert(kRecA + kRecB + 2 * kMaxPub <= kSlotWords, "record too large");
static_assert(kSlotWords <= 32, "one record word per lane of the communication warp");

struct PanelArgs {
  int n;
  int panel;
  int nominal_end;  // min((panel+1)*b, n)
  int can_shift;    // another panel follows
  int win_rows;     // b + 2: panel rows staged per slot
  int win_pad;      // ints reserved for the window map
  double* a;
  long long lda;
  double* w;         // W rows, final column order (for the trailing update)
  long long ldw;
  double* wslot;     // W rows by slot when shared memory cannot hold them
  double* uslot;     // U by slot
  double* ucm;       // U, final column order: ucm[x * ldu + q]
  int ldu;
  double* dlog;      // dlog[2l] = D(l, l); dlog[2l+1] = D(l, l+1) of a 2x2
  int* srcmap;       // slot of index x at the end of the panel
  int* moved;        // 2 x move_cap
  int move_cap;
  double* gbuf;      // move_cap x ldw
  int* moves;        // nb x 2 x move_cap: each panel's moves, for the deferred column exchanges
  int* move_counts;  // nb
  int* bounds;       // 2 nb: each panel's [start, end)
  int* permbuf;
  int* perm;
  int* ptype;
  int* panel_end;
  unsigned long long* slots;
  DeviceState* st;
  int nslots;        // records each exchange waits for (gridDim.x normally)
  int slot_stride;   // records per parity in `slots` (>= nslots)
  unsigned long long timeout_ns;
  int coef_cap;      // doubles reserved for each coefficient column
  int w_smem;        // keep this CTA's panel rows in shared memory
  int smem_cols;     // slice width the shared-memory allocation holds
  int wcap;          // doubles of shared memory for panel rows: all of them (w_smem), else the
                     // first wcap / S rows of the slice (the rest in wslot)
  unsigned long long* stats;  // optional per-phase nanoseconds (CTA 0)
  unsigned poll_ns;           // pause between polls of the arrival counter
  double* pivlog;             // optional decision log, kPivLogWords per position
};

__device__ __forceinline__ void fail(DeviceState* st, int code) {
  atomicCAS(&st->status, 0, code);
  atomicExch(&st->abort, 1);
}

__device__ __forceinline__ double join_hi_lo(unsigned long long hi, unsigned long long lo) {
  const unsigned long long bits = ((hi & 0xffffffffull) << 32) | (lo & 0xffffffffull);
  return __longlong_as_double(static_cast<long long>(bits));
}

__device__ __forceinline__ unsigned half_of(double x, bool high) {
  const unsigned long long bits = static_cast<unsigned long long>(__double_as_longlong(x));
  return high ? static_cast<unsigned>(bits >> 32) : static_cast<unsigned>(bits);
}

// Argmax candidate of an exchange: value, index, the slot holding the index,
// and (second channel) a payload double that travels with the winner.
struct Cand {
  double v;
  int i;
  int s;
  double pay;
};
__device__ __forceinline__ Cand no_cand() { return Cand{0.0, INT_MAX, -1, 0.0}; }

// Argmax combine with the reference's tie rule (src/block_ldlt_decomposition.cc:
// 164-182 scans ascending columns with a strict '>'): larger value wins, equal
// values keep the lower index.  NaN never enters (callers skip it).  With
// distinct indices this is a total order, so any combine tree gives the same
// winner.
__device__ __forceinline__ void argmax_join(Cand& a, const Cand& b) {
  if (b.v > a.v || (b.v == a.v && b.i < a.i)) a = b;
}

// Warp-wide argmax_join, every lane gets the result.  The values are never
// negative or NaN, so their bit patterns order like the values: the maximum
// comes from two integer reductions (high word, then low word among the
// lanes that hold the highest high word), the index from a third.
template <bool kPay>
__device__ __forceinline__ void warp_argmax(Cand& c) {
  const unsigned long long key = static_cast<unsigned long long>(__double_as_longlong(c.v));
  const unsigned hi = static_cast<unsigned>(key >> 32), lo = static_cast<unsigned>(key);
  const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
  const unsigned mlo = __reduce_max_sync(0xffffffffu, hi == mhi ? lo : 0u);
  const bool top = hi == mhi && lo == mlo;
  const unsigned midx = __reduce_min_sync(0xffffffffu, top ? static_cast<unsigned>(c.i) : 0xffffffffu);
  const int who = __ffs(__ballot_sync(0xffffffffu, top && static_cast<unsigned>(c.i) == midx)) - 1;
  c.v = __longlong_as_double(static_cast<long long>((static_cast<unsigned long long>(mhi) << 32) | mlo));
  c.i = static_cast<int>(midx);
  c.s = __shfl_sync(0xffffffffu, c.s, who);
  if (kPay) c.pay = __shfl_sync(0xffffffffu, c.pay, who);
}

// Shared memory of the exchanges.
struct XShared {
  Cand pa[kWarps], pb[kWarps];        // this CTA's record: the compute warps' partials
  Cand ra[kAllWarps], rb[kAllWarps];  // the grid's records: one partial per warp
  int ok[kAllWarps];
  double pub[kMaxPub];                // published doubles of this exchange
};

struct XResult {
  Cand a, b;
  bool ok;
};

// Barrier of the compute warps only (named barrier 1): the communication
// warp may be inside a release fence meanwhile.
__device__ __forceinline__ void compute_warps_sync() {
  asm volatile("bar.sync 1, %0;" ::"n"(kThreads) : "memory");
}

__device__ __forceinline__ void cp_async_8(double* smem_dst, const double* gsrc) {
  const unsigned saddr = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(saddr), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// CTA-collective grid exchange: reduce this CTA's argmax candidate `ca` (and
// `cb` with kTwo) over the CTA, publish the CTA's record (the reductions plus
// the npub doubles of pub_in), and return the grid-wide argmax of every
// channel once all `nslots` CTAs of this exchange have arrived; X.pub[k] then
// holds pub_in[k] of CTA pub_owner[k].  Must be called by every thread.
//
// Records are structure-of-arrays: word w of CTA c lives at
// slots[((tag & 1) * kSlotWords + w) * slot_stride + c], so one warp load
// reads word w of 32 consecutive CTAs.  A CTA stores its record, then adds
// one to the arrival counter; the communication warp polls that single word
// (acquire loads) until it reaches `target`, and after a CTA barrier thread
// c reads the record of CTA c.  Polling the records themselves instead is
// about three times slower (every SM hammering lines that are being
// written).  Every record word also carries the exchange's tag in its high
// half, which the reader checks: the record stores are not ordered before
// the arrival.  Two record sets alternate (tag parity): no CTA can be two
// exchanges ahead of another.
//
// Ordering.  The arrival is issued by the thread that issued the CTA's
// release fence (here when `release`, or earlier by the caller, after a CTA
// barrier that follows the writes to publish), so after the exchange this
// CTA sees everything the other CTAs wrote before their fence.
template <bool kTwo>
__device__ __forceinline__ XResult exchange(const PanelArgs& P, unsigned tag, bool release, Cand ca, Cand cb,
                                            const double* pub_in, const int (&pub_owner)[kMaxPub], int npub,
                                            XShared& X) {
  constexpr int kRec = kRecA + (kTwo ? kRecB : 0);
  const int t = threadIdx.x;
  const int lane = t & 31, warp = t >> 5;
  warp_argmax<false>(ca);
  if (kTwo) warp_argmax<true>(cb);
  if (lane == 0 && warp < kWarps) {
    X.pa[warp] = ca;
    if (kTwo) X.pb[warp] = cb;
  }
  __syncthreads();  // also orders this CTA's global writes before a release
  const unsigned long long t_stat = P.stats ? globaltimer_ns() : 0;
  unsigned long long* par_base =
      P.slots + static_cast<size_t>(tag & 1u) * kSlotWords * P.slot_stride;
  const size_t st = P.slot_stride;
  unsigned long long t0 = 0;  // read when a wait turns out to be long
  if (warp == kCommWarp) {
    // one compute warp's partial per lane, reduced across the warp
    Cand a = lane < kWarps ? X.pa[lane] : no_cand();
    Cand b = kTwo && lane < kWarps ? X.pb[lane] : no_cand();
    warp_argmax<false>(a);
    if (kTwo) warp_argmax<true>(b);
    if (lane == 0 && release) fence_acq_rel_gpu();
    if (lane < kRec + 2 * npub) {
      unsigned word;
      if (lane == 0) {
        word = static_cast<unsigned>(a.i);
      } else if (lane < 3) {
        word = half_of(a.v, lane == 1);
      } else if (lane == 3) {
        word = static_cast<unsigned>(a.s);
      } else if (kTwo && lane == 4) {
        word = static_cast<unsigned>(b.i);
      } else if (kTwo && lane < 7) {
        word = half_of(b.v, lane == 5);
      } else if (kTwo && lane == 7) {
        word = static_cast<unsigned>(b.s);
      } else if (kTwo && lane < kRec) {
        word = half_of(b.pay, lane == 8);
      } else {
        word = half_of(pub_in[(lane - kRec) >> 1], ((lane - kRec) & 1) == 0);
      }
      st_relaxed_u64(par_base + static_cast<size_t>(lane) * st + blockIdx.x, tag_word(tag, word));
    }
    // arrive, then wait for every CTA of this exchange
    if (lane == 0) red_relaxed_add_u64(&P.st->xcount, 1ull);
    const unsigned long long target = static_cast<unsigned long long>(P.nslots) * tag;
    bool ok = true;
    for (unsigned iter = 1;; ++iter) {
      if (__all_sync(0xffffffffu, ld_acquire_u64(&P.st->xcount) >= target)) break;
      if (P.poll_ns) __nanosleep(P.poll_ns);
      if ((iter & 31u) == 0) {
        if (iter == 32) t0 = globaltimer_ns();
        const bool stop = __any_sync(0xffffffffu, ld_relaxed_s32(&P.st->abort) != 0);
        const bool late = __any_sync(0xffffffffu, globaltimer_ns() - t0 > P.timeout_ns);
        if (stop || late) {
          if (lane == 0 && !stop) fail(P.st, BBK_ERR_TIMEOUT);
          ok = false;
          break;
        }
      }
    }
    if (lane == 0) X.ok[kAllWarps - 1] = ok;
  }
  __syncthreads();
  XResult r;
  r.ok = X.ok[kAllWarps - 1] != 0;
  if (!r.ok) return r;  // uniform over the CTA
  // ---- read: thread c reads the record of CTA c; lanes of the communication
  // warp below npub also read published word pairs.  A word whose tag is not
  // yet this exchange's is read again (its store may land after the arrival).
  const bool has_rec = t < P.nslots;
  const bool has_pub = warp == kCommWarp && lane < npub;
  int owner = 0;
#pragma unroll
  for (int k = 0; k < kMaxPub; ++k)
    if (lane == k) owner = pub_owner[k];
  const unsigned long long* rsrc = par_base + (has_rec ? t : 0);
  const unsigned long long* psrc =
      par_base + static_cast<size_t>(kRec + 2 * (has_pub ? lane : 0)) * st + (has_pub ? owner : 0);
  unsigned long long w[kRec];
  unsigned long long pw0 = 0, pw1 = 0;
  bool rec_pending = has_rec, pub_pending = has_pub, ok = true;
  for (unsigned iter = 1;; ++iter) {
    if (rec_pending) {
#pragma unroll
      for (int k = 0; k < kRec; ++k) w[k] = __ldcg(rsrc + k * st);
    }
    if (pub_pending) {
      pw0 = __ldcg(psrc);
      pw1 = __ldcg(psrc + st);
    }
    if (rec_pending) {
      bool all = true;
#pragma unroll
      for (int k = 0; k < kRec; ++k) all = all && static_cast<unsigned>(w[k] >> 32) == tag;
      rec_pending = !all;
    }
    if (pub_pending && static_cast<unsigned>(pw0 >> 32) == tag && static_cast<unsigned>(pw1 >> 32) == tag)
      pub_pending = false;
    if (!__any_sync(0xffffffffu, rec_pending || pub_pending)) break;
    if (iter == 32) t0 = globaltimer_ns();
    if ((iter & 31u) == 0 && __any_sync(0xffffffffu, globaltimer_ns() - t0 > P.timeout_ns)) {
      if (lane == 0) fail(P.st, BBK_ERR_TIMEOUT);
      ok = false;
      break;
    }
  }
  if (P.stats && blockIdx.x == 0 && t == kThreads) atomicAdd(P.stats + 7, globaltimer_ns() - t_stat);
  // ---- reduce the records: per warp, then every thread over the warps
  Cand ra = no_cand(), rb = no_cand();
  if (has_rec && ok) {
    ra = Cand{join_hi_lo(w[1], w[2]), static_cast<int>(w[0] & 0xffffffffu),
              static_cast<int>(w[3] & 0xffffffffu), 0.0};
    if (kTwo)
      rb = Cand{join_hi_lo(w[5], w[6]), static_cast<int>(w[4] & 0xffffffffu),
                static_cast<int>(w[7] & 0xffffffffu), join_hi_lo(w[8], w[9])};
  }
  warp_argmax<false>(ra);
  if (kTwo) warp_argmax<true>(rb);
  const int wok = __all_sync(0xffffffffu, ok);
  if (lane == 0) {
    X.ra[warp] = ra;
    if (kTwo) X.rb[warp] = rb;
    X.ok[warp] = wok;
  }
  if (has_pub) X.pub[lane] = join_hi_lo(pw0, pw1);
  __syncthreads();
  // every warp reduces the per-warp partials (one per lane)
  r.a = lane < kAllWarps ? X.ra[lane] : no_cand();
  r.b = kTwo && lane < kAllWarps ? X.rb[lane] : no_cand();
  warp_argmax<false>(r.a);
  if (kTwo) warp_argmax<true>(r.b);
  r.ok = __all_sync(0xffffffffu, lane >= kAllWarps || X.ok[lane] != 0);
  return r;
}

// kOrdered: the row and candidate dot products in the reference's order
// (bitwise the reference); otherwise reassociated (split_dot).
// kSmemW: the CTA's panel rows live in shared memory (else in global memory,
// for orders whose slice does not fit).
template <bool kOrdered, bool kSmemW>
__global__ void __launch_bounds__(kBlock, 1) panel_kernel(PanelArgs P) {
  extern __shared__ double dsm[];
  __shared__ XShared X;
  __shared__ double s_pub[kMaxPub];

  if (ld_relaxed_s32(&P.st->abort)) return;
  const int G = gridDim.x;
  const int c = blockIdx.x;
  const int t = threadIdx.x;
  // slot-mapped work uses the compute threads only: the communication warp's
  // tz puts its slots beyond every range
  const int tz = t < kThreads ? t : (1 << 28);
  const int n = P.n;
  const int kstart = ldcg(&P.st->kstart[P.panel & 1]);
  const int S = (n - kstart + G - 1) / G;  // slots per CTA
  // reassociated modes with at most kPairSlots slots per CTA: the compute
  // warps split the rows of the candidate and look-ahead sums
  const bool paired = !kOrdered && S <= kPairSlots;
  const int lo = kstart + c * S;
  const int hi = min(n, lo + S);
  const int width = max(0, hi - lo);
  const int nwin = min(P.win_rows, n - kstart);  // panel rows staged per slot
  const long long lda = P.lda, ldw = P.ldw;
  const int ldu = P.ldu;
  auto owner = [&](int z) -> int { return (z - kstart) / S; };
  // shared memory: two coefficient columns, candidate column and row computed
  // ahead of this CTA's slots, the per-warp partial sums, the slots' panel
  // rows wsm[m*S + (z - lo)] (all of them, or the first srows), then the maps
  double* coef = dsm;
  double* coef2 = dsm + P.coef_cap;  // coefficients of a row computed ahead
  double* wcs = dsm + 2 * P.coef_cap;
  double* svs = wcs + P.smem_cols;   // the row computed ahead, by slot
  double* wpart = svs + P.smem_cols;  // per-warp partial sums: 2 x kWarps x kPairSlots
  double* wsm = wpart + 2 * kWarps * kPairSlots;  // wcap doubles
  int* win = reinterpret_cast<int*>(wsm + P.wcap);
  int* mypos = win + P.win_pad;  // index held by slot lo + zz
  // panel rows kept in shared memory: all of them, or as many rows of this
  // panel's slot width as the allocation holds
  const int srows = kSmemW ? P.win_rows : min(P.win_rows, P.wcap / max(S, 1));
  auto wat = [&](int m, int z) -> double& {
    if (kSmemW || m < srows) return wsm[m * S + (z - lo)];
    return P.wslot[m * ldw + z];
  };
  // the same, split by where the rows live (the hot dot products run over
  // the shared-memory rows and then the global ones)
  auto wat_s = [&](int m, int z) -> double { return wsm[m * S + (z - lo)]; };
  auto wat_g = [&](int m, int z) -> double { return P.wslot[m * ldw + z]; };
  // A(x, z) of the symmetric matrix from its upper triangle (A is not written
  // while the panel runs)
  auto asym = [&](int x, int z) -> double {
    return x <= z ? __ldg(P.a + static_cast<long long>(x) * lda + z)
                  : __ldg(P.a + static_cast<long long>(z) * lda + x);
  };
  auto aptr = [&](int x, int z) -> const double* {
    return x <= z ? P.a + static_cast<long long>(x) * lda + z : P.a + static_cast<long long>(z) * lda + x;
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

  for (int m = t; m < nwin; m += kBlock) win[m] = kstart + m;
  for (int zz = t; zz < width; zz += kBlock) mypos[zz] = lo + zz;
  // stage the panel rows of A for this CTA's slots
  for (int idx = t; idx < nwin * width; idx += kBlock) {
    const int m = idx / width, zz = idx - m * width;
    const int x = kstart + m, z = lo + zz;
    const double* src = x <= z ? P.a + static_cast<long long>(x) * lda + z
                               : P.a + static_cast<long long>(z) * lda + x;
    if (kSmemW || m < srows)
      cp_async_8(&wsm[m * S + zz], src);
    else
      P.wslot[m * ldw + z] = __ldg(src);
  }
  cp_async_wait_all();
  __syncthreads();

  // exchanges are numbered across the factorization; the k-th (from 1) uses
  // tag k
  unsigned seq = static_cast<unsigned>(ldcg(&P.st->xseq[P.panel & 1]));
  int p = kstart;
  // coefficients U[q, p] of the current row: rows q < n_old from the Uslot
  // column of p's slot, then lp - n_old (<= 2) values computed by every CTA.
  int n_old = 0;
  double extra0 = 0.0, extra1 = 0.0;
  int ncand = 0, nahead = 0;
  // the next row's coefficient column, loaded during the scaling phase when
  // it has at most 2 * kThreads rows
  double cpre[2] = {0.0, 0.0};
  bool coef_pre = false;
  // Rows computed ahead.  A candidate step whose outcome may be "keep the
  // 1x1 pivot p" (r != p+1) also updates row p+1 during its candidate phase,
  // as that outcome would leave it, and reduces that row's argmax in the
  // candidate exchange.  When the pivot is kept, the next step starts with
  // its row and argmax known and skips its row update and first exchange.
  // Its U row (written by this step's scaling, after the last exchange) is
  // then not yet visible to other CTAs: the two values of that row the next
  // step needs travel as scalars (u_prev_r = U[p, r'] for its candidate
  // column, carry = U[p, p+2] for the row after it), and its candidate phase
  // releases the row.  In the ordered mode row p+1 is summed in the
  // reference's order (the last term, which involves the candidate's result
  // at column r, is added after the exchange), so results do not change.
  bool ahead = false;
  // loaded one step ahead: the next row's coefficient column (ca) and the
  // candidate's U column (cr), at most 2 * kThreads rows each
  double ca0 = 0.0, ca1 = 0.0, cr0 = 0.0, cr1 = 0.0;
  double nx_omega = 0.0, nx_dpp = 0.0, nx_w1 = 0.0, nx_w2 = 0.0;
  int nx_r = 0, nx_rs = 0;
  double u_prev_r = 0.0, carry = 0.0;

  while (p < P.nominal_end) {
    const int lp = p - kstart;
    const int sp = win[lp];
    const bool was_ahead = ahead;
    ahead = false;
    // U rows whose writes by other CTAs this CTA may read: every row before
    // lp, except the previous one when this row was computed ahead
    const int nrel = was_ahead ? lp - 1 : lp;
    double omega, dpp, w_p1, w_p2;
    int r, rs;
    if (!was_ahead) {
      // the row of p is staged in shared memory unless an interchange gave p a
      // slot whose staged row was already consumed
      const bool staged = (sp - kstart) == lp;
      // ---- row update: W[p, j] = A[p, j] - sum_q U[q, p] W[q, j]
      // (CopyCurrentRowToWorkspace + UpdateCurrentRowInWorkspace, :122-162)
      double av[kCols];
#pragma unroll
      for (int k = 0; k < kCols; ++k) {
        const int z = lo + tz + k * kThreads;
        double v = 0.0;
        if (z < hi && mypos[z - lo] >= p) v = staged ? wat(lp, z) : asym(sp, z);
        av[k] = v;
      }
      {
        if (coef_pre) {
          if (tz < n_old) coef[tz] = cpre[0];
          if (tz + kThreads < n_old) coef[tz + kThreads] = cpre[1];
        } else {
          const double* ucol = P.uslot + static_cast<size_t>(sp) * ldu;
          for (int q = t; q < n_old; q += kBlock) coef[q] = ldcg(ucol + q);
        }
        if (t == 0) {
          coef[n_old] = extra0;
          coef[n_old + 1] = extra1;
        }
        if (t < kMaxPub) s_pub[t] = 0.0;
      }
      __syncthreads();
      // release the previous steps' U rows while the compute warps update the row
      if (t == kThreads) fence_acq_rel_gpu();
      Cand best = no_cand();
      auto finish_row = [&](int z, int j, double a_val, double acc) {
        const double wv = xsub(a_val, acc);
        wat(lp, z) = wv;
        if (j > p)
          argmax_join(best, Cand{fabs(wv), j, z, 0.0});  // FindCurrentRowMax, :164-182
        else
          s_pub[0] = wv;  // W[p, p]
        if (j == p + 1) s_pub[1] = wv;
        if (j == p + 2) s_pub[2] = wv;
      };
      if (paired) {
        // the compute warps split the rows q < lp (see the candidate phase)
        if (t < kThreads) {
          const int w = t >> 5, ln = t & 31;
          const int qa = (lp * w) / kWarps, qb = (lp * (w + 1)) / kWarps;
          double s1[3] = {0.0, 0.0, 0.0};
          auto rows = [&](int q0, int q1, auto&& wget) {
            for (int q = q0; q < q1; ++q) {
              const double c1 = coef[q];
#pragma unroll
              for (int k = 0; k < 3; ++k) {
                const int zz = ln + 32 * k;
                if (zz < width) s1[k] = __fma_rn(c1, wget(q, lo + zz), s1[k]);
              }
            }
          };
          const int qm = kSmemW ? qb : min(max(qa, srows), qb);
          rows(qa, qm, wat_s);
          if (!kSmemW) rows(qm, qb, wat_g);
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            const int zz = ln + 32 * k;
            if (zz < width) wpart[w * kPairSlots + zz] = s1[k];
          }
          compute_warps_sync();
        }
        if (t < width) {
          const int j = mypos[t];
          if (j >= p) {
            double acc = wpart[t];
#pragma unroll
            for (int w = 1; w < kWarps; ++w) acc += wpart[w * kPairSlots + t];
            finish_row(lo + t, j, av[0], acc);
          }
        }
      } else {
#pragma unroll
        for (int k = 0; k < kCols; ++k) {
          const int z = lo + tz + k * kThreads;
          if (z < hi) {
            const int j = mypos[z - lo];
            if (j >= p) {
              double acc;
              if (kSmemW) {
                acc = kOrdered ? ordered_dot(coef, lp, [&](int q) { return wat(q, z); })
                               : split_dot(coef, lp, [&](int q) { return wat(q, z); });
              } else {
                const int qs = min(lp, srows);
                auto ws = [&](int q) { return wat_s(q, z); };
                auto wg = [&](int q) { return wat_g(q, z); };
                acc = kOrdered ? ordered_dot_range(ordered_dot_range(0.0, coef, 0, qs, ws), coef, qs, lp, wg)
                               : split_dot_range(coef, 0, qs, ws) + split_dot_range(coef, qs, lp, wg);
              }
              finish_row(z, j, av[k], acc);
            }
          }
        }
      }
      lap(0);
      int owners[kMaxPub] = {};
      owners[0] = owner(sp);
      owners[1] = lp + 1 < nwin ? owner(win[lp + 1]) : 0;
      owners[2] = lp + 2 < nwin ? owner(win[lp + 2]) : 0;
      const XResult x1 = exchange<false>(P, ++seq, false, best, no_cand(), s_pub, owners, 3, X);
      if (!x1.ok) return;
      omega = x1.a.v;
      r = x1.a.i;
      rs = x1.a.s;  // slot of r
      dpp = X.pub[0];
      w_p1 = X.pub[1];  // W[p, p+1] (current-row version)
      w_p2 = X.pub[2];  // W[p, p+2]
    } else {
      ++nahead;
      omega = nx_omega;
      r = nx_r;
      rs = nx_rs;
      dpp = nx_dpp;
      w_p1 = nx_w1;
      w_p2 = nx_w2;
    }
    lap(1);
    // The next row's coefficient column (the visible rows q < nrel) is loaded
    // now for every slot the next row may have, so its latency hides behind
    // the rest of the step: A = slot of p+1, B = slot of p+2 (2x2 pivot),
    // C = slot of p (r = p+1).  After a row computed ahead, A (and the
    // candidate's operands) were loaded by the previous step.
    const bool prefetch = lp <= 2 * kThreads;
    auto preload = [&](int slot, int rows, double& c0, double& c1) {
      const double* ucol = P.uslot + static_cast<size_t>(slot) * ldu;
      c0 = tz < rows ? ldcg(ucol + tz) : 0.0;
      c1 = tz + kThreads < rows ? ldcg(ucol + tz + kThreads) : 0.0;
    };
    // the candidate column's operands for pivot row pp with candidate slot
    // rslot: A(z, r) of this CTA's active slots into wcs, each copied by the
    // thread that later finishes that slot; U[q, r] (q < rows) into cr
    auto issue_cand = [&](int pp, int rslot, int rows) {
#pragma unroll
      for (int k = 0; k < kCols; ++k) {
        const int z = lo + tz + k * kThreads;
        if (z < hi && mypos[z - lo] >= pp) cp_async_8(&wcs[z - lo], aptr(z, rslot));
      }
      if (prefetch) preload(rslot, rows, cr0, cr1);
    };
    const int slot_a = lp + 1 < nwin ? win[lp + 1] : -1;
    int slot_b = -1, slot_c = -1;
    double cb0 = 0.0, cb1 = 0.0, cc0 = 0.0, cc1 = 0.0;
    if (!was_ahead && prefetch && slot_a >= 0) preload(slot_a, nrel, ca0, ca1);

    int kind = 1;  // 1: 1x1 at p; -1: 1x1 after p<->r; 2: 2x2 with p+1<->r
    bool cand = false, spec = false;
    double log_sigma = __longlong_as_double(0x7ff8000000000000ll);  // NaN: no candidate
    double log_arr = log_sigma;
    double wc_r = 0.0, wc_p = 0.0, wc_p1 = 0.0, wc_p2 = 0.0;
    double nx_ar = 0.0, nx_part = 0.0, nx_d = 0.0, nx_1 = 0.0, nx_2 = 0.0;
    double e0 = 0.0;  // U[p, p+1] when p stays a 1x1 pivot (row computed ahead)
    Cand nx_best = no_cand();
    // FactorPanel's test, :90-92
    if (!(fabs(dpp) >= xmul(kAlpha, omega) || omega == 0.0)) {
      cand = true;
      ++ncand;
      if (!was_ahead) issue_cand(p, rs, nrel);
      slot_b = lp + 2 < nwin ? win[lp + 2] : -1;
      slot_c = r == p + 1 ? sp : -1;
      if (prefetch && slot_b >= 0) preload(slot_b, nrel, cb0, cb1);
      if (prefetch && slot_c >= 0) preload(slot_c, nrel, cc0, cc1);
      spec = r != p + 1 && p + 1 < P.nominal_end && slot_a >= 0;
      // coefficients: coef = U[q, r] (the candidate column), coef2 = U[q, p+1]
      // (row p+1, when computed ahead; U[lp, p+1] is applied last); the
      // visible rows from the slots' columns, then row lp - 1 passed along
      if (prefetch) {
        if (tz < nrel) {
          coef[tz] = cr0;
          coef2[tz] = ca0;
        }
        if (tz + kThreads < nrel) {
          coef[tz + kThreads] = cr1;
          coef2[tz + kThreads] = ca1;
        }
      } else {
        const double* ucol = P.uslot + static_cast<size_t>(rs) * ldu;
        for (int q = t; q < nrel; q += kBlock) coef[q] = ldcg(ucol + q);
        if (spec) {
          const double* ucol2 = P.uslot + static_cast<size_t>(slot_a) * ldu;
          for (int q = t; q < nrel; q += kBlock) coef2[q] = ldcg(ucol2 + q);
        }
      }
      if (was_ahead && t == 0) {
        coef[lp - 1] = u_prev_r;
        coef2[lp - 1] = carry;
      }
      if (t < kMaxPub) s_pub[t] = 0.0;
      __syncthreads();
      // release U row lp - 1 (written by the previous step, after its last exchange)
      if (was_ahead && t == kThreads) fence_acq_rel_gpu();
      // ---- candidate column W(i, r) = A(i, r) - sum_q U[q, r] W[q, i]
      // (CopyCandidateToWorkspace + UpdateCandidateInWorkspace, :184-352), and
      // row p+1 as keeping pivot p leaves it: W[p+1, j] = A(p+1, j) -
      // (sum_{q < lp} U[q, p+1] W[q, j] + U[lp, p+1] W[lp, j]).  At j = r,
      // W[lp, r] becomes the candidate's W(p, r), so the owner publishes
      // A(p+1, r) and the partial sum instead.
      const bool staged1 = spec && (slot_a - kstart) == lp + 1;
      if (spec) e0 = div_or_zero(w_p1, safe_denominator(dpp));
      Cand best = no_cand();
      double sig = 0.0;
      // slot z holding index i >= p, with its candidate sum acc and (two) the
      // partial sum of row p+1
      auto finish = [&](int z, int i, double acc, double part, bool two) {
        cp_async_wait_all();  // this thread's copy of A(z, r)
        const double v = xsub(wcs[z - lo], acc);
        wcs[z - lo] = v;
        if (i != r) {
          const double av2 = fabs(v);
          sig = (sig < av2) ? av2 : sig;  // std::max, FindCandidateColumnMax :354-367
        } else {
          s_pub[0] = v;
        }
        if (i == p) s_pub[1] = v;
        if (i == p + 1) s_pub[2] = v;
        if (i == p + 2) s_pub[3] = v;
        if (two) {
          const double a1 = staged1 ? wat(lp + 1, z) : asym(slot_a, z);
          if (i != r) {
            const double wp = wat(lp, z);
            const double v1 = xsub(a1, xadd(part, xmul(e0, wp)));
            svs[z - lo] = v1;
            if (i > p + 1)
              argmax_join(best, Cand{fabs(v1), i, z, wp});
            else
              s_pub[4] = v1;  // W[p+1, p+1]
            if (i == p + 2) s_pub[5] = v1;
            if (i == p + 3) s_pub[6] = v1;
          } else {
            s_pub[7] = a1;
            s_pub[8] = part;
          }
        }
      };
      if (paired) {
        // each compute warp sums a range of rows for every slot (lanes l,
        // l + 32, l + 64), so each coefficient is read by one warp only; the
        // per-warp partial sums are then added in warp order
        if (t < kThreads) {
          const int w = t >> 5, ln = t & 31;
          const int qa = (lp * w) / kWarps, qb = (lp * (w + 1)) / kWarps;
          double sa[3] = {0.0, 0.0, 0.0}, sb[3] = {0.0, 0.0, 0.0};
          auto rows = [&](int q0, int q1, auto&& wget) {
            for (int q = q0; q < q1; ++q) {
              const double c1 = coef[q], c2 = coef2[q];
#pragma unroll
              for (int k = 0; k < 3; ++k) {
                const int zz = ln + 32 * k;
                if (zz < width) {
                  const double x = wget(q, lo + zz);
                  sa[k] = __fma_rn(c1, x, sa[k]);
                  sb[k] = __fma_rn(c2, x, sb[k]);
                }
              }
            }
          };
          const int qm = kSmemW ? qb : min(max(qa, srows), qb);
          rows(qa, qm, wat_s);
          if (!kSmemW) rows(qm, qb, wat_g);
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            const int zz = ln + 32 * k;
            if (zz < width) {
              wpart[(2 * w) * kPairSlots + zz] = sa[k];
              wpart[(2 * w + 1) * kPairSlots + zz] = sb[k];
            }
          }
          compute_warps_sync();
        }
        if (t < width) {
          const int i = mypos[t];
          if (i >= p) {
            double acc = wpart[t], part = wpart[kPairSlots + t];
#pragma unroll
            for (int w = 1; w < kWarps; ++w) {
              acc += wpart[(2 * w) * kPairSlots + t];
              part += wpart[(2 * w + 1) * kPairSlots + t];
            }
            finish(lo + t, i, acc, part, spec && i > p);
          }
        }
      } else {
#pragma unroll
        for (int k = 0; k < kCols; ++k) {
          const int z = lo + tz + k * kThreads;
          if (z < hi) {
            const int i = mypos[z - lo];
            if (i >= p) {
              const bool two = spec && i > p;
              double acc, part = 0.0;
              auto wq = [&](int q) { return wat(q, z); };
              if (kSmemW) {
                if (two) {
                  if (kOrdered)
                    ordered_dot2(coef, coef2, lp, wq, acc, part);
                  else
                    split_dot2(coef, coef2, lp, wq, acc, part);
                } else {
                  acc = kOrdered ? ordered_dot(coef, lp, wq) : split_dot(coef, lp, wq);
                }
              } else {
                // shared-memory rows first, then the global ones (the
                // ordered mode continues the same sums: same order)
                const int qs = min(lp, srows);
                auto ws = [&](int q) { return wat_s(q, z); };
                auto wg = [&](int q) { return wat_g(q, z); };
                if (two) {
                  if (kOrdered) {
                    acc = 0.0;
                    ordered_dot2_range(coef, coef2, 0, qs, ws, acc, part);
                    ordered_dot2_range(coef, coef2, qs, lp, wg, acc, part);
                  } else {
                    double a2, p2;
                    split_dot2_range(coef, coef2, 0, qs, ws, acc, part);
                    split_dot2_range(coef, coef2, qs, lp, wg, a2, p2);
                    acc += a2;
                    part += p2;
                  }
                } else {
                  acc = kOrdered ? ordered_dot_range(ordered_dot_range(0.0, coef, 0, qs, ws), coef, qs, lp, wg)
                                 : split_dot_range(coef, 0, qs, ws) + split_dot_range(coef, qs, lp, wg);
                }
              }
              finish(z, i, acc, part, two);
            }
          }
        }
      }
      nx_best = best;
      lap(2);
      int owners[kMaxPub] = {};
      owners[0] = owner(rs);
      owners[1] = owner(sp);
      owners[2] = lp + 1 < nwin ? owner(win[lp + 1]) : 0;
      owners[3] = lp + 2 < nwin ? owner(win[lp + 2]) : 0;
      if (spec) {
        owners[4] = owner(slot_a);
        owners[5] = owners[3];
        owners[6] = lp + 3 < nwin ? owner(win[lp + 3]) : 0;
        owners[7] = owners[0];
        owners[8] = owners[0];
      }
      const XResult x2 = exchange<true>(P, ++seq, false, Cand{sig, 0, 0, 0.0}, nx_best, s_pub, owners,
                                        spec ? 9 : 4, X);
      if (!x2.ok) return;
      const double sigma = x2.a.v;
      wc_r = X.pub[0];
      wc_p = X.pub[1];
      wc_p1 = X.pub[2];
      wc_p2 = X.pub[3];
      if (spec) {
        nx_best = x2.b;
        nx_d = X.pub[4];
        nx_1 = X.pub[5];
        nx_2 = X.pub[6];
        nx_ar = X.pub[7];
        nx_part = X.pub[8];
      }
      lap(3);
      log_sigma = sigma;
      log_arr = fabs(wc_r);
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
    if (P.pivlog != nullptr && c == 0 && t == 0) {
      // the quantities this step's decision compared (FactorPanel :90-92,
      // SelectPivot :369-390), at the position where its pivot starts
      double* lg = P.pivlog + static_cast<size_t>(p) * kPivLogWords;
      lg[0] = fabs(dpp);
      lg[1] = omega;
      lg[2] = log_sigma;
      lg[3] = log_arr;
    }

    if (kind == 1) {
      // ScaleOneByOnePivot (:633-656); after a candidate evaluation the
      // reference's W(p, r) holds the column version of that entry.
      const double d = dpp;
      const double den = safe_denominator(d);
      double wr = 0.0;  // W[p+1, r] of the row computed ahead
      if (spec) {
        wr = xsub(nx_ar, xadd(nx_part, xmul(e0, wc_p)));
        // the next step starts from row p+1 and its argmax
        Cand best = nx_best;
        argmax_join(best, Cand{fabs(wr), r, rs, wc_p});
        nx_omega = best.v;
        nx_r = best.i;
        nx_rs = best.s;
        nx_dpp = nx_d;
        nx_w1 = r == p + 2 ? wr : nx_1;
        nx_w2 = r == p + 3 ? wr : nx_2;
        u_prev_r = div_or_zero(best.pay, den);
        carry = div_or_zero(r == p + 2 ? wc_p : w_p2, den);
        ahead = true;
        // the next step's operands load while this step scales: its next
        // row's coefficient column (slot of p+2) and, when it evaluates a
        // candidate, that candidate's A and U columns (visible rows q < lp)
        const int slot_a2 = lp + 2 < nwin ? win[lp + 2] : -1;
        if (prefetch && slot_a2 >= 0) preload(slot_a2, lp, ca0, ca1);
        if (!(fabs(nx_dpp) >= xmul(kAlpha, nx_omega) || nx_omega == 0.0)) issue_cand(p + 1, nx_rs, lp);
      }
#pragma unroll
      for (int k = 0; k < kCols; ++k) {
        const int z = lo + tz + k * kThreads;
        if (z < hi) {
          const int j = mypos[z - lo];
          if (j > p) {
            double wv;
            if (cand && j == r) {
              wv = wc_p;
              wat(lp, z) = wv;
            } else {
              wv = wat(lp, z);
            }
            P.uslot[static_cast<size_t>(z) * ldu + lp] = div_or_zero(wv, den);
            if (spec) wat(lp + 1, z) = j == r ? wr : svs[z - lo];
          }
        }
      }
      if (c == 0 && t == 0) {
        P.dlog[2 * lp] = d;
        P.ptype[p] = 1;
      }
      if (was_ahead && !cand) {
        // next row's coefficients: U[q, p+1] for q < lp - 1, then U[lp - 1, p+1]
        // (passed along) and U[p, p+1]
        n_old = lp - 1;
        extra0 = carry;
        extra1 = div_or_zero(w_p1, den);
      } else {
        // next row's coefficients: U[q, p+1] for q < p, then U[p, p+1]
        n_old = lp;
        extra0 = div_or_zero((cand && r == p + 1) ? wc_p : w_p1, den);
      }
      p += 1;
    } else if (kind == -1) {
      // SwapOneByOnePivot (:392-401, :414-498) + ScaleOneByOnePivot: p and r
      // exchange slots; the new row p is the candidate column.
      const double d = wc_r;
      const double den = safe_denominator(d);
      if (t == 0) {
        win[lp] = rs;
        if (r - kstart < nwin) win[r - kstart] = sp;
        if (sp >= lo && sp < hi) mypos[sp - lo] = r;
        if (rs >= lo && rs < hi) mypos[rs - lo] = p;
      }
      __syncthreads();
#pragma unroll
      for (int k = 0; k < kCols; ++k) {
        const int z = lo + tz + k * kThreads;
        if (z < hi && mypos[z - lo] > p) {
          const double wv = wcs[z - lo];
          wat(lp, z) = wv;
          P.uslot[static_cast<size_t>(z) * ldu + lp] = div_or_zero(wv, den);
        }
      }
      if (c == 0 && t == 0) {
        P.dlog[2 * lp] = d;
        P.ptype[p] = 1;
      }
      n_old = lp;
      extra0 = div_or_zero((r == p + 1) ? wc_p : wc_p1, den);
      p += 1;
    } else {
      // SwapTwoByTwoPivot (:403-412, :500-587) + ScaleTwoByTwoPivot (:658-704):
      // p+1 and r exchange slots; row p+1 is the candidate column.
      const int ls = lp + 1;
      const int ss = win[ls];
      const double d11 = dpp, d21 = wc_p, d22 = wc_r;
      const double det = xsub(xmul(d11, d22), xmul(d21, d21));
      const double i11 = xdiv(d22, det);
      const double i22 = xdiv(d11, det);
      const double i21 = xdiv(-d21, det);
      __syncthreads();  // every thread has read win[ls]
      if (r != p + 1 && t == 0) {
        win[ls] = rs;
        if (r - kstart < nwin) win[r - kstart] = ss;
        if (ss >= lo && ss < hi) mypos[ss - lo] = r;
        if (rs >= lo && rs < hi) mypos[rs - lo] = p + 1;
      }
      __syncthreads();
#pragma unroll
      for (int k = 0; k < kCols; ++k) {
        const int z = lo + tz + k * kThreads;
        if (z < hi && mypos[z - lo] > p + 1) {
          const double x = wat(lp, z);
          const double y = wcs[z - lo];
          wat(ls, z) = y;
          P.uslot[static_cast<size_t>(z) * ldu + lp] = xadd(xmul(i11, x), xmul(i21, y));
          P.uslot[static_cast<size_t>(z) * ldu + ls] = xadd(xmul(i21, x), xmul(i22, y));
        }
      }
      if (c == 0 && t == 0) {
        P.dlog[2 * lp] = d11;
        P.dlog[2 * lp + 1] = d21;
        P.dlog[2 * ls] = d22;
        P.ptype[p] = 2;
        P.ptype[p + 1] = -2;
      }
      // next row p+2: coefficients U[q, p+2], q < p, then U[p, p+2], U[p+1, p+2]
      const double x = (r == p + 2) ? w_p1 : w_p2;
      const double y = (r == p + 2) ? wc_p1 : wc_p2;
      n_old = lp;
      extra0 = xadd(xmul(i11, x), xmul(i21, y));
      extra1 = xadd(xmul(i21, x), xmul(i22, y));
      p += 2;
    }
    coef_pre = prefetch && p < P.nominal_end && !ahead;
    if (coef_pre) {
      const int next = win[p - kstart];
      if (next == slot_a) {
        cpre[0] = ca0;
        cpre[1] = ca1;
      } else if (next == slot_b) {
        cpre[0] = cb0;
        cpre[1] = cb1;
      } else if (next == slot_c) {
        cpre[0] = cc0;
        cpre[1] = cc1;
      } else {
        preload(next, nrel, cpre[0], cpre[1]);
      }
      // U row nrel, released by this step's candidate exchange
      if (n_old > nrel) {
        const double* ucol = P.uslot + static_cast<size_t>(next) * ldu;
        if (tz == nrel) cpre[0] = ldcg(ucol + nrel);
        if (tz + kThreads == nrel) cpre[1] = ldcg(ucol + nrel);
      }
    }
    __syncthreads();
    lap(4);
  }

  cp_async_wait_all();
  if (P.stats && t == 0)
    for (int k = 0; k < 5; ++k) atomicAdd(P.stats + 16 + 2048 + c * 5 + k, tm[k]);
  const int e = p;
  const int kb = e - kstart;
  // ---- the panel's W and U in final column order, the slot of every index,
  // and the list of indices whose slot changed
  __syncthreads();
  for (int idx = t; idx < width * kb; idx += kBlock) {
    const int zz = idx / kb, q = idx - zz * kb;
    P.ucm[static_cast<size_t>(mypos[zz]) * ldu + q] = P.uslot[static_cast<size_t>(lo + zz) * ldu + q];
  }
  for (int idx = t; idx < width * kb; idx += kBlock) {
    const int q = idx / width, zz = idx - q * width;
    const int x = mypos[zz];
    if (x >= e) P.w[q * ldw + x] = wat(q, lo + zz);
  }
  for (int zz = t; zz < width; zz += kBlock) {
    const int x = mypos[zz], z = lo + zz;
    P.srcmap[x] = z;
    if (x != z) {
      const int slot_i = atomicAdd(&P.st->moved[P.panel & 1], 1);
      P.moved[(P.panel & 1) * P.move_cap + slot_i] = x;
    }
  }
  if (c == 0 && t == 0) {
    // panel range [kstart, e); the next panel starts at e.
    P.st->kstart[(P.panel + 1) & 1] = e;
    P.st->xseq[(P.panel + 1) & 1] = static_cast<int>(seq + 1);  // + the barrier below
    if (P.panel_end) P.panel_end[P.panel] = e;
    P.bounds[2 * P.panel] = kstart;
    P.bounds[2 * P.panel + 1] = e;
    if (P.stats) {
      for (int k = 0; k < 5; ++k) atomicAdd(P.stats + k, tm[k]);
      atomicAdd(P.stats + 5, static_cast<unsigned long long>(kb));
      atomicAdd(P.stats + 6, static_cast<unsigned long long>(ncand));
      atomicAdd(P.stats + 9, static_cast<unsigned long long>(nahead));
    }
  }
  // grid barrier: every CTA's maps and lists are visible after it
  {
    const int owners0[kMaxPub] = {};
    const XResult xb = exchange<false>(P, ++seq, true, no_cand(), no_cand(), s_pub, owners0, 0, X);
    if (!xb.ok) return;
  }
  // ---- gather the interchanged data (written back by finalize_kernel)
  const int cnt = ldcg(&P.st->moved[P.panel & 1]);
  if (c == 0 && t == 0) P.move_counts[P.panel] = cnt;
  if (cnt == 0) return;
  const int* list = P.moved + (P.panel & 1) * P.move_cap;
  const long long m = n - kstart;
  const long long nthreads = static_cast<long long>(G) * kBlock;
  const long long gtid = static_cast<long long>(c) * kBlock + t;
  // rows of the moved indices over the active columns: gbuf[ix][y - k0] = A(src x, src y)
  for (long long idx = gtid; idx < cnt * m; idx += nthreads) {
    const int ix = static_cast<int>(idx / m);
    const int y = kstart + static_cast<int>(idx - ix * m);
    const int sx = ldcg(P.srcmap + ldcg(list + ix));
    const int sy = ldcg(P.srcmap + y);
    P.gbuf[ix * ldw + (y - kstart)] = asym(sx, sy);
  }
  // the moves (position dst receives what position src held): the factored
  // rows q < k0 take the same column exchanges (:472-491), applied once
  // after the last panel (launch_left_swaps)
  int* rec = P.moves + static_cast<size_t>(P.panel) * 2 * P.move_cap;
  for (long long ix = gtid; ix < cnt; ix += nthreads) {
    const int x = ldcg(list + ix);
    rec[ix] = x;
    rec[P.move_cap + ix] = ldcg(P.srcmap + x);
  }
  for (long long ix = gtid; ix < cnt; ix += nthreads)
    P.permbuf[ix] = ldcg(P.perm + ldcg(P.srcmap + ldcg(list + ix)));
}

// Writes back what the panel's interchanges moved, the permutation, and the
// panel's compact factor rows [k0, e):
//   A[x, y]  (moved x >= e, y >= e)        from the gathered rows
//   perm[x]  (moved x)                     = perm[slot of x] before the panel
//   A[q, j]  (k0 <= q < e, j >= q)         D entries (dlog) or U[q, j] (ucm)
struct FinArgs {
  double* a;
  long long lda;
  const double* ucm;
  int ldu;
  const double* dlog;
  const int* ptype;
  const int* moved;
  int move_cap;
  const double* gbuf;
  long long ldg;
  const int* permbuf;
  int* perm;
  int n;
  DeviceState* st;
  int panel;
};

constexpr int kFinTile = 32;
constexpr int kFinUnroll = 4;  // loads in flight per thread in the write-back loops
constexpr int kFinCtasPerSm = 6;  // resident at 40 registers per thread
__global__ void __launch_bounds__(256) finalize_kernel(FinArgs F) {
  __shared__ double tile[kFinTile][kFinTile + 1];
  if (ld_relaxed_s32(&F.st->abort)) return;
  const int k0 = ldcg(&F.st->kstart[F.panel & 1]);
  const int e = ldcg(&F.st->kstart[(F.panel + 1) & 1]);
  const int kb = e - k0;
  const int n = F.n;
  const long long lda = F.lda;
  const long long nthreads = static_cast<long long>(gridDim.x) * blockDim.x;
  const long long gtid = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  // the next panel counts its moved indices from zero
  if (gtid == 0) F.st->moved[(F.panel + 1) & 1] = 0;
  const int cnt = ldcg(&F.st->moved[F.panel & 1]);
  const int* list = F.moved + (F.panel & 1) * F.move_cap;
  if (cnt > 0) {
    // each thread keeps kFinUnroll loads in flight before its stores
    const long long m = n - e, total1 = cnt * m;
    for (long long base = gtid; base < total1; base += nthreads * kFinUnroll) {
      double v[kFinUnroll];
      long long dst[kFinUnroll];
#pragma unroll
      for (int u = 0; u < kFinUnroll; ++u) {
        const long long idx = base + u * nthreads;
        dst[u] = -1;
        v[u] = 0.0;
        if (idx < total1) {
          const int ix = static_cast<int>(idx / m), y = e + static_cast<int>(idx - ix * m);
          const int x = list[ix];
          if (x >= e) {
            v[u] = F.gbuf[ix * F.ldg + (y - k0)];
            dst[u] = x <= y ? static_cast<long long>(x) * lda + y : static_cast<long long>(y) * lda + x;
          }
        }
      }
#pragma unroll
      for (int u = 0; u < kFinUnroll; ++u)
        if (dst[u] >= 0) F.a[dst[u]] = v[u];
    }
    for (long long ix = gtid; ix < cnt; ix += nthreads) F.perm[list[ix]] = F.permbuf[ix];
  }
  if (kb <= 0) return;
  // compact rows: tiles over (q in [0, kb), j in [k0, n))
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
      if (j < n && q < kb && j >= k0 + q) {
        const int lj = j - k0;
        if (j < e && q == lj)
          v = F.dlog[2 * lj];  // D(l, l)
        else if (j < e && q == lj - 1 && F.ptype[j] == -2)
          v = F.dlog[2 * q + 1];  // D(l, l+1) of a 2x2
        else
          v = F.ucm[static_cast<size_t>(j) * F.ldu + q];
      }
      tile[jj][tx] = v;
    }
    __syncthreads();
    for (int qq = ty; qq < kFinTile; qq += 8) {
      const int q = q0 + qq, j = j0 + tx;
      if (q < kb && j < n && j >= k0 + q) F.a[static_cast<size_t>(k0 + q) * lda + j] = tile[tx][qq];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// The factored rows' column exchanges, applied once after the last panel.
// Each panel's interchanges move indices at positions >= its start, and the
// reference exchanges the same columns of every row factored before, as it
// goes (:472-491).  Those rows are not read again while the factorization
// runs, so each panel only records its moves (position dst receives what
// position src held); from the last panel back, inv maps a position at the
// end of panel k to its final position, and panel k's rows are scattered in
// final column order into the gbuf scratch and copied back.  Every entry
// moves once, by copies coalesced on one side, instead of a scattered read
// and write per moved column and earlier row at every panel.  pend[parity]
// counts the moves after panel k: while it is zero the rows stay as they are.
struct SwapArgs {
  const int* moves;
  const int* counts;
  const int* bounds;
  int move_cap;
  int n;
  int* inv;
  int* tmp;   // move_cap values, then pend[2]
  double* a;
  long long lda;
  double* scratch;
  long long lds;
  const DeviceState* st;
};

__device__ __forceinline__ void panel_range(const int* bounds, int panel, int n, int& k0, int& e) {
  k0 = min(max(bounds[2 * panel], 0), n);
  e = min(max(bounds[2 * panel + 1], k0), n);
}

// inv_{k-1} = inv_k composed with panel k's moves (inv[src] = inv[dst]); the
// moves permute the moved positions among themselves.  One CTA.
__device__ void moves_into_inv(const SwapArgs& S, int panel) {
  const int cnt = min(max(S.counts[panel], 0), S.move_cap);
  const int* dst = S.moves + static_cast<size_t>(panel) * 2 * S.move_cap;
  const int* src = dst + S.move_cap;
  int* pend = S.tmp + S.move_cap;
  for (int ix = threadIdx.x; ix < cnt; ix += blockDim.x) {
    const int d = dst[ix];
    S.tmp[ix] = d >= 0 && d < S.n ? S.inv[d] : 0;
  }
  __syncthreads();
  for (int ix = threadIdx.x; ix < cnt; ix += blockDim.x) {
    const int sidx = src[ix];
    if (sidx >= 0 && sidx < S.n) S.inv[sidx] = S.tmp[ix];
  }
  if (threadIdx.x == 0) pend[(panel - 1) & 1] = pend[panel & 1] + cnt;
}

// inv = identity, pend = 0, then the last panel's moves
__global__ void swaps_start_kernel(SwapArgs S, int last) {
  if (ld_relaxed_s32(&S.st->abort)) return;
  for (int i = threadIdx.x; i < S.n; i += blockDim.x) S.inv[i] = i;
  if (threadIdx.x == 0) S.tmp[S.move_cap + (last & 1)] = 0;
  __syncthreads();
  moves_into_inv(S, last);
}

// scratch[r][inv[x] - e] = A[k0 + r, x] for panel k's rows
__global__ void rows_scatter_kernel(SwapArgs S, int panel) {
  if (ld_relaxed_s32(&S.st->abort) || S.tmp[S.move_cap + (panel & 1)] == 0) return;
  int k0, e;
  panel_range(S.bounds, panel, S.n, k0, e);
  const long long cols = S.n - e, total = static_cast<long long>(e - k0) * cols;
  for (long long idx = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; idx < total;
       idx += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int r = static_cast<int>(idx / cols), x = e + static_cast<int>(idx - r * cols);
    const int f = S.inv[x];
    if (f >= e && f < S.n) S.scratch[r * S.lds + (f - e)] = S.a[static_cast<long long>(k0 + r) * S.lda + x];
  }
}

// A[k0 + r, j] = scratch[r][j - e]; block 0 then folds panel k's moves into
// inv for panel k - 1 (nothing here reads inv)
__global__ void rows_back_kernel(SwapArgs S, int panel) {
  if (ld_relaxed_s32(&S.st->abort)) return;
  if (S.tmp[S.move_cap + (panel & 1)] != 0) {
    int k0, e;
    panel_range(S.bounds, panel, S.n, k0, e);
    const long long cols = S.n - e, total = static_cast<long long>(e - k0) * cols;
    for (long long idx = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; idx < total;
         idx += static_cast<long long>(gridDim.x) * blockDim.x) {
      const int r = static_cast<int>(idx / cols), j = e + static_cast<int>(idx - r * cols);
      S.a[static_cast<long long>(k0 + r) * S.lda + j] = S.scratch[r * S.lds + (j - e)];
    }
  }
  if (blockIdx.x == 0 && panel > 0) moves_into_inv(S, panel);
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
    st->moved[0] = 0;
    st->moved[1] = 0;
    st->xseq[0] = 0;
    st->xseq[1] = 0;
    st->xcount = 0ull;
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
__global__ void __launch_bounds__(kBlock) probe_kernel(PanelArgs P) {
  __shared__ XShared X;
  __shared__ double s_pub[kMaxPub];
  if (threadIdx.x < kMaxPub) s_pub[threadIdx.x] = 0.0;
  const int owners[kMaxPub] = {};
  __syncthreads();
  const unsigned long long t0 = globaltimer_ns();
  for (int it = 0; it < P.n; ++it) {
    const Cand mine{static_cast<double>(blockIdx.x), static_cast<int>(blockIdx.x), static_cast<int>(blockIdx.x), 0.0};
    const XResult x = exchange<false>(P, static_cast<unsigned>(it) + 1u, true, mine, no_cand(), s_pub,
                                      owners, 3, X);
    if (!x.ok) return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && P.stats) P.stats[0] = globaltimer_ns() - t0;
}

}  // namespace

static int cooperative_launch(const void* fn, int grid, PanelArgs* args, cudaStream_t s) {
  void* kargs[] = {args};
  cudaError_t err = cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kBlock), kargs, 0, s);
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
  P.win_rows = plan.b + 2;
  P.win_pad = static_cast<int>(align_up(static_cast<size_t>(plan.b) + 2, 2));
  P.a = plan.a;
  P.lda = plan.lda;
  P.w = plan.w;
  P.ldw = plan.ldw;
  P.wslot = plan.wslot;
  P.uslot = plan.uslot;
  P.ucm = plan.ucm;
  P.ldu = plan.ldu;
  P.dlog = plan.dlog;
  P.srcmap = plan.srcmap;
  P.moved = plan.moved;
  P.move_cap = plan.move_cap;
  P.gbuf = plan.gbuf;
  P.moves = plan.moves;
  P.move_counts = plan.move_counts;
  P.bounds = plan.bounds;
  P.permbuf = plan.permbuf;
  P.perm = plan.perm;
  P.ptype = plan.pivot_types;
  P.panel_end = plan.panel_end;
  P.slots = plan.slots;
  P.st = plan.state;
  P.nslots = plan.grid;
  P.slot_stride = plan.grid;
  P.timeout_ns = plan.timeout_ns;
  P.stats = plan.stats;
  P.pivlog = plan.pivlog;
  static const unsigned poll_ns = [] {
    const char* e = getenv("BBK_POLL_NS");
    return e ? static_cast<unsigned>(atoi(e)) : 0u;
  }();
  P.poll_ns = poll_ns;
  if (plan.grid > kMaxGrid)
    return set_error(BBK_ERR_INVALID_ARGUMENT, "panel grid %d exceeds %d", plan.grid, kMaxGrid);
  // shared memory: two coefficient columns + candidate column + row computed
  // ahead + per-warp partial sums + the slots' panel rows (all, or as many
  // as fit), then the window map and the slot -> index map
  const int smax = (plan.n + plan.grid - 1) / plan.grid;
  P.coef_cap = static_cast<int>(align_up(static_cast<size_t>(plan.b) + 4, 2));
  P.smem_cols = smax;
  const size_t base = (2 * static_cast<size_t>(P.coef_cap) + 2 * static_cast<size_t>(smax) +
                       2 * static_cast<size_t>(kWarps) * kPairSlots) * sizeof(double) +
                      (static_cast<size_t>(P.win_pad) + smax) * sizeof(int);
  const size_t wbytes = static_cast<size_t>(P.win_rows) * smax * sizeof(double);
  const size_t limit = 220 * 1024;
  P.w_smem = base + wbytes <= limit;
  // a slice too wide for shared memory keeps its first rows there (the rows
  // every pivot step of the panel reads) and the rest in global memory; the
  // kernel divides the room by its own slot width, which shrinks as the
  // factorization proceeds
  size_t wroom = P.w_smem ? wbytes : (base < limit ? (limit - base) & ~static_cast<size_t>(7) : 0);
  if (const char* e = getenv("BBK_PANEL_SMEM_ROWS")) {
    // testing and tuning: at most this many rows of the widest slice in
    // shared memory (the split layout at any size)
    const size_t cap = static_cast<size_t>(std::max(0, atoi(e))) * smax * sizeof(double);
    if (cap < wroom) {
      P.w_smem = 0;
      wroom = cap;
    }
  }
  P.wcap = static_cast<int>(wroom / sizeof(double));
  const size_t bytes = base + wroom;
  const bool ordered = plan.mode == BBK_UPDATE_FP64_ORDERED;
  const void* fn = ordered ? (P.w_smem ? reinterpret_cast<const void*>(panel_kernel<true, true>)
                                       : reinterpret_cast<const void*>(panel_kernel<true, false>))
                           : (P.w_smem ? reinterpret_cast<const void*>(panel_kernel<false, true>)
                                       : reinterpret_cast<const void*>(panel_kernel<false, false>));
  BBK_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)));
  void* kargs[] = {&P};
  cudaError_t err = cudaLaunchCooperativeKernel(fn, dim3(plan.grid), dim3(kBlock), kargs, bytes, s);
  if (err != cudaSuccess) return cuda_error(err, "cudaLaunchCooperativeKernel(panel)");
  count_launch();
  return BBK_OK;
}

namespace {
// The panel's W rows at the trailing columns (x >= e, final column order,
// as the panel kernel left them for the update) into the caller's array.
__global__ void wrows_kernel(const DeviceState* st, int panel, int n, const double* w, long long ldw,
                             double* out, long long ldo) {
  if (ld_relaxed_s32(&st->abort)) return;
  const int k0 = ldcg(&st->kstart[panel & 1]);
  const int e = ldcg(&st->kstart[(panel + 1) & 1]);
  const long long width = n - e, total = static_cast<long long>(e - k0) * width;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int q = static_cast<int>(t / width), x = e + static_cast<int>(t % width);
    out[static_cast<long long>(k0 + q) * ldo + x] = w[q * ldw + x];
  }
}
}  // namespace

int launch_wrows(const FactorPlan& plan, int panel, cudaStream_t s) {
  const long long work = static_cast<long long>(plan.b + 1) * plan.n;
  const int grid = static_cast<int>(std::max(1LL, std::min(4096LL, (work + 255) / 256)));
  wrows_kernel<<<grid, 256, 0, s>>>(plan.state, panel, plan.n, plan.w, plan.ldw, plan.wrows, plan.ld_wrows);
  BBK_CUDA_TRY(cudaGetLastError());
  count_launch();
  return BBK_OK;
}

int launch_left_swaps(const FactorPlan& plan, cudaStream_t s) {
  if (plan.nb < 2) return BBK_OK;
  const int sms = device_sm_count();
  SwapArgs S{plan.moves, plan.move_counts, plan.bounds, plan.move_cap, plan.n, plan.posinv, plan.movetmp,
             plan.a, plan.lda, plan.gbuf, plan.ldw, plan.state};
  swaps_start_kernel<<<1, 1024, 0, s>>>(S, plan.nb - 1);
  BBK_CUDA_TRY(cudaGetLastError());
  count_launch();
  for (int k = plan.nb - 2; k >= 0; --k) {
    rows_scatter_kernel<<<4 * sms, 256, 0, s>>>(S, k);
    rows_back_kernel<<<4 * sms, 256, 0, s>>>(S, k);
    BBK_CUDA_TRY(cudaGetLastError());
    count_launch(2);
  }
  return BBK_OK;
}

int launch_finalize(const FactorPlan& plan, int panel, cudaStream_t s) {
  const int sms = device_sm_count();
  FinArgs F{};
  F.a = plan.a;
  F.lda = plan.lda;
  F.ucm = plan.ucm;
  F.ldu = plan.ldu;
  F.dlog = plan.dlog;
  F.ptype = plan.pivot_types;
  F.moved = plan.moved;
  F.move_cap = plan.move_cap;
  F.gbuf = plan.gbuf;
  F.ldg = plan.ldw;
  F.permbuf = plan.permbuf;
  F.perm = plan.perm;
  F.n = plan.n;
  F.st = plan.state;
  F.panel = panel;
  // large orders: a full SM of threads (n=40000: 38.4 -> 35.1 ms per
  // factorization); small ones keep 2 CTAs per SM (n=10000: 1.06 ms, 1.12
  // with the full grid)
  const int ctas = (plan.n >= 16384 ? kFinCtasPerSm : 2) * sms;
  finalize_kernel<<<ctas, 256, 0, s>>>(F);
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
  if (nslots > kMaxGrid + 1 || ctas > kMaxGrid)
    return set_error(BBK_ERR_INVALID_ARGUMENT, "probe: %d blocks exceed %d", ctas, kMaxGrid);
  PanelArgs P{};
  P.slots = slots;
  P.st = st;
  P.nslots = nslots;
  P.slot_stride = ctas + 1;
  P.timeout_ns = timeout_ns;
  P.n = iters;
  P.stats = stats;
  return cooperative_launch(reinterpret_cast<const void*>(probe_kernel), ctas, &P, s);
}

}  // namespace bbk
