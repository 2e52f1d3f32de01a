// Internal declarations shared by the CUDA translation units of libbbk_b200.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstddef>

#include "bbk_ldlt.h"

namespace bbk {

// ---------------------------------------------------------------------------
// Host-side helpers (capi.cu)
// ---------------------------------------------------------------------------
int set_error(int status, const char* fmt, ...);
int cuda_error(cudaError_t err, const char* what);
void count_launch(unsigned n = 1);
unsigned long long wait_timeout_ns();
int device_sm_count();
int check_device();  // BBK_OK on an sm_10x device, else BBK_ERR_NO_DEVICE

#define BBK_CUDA_TRY(expr)                                            \
  do {                                                                \
    cudaError_t bbk_err_ = (expr);                                    \
    if (bbk_err_ != cudaSuccess) return ::bbk::cuda_error(bbk_err_, #expr); \
  } while (0)

inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Bunch-Kaufman threshold (1 + sqrt(17)) / 8, the reference's literal
// (src/block_ldlt_decomposition.cc:14).
constexpr double kAlpha = 0.6403882032022076;
constexpr double kDblEpsilon = 2.220446049250313080847e-16;  // DBL_EPSILON

// ---------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------
// Exactly-rounded arithmetic that the compiler may not contract into FMAs:
// the panel reproduces the reference's operation order bit for bit.
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double xdiv(double a, double b) { return __ddiv_rn(a, b); }

// L2-coherent load (bypasses L1): data written by other CTAs of the same
// grid is read through these after an exchange.
__device__ __forceinline__ double ldcg(const double* p) { return __ldcg(p); }
__device__ __forceinline__ int ldcg(const int* p) { return __ldcg(p); }

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ int ld_relaxed_s32(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void red_release_add_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void red_relaxed_add_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("red.relaxed.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void fence_acq_rel_gpu() {
  asm volatile("fence.acq_rel.gpu;" ::: "memory");
}
__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// ---------------------------------------------------------------------------
// Pivot arithmetic shared by the panel and batched kernels
// (src/block_ldlt_decomposition.cc in wentianshu/BlockedBunchKaufmanLDLT)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double safe_denominator(double d) {
  // src/block_ldlt_decomposition.cc:21-26 (absolute threshold)
  return fabs(d) <= kDblEpsilon ? 0.0 : d;
}

__device__ __forceinline__ double div_or_zero(double x, double den) {
  return den == 0.0 ? 0.0 : xdiv(x, den);
}

// acc + sum_{q0 <= q < q1} c[q] * w(q) in ascending q, every product and sum
// rounded separately (the reference's order: its sums start at 0.0 and add
// one product at a time, so a sum over [0, q1) split at any q0 and continued
// from the first part's result is the same sum bit for bit).  The products
// do not depend on the running sum: each batch of eight is loaded and
// multiplied while the previous batch is being added.
template <typename WGet>
__device__ __forceinline__ double ordered_dot_range(double acc, const double* c, int q0, int q1, WGet&& w) {
  int q = q0;
  if (q1 - q0 >= 8) {
    double cur[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) cur[u] = xmul(c[q0 + u], w(q0 + u));
    for (q = q0 + 8; q + 8 <= q1; q += 8) {
      double nxt[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) nxt[u] = xmul(c[q + u], w(q + u));
#pragma unroll
      for (int u = 0; u < 8; ++u) acc = xadd(acc, cur[u]);
#pragma unroll
      for (int u = 0; u < 8; ++u) cur[u] = nxt[u];
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) acc = xadd(acc, cur[u]);
  }
  for (; q < q1; ++q) acc = xadd(acc, xmul(c[q], w(q)));
  return acc;
}

template <typename WGet>
__device__ __forceinline__ double ordered_dot(const double* c, int count, WGet&& w) {
  return ordered_dot_range(0.0, c, 0, count, w);
}

// Two sums over the same w(q) at once, continued from s1 / s2: s1 += sum
// c1[q] w(q), s2 += sum c2[q] w(q), q in [q0, q1), each added in ascending q
// with every product and sum rounded separately, so each is bitwise
// ordered_dot of its coefficients; w(q) is read once.
template <typename WGet>
__device__ __forceinline__ void ordered_dot2_range(const double* c1, const double* c2, int q0, int q1, WGet&& w,
                                                   double& s1, double& s2) {
  double a1 = s1, a2 = s2;
  int q = q0;
  for (; q + 4 <= q1; q += 4) {
    double p1[4], p2[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const double x = w(q + u);
      p1[u] = xmul(c1[q + u], x);
      p2[u] = xmul(c2[q + u], x);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      a1 = xadd(a1, p1[u]);
      a2 = xadd(a2, p2[u]);
    }
  }
  for (; q < q1; ++q) {
    const double x = w(q);
    a1 = xadd(a1, xmul(c1[q], x));
    a2 = xadd(a2, xmul(c2[q], x));
  }
  s1 = a1;
  s2 = a2;
}

template <typename WGet>
__device__ __forceinline__ void ordered_dot2(const double* c1, const double* c2, int count, WGet&& w,
                                             double& s1, double& s2) {
  s1 = 0.0;
  s2 = 0.0;
  ordered_dot2_range(c1, c2, 0, count, w, s1, s2);
}

// The reassociated counterpart of ordered_dot2: four FMA accumulators per
// sum over q in [q0, q1).
template <typename WGet>
__device__ __forceinline__ void split_dot2_range(const double* c1, const double* c2, int q0, int q1, WGet&& w,
                                                 double& s1, double& s2) {
  double a[4] = {0.0, 0.0, 0.0, 0.0}, b[4] = {0.0, 0.0, 0.0, 0.0};
  int q = q0;
  for (; q + 4 <= q1; q += 4) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const double x = w(q + u);
      a[u] = __fma_rn(c1[q + u], x, a[u]);
      b[u] = __fma_rn(c2[q + u], x, b[u]);
    }
  }
#pragma unroll
  for (int u = 0; u < 4; ++u)
    if (q + u < q1) {
      const double x = w(q + u);
      a[u] = __fma_rn(c1[q + u], x, a[u]);
      b[u] = __fma_rn(c2[q + u], x, b[u]);
    }
  s1 = (a[0] + a[1]) + (a[2] + a[3]);
  s2 = (b[0] + b[1]) + (b[2] + b[3]);
}

template <typename WGet>
__device__ __forceinline__ void split_dot2(const double* c1, const double* c2, int count, WGet&& w,
                                           double& s1, double& s2) {
  split_dot2_range(c1, c2, 0, count, w, s1, s2);
}

// sum_{q0 <= q < q1} c[q] * w(q) with eight independent FMA accumulators
// combined pairwise: the same sum, reassociated, with an eighth of the
// dependent-latency chain (update modes that do not reproduce the
// reference's rounding).
template <typename WGet>
__device__ __forceinline__ double split_dot_range(const double* c, int q0, int q1, WGet&& w) {
  double a[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  int q = q0;
  for (; q + 8 <= q1; q += 8) {
#pragma unroll
    for (int u = 0; u < 8; ++u) a[u] = __fma_rn(c[q + u], w(q + u), a[u]);
  }
#pragma unroll
  for (int u = 0; u < 8; ++u)
    if (q + u < q1) a[u] = __fma_rn(c[q + u], w(q + u), a[u]);
  return ((a[0] + a[1]) + (a[2] + a[3])) + ((a[4] + a[5]) + (a[6] + a[7]));
}

template <typename WGet>
__device__ __forceinline__ double split_dot(const double* c, int count, WGet&& w) {
  return split_dot_range(c, 0, count, w);
}

// Device status words shared by every kernel of one factorization.
struct DeviceState {
  int kstart[2];  // first row of panel P is kstart[P & 1]; panel P writes
                  // its end (= start of P + 1) into kstart[(P + 1) & 1]
  int abort;      // nonzero: a kernel gave up; every later kernel returns
  int status;     // bbk_status of the factorization
  int moved[2];   // panel P: count of indices its interchanges moved, in moved[P & 1]
  int xseq[2];    // exchanges completed before panel P, in xseq[P & 1]
  int pad[24];    // the arrival counter gets a cache line of its own
  unsigned long long xcount;  // arrivals at grid exchanges (one per CTA per exchange)
};

// ---------------------------------------------------------------------------
// Grid exchange: a grid-wide barrier fused with an all-gather of one small
// record per CTA.  Each CTA stores its record, then adds one to an arrival
// counter; one warp per CTA polls that single word with acquire loads until
// all CTAs of this exchange have arrived, and then the CTA reads the records
// (one pass).  Every record word also carries the exchange's 32-bit tag in
// its high half, which the reader checks.  Two record sets alternate (tag
// parity): no CTA can be two exchanges ahead of another.
// ---------------------------------------------------------------------------
constexpr int kSlotWords = 32;   // words per CTA record
constexpr int kPivLogWords = 4;  // decision log: |W(p,p)|, omega, sigma, |W(r,r)|
constexpr int kMaxPub = 10;      // published doubles per record

__device__ __forceinline__ unsigned long long tag_word(unsigned tag, unsigned v) {
  return (static_cast<unsigned long long>(tag) << 32) | v;
}

}  // namespace bbk

// Launch entry points implemented in the .cu files (host side).
namespace bbk {
struct FactorPlan;
int panel_grid_size(int n);
int panel_max_n();
int launch_init(int n, int* perm, int* pivot_types, DeviceState* st,
                unsigned long long* slots, size_t slot_words, cudaStream_t s);
int launch_panel(const FactorPlan& plan, int panel, cudaStream_t s);
int launch_finalize(const FactorPlan& plan, int panel, cudaStream_t s);
int launch_left_swaps(const FactorPlan& plan, cudaStream_t s);
int launch_wrows(const FactorPlan& plan, int panel, cudaStream_t s);
int launch_update(const FactorPlan& plan, int panel, cudaStream_t s);
int launch_status_copy(const DeviceState* st, int* status_out, cudaStream_t s);
int launch_probe_wait(int ctas, int nslots, int iters, unsigned long long timeout_ns,
                      DeviceState* st, unsigned long long* slots, unsigned long long* stats,
                      cudaStream_t s);
int launch_update_block(int rows, int cols, int inner, const double* left, int ls,
                        const double* ws, int wss, double* target, int ts, int mode,
                        cudaStream_t s);
int launch_scale_1x1(int count, double pivot, const double* src, int ss, double* dst,
                     int ds, cudaStream_t s);
int launch_scale_2x2(int count, double a, double b, double c, const double* s1, int s1s,
                     const double* s2, int s2s, double* d1, int d1s, double* d2, int d2s,
                     cudaStream_t s);
int solve_enqueue(int n, const double* f, long long ldf, const int* perm,
                  const int* pivot_types, int nrhs, double* b, long long ldb,
                  double* work, cudaStream_t s);
size_t solve_work_doubles(int n, int nrhs);
// The status word solve_enqueue keeps inside its scratch (BBK_OK, or
// BBK_ERR_TIMEOUT when a sweep's bounded wait ran out), and a synchronous
// read of it after the solve (waits for the stream).
int* solve_status_word(double* work, int n, int nrhs);
int solve_status(double* work, int n, int nrhs, cudaStream_t s);
// solve_enqueue under the library's per-kernel-class timing (capi.cu).
int enqueue_solve(int n, const double* f, long long ldf, const int* perm, const int* pt,
                  int nrhs, double* b, long long ldb, double* work, cudaStream_t s);
size_t refine_work_doubles(int n, int nrhs, int restart);
int refine_enqueue(int n, const double* a, long long lda, const double* f, long long ldf,
                   const int* perm, const int* pt, int nrhs, const double* b, double* x, double tol,
                   int max_iter, int method, int restart, double* work, bbk_refine_info* info,
                   cudaStream_t s);
size_t reconstruct_work_doubles(int n);
int reconstruct_enqueue(int n, const double* f, long long ldf, const int* perm,
                        const int* pivot_types, double* out, long long ldo,
                        double* work, cudaStream_t s);
int extract_ld_enqueue(int n, const double* f, long long ldf, const int* pivot_types, double* l,
                       long long ldl, double* d, long long ldd, cudaStream_t s);
int launch_upper_product(int n, const double* m, const double* u, long long ld, double* c,
                         cudaStream_t s);

// Everything a factorization's kernels need: the caller's matrix and the
// carved-up workspace.
struct FactorPlan {
  int n = 0;
  int b = 0;           // reference block size (nominal panel width)
  int nb = 0;          // number of panels
  int mode = 0;        // bbk_update_mode
  double* a = nullptr;
  long long lda = 0;
  int* perm = nullptr;
  int* pivot_types = nullptr;
  int* panel_end = nullptr;  // may be null
  // workspace
  double* w = nullptr;       // (b+2) rows x ldw: the panel's W rows, final column order
  long long ldw = 0;
  double* ucm = nullptr;     // n x ldu column-major U rows of the panel, final column order
  int ldu = 0;
  double* uslot = nullptr;   // n x ldu: U by column slot while the panel runs
  double* wslot = nullptr;   // (b+2) x ldw: W by slot when shared memory cannot hold it
  double* dlog = nullptr;    // 2 x (b+2): D entries of the panel's pivots
  int* srcmap = nullptr;     // n: slot holding each index at the end of a panel
  int* moved = nullptr;      // 2 x move_cap: indices a panel's interchanges moved
  int move_cap = 0;
  double* gbuf = nullptr;    // move_cap x ldw: gathered rows of the moved indices
  int* moves = nullptr;      // nb x 2 x move_cap: each panel's moves (positions dst, then src)
  int* move_counts = nullptr;  // nb: moves per panel
  int* bounds = nullptr;     // 2 nb: each panel's [start, end)
  int* posinv = nullptr;     // n: position at the end of a panel -> final position
  int* movetmp = nullptr;    // move_cap + 2
  int* permbuf = nullptr;    // move_cap: gathered permutation entries
  unsigned long long* slots = nullptr;  // 2 x grid x kSlotWords
  DeviceState* state = nullptr;
  int grid = 0;              // CTAs of the panel kernel
  unsigned long long timeout_ns = 0;
  unsigned long long* stats = nullptr;  // optional per-phase panel timing
  double* scales = nullptr;  // BF16 update: 2 x (n/64 + 2) power-of-two scales
  void* hsplit = nullptr;    // BF16 update: 2 operands x 3 terms x hstride BF16, split once per panel
  int kpad = 0;              // BF16 update: panel width rounded up to 32 (k pitch of hsplit)
  size_t hstride = 0;        // BF16 update: elements per operand term (n_pad x kpad)
  double* pivlog = nullptr;  // optional decision log (kPivLogWords doubles per position)
  double* wrows = nullptr;   // optional copy of each panel's W rows at its trailing columns
  long long ld_wrows = 0;
};
}  // namespace bbk
