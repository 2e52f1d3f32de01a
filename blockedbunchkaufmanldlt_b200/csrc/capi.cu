// extern "C" entry points of libbbk_b200 (declared in include/bbk_ldlt.h).
#include <atomic>
#include <cstdarg>
#include <mutex>
#include <vector>
#include <cstdio>
#include <cstring>

#include "bbk_internal.cuh"

namespace bbk {
namespace {

thread_local char g_error[1024] = "";
std::atomic<unsigned long long> g_launches{0};
std::atomic<unsigned long long> g_timeout_ns{5000000000ull};

constexpr int kMaxPanelGrid = 1024;
constexpr size_t kAlign = 256;

int g_sm_count[64] = {0};

// Optional per-class device timing (bbk_profile_begin/end).
enum ProfClass { kProfInit = 0, kProfPanel, kProfFinalize, kProfUpdate, kProfSolve, kProfClasses };
struct ProfRecord {
  int cls;
  cudaEvent_t start, stop;
};
std::mutex g_prof_mu;
bool g_prof_on = false;
std::vector<ProfRecord> g_prof;
std::vector<cudaEvent_t> g_event_pool;

cudaEvent_t pool_event() {
  if (!g_event_pool.empty()) {
    cudaEvent_t e = g_event_pool.back();
    g_event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// Runs `launch` between two events on stream s when profiling is on.
template <typename F>
int profiled(int cls, cudaStream_t s, F&& launch) {
  if (!g_prof_on) return launch();
  std::lock_guard<std::mutex> lk(g_prof_mu);
  ProfRecord r{cls, pool_event(), pool_event()};
  cudaEventRecord(r.start, s);
  const int rc = launch();
  cudaEventRecord(r.stop, s);
  g_prof.push_back(r);
  return rc;
}


struct Carver {
  char* base;
  size_t off = 0;
  template <typename T>
  T* take(size_t count) {
    T* p = reinterpret_cast<T*>(base ? base + off : nullptr);
    off = align_up(off + count * sizeof(T), kAlign);
    return p;
  }
};

// Lays out (or, with base == nullptr, measures) the factorization workspace.
size_t carve_factor(FactorPlan& plan, char* base) {
  const int n = plan.n, b = plan.b;
  // 128-aligned: the update's 128 x 128 tiles read W columns and U rows up
  // to the next multiple of 128
  const long long npad = static_cast<long long>(align_up(static_cast<size_t>(n), 128));
  plan.ldw = npad;
  plan.ldu = static_cast<int>(align_up(static_cast<size_t>(b) + 2, 4));
  Carver c{base};
  plan.state = c.take<DeviceState>(1);
  plan.slots = c.take<unsigned long long>(2ull * kMaxPanelGrid * kSlotWords);
  plan.w = c.take<double>(static_cast<size_t>(b + 2) * npad);
  plan.ucm = c.take<double>(static_cast<size_t>(npad) * plan.ldu);
  plan.uslot = c.take<double>(static_cast<size_t>(npad) * plan.ldu);
  plan.wslot = c.take<double>(static_cast<size_t>(b + 2) * npad);
  plan.dlog = c.take<double>(2 * static_cast<size_t>(b + 2));
  plan.srcmap = c.take<int>(static_cast<size_t>(npad));
  // each pivot step moves at most two indices
  plan.move_cap = static_cast<int>(align_up(2 * static_cast<size_t>(b) + 4, 4));
  plan.moved = c.take<int>(2 * static_cast<size_t>(plan.move_cap));
  plan.gbuf = c.take<double>(static_cast<size_t>(plan.move_cap) * npad);
  const size_t nb = (static_cast<size_t>(n) + b - 1) / b;
  plan.moves = c.take<int>(nb * 2 * plan.move_cap);
  plan.move_counts = c.take<int>(nb);
  plan.bounds = c.take<int>(2 * nb);
  plan.posinv = c.take<int>(static_cast<size_t>(npad));
  plan.movetmp = c.take<int>(static_cast<size_t>(plan.move_cap) + 2);
  plan.permbuf = c.take<int>(static_cast<size_t>(plan.move_cap));
  plan.scales = c.take<double>(2 * (static_cast<size_t>(n) / 64 + 2));
  plan.kpad = static_cast<int>(align_up(static_cast<size_t>(b) + 1, 32));
  plan.hstride = static_cast<size_t>(npad) * plan.kpad;
  plan.hsplit = c.take<unsigned short>(2 * 3 * plan.hstride);
  c.take<int>(4);  // status word for the synchronous entry point
  return c.off;
}

constexpr size_t kPanelStatsWords = 16 + 1024 + 1024 + 5 * 1024;
unsigned long long* g_panel_stats = nullptr;  // device counters (diagnostics)
bool g_panel_stats_on = false;

int validate_factor_args(int n, int block_size, const double* a, long long lda, const int* perm,
                         const int* pivot_types, int mode) {
  if (n <= 0) return set_error(BBK_ERR_INVALID_ARGUMENT, "matrix size must be positive");
  if (block_size <= 0) return set_error(BBK_ERR_INVALID_ARGUMENT, "block size must be positive");
  if (lda < n) return set_error(BBK_ERR_INVALID_ARGUMENT, "lda (%lld) < n (%d)", lda, n);
  if (!a || !perm || !pivot_types)
    return set_error(BBK_ERR_INVALID_ARGUMENT, "null matrix, permutation or pivot array");
  if (mode != BBK_UPDATE_FP64 && mode != BBK_UPDATE_FP64_ORDERED && mode != BBK_UPDATE_FP32 &&
      mode != BBK_UPDATE_BF16 && mode != BBK_UPDATE_BF16X3)
    return set_error(BBK_ERR_INVALID_ARGUMENT, "unknown update mode %d", mode);
  return BBK_OK;
}

}  // namespace

int set_error(int status, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_error, sizeof(g_error), fmt, ap);
  va_end(ap);
  return status;
}

int cuda_error(cudaError_t err, const char* what) {
  snprintf(g_error, sizeof(g_error), "%s: %s", what, cudaGetErrorString(err));
  return err == cudaErrorMemoryAllocation ? BBK_ERR_ALLOC : BBK_ERR_CUDA;
}

// Copies the upper triangle of an n x ld row-major matrix between host and
// device as 64-row block wedges (rows [k, k+64), columns [k, n)): about half
// the bytes of the full matrix.  The few strictly-lower entries inside each
// wedge are copied unchanged (the factorization never writes them).
cudaError_t copy_upper(double* dst, const double* src, int n, long long ld, cudaMemcpyKind kind,
                       cudaStream_t s) {
  constexpr int kRows = 64;
  const size_t pitch = static_cast<size_t>(ld) * sizeof(double);
  for (int k = 0; k < n; k += kRows) {
    const int h = n - k < kRows ? n - k : kRows;
    const size_t off = static_cast<size_t>(k) * ld + k;
    cudaError_t err = cudaMemcpy2DAsync(dst + off, pitch, src + off, pitch,
                                        static_cast<size_t>(n - k) * sizeof(double), h, kind, s);
    if (err != cudaSuccess) return err;
  }
  return cudaSuccess;
}

int check_device() {
  int dev = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err != cudaSuccess) return set_error(BBK_ERR_NO_DEVICE, "no CUDA device: %s", cudaGetErrorString(err));
  int major = 0;
  err = cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  if (err != cudaSuccess) return cuda_error(err, "cudaDeviceGetAttribute");
  if (major != 10)
    return set_error(BBK_ERR_NO_DEVICE,
                     "libbbk_b200 is built for sm_100a only; device %d is sm_%d0", dev, major);
  // Workspace this library allocates with cudaMallocAsync goes back to the
  // device's default pool; keep it there instead of releasing it to the
  // driver at every synchronization, so repeated calls reuse it.
  static bool pool_kept[64] = {};
  if (dev >= 0 && dev < 64 && !pool_kept[dev]) {
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
      unsigned long long keep = ~0ull;  // the attribute is a 64-bit byte count
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    pool_kept[dev] = true;
  }
  return BBK_OK;
}

void count_launch(unsigned n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

unsigned long long wait_timeout_ns() { return g_timeout_ns.load(std::memory_order_relaxed); }

int device_sm_count() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (g_sm_count[dev] == 0) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
      v = 148;
    g_sm_count[dev] = v;
  }
  return g_sm_count[dev];
}

// Enqueue a whole factorization for an already carved plan.
static int enqueue_factor(FactorPlan& plan, int* status_device, cudaStream_t s) {
  int rc = profiled(kProfInit, s, [&] {
    return launch_init(plan.n, plan.perm, plan.pivot_types, plan.state, plan.slots,
                       2ull * kMaxPanelGrid * kSlotWords, s);
  });
  if (rc) return rc;
  for (int panel = 0; panel < plan.nb; ++panel) {
    if ((rc = profiled(kProfPanel, s, [&] { return launch_panel(plan, panel, s); }))) return rc;
    if ((rc = profiled(kProfFinalize, s, [&] { return launch_finalize(plan, panel, s); }))) return rc;
    if (plan.wrows && (rc = launch_wrows(plan, panel, s))) return rc;
    if ((rc = profiled(kProfUpdate, s, [&] { return launch_update(plan, panel, s); }))) return rc;
  }
  if ((rc = profiled(kProfFinalize, s, [&] { return launch_left_swaps(plan, s); }))) return rc;
  return launch_status_copy(plan.state, status_device, s);
}

int enqueue_solve(int n, const double* f, long long ldf, const int* perm, const int* pt,
                  int nrhs, double* b, long long ldb, double* work, cudaStream_t s) {
  return profiled(kProfSolve, s, [&] {
    return solve_enqueue(n, f, ldf, perm, pt, nrhs, b, ldb, work, s);
  });
}

}  // namespace bbk

using namespace bbk;

extern "C" {

int bbk_abi_version(void) { return BBK_ABI_VERSION; }

const char* bbk_last_error(void) { return g_error; }

const char* bbk_status_string(int status) {
  switch (status) {
    case BBK_OK: return "ok";
    case BBK_ERR_INVALID_ARGUMENT: return "invalid argument";
    case BBK_ERR_OUT_OF_RANGE: return "out of range";
    case BBK_ERR_LOGIC: return "logic error";
    case BBK_ERR_ALLOC: return "allocation failed";
    case BBK_ERR_CUDA: return "CUDA error";
    case BBK_ERR_TIMEOUT: return "device-side wait timed out";
    case BBK_ERR_NO_DEVICE: return "no usable sm_100 device";
    case BBK_ERR_WORKSPACE: return "workspace too small";
    default: return "unknown status";
  }
}

unsigned long long bbk_kernel_launch_count(void) {
  return g_launches.load(std::memory_order_relaxed);
}

int bbk_profile_begin(void) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  for (auto& r : g_prof) {
    g_event_pool.push_back(r.start);
    g_event_pool.push_back(r.stop);
  }
  g_prof.clear();
  g_prof_on = true;
  return BBK_OK;
}

int bbk_profile_end(double* ms, long long* counts) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  g_prof_on = false;
  double tot[kProfClasses] = {0};
  long long cnt[kProfClasses] = {0};
  int rc = BBK_OK;
  for (auto& r : g_prof) {
    cudaError_t err = cudaEventSynchronize(r.stop);
    float t = 0.f;
    if (err == cudaSuccess) err = cudaEventElapsedTime(&t, r.start, r.stop);
    if (err != cudaSuccess && rc == BBK_OK) rc = cuda_error(err, "profile events");
    tot[r.cls] += t;
    cnt[r.cls] += 1;
    g_event_pool.push_back(r.start);
    g_event_pool.push_back(r.stop);
  }
  g_prof.clear();
  for (int i = 0; i < kProfClasses; ++i) {
    if (ms) ms[i] = tot[i];
    if (counts) counts[i] = cnt[i];
  }
  return rc;
}

int bbk_panel_stats(int enable, unsigned long long* out) {
  int rc = check_device();
  if (rc) return rc;
  if (enable) {
    if (!g_panel_stats) BBK_CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(&g_panel_stats), kPanelStatsWords * 8));
    BBK_CUDA_TRY(cudaMemset(g_panel_stats, 0, kPanelStatsWords * 8));
    g_panel_stats_on = true;
    return BBK_OK;
  }
  g_panel_stats_on = false;
  if (out && g_panel_stats) {
    BBK_CUDA_TRY(cudaDeviceSynchronize());
    BBK_CUDA_TRY(cudaMemcpy(out, g_panel_stats, 10 * 8, cudaMemcpyDeviceToHost));
  }
  return BBK_OK;
}

int bbk_panel_stats_raw(unsigned long long* out, size_t words) {
  if (!g_panel_stats || !out) return set_error(BBK_ERR_LOGIC, "panel stats never armed");
  if (words > kPanelStatsWords) words = kPanelStatsWords;
  BBK_CUDA_TRY(cudaDeviceSynchronize());
  BBK_CUDA_TRY(cudaMemcpy(out, g_panel_stats, words * 8, cudaMemcpyDeviceToHost));
  return BBK_OK;
}

int bbk_set_wait_timeout_ns(unsigned long long timeout_ns) {
  if (timeout_ns == 0) return set_error(BBK_ERR_INVALID_ARGUMENT, "timeout must be positive");
  g_timeout_ns.store(timeout_ns, std::memory_order_relaxed);
  return BBK_OK;
}

size_t bbk_factor_workspace_size(int n, int block_size) {
  if (n <= 0 || block_size <= 0) return 0;
  FactorPlan plan;
  plan.n = n;
  plan.b = block_size;
  return carve_factor(plan, nullptr);
}

static int factor_async(int n, int block_size, double* a, long long lda, int* perm,
                        int* pivot_types, int* panel_end, int update_mode, const bbk_factor_extras* extras,
                        void* workspace, size_t workspace_bytes, int* status_device,
                        void* stream) {
  int rc = validate_factor_args(n, block_size, a, lda, perm, pivot_types, update_mode);
  if (rc) return rc;
  double* pivot_log = extras ? extras->pivot_log : nullptr;
  if (extras && extras->workspace_rows && extras->workspace_ld < n)
    return set_error(BBK_ERR_INVALID_ARGUMENT, "workspace_ld (%lld) < n (%d)", extras->workspace_ld, n);
  if ((rc = check_device())) return rc;
  if (n > panel_max_n())
    return set_error(BBK_ERR_INVALID_ARGUMENT, "n = %d exceeds this device's panel limit %d", n,
                     panel_max_n());
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  FactorPlan plan;
  plan.n = n;
  plan.b = block_size;
  plan.nb = (n + block_size - 1) / block_size;
  plan.mode = update_mode;
  plan.a = a;
  plan.lda = lda;
  plan.perm = perm;
  plan.pivot_types = pivot_types;
  plan.panel_end = panel_end;
  plan.grid = panel_grid_size(n);
  plan.timeout_ns = wait_timeout_ns();
  plan.stats = g_panel_stats_on ? g_panel_stats : nullptr;
  plan.pivlog = pivot_log;
  plan.wrows = extras ? extras->workspace_rows : nullptr;
  plan.ld_wrows = extras ? extras->workspace_ld : 0;
  if (pivot_log) {
    // all-ones bytes: NaN at every position no decision writes
    BBK_CUDA_TRY(cudaMemsetAsync(pivot_log, 0xff, static_cast<size_t>(n) * kPivLogWords * sizeof(double), s));
  }
  const size_t need = carve_factor(plan, nullptr);
  char* base = static_cast<char*>(workspace);
  bool owned = false;
  if (base == nullptr) {
    BBK_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void**>(&base), need, s));
    owned = true;
  } else if (workspace_bytes < need) {
    return set_error(BBK_ERR_WORKSPACE, "factor workspace needs %zu bytes, got %zu", need,
                     workspace_bytes);
  }
  carve_factor(plan, base);
  int* status = status_device;
  if (status == nullptr) {
    Carver c{base};
    c.off = need - kAlign;
    status = c.take<int>(1);
  }
  rc = enqueue_factor(plan, status, s);
  if (owned) {
    cudaError_t err = cudaFreeAsync(base, s);
    if (!rc && err != cudaSuccess) rc = cuda_error(err, "cudaFreeAsync");
  }
  return rc;
}

int bbk_factor_device_async(int n, int block_size, double* a, long long lda, int* perm,
                            int* pivot_types, int* panel_end, int update_mode, void* workspace,
                            size_t workspace_bytes, int* status_device, void* stream) {
  return factor_async(n, block_size, a, lda, perm, pivot_types, panel_end, update_mode, nullptr,
                      workspace, workspace_bytes, status_device, stream);
}

int bbk_factor_device_ex(int n, int block_size, double* a, long long lda, int* perm, int* pivot_types,
                         int* panel_end, int update_mode, const bbk_factor_extras* extras, void* workspace,
                         size_t workspace_bytes, int* status_device, void* stream) {
  return factor_async(n, block_size, a, lda, perm, pivot_types, panel_end, update_mode, extras,
                      workspace, workspace_bytes, status_device, stream);
}

int bbk_factor_device(int n, int block_size, double* a, long long lda, int* perm,
                      int* pivot_types, int* panel_end, int update_mode, void* workspace,
                      size_t workspace_bytes, void* stream) {
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int* d_status = nullptr;
  int rc = validate_factor_args(n, block_size, a, lda, perm, pivot_types, update_mode);
  if (rc) return rc;
  if ((rc = check_device())) return rc;
  BBK_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void**>(&d_status), sizeof(int), s));
  rc = bbk_factor_device_async(n, block_size, a, lda, perm, pivot_types, panel_end, update_mode,
                               workspace, workspace_bytes, d_status, s);
  int h_status = BBK_OK;
  if (!rc) {
    cudaError_t err = cudaMemcpyAsync(&h_status, d_status, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) rc = cuda_error(err, "factorization");
  }
  cudaFreeAsync(d_status, s);
  if (rc) return rc;
  if (h_status != BBK_OK)
    return set_error(h_status, "factorization aborted on the device: %s", bbk_status_string(h_status));
  return BBK_OK;
}

int bbk_factor_host(int n, int block_size, double* a, long long lda, int* perm, int* pivot_types,
                    int* panel_end, int update_mode) {
  return bbk_factor_solve_host(n, block_size, a, lda, perm, pivot_types, panel_end, 0, nullptr, 0,
                               update_mode);
}

size_t bbk_solve_workspace_size(int n, int nrhs) {
  if (n <= 0 || nrhs <= 0) return 0;
  return solve_work_doubles(n, nrhs) * sizeof(double);
}

static int validate_solve(int n, const double* f, long long ldf, const int* perm, const int* pt,
                          int nrhs, const double* b, long long ldb) {
  if (n <= 0) return set_error(BBK_ERR_INVALID_ARGUMENT, "matrix size must be positive");
  if (nrhs < 0) return set_error(BBK_ERR_INVALID_ARGUMENT, "nrhs must be non-negative");
  if (ldf < n || (nrhs > 0 && ldb < n))
    return set_error(BBK_ERR_INVALID_ARGUMENT, "leading dimension smaller than n");
  if (!f || !perm || !pt || (nrhs > 0 && !b))
    return set_error(BBK_ERR_INVALID_ARGUMENT, "null factor, permutation, pivot or rhs array");
  return BBK_OK;
}

int bbk_solve_device(int n, const double* factors, long long ldf, const int* perm,
                     const int* pivot_types, int nrhs, double* b, long long ldb, void* workspace,
                     size_t workspace_bytes, void* stream) {
  int rc = validate_solve(n, factors, ldf, perm, pivot_types, nrhs, b, ldb);
  if (rc) return rc;
  if (nrhs == 0) return BBK_OK;
  if ((rc = check_device())) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t need = bbk_solve_workspace_size(n, nrhs);
  double* work = static_cast<double*>(workspace);
  bool owned = false;
  if (work == nullptr) {
    BBK_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void**>(&work), need, s));
    owned = true;
  } else if (workspace_bytes < need) {
    return set_error(BBK_ERR_WORKSPACE, "solve workspace needs %zu bytes, got %zu", need,
                     workspace_bytes);
  }
  rc = enqueue_solve(n, factors, ldf, perm, pivot_types, nrhs, b, ldb, work, s);
  if (!rc) rc = solve_status(work, n, nrhs, s);  // waits for the solve
  if (owned) cudaFreeAsync(work, s);
  return rc;
}

int bbk_solve_host(int n, const double* factors, long long ldf, const int* perm,
                   const int* pivot_types, int nrhs, double* b, long long ldb) {
  int rc = validate_solve(n, factors, ldf, perm, pivot_types, nrhs, b, ldb);
  if (rc) return rc;
  if (nrhs == 0) return BBK_OK;
  if ((rc = check_device())) return rc;
  cudaStream_t s;
  BBK_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  double *d_f = nullptr, *d_b = nullptr, *work = nullptr;
  int *d_perm = nullptr, *d_pt = nullptr;
  const size_t fbytes = static_cast<size_t>(n) * ldf * sizeof(double);
  const size_t bbytes = static_cast<size_t>(nrhs) * ldb * sizeof(double);
  cudaError_t err = cudaMallocAsync(reinterpret_cast<void**>(&d_f), fbytes, s);
  if (err == cudaSuccess) err = cudaMallocAsync(reinterpret_cast<void**>(&d_b), bbytes, s);
  if (err == cudaSuccess) err = cudaMallocAsync(reinterpret_cast<void**>(&d_perm), n * sizeof(int), s);
  if (err == cudaSuccess) err = cudaMallocAsync(reinterpret_cast<void**>(&d_pt), n * sizeof(int), s);
  if (err == cudaSuccess)
    err = cudaMallocAsync(reinterpret_cast<void**>(&work), bbk_solve_workspace_size(n, nrhs), s);
  if (err == cudaSuccess) err = copy_upper(d_f, factors, n, ldf, cudaMemcpyHostToDevice, s);
  if (err == cudaSuccess) err = cudaMemcpyAsync(d_b, b, bbytes, cudaMemcpyHostToDevice, s);
  if (err == cudaSuccess) err = cudaMemcpyAsync(d_perm, perm, n * sizeof(int), cudaMemcpyHostToDevice, s);
  if (err == cudaSuccess) err = cudaMemcpyAsync(d_pt, pivot_types, n * sizeof(int), cudaMemcpyHostToDevice, s);
  if (err != cudaSuccess) {
    rc = cuda_error(err, "solve setup");
  } else {
    rc = enqueue_solve(n, d_f, ldf, d_perm, d_pt, nrhs, d_b, ldb, work, s);
    if (!rc) rc = solve_status(work, n, nrhs, s);
    if (!rc) {
      err = cudaMemcpyAsync(b, d_b, bbytes, cudaMemcpyDeviceToHost, s);
      if (err == cudaSuccess) err = cudaStreamSynchronize(s);
      if (err != cudaSuccess) rc = cuda_error(err, "solve");
    }
  }
  cudaFreeAsync(d_f, s);
  cudaFreeAsync(d_b, s);
  cudaFreeAsync(d_perm, s);
  cudaFreeAsync(d_pt, s);
  cudaFreeAsync(work, s);
  cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  return rc;
}

int bbk_factor_solve_host(int n, int block_size, double* a, long long lda, int* perm,
                          int* pivot_types, int* panel_end, int nrhs, double* b, long long ldb,
                          int update_mode) {
  int rc = validate_factor_args(n, block_size, a, lda, perm, pivot_types, update_mode);
  if (rc) return rc;
  if (nrhs < 0 || (nrhs > 0 && (!b || ldb < n)))
    return set_error(BBK_ERR_INVALID_ARGUMENT, "bad right-hand side arguments");
  if ((rc = check_device())) return rc;
  cudaStream_t s;
  BBK_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  const int nb = (n + block_size - 1) / block_size;
  const size_t abytes = static_cast<size_t>(n) * lda * sizeof(double);
  const size_t bbytes = static_cast<size_t>(nrhs) * ldb * sizeof(double);
  const size_t fws = bbk_factor_workspace_size(n, block_size);
  const size_t sws = nrhs > 0 ? bbk_solve_workspace_size(n, nrhs) : 0;
  double *d_a = nullptr, *d_b = nullptr;
  int *d_perm = nullptr, *d_pt = nullptr, *d_pe = nullptr, *d_status = nullptr;
  char* ws = nullptr;
  int h_status = BBK_OK;
  cudaError_t err = cudaMallocAsync(reinterpret_cast<void**>(&d_a), abytes, s);
  if (err == cudaSuccess && nrhs > 0) err = cudaMallocAsync(reinterpret_cast<void**>(&d_b), bbytes, s);
  if (err == cudaSuccess) err = cudaMallocAsync(reinterpret_cast<void**>(&d_perm), n * sizeof(int), s);
  if (err == cudaSuccess) err = cudaMallocAsync(reinterpret_cast<void**>(&d_pt), n * sizeof(int), s);
  if (err == cudaSuccess) err = cudaMallocAsync(reinterpret_cast<void**>(&d_pe), nb * sizeof(int), s);
  if (err == cudaSuccess) err = cudaMallocAsync(reinterpret_cast<void**>(&d_status), sizeof(int), s);
  if (err == cudaSuccess)
    err = cudaMallocAsync(reinterpret_cast<void**>(&ws), fws > sws ? fws : sws, s);
  if (err == cudaSuccess) err = copy_upper(d_a, a, n, lda, cudaMemcpyHostToDevice, s);
  if (err == cudaSuccess && nrhs > 0) err = cudaMemcpyAsync(d_b, b, bbytes, cudaMemcpyHostToDevice, s);
  if (err != cudaSuccess) {
    rc = cuda_error(err, "factorization setup");
  } else {
    rc = bbk_factor_device_async(n, block_size, d_a, lda, d_perm, d_pt, d_pe, update_mode, ws, fws,
                                 d_status, s);
    // The solve only reads the factors, so their copy back to the host runs
    // on a second stream, concurrently with the solve.
    cudaStream_t s2 = nullptr;
    cudaEvent_t factored = nullptr, copied = nullptr;
    if (!rc) {
      err = cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking);
      if (err == cudaSuccess) err = cudaEventCreateWithFlags(&factored, cudaEventDisableTiming);
      if (err == cudaSuccess) err = cudaEventCreateWithFlags(&copied, cudaEventDisableTiming);
      if (err == cudaSuccess) err = cudaEventRecord(factored, s);
      if (err != cudaSuccess) rc = cuda_error(err, "factorization copy stream");
    }
    int* solve_st = nullptr;
    int h_solve = BBK_OK;
    if (!rc && nrhs > 0) {
      rc = enqueue_solve(n, d_a, lda, d_perm, d_pt, nrhs, d_b, ldb, reinterpret_cast<double*>(ws), s);
      solve_st = solve_status_word(reinterpret_cast<double*>(ws), n, nrhs);
    }
    if (!rc) {
      // the second stream's copies are enqueued first: a copy into pageable
      // memory (the status word below, or a caller's pageable buffer) can
      // block this thread until its stream reaches it
      err = cudaStreamWaitEvent(s2, factored, 0);
      if (err == cudaSuccess) err = copy_upper(a, d_a, n, lda, cudaMemcpyDeviceToHost, s2);
      if (err == cudaSuccess) err = cudaMemcpyAsync(perm, d_perm, n * sizeof(int), cudaMemcpyDeviceToHost, s2);
      if (err == cudaSuccess) err = cudaMemcpyAsync(pivot_types, d_pt, n * sizeof(int), cudaMemcpyDeviceToHost, s2);
      if (err == cudaSuccess && panel_end)
        err = cudaMemcpyAsync(panel_end, d_pe, nb * sizeof(int), cudaMemcpyDeviceToHost, s2);
      if (err == cudaSuccess && nrhs > 0) err = cudaMemcpyAsync(b, d_b, bbytes, cudaMemcpyDeviceToHost, s);
      if (err == cudaSuccess) err = cudaMemcpyAsync(&h_status, d_status, sizeof(int), cudaMemcpyDeviceToHost, s);
      if (err == cudaSuccess && solve_st)
        err = cudaMemcpyAsync(&h_solve, solve_st, sizeof(int), cudaMemcpyDeviceToHost, s);
      if (err == cudaSuccess) err = cudaStreamSynchronize(s2);
      if (err == cudaSuccess) err = cudaStreamSynchronize(s);
      if (err != cudaSuccess) rc = cuda_error(err, "factorization");
      if (!rc && h_status == BBK_OK && h_solve != BBK_OK)
        rc = set_error(h_solve, "solve aborted on the device: %s", bbk_status_string(h_solve));
    }
    if (s2) {
      // the frees below are ordered on s: s waits for s2's copies first
      if (copied && cudaEventRecord(copied, s2) == cudaSuccess) cudaStreamWaitEvent(s, copied, 0);
      cudaStreamSynchronize(s2);
      cudaStreamDestroy(s2);
    }
    if (factored) cudaEventDestroy(factored);
    if (copied) cudaEventDestroy(copied);
  }
  cudaFreeAsync(d_a, s);
  if (d_b) cudaFreeAsync(d_b, s);
  cudaFreeAsync(d_perm, s);
  cudaFreeAsync(d_pt, s);
  cudaFreeAsync(d_pe, s);
  cudaFreeAsync(d_status, s);
  cudaFreeAsync(ws, s);
  cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  if (rc) return rc;
  if (h_status != BBK_OK)
    return set_error(h_status, "factorization aborted on the device: %s", bbk_status_string(h_status));
  return BBK_OK;
}

size_t bbk_solve_refined_workspace_size(int n, int nrhs, int restart) {
  if (n <= 0 || nrhs <= 0 || restart < 0) return 0;
  const size_t vec = static_cast<size_t>(n) * nrhs;
  return (refine_work_doubles(n, nrhs, restart > 0 ? restart : 1) + 2 * vec) * sizeof(double) + kAlign;
}

int bbk_solve_refined_device(int n, const double* a, long long lda, const double* factors,
                             long long ldf, const int* perm, const int* pivot_types, int nrhs,
                             const double* b, long long ldb, double* x, long long ldx, double tol,
                             int max_iter, int method, int restart, bbk_refine_info* info,
                             void* workspace, size_t workspace_bytes, void* stream) {
  int rc = validate_solve(n, factors, ldf, perm, pivot_types, nrhs, b, ldb);
  if (rc) return rc;
  if (!a || lda < n || !x || (nrhs > 0 && ldx < n) || !info)
    return set_error(BBK_ERR_INVALID_ARGUMENT, "bad refinement arguments");
  if (method != BBK_REFINE_CLASSICAL && method != BBK_REFINE_GMRES)
    return set_error(BBK_ERR_INVALID_ARGUMENT, "unknown refinement method %d", method);
  if (max_iter < 0 || !(tol >= 0.0) || (method == BBK_REFINE_GMRES && restart <= 0))
    return set_error(BBK_ERR_INVALID_ARGUMENT, "bad refinement controls");
  *info = bbk_refine_info{};
  if (nrhs == 0) {
    info->converged = 1;
    return BBK_OK;
  }
  if ((rc = check_device())) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int m = method == BBK_REFINE_GMRES ? restart : 1;
  const size_t need = bbk_solve_refined_workspace_size(n, nrhs, m);
  char* base = static_cast<char*>(workspace);
  bool owned = false;
  if (base == nullptr) {
    BBK_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void**>(&base), need, s));
    owned = true;
  } else if (workspace_bytes < need) {
    return set_error(BBK_ERR_WORKSPACE, "refinement workspace needs %zu bytes, got %zu", need,
                     workspace_bytes);
  }
  double* bc = reinterpret_cast<double*>(align_up(reinterpret_cast<uintptr_t>(base), kAlign));
  const size_t vec = static_cast<size_t>(n) * nrhs;
  double* xc = bc + vec;
  double* work = xc + vec;
  const size_t pitch_b = static_cast<size_t>(ldb) * sizeof(double);
  const size_t pitch_x = static_cast<size_t>(ldx) * sizeof(double);
  const size_t row = static_cast<size_t>(n) * sizeof(double);
  cudaError_t err = cudaMemcpy2DAsync(bc, row, b, pitch_b, row, nrhs, cudaMemcpyDeviceToDevice, s);
  if (err == cudaSuccess) err = cudaMemcpy2DAsync(xc, row, b, pitch_b, row, nrhs, cudaMemcpyDeviceToDevice, s);
  if (err != cudaSuccess) {
    rc = cuda_error(err, "refinement setup");
  } else {
    // x0 from the factors, then FP64 refinement (the solve scratch sits at
    // the end of the refinement workspace)
    double* swork = work + refine_work_doubles(n, nrhs, m) - solve_work_doubles(n, nrhs);
    rc = enqueue_solve(n, factors, ldf, perm, pivot_types, nrhs, xc, n, swork, s);
    if (!rc) rc = solve_status(swork, n, nrhs, s);
    if (!rc)
      rc = refine_enqueue(n, a, lda, factors, ldf, perm, pivot_types, nrhs, bc, xc, tol, max_iter,
                          method, m, work, info, s);
    if (!rc) {
      err = cudaMemcpy2DAsync(x, pitch_x, xc, row, row, nrhs, cudaMemcpyDeviceToDevice, s);
      if (err == cudaSuccess) err = cudaStreamSynchronize(s);
      if (err != cudaSuccess) rc = cuda_error(err, "refinement");
    }
  }
  if (owned) cudaFreeAsync(base, s);
  return rc;
}

int bbk_reconstruct_device(int n, const double* factors, long long ldf, const int* perm,
                           const int* pivot_types, double* out, long long ldo, void* stream) {
  if (n <= 0) return set_error(BBK_ERR_INVALID_ARGUMENT, "matrix size must be positive");
  if (!factors || !perm || !pivot_types || !out || ldf < n || ldo < n)
    return set_error(BBK_ERR_INVALID_ARGUMENT, "bad reconstruction arguments");
  int rc = check_device();
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double* m = nullptr;
  BBK_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void**>(&m), reconstruct_work_doubles(n) * sizeof(double), s));
  rc = reconstruct_enqueue(n, factors, ldf, perm, pivot_types, out, ldo, m, s);
  cudaFreeAsync(m, s);
  if (rc) return rc;
  BBK_CUDA_TRY(cudaStreamSynchronize(s));
  return BBK_OK;
}

int bbk_extract_ld_device(int n, const double* factors, long long ldf, const int* pivot_types, double* l,
                          long long ldl, double* d, long long ldd, void* stream) {
  if (n <= 0) return set_error(BBK_ERR_INVALID_ARGUMENT, "matrix size must be positive");
  if (!factors || !pivot_types || (!l && !d) || ldf < n || (l && ldl < n) || (d && ldd < n))
    return set_error(BBK_ERR_INVALID_ARGUMENT, "bad extraction arguments");
  int rc = check_device();
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  rc = extract_ld_enqueue(n, factors, ldf, pivot_types, l, ldl, d, ldd, s);
  if (rc) return rc;
  BBK_CUDA_TRY(cudaStreamSynchronize(s));
  return BBK_OK;
}

int bbk_scale_one_by_one(int count, double pivot, const double* source, int source_stride,
                         double* destination, int destination_stride, void* stream) {
  if (count <= 0) return BBK_OK;
  if (!source || !destination) return set_error(BBK_ERR_INVALID_ARGUMENT, "null pointer");
  int rc = check_device();
  if (rc) return rc;
  return launch_scale_1x1(count, pivot, source, source_stride, destination, destination_stride,
                          static_cast<cudaStream_t>(stream));
}

int bbk_scale_two_by_two(int count, double a, double b, double c, const double* first_source,
                         int first_source_stride, const double* second_source,
                         int second_source_stride, double* first_destination,
                         int first_destination_stride, double* second_destination,
                         int second_destination_stride, void* stream) {
  if (count <= 0) return BBK_OK;
  if (!first_source || !second_source || !first_destination || !second_destination)
    return set_error(BBK_ERR_INVALID_ARGUMENT, "null pointer");
  int rc = check_device();
  if (rc) return rc;
  return launch_scale_2x2(count, a, b, c, first_source, first_source_stride, second_source,
                          second_source_stride, first_destination, first_destination_stride,
                          second_destination, second_destination_stride,
                          static_cast<cudaStream_t>(stream));
}

int bbk_update_trailing_block(int rows, int cols, int inner_dim, const double* left_panel,
                              int left_panel_stride, const double* workspace_panel,
                              int workspace_panel_stride, double* target, int target_stride,
                              int update_mode, void* stream) {
  if (rows <= 0 || cols <= 0 || inner_dim <= 0) return BBK_OK;
  if (!left_panel || !workspace_panel || !target)
    return set_error(BBK_ERR_INVALID_ARGUMENT, "null pointer");
  if (update_mode != BBK_UPDATE_FP64 && update_mode != BBK_UPDATE_FP64_ORDERED &&
      update_mode != BBK_UPDATE_FP32)
    return set_error(BBK_ERR_INVALID_ARGUMENT, "unknown update mode %d", update_mode);
  int rc = check_device();
  if (rc) return rc;
  return launch_update_block(rows, cols, inner_dim, left_panel, left_panel_stride, workspace_panel,
                             workspace_panel_stride, target, target_stride, update_mode,
                             static_cast<cudaStream_t>(stream));
}

static int run_probe(int ctas, int nslots, int iters, unsigned long long timeout_ns,
                     unsigned long long* elapsed_ns, int* device_status, cudaStream_t s) {
  const size_t slot_words = 2ull * (ctas + 1) * kSlotWords;
  const size_t off_slots = align_up(sizeof(DeviceState), kAlign);
  const size_t off_stats = off_slots + align_up(slot_words * 8, kAlign);
  const size_t bytes = off_stats + kAlign;
  char* base = nullptr;
  BBK_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void**>(&base), bytes, s));
  DeviceState* st = reinterpret_cast<DeviceState*>(base);
  auto* slots = reinterpret_cast<unsigned long long*>(base + off_slots);
  auto* stats = reinterpret_cast<unsigned long long*>(base + off_stats);
  int rc = BBK_OK;
  cudaError_t err = cudaMemsetAsync(base, 0, bytes, s);
  if (err != cudaSuccess) {
    rc = cuda_error(err, "cudaMemsetAsync");
  } else {
    rc = launch_probe_wait(ctas, nslots, iters, timeout_ns, st, slots, stats, s);
    if (!rc) {
      err = cudaMemcpyAsync(device_status, &st->status, sizeof(int), cudaMemcpyDeviceToHost, s);
      if (err == cudaSuccess && elapsed_ns)
        err = cudaMemcpyAsync(elapsed_ns, stats, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s);
      if (err == cudaSuccess) err = cudaStreamSynchronize(s);
      if (err != cudaSuccess) rc = cuda_error(err, "probe");
    }
  }
  cudaFreeAsync(base, s);
  cudaStreamSynchronize(s);
  return rc;
}

int bbk_probe_bounded_wait(int ctas, unsigned long long timeout_ns, void* stream) {
  if (ctas <= 0 || ctas > 223 || timeout_ns == 0)
    return set_error(BBK_ERR_INVALID_ARGUMENT, "bad probe arguments");
  int rc = check_device();
  if (rc) return rc;
  int h_status = BBK_OK;
  rc = run_probe(ctas, ctas + 1, 1, timeout_ns, nullptr, &h_status, static_cast<cudaStream_t>(stream));
  if (rc) return rc;
  if (h_status != BBK_OK) return set_error(h_status, "bounded wait expired as designed");
  return set_error(BBK_ERR_LOGIC, "bounded-wait probe finished without timing out");
}

int bbk_probe_exchange_ns(int ctas, int iters, double* ns_per_exchange, void* stream) {
  if (ctas <= 0 || ctas > 224 || iters <= 0 || !ns_per_exchange)
    return set_error(BBK_ERR_INVALID_ARGUMENT, "bad probe arguments");
  int rc = check_device();
  if (rc) return rc;
  int h_status = BBK_OK;
  unsigned long long ns = 0;
  rc = run_probe(ctas, ctas, iters, wait_timeout_ns(), &ns, &h_status, static_cast<cudaStream_t>(stream));
  if (rc) return rc;
  if (h_status != BBK_OK) return set_error(h_status, "exchange probe aborted");
  *ns_per_exchange = static_cast<double>(ns) / iters;
  return BBK_OK;
}

}  // extern "C"
