// Solve entry point for callers that must not allocate device memory.
//
// Some callers cannot call cudaMalloc (or any allocating routine): a
// framework whose caching allocator owns all of the device's memory and must
// not be bypassed, a fixed-size memory pool set up once at start-up, or a
// latency-critical loop where the device-wide synchronisation that
// cudaMalloc/cudaFree imply is not acceptable.  bbk_solve_device needs
// 2 * n * nrhs doubles of scratch and otherwise allocates them; this variant
// takes that scratch from the array below instead.
//
// The array is a file-scope __device__ variable: every GPU that loads the
// library holds its 8 MiB until the process exits.  In host code its name is
// only a host-side stand-in, so the device address is looked up with
// cudaGetSymbolAddress once per device (with that device current) and only
// that address is ever handed to kernels.
#include <mutex>

#include "bbk_internal.cuh"

namespace bbk {
namespace {

constexpr long long kNoAllocMaxElements = BBK_SOLVE_NOALLOC_MAX_ELEMENTS;  // n * nrhs

// Two ping-pong copies of the right-hand sides (see solve_enqueue).
static __device__ __align__(256) double g_solve_scratch[2 * kNoAllocMaxElements];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
double* g_scratch_addr[kMaxDevices] = {nullptr};

// Device address of g_solve_scratch on the current device (looked up once).
int scratch_address(double** out) {
  int dev = 0;
  BBK_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return set_error(BBK_ERR_NO_DEVICE, "device %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (g_scratch_addr[dev] == nullptr) {
    void* p = nullptr;
    const cudaError_t err = cudaGetSymbolAddress(&p, g_solve_scratch);
    if (err != cudaSuccess) return cuda_error(err, "cudaGetSymbolAddress(solve scratch)");
    g_scratch_addr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_addr[dev];
  return BBK_OK;
}

}  // namespace
}  // namespace bbk

using namespace bbk;

extern "C" int bbk_solve_device_noalloc(int n, const double* factors, long long ldf,
                                        const int* perm, const int* pivot_types, int nrhs,
                                        double* b, long long ldb, void* stream) {
  if (n <= 0) return set_error(BBK_ERR_INVALID_ARGUMENT, "matrix size must be positive");
  if (nrhs < 0) return set_error(BBK_ERR_INVALID_ARGUMENT, "nrhs must be non-negative");
  if (ldf < n || (nrhs > 0 && ldb < n))
    return set_error(BBK_ERR_INVALID_ARGUMENT, "leading dimension smaller than n");
  if (!factors || !perm || !pivot_types || (nrhs > 0 && !b))
    return set_error(BBK_ERR_INVALID_ARGUMENT, "null factor, permutation, pivot or rhs array");
  if (static_cast<long long>(n) * nrhs > kNoAllocMaxElements)
    return set_error(BBK_ERR_INVALID_ARGUMENT,
                     "n * nrhs = %lld exceeds the fixed scratch of bbk_solve_device_noalloc "
                     "(at most %lld); use bbk_solve_device",
                     static_cast<long long>(n) * nrhs, kNoAllocMaxElements);
  if (nrhs == 0) return BBK_OK;
  int dev = 0, major = 0;
  BBK_CUDA_TRY(cudaGetDevice(&dev));
  BBK_CUDA_TRY(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
  if (major != 10)
    return set_error(BBK_ERR_NO_DEVICE, "libbbk_b200 is built for sm_100a only; device %d is sm_%d0",
                     dev, major);
  double* scratch = nullptr;
  int rc = scratch_address(&scratch);
  if (rc) return rc;
  // Every element of the scratch is written before it is read, so the
  // previous call's contents need no clearing.
  return solve_enqueue(n, factors, ldf, perm, pivot_types, nrhs, b, ldb, scratch,
                       static_cast<cudaStream_t>(stream));
}
