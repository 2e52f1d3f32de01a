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
// only a host-side stand-in, so on every call the device address is looked
// up with cudaGetSymbolAddress (with the call's device current) and only
// that address is handed to kernels.  The lookup is not cached: after a
// cudaDeviceReset, or in another context on the same device, the library's
// module is loaded again and the array can sit elsewhere.  The first lookup
// on a device may load the module, so the first call should come before any
// stream capture.
#include "bbk_internal.cuh"

namespace bbk {
namespace {

constexpr long long kNoAllocMaxElements = BBK_SOLVE_NOALLOC_MAX_ELEMENTS;  // n * nrhs

// The solve's scratch, laid out as solve_enqueue uses it: the right-hand
// sides being solved (n * nrhs doubles), then one flag per 64-row block and
// the status word.  Sized like solve_work_doubles(n, nrhs) at the limit.
static __device__ __align__(256) double g_solve_scratch[2 * kNoAllocMaxElements];

// Device address of g_solve_scratch in the current context.
int scratch_address(double** out) {
  void* p = nullptr;
  const cudaError_t err = cudaGetSymbolAddress(&p, g_solve_scratch);
  if (err != cudaSuccess) return cuda_error(err, "cudaGetSymbolAddress(solve scratch)");
  *out = static_cast<double*>(p);
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
  // Every element of the scratch is written before it is read (the block
  // flags and the status word are cleared by the solve's first kernel), so
  // the previous call's contents need no clearing.
  return enqueue_solve(n, factors, ldf, perm, pivot_types, nrhs, b, ldb, scratch,
                       static_cast<cudaStream_t>(stream));
}
