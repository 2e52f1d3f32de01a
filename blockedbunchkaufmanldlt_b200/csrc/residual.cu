// Sampled relative residual of compact Bunch-Kaufman factors, on the device.
//
// The reference checks its large factorizations without forming L D L^T:
// SampledRelativeResidual (tests/block_ldlt_large_stress_test.cc:220-244 in
// wentianshu/BlockedBunchKaufmanLDLT) evaluates, for a set of sampled
// entries (row, col) of the original matrix, the same entry of
// P^T L D L^T P straight from the compact factors (CompactLValue and
// ReconstructedPermutedEntry, :160-194) and returns
//   sqrt(sum (reconstructed - original)^2) / max(sqrt(sum original^2), 1).
// Here one thread evaluates one sample, summing over the pivots in the
// reference's order with every product and sum rounded separately, and one
// thread then forms the two sums in sample order, so the result is bit for
// bit the reference's for the same (finite) factors.  Only pivots
// p <= min(i, j) of the factored positions (i, j) contribute
// (L(i, p) = 0 for p > i).
#include <algorithm>

#include "bbk_internal.cuh"

namespace bbk {
namespace {

// inv[perm[i]] = i; inv starts at -1, and entries of perm outside [0, n)
// are skipped, so a caller's invalid permutation cannot reach memory
// outside the arrays (its samples then come out NaN)
__global__ void inverse_perm_kernel(int n, const int* perm, int* inv) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int p = perm[i];
    if (p >= 0 && p < n) inv[p] = i;
  }
}

// CompactLValue (:160-172): L(row, col) from the compact upper factor.
__device__ __forceinline__ double compact_l(const double* f, long long ldf, const int* pt, int row, int col) {
  if (row == col) return 1.0;
  if (row < col) return 0.0;
  if (pt[col] == 2 && row == col + 1) return 0.0;
  return f[static_cast<long long>(col) * ldf + row];
}

// ReconstructedPermutedEntry (:174-194) at factored positions (r, c), and
// the difference to the original entry; diff[k], orig[k] per sample.
__global__ void sampled_entry_kernel(int n, const double* a, long long lda, const double* f, long long ldf,
                                     const int* pt, const int* inv, int count, const int* rows,
                                     const int* cols, double* diff, double* orig) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const int orow = rows[k], ocol = cols[k];
  const bool in_range = orow >= 0 && orow < n && ocol >= 0 && ocol < n;
  const int r = in_range ? inv[orow] : -1, c = in_range ? inv[ocol] : -1;
  if (r < 0 || c < 0) {  // a sample outside the matrix, or a position no index maps to
    diff[k] = __longlong_as_double(0x7ff8000000000000ll);
    orig[k] = 0.0;
    return;
  }
  const int last = min(r, c);
  double value = 0.0;
  for (int p = 0; p <= last; ++p) {
    const double row_left = compact_l(f, ldf, pt, r, p);
    const double col_left = compact_l(f, ldf, pt, c, p);
    const double d = f[static_cast<long long>(p) * ldf + p];
    value = xadd(value, xmul(xmul(row_left, d), col_left));
    if (pt[p] == 2) {
      const double off = f[static_cast<long long>(p) * ldf + p + 1];
      const double row_next = compact_l(f, ldf, pt, r, p + 1);
      const double col_next = compact_l(f, ldf, pt, c, p + 1);
      value = xadd(value, xmul(off, xadd(xmul(row_left, col_next), xmul(row_next, col_left))));
    }
  }
  // the original symmetric matrix from its upper triangle
  const int lo = min(orow, ocol), hi = max(orow, ocol);
  const double expected = a[static_cast<long long>(lo) * lda + hi];
  diff[k] = xsub(value, expected);
  orig[k] = expected;
}

// The two sums of SampledRelativeResidual (:236-243), in sample order.
__global__ void sampled_norm_kernel(int count, const double* diff, const double* orig, double* out) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  double rs = 0.0, os = 0.0;
  for (int k = 0; k < count; ++k) {
    rs = xadd(rs, xmul(diff[k], diff[k]));
    os = xadd(os, xmul(orig[k], orig[k]));
  }
  const double on = __dsqrt_rn(os);
  out[0] = __ddiv_rn(__dsqrt_rn(rs), on < 1.0 ? 1.0 : on);  // std::max(on, 1.0)
}

}  // namespace

size_t sampled_residual_work_bytes(int n, int count) {
  return align_up(static_cast<size_t>(n) * sizeof(int), 256) + 3 * align_up(static_cast<size_t>(count) * 8, 256);
}

int sampled_residual_enqueue(int n, const double* a, long long lda, const double* f, long long ldf,
                             const int* perm, const int* pt, int count, const int* rows, const int* cols,
                             double* out, void* work, cudaStream_t s) {
  char* w = static_cast<char*>(work);
  int* inv = reinterpret_cast<int*>(w);
  BBK_CUDA_TRY(cudaMemsetAsync(inv, 0xff, static_cast<size_t>(n) * sizeof(int), s));
  w += align_up(static_cast<size_t>(n) * sizeof(int), 256);
  double* diff = reinterpret_cast<double*>(w);
  w += align_up(static_cast<size_t>(count) * 8, 256);
  double* orig = reinterpret_cast<double*>(w);
  inverse_perm_kernel<<<std::max(1, std::min(1024, (n + 255) / 256)), 256, 0, s>>>(n, perm, inv);
  BBK_CUDA_TRY(cudaGetLastError());
  sampled_entry_kernel<<<(count + 127) / 128, 128, 0, s>>>(n, a, lda, f, ldf, pt, inv, count, rows, cols,
                                                            diff, orig);
  BBK_CUDA_TRY(cudaGetLastError());
  sampled_norm_kernel<<<1, 32, 0, s>>>(count, diff, orig, out);
  BBK_CUDA_TRY(cudaGetLastError());
  count_launch(3);
  return BBK_OK;
}

}  // namespace bbk

using namespace bbk;

extern "C" int bbk_sampled_residual_device(int n, const double* a, long long lda, const double* factors,
                                           long long ldf, const int* perm, const int* pivot_types, int count,
                                           const int* rows, const int* cols, double* residual, void* stream) {
  if (n <= 0 || count <= 0) return set_error(BBK_ERR_INVALID_ARGUMENT, "matrix size and sample count must be positive");
  if (!a || !factors || !perm || !pivot_types || !rows || !cols || !residual)
    return set_error(BBK_ERR_INVALID_ARGUMENT, "null pointer");
  if (lda < n || ldf < n) return set_error(BBK_ERR_INVALID_ARGUMENT, "leading dimension smaller than n");
  int rc = check_device();
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t bytes = sampled_residual_work_bytes(n, count);
  char* work = nullptr;
  BBK_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void**>(&work), bytes, s));
  double* d_out = reinterpret_cast<double*>(work + bytes - align_up(static_cast<size_t>(count) * 8, 256));
  rc = sampled_residual_enqueue(n, a, lda, factors, ldf, perm, pivot_types, count, rows, cols, d_out, work, s);
  if (!rc) {
    cudaError_t err = cudaMemcpyAsync(residual, d_out, sizeof(double), cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if (err != cudaSuccess) rc = cuda_error(err, "sampled residual");
  }
  cudaFreeAsync(work, s);
  return rc;
}
