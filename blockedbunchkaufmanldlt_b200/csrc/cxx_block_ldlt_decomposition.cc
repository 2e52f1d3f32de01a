// BlockLdltDecomposition (include/block_ldlt_decomposition.h): the
// reference's class over the C ABI.  Factorize() streams the upper blocks to
// the GPU one block row at a time through two pinned staging buffers (packing
// one block row while the previous one is copied), factors there
// (bbk_factor_device_ex), rebuilds the reference's block geometry from the
// panel ends (the same sequence of tile edits as
// ShiftBoundaryColumnToNextBlock, src/block_ldlt_decomposition.cc:589-631)
// and streams the compact factors and the workspace rows back into it the
// same way.  The factors stay on the GPU for Solve() and
// ReconstructOriginal(); in the kFull mode L and D are extracted there too
// (ExtractRegularFactorsFromCompact, :746-763).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>

#include "bbk_ldlt.h"
#include "block_ldlt_decomposition.h"

namespace naive_block_ldlt {
namespace {

// bbk_status -> the reference's exception types
[[noreturn]] void Throw(int status, const char* what) {
  const std::string msg = std::string(what) + ": " + bbk_last_error();
  switch (status) {
    case BBK_ERR_INVALID_ARGUMENT: throw std::invalid_argument(msg);
    case BBK_ERR_OUT_OF_RANGE: throw std::out_of_range(msg);
    case BBK_ERR_LOGIC: throw std::logic_error(msg);
    case BBK_ERR_ALLOC: throw std::bad_alloc();
    default: throw std::runtime_error(msg);
  }
}

void CheckCuda(cudaError_t err, const char* what) {
  if (err == cudaErrorMemoryAllocation) throw std::bad_alloc();
  if (err != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(err));
}

template <typename T>
struct DeviceArray {
  T* ptr = nullptr;
  explicit DeviceArray(size_t n) { CheckCuda(cudaMalloc(reinterpret_cast<void**>(&ptr), n * sizeof(T)), "cudaMalloc"); }
  ~DeviceArray() { cudaFree(ptr); }
  T* release() {
    T* p = ptr;
    ptr = nullptr;
    return p;
  }
  DeviceArray(const DeviceArray&) = delete;
  DeviceArray& operator=(const DeviceArray&) = delete;
};

struct Stream {
  cudaStream_t s = nullptr;
  Stream() { CheckCuda(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate"); }
  ~Stream() {
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
  }
  Stream(const Stream&) = delete;
  Stream& operator=(const Stream&) = delete;
};

// Two pinned buffers of one block row each, and the events that say when
// the copy out of (or into) each is done.
struct PinnedPair {
  double* buf[2] = {nullptr, nullptr};
  cudaEvent_t done[2] = {nullptr, nullptr};
  bool used[2] = {false, false};
  explicit PinnedPair(size_t elems) {
    for (int k = 0; k < 2; ++k) {
      CheckCuda(cudaMallocHost(reinterpret_cast<void**>(&buf[k]), elems * sizeof(double)), "cudaMallocHost");
      CheckCuda(cudaEventCreateWithFlags(&done[k], cudaEventDisableTiming), "cudaEventCreate");
    }
  }
  ~PinnedPair() {
    for (int k = 0; k < 2; ++k) {
      if (done[k]) {
        cudaEventSynchronize(done[k]);
        cudaEventDestroy(done[k]);
      }
      cudaFreeHost(buf[k]);
    }
  }
  // buffer k, once the copy that last used it has finished
  double* take(int k) {
    if (used[k]) CheckCuda(cudaEventSynchronize(done[k]), "staging copy");
    used[k] = true;
    return buf[k];
  }
  PinnedPair(const PinnedPair&) = delete;
  PinnedPair& operator=(const PinnedPair&) = delete;
};

// Rows of the tallest block row of `m` (the staging buffers hold one block
// row of the upper triangle: rows x (n - row0) doubles).
int MaxBlockRows(const BlockMatrix& m) {
  int h = 0;
  for (int br = 0; br < m.num_blocks(); ++br) h = std::max(h, m.GetBlock(br, br).rows());
  return h;
}

// Upper blocks of `m` -> the device's dense row-major upper triangle (ld n),
// one block row (rows [row0, row0 + h), columns [row0, n)) per copy.
void UploadUpper(const BlockMatrix& m, double* dev, cudaStream_t s) {
  const int n = m.Rows(), nb = m.num_blocks();
  PinnedPair stage(static_cast<size_t>(std::max(1, MaxBlockRows(m))) * n);
  for (int br = 0; br < nb; ++br) {
    const Block& diag = m.GetBlock(br, br);
    const int r0 = diag.row0(), h = diag.rows(), width = n - r0;
    if (h <= 0) continue;
    double* st = stage.take(br & 1);
    for (int bc = br; bc < nb; ++bc) {
      const Block& blk = m.GetBlock(br, bc);
      for (int r = 0; r < blk.rows(); ++r)
        std::memcpy(st + static_cast<size_t>(r) * width + (blk.col0() - r0), &blk(r, 0),
                    static_cast<size_t>(blk.cols()) * sizeof(double));
    }
    const size_t pitch = static_cast<size_t>(width) * sizeof(double);
    CheckCuda(cudaMemcpy2DAsync(dev + static_cast<size_t>(r0) * n + r0, static_cast<size_t>(n) * sizeof(double),
                                st, pitch, pitch, h, cudaMemcpyHostToDevice, s),
              "upload");
    CheckCuda(cudaEventRecord(stage.done[br & 1], s), "cudaEventRecord");
  }
  CheckCuda(cudaStreamSynchronize(s), "upload");
}

// The device's dense upper triangle -> the upper blocks of `m` (its
// geometry already final); entries below the diagonal of diagonal blocks
// are set to zero.  The copy of block row br + 1 runs while br is unpacked.
void DownloadUpper(const double* dev, BlockMatrix* m, cudaStream_t s) {
  const int n = m->Rows(), nb = m->num_blocks();
  PinnedPair stage(static_cast<size_t>(std::max(1, MaxBlockRows(*m))) * n);
  auto issue = [&](int br) {
    const Block& diag = m->GetBlock(br, br);
    const int r0 = diag.row0(), h = diag.rows(), width = n - r0;
    if (h <= 0) return;
    double* st = stage.take(br & 1);
    const size_t pitch = static_cast<size_t>(width) * sizeof(double);
    CheckCuda(cudaMemcpy2DAsync(st, pitch, dev + static_cast<size_t>(r0) * n + r0,
                                static_cast<size_t>(n) * sizeof(double), pitch, h, cudaMemcpyDeviceToHost, s),
              "download");
    CheckCuda(cudaEventRecord(stage.done[br & 1], s), "cudaEventRecord");
  };
  if (nb > 0) issue(0);
  for (int br = 0; br < nb; ++br) {
    const Block& diag = m->GetBlock(br, br);
    const int r0 = diag.row0(), h = diag.rows(), width = n - r0;
    if (h > 0) CheckCuda(cudaEventSynchronize(stage.done[br & 1]), "download");
    const double* st = stage.buf[br & 1];
    // the other buffer is free: block row br - 1 was unpacked already
    if (br + 1 < nb) issue(br + 1);
    if (h <= 0) continue;
    for (int bc = br; bc < nb; ++bc) {
      Block& blk = m->GetBlock(br, bc);
      for (int r = 0; r < blk.rows(); ++r) {
        const int gi = r0 + r;
        for (int c = 0; c < blk.cols(); ++c) {
          const int gj = blk.col0() + c;
          blk(r, c) = gi <= gj ? st[static_cast<size_t>(r) * width + (gj - r0)] : 0.0;
        }
      }
    }
  }
}

}  // namespace

struct BlockLdltDecomposition::DeviceFactors {
  int n = 0;
  double* a = nullptr;  // n x n row-major, compact factors in the upper triangle
  int* perm = nullptr;
  int* pt = nullptr;
  ~DeviceFactors() {
    cudaFree(a);
    cudaFree(perm);
    cudaFree(pt);
  }
};

BlockLdltDecomposition::BlockLdltDecomposition(const BlockMatrix& matrix, FactorizationMode mode)
    : original_(mode == FactorizationMode::kFull ? matrix.ToRegular() : RegularMatrix()),
      factors_(matrix),
      workspace_(matrix.Rows(), matrix.block_size()),
      l_factor_(mode == FactorizationMode::kFull ? RegularMatrix::Identity(matrix.Rows())
                                                 : RegularMatrix()),
      d_factor_(mode == FactorizationMode::kFull ? RegularMatrix(matrix.Rows(), matrix.Rows())
                                                 : RegularMatrix()),
      permutation_(matrix.Rows()),
      pivot_types_(matrix.Rows(), 0),
      mode_(mode) {
  for (int i = 0; i < matrix.Rows(); ++i) permutation_[i] = i;
}

void BlockLdltDecomposition::RebuildGeometry(BlockMatrix* m, const std::vector<int>& panel_end) const {
  const int n = factors_.Rows(), b = factors_.block_size();
  *m = BlockMatrix(n, b);
  const int nb = m->num_blocks();
  for (int panel = 0; panel + 1 < nb; ++panel) {
    const int nominal = std::min((panel + 1) * b, n);
    if (panel_end[panel] >= nominal) continue;
    const int next = panel + 1;
    for (int bc = next; bc < nb; ++bc) m->ExpandBlock(next, bc);
    m->AddColumnLeft(panel, next);
    for (int bc = next; bc < nb; ++bc) m->ShrinkBlock(panel, bc);
    m->ShrinkBlock(panel, panel);
  }
}

void BlockLdltDecomposition::Factorize() {
  const int n = factors_.Rows(), b = factors_.block_size();
  const int nb = factors_.num_blocks();
  const size_t nn = static_cast<size_t>(n) * n;
  Stream stream;
  DeviceArray<double> a(nn), w(nn);
  DeviceArray<int> perm(n), pt(n), pe(nb), status(1);
  CheckCuda(cudaMemsetAsync(w.ptr, 0, nn * sizeof(double), stream.s), "cudaMemset");
  UploadUpper(factors_, a.ptr, stream.s);
  bbk_factor_extras extras{};
  extras.workspace_rows = w.ptr;  // the W rows Workspace() returns
  extras.workspace_ld = n;
  int rc = bbk_factor_device_ex(n, b, a.ptr, n, perm.ptr, pt.ptr, pe.ptr, update_mode_, &extras, nullptr, 0,
                                status.ptr, stream.s);
  if (rc != BBK_OK) Throw(rc, "Factorize");
  std::vector<int> panel_end(nb, 0);
  int h_status = BBK_OK;
  CheckCuda(cudaMemcpyAsync(permutation_.data(), perm.ptr, n * sizeof(int), cudaMemcpyDeviceToHost, stream.s),
            "download");
  CheckCuda(cudaMemcpyAsync(pivot_types_.data(), pt.ptr, n * sizeof(int), cudaMemcpyDeviceToHost, stream.s),
            "download");
  CheckCuda(cudaMemcpyAsync(panel_end.data(), pe.ptr, nb * sizeof(int), cudaMemcpyDeviceToHost, stream.s),
            "download");
  CheckCuda(cudaMemcpyAsync(&h_status, status.ptr, sizeof(int), cudaMemcpyDeviceToHost, stream.s), "download");
  CheckCuda(cudaStreamSynchronize(stream.s), "Factorize");
  if (h_status != BBK_OK) Throw(h_status, "Factorize");

  RebuildGeometry(&factors_, panel_end);
  RebuildGeometry(&workspace_, panel_end);
  DownloadUpper(a.ptr, &factors_, stream.s);
  DownloadUpper(w.ptr, &workspace_, stream.s);

  if (mode_ == FactorizationMode::kFull) {
    // ExtractRegularFactorsFromCompact (src/block_ldlt_decomposition.cc:746-763)
    rc = bbk_extract_ld_device(n, a.ptr, n, pt.ptr, w.ptr, n, nullptr, 0, stream.s);
    if (rc != BBK_OK) Throw(rc, "Factorize");
    CheckCuda(cudaMemcpy(l_factor_.Data(), w.ptr, nn * sizeof(double), cudaMemcpyDeviceToHost), "download");
    rc = bbk_extract_ld_device(n, a.ptr, n, pt.ptr, nullptr, 0, w.ptr, n, stream.s);
    if (rc != BBK_OK) Throw(rc, "Factorize");
    CheckCuda(cudaMemcpy(d_factor_.Data(), w.ptr, nn * sizeof(double), cudaMemcpyDeviceToHost), "download");
  }
  auto dev = std::make_shared<DeviceFactors>();
  dev->n = n;
  dev->a = a.release();
  dev->perm = perm.release();
  dev->pt = pt.release();
  device_ = std::move(dev);
  factorized_ = true;
}

RegularMatrix BlockLdltDecomposition::ReconstructOriginal() const {
  if (mode_ != FactorizationMode::kFull)
    throw std::logic_error("ReconstructOriginal() requires full factor storage");
  if (!factorized_) throw std::logic_error("Factorize() must be called before ReconstructOriginal()");
  const int n = factors_.Rows();
  const size_t nn = static_cast<size_t>(n) * n;
  DeviceArray<double> out(nn);
  const int rc = bbk_reconstruct_device(n, device_->a, n, device_->perm, device_->pt, out.ptr, n, nullptr);
  if (rc != BBK_OK) Throw(rc, "ReconstructOriginal");
  RegularMatrix result(n, n);
  CheckCuda(cudaMemcpy(result.Data(), out.ptr, nn * sizeof(double), cudaMemcpyDeviceToHost), "download");
  return result;
}

std::vector<double> BlockLdltDecomposition::Solve(const std::vector<double>& b, int nrhs) const {
  if (!factorized_) throw std::logic_error("Factorize() must be called before Solve()");
  const int n = factors_.Rows();
  if (nrhs < 0 || b.size() != static_cast<size_t>(n) * nrhs)
    throw std::invalid_argument("right-hand side size does not match");
  std::vector<double> x(b);
  if (nrhs == 0) return x;
  DeviceArray<double> db(x.size());
  CheckCuda(cudaMemcpy(db.ptr, x.data(), x.size() * sizeof(double), cudaMemcpyHostToDevice), "upload");
  const int rc = bbk_solve_device(n, device_->a, n, device_->perm, device_->pt, nrhs, db.ptr, n, nullptr, 0,
                                  nullptr);
  if (rc != BBK_OK) Throw(rc, "Solve");
  CheckCuda(cudaMemcpy(x.data(), db.ptr, x.size() * sizeof(double), cudaMemcpyDeviceToHost), "download");
  return x;
}

}  // namespace naive_block_ldlt
