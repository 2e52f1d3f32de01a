// BlockLdltDecomposition (include/block_ldlt_decomposition.h): the
// reference's class over the C ABI.  Factorize() packs the upper blocks into
// the dense row-major form, factors on the GPU (bbk_factor_host), rebuilds the
// reference's block geometry from the panel ends (the same sequence of tile
// edits as ShiftBoundaryColumnToNextBlock, src/block_ldlt_decomposition.cc:
// 589-631) and unpacks the compact factors into it.
#include <cuda_runtime.h>

#include <algorithm>
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
  if (err != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(err));
}

template <typename T>
struct DeviceArray {
  T* ptr = nullptr;
  explicit DeviceArray(size_t n) { CheckCuda(cudaMalloc(reinterpret_cast<void**>(&ptr), n * sizeof(T)), "cudaMalloc"); }
  ~DeviceArray() { cudaFree(ptr); }
  DeviceArray(const DeviceArray&) = delete;
  DeviceArray& operator=(const DeviceArray&) = delete;
};

}  // namespace

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
  dense_.assign(static_cast<size_t>(n) * n, 0.0);
  for (int bc = 0; bc < nb; ++bc)
    for (int br = 0; br <= bc; ++br) {
      const Block& blk = factors_.GetBlock(br, bc);
      for (int r = 0; r < blk.rows(); ++r)
        for (int c = 0; c < blk.cols(); ++c) {
          const int gi = blk.row0() + r, gj = blk.col0() + c;
          if (gi >= 0 && gj < n && gi <= gj) dense_[static_cast<size_t>(gi) * n + gj] = blk(r, c);
        }
    }
  std::vector<int> panel_end(nb, 0);
  const int rc = bbk_factor_host(n, b, dense_.data(), n, permutation_.data(), pivot_types_.data(),
                                 panel_end.data(), update_mode_);
  if (rc != BBK_OK) Throw(rc, "Factorize");

  RebuildGeometry(&factors_, panel_end);
  RebuildGeometry(&workspace_, panel_end);
  for (int bc = 0; bc < nb; ++bc)
    for (int br = 0; br <= bc; ++br) {
      Block& blk = factors_.GetBlock(br, bc);
      for (int r = 0; r < blk.rows(); ++r)
        for (int c = 0; c < blk.cols(); ++c) {
          const int gi = blk.row0() + r, gj = blk.col0() + c;
          blk(r, c) = (gi <= gj) ? dense_[static_cast<size_t>(gi) * n + gj] : 0.0;
        }
    }

  if (mode_ == FactorizationMode::kFull) {
    // ExtractRegularFactorsFromCompact (src/block_ldlt_decomposition.cc:746-763)
    l_factor_.Fill(0.0);
    d_factor_.Fill(0.0);
    for (int row = 0; row < n; ++row) {
      l_factor_(row, row) = 1.0;
      d_factor_(row, row) = dense_[static_cast<size_t>(row) * n + row];
      for (int col = row + 1; col < n; ++col) {
        const double v = dense_[static_cast<size_t>(row) * n + col];
        if (col == row + 1 && pivot_types_[row] == 2) {
          d_factor_(row, col) = v;
          d_factor_(col, row) = v;
        } else {
          l_factor_(col, row) = v;
        }
      }
    }
  }
  factorized_ = true;
}

RegularMatrix BlockLdltDecomposition::ReconstructOriginal() const {
  if (mode_ != FactorizationMode::kFull)
    throw std::logic_error("ReconstructOriginal() requires full factor storage");
  if (!factorized_) throw std::logic_error("Factorize() must be called before ReconstructOriginal()");
  const int n = factors_.Rows();
  const size_t nn = static_cast<size_t>(n) * n;
  DeviceArray<double> f(nn), out(nn);
  DeviceArray<int> perm(n), pt(n);
  CheckCuda(cudaMemcpy(f.ptr, dense_.data(), nn * sizeof(double), cudaMemcpyHostToDevice), "upload");
  CheckCuda(cudaMemcpy(perm.ptr, permutation_.data(), n * sizeof(int), cudaMemcpyHostToDevice), "upload");
  CheckCuda(cudaMemcpy(pt.ptr, pivot_types_.data(), n * sizeof(int), cudaMemcpyHostToDevice), "upload");
  const int rc = bbk_reconstruct_device(n, f.ptr, n, perm.ptr, pt.ptr, out.ptr, n, nullptr);
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
  const int rc = bbk_solve_host(n, dense_.data(), n, permutation_.data(), pivot_types_.data(), nrhs,
                                x.data(), n);
  if (rc != BBK_OK) Throw(rc, "Solve");
  return x;
}

}  // namespace naive_block_ldlt
