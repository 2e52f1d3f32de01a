// Drop-in for the reference's BlockLdltDecomposition
// (include/block_ldlt_decomposition.h): P A P^T = L D L^T by blocked
// Bunch-Kaufman pivoting, with the same compact factor layout, permutation,
// pivot types and block geometry.  Factorize() runs on the GPU through the C
// ABI of bbk_ldlt.h; the public interface is the reference's, plus
// SetUpdateMode() and Solve(), which the reference does not have.
#ifndef NAIVE_BLOCK_LDLT_BLOCK_LDLT_DECOMPOSITION_H_
#define NAIVE_BLOCK_LDLT_BLOCK_LDLT_DECOMPOSITION_H_

#include <memory>
#include <vector>

#include "block_matrix.h"
#include "regular_matrix.h"

namespace naive_block_ldlt {

class BlockLdltDecomposition {
 public:
  enum class FactorizationMode {
    kFull,
    kCompactOnly,
  };

  explicit BlockLdltDecomposition(const BlockMatrix& matrix,
                                  FactorizationMode mode = FactorizationMode::kFull);

  void Factorize();
  RegularMatrix ReconstructOriginal() const;

  const RegularMatrix& LFactor() const { return l_factor_; }
  const RegularMatrix& DFactor() const { return d_factor_; }
  const BlockMatrix& CompactFactors() const { return factors_; }
  // Same geometry as CompactFactors().  Outside the diagonal blocks it holds,
  // like the reference's, each panel's workspace rows W = D U (the unscaled
  // updated pivot rows the trailing update reads) in the column order at the
  // panel's end; the diagonal blocks, where the reference also keeps
  // intermediate candidate copies, read as zero.
  const BlockMatrix& Workspace() const { return workspace_; }
  const std::vector<int>& Permutation() const { return permutation_; }
  const std::vector<int>& PivotTypes() const { return pivot_types_; }

  // Extensions.  Trailing-update arithmetic (a bbk_update_mode): the default
  // BBK_UPDATE_FP64 uses FP64 tensor cores; BBK_UPDATE_FP64_ORDERED
  // reproduces the reference bit for bit.
  void SetUpdateMode(int update_mode) { update_mode_ = update_mode; }
  // Solves A x = b for nrhs right-hand sides stored one after another (each
  // of length Rows()); after Factorize().
  std::vector<double> Solve(const std::vector<double>& b, int nrhs = 1) const;

 private:
  struct DeviceFactors;  // the compact factors, permutation and pivot types on the GPU
  void RebuildGeometry(BlockMatrix* matrix, const std::vector<int>& panel_end) const;

  RegularMatrix original_;
  BlockMatrix factors_;
  BlockMatrix workspace_;
  RegularMatrix l_factor_;
  RegularMatrix d_factor_;
  std::vector<int> permutation_;
  std::vector<int> pivot_types_;
  // after Factorize(): the device copy Solve() and ReconstructOriginal() use
  // (shared by copies of this object; never modified after Factorize())
  std::shared_ptr<const DeviceFactors> device_;
  FactorizationMode mode_ = FactorizationMode::kFull;
  int update_mode_ = 0;
  bool factorized_ = false;
};

}  // namespace naive_block_ldlt

#endif  // NAIVE_BLOCK_LDLT_BLOCK_LDLT_DECOMPOSITION_H_
