// Drop-in for the reference's BlockMatrix (include/block_matrix.h): a
// symmetric matrix stored as its upper blocks (block_row <= block_col), each
// tile row-major in its own 64-byte aligned buffer with one row/column of
// slack (for every block but the first row/column) so a panel boundary can
// move by one column, exactly the geometry rules of the reference
// (src/block_matrix.cc:209-231).  Element access finds the owning tile by
// binary search instead of the reference's scan over all tiles.
#ifndef NAIVE_BLOCK_LDLT_BLOCK_MATRIX_H_
#define NAIVE_BLOCK_LDLT_BLOCK_MATRIX_H_

#include <vector>

#include "aligned_buffer.h"
#include "block.h"
#include "matrix.h"
#include "regular_matrix.h"

namespace naive_block_ldlt {

struct BlockColumnLocation {
  int block_row = 0;
  int block_col = 0;
  int local_col = 0;
};

enum class MatrixTriangle {
  kUpper,
  kLower,
};

class BlockMatrix : public Matrix {
 public:
  BlockMatrix() = default;
  BlockMatrix(int size, int block_size);
  BlockMatrix(const RegularMatrix& matrix, int block_size,
              MatrixTriangle input_triangle = MatrixTriangle::kUpper);
  BlockMatrix(const BlockMatrix& other);
  BlockMatrix& operator=(const BlockMatrix& other);
  BlockMatrix(BlockMatrix&& other) noexcept = default;
  BlockMatrix& operator=(BlockMatrix&& other) noexcept = default;

  int Rows() const override { return size_; }
  int Cols() const override { return size_; }
  int block_size() const { return block_size_; }
  int num_blocks() const { return num_blocks_; }

  // Symmetric access: (row, col) with row > col reads (col, row).
  double& operator()(int row, int col) override;
  const double& operator()(int row, int col) const override;

  int BlockId(int block_row, int block_col) const;
  Block& GetBlock(int block_row, int block_col);
  const Block& GetBlock(int block_row, int block_col) const;
  BlockColumnLocation GlobalColumnToBlockColumn(int block_row, int preferred_block_col,
                                                int column) const;

  RegularMatrix ToRegular() const;
  RegularMatrix ToUpperRegular() const;

  // Geometry edits used when a panel boundary moves (the reference's
  // ShiftBoundaryColumnToNextBlock): grow a tile by one row at the top (and,
  // on the diagonal, col_size columns at the left), shrink it by its last
  // row (and column on the diagonal), or add columns at its left.
  void ExpandBlock(int block_row, int block_col, int col_size = 1);
  void ShrinkBlock(int block_row, int block_col);
  void AddColumnLeft(int block_row, int block_col, int col_size = 1);

 private:
  void AllocateBlocks();
  Block* Locate(int row, int col);
  void Reshape(int block_row, int block_col, int rows, int cols, int row_shift, int col_shift,
               int row0, int col0);

  int size_ = 0;
  int block_size_ = 0;
  int num_blocks_ = 0;
  std::vector<AlignedBuffer> storage_;
  std::vector<Block> blocks_;        // indexed by BlockId
  std::vector<int> row_capacity_;
  std::vector<int> col_capacity_;
};

}  // namespace naive_block_ldlt

#endif  // NAIVE_BLOCK_LDLT_BLOCK_MATRIX_H_
