// BlockMatrix (include/block_matrix.h): the reference's upper-block storage
// and its geometry rules (src/block_matrix.cc in
// wentianshu/BlockedBunchKaufmanLDLT), host side.
#include <algorithm>
#include <stdexcept>
#include <vector>

#include "block_matrix.h"

namespace naive_block_ldlt {

BlockMatrix::BlockMatrix(int size, int block_size) : size_(size), block_size_(block_size) {
  if (size <= 0) throw std::invalid_argument("matrix size must be positive");
  if (block_size <= 0) throw std::invalid_argument("block size must be positive");
  num_blocks_ = (size + block_size - 1) / block_size;
  AllocateBlocks();
}

BlockMatrix::BlockMatrix(const RegularMatrix& matrix, int block_size, MatrixTriangle input_triangle)
    : BlockMatrix(matrix.Rows(), block_size) {
  if (matrix.Rows() != matrix.Cols()) throw std::invalid_argument("block matrix input must be square");
  // only the chosen triangle is read
  const bool upper = input_triangle == MatrixTriangle::kUpper;
  for (Block& blk : blocks_) {
    for (int r = 0; r < blk.rows(); ++r) {
      const int gi = blk.row0() + r;
      for (int c = 0; c < blk.cols(); ++c) {
        const int gj = blk.col0() + c;
        if (gi <= gj) blk(r, c) = upper ? matrix(gi, gj) : matrix(gj, gi);
      }
    }
  }
}

BlockMatrix::BlockMatrix(const BlockMatrix& other)
    : size_(other.size_),
      block_size_(other.block_size_),
      num_blocks_(other.num_blocks_),
      row_capacity_(other.row_capacity_),
      col_capacity_(other.col_capacity_) {
  storage_.reserve(other.storage_.size());
  blocks_.reserve(other.blocks_.size());
  for (size_t id = 0; id < other.blocks_.size(); ++id) {
    const AlignedBuffer& src = other.storage_[id];
    storage_.emplace_back(src.size());
    std::copy(src.data(), src.data() + src.size(), storage_.back().data());
    const Block& b = other.blocks_[id];
    blocks_.emplace_back(storage_.back().data(), b.rows(), b.cols(), b.leading_dimension(), b.row0(),
                         b.col0(), b.block_row(), b.block_col());
  }
}

BlockMatrix& BlockMatrix::operator=(const BlockMatrix& other) {
  if (this != &other) {
    BlockMatrix copy(other);
    *this = std::move(copy);
  }
  return *this;
}

void BlockMatrix::AllocateBlocks() {
  const int count = num_blocks_ * (num_blocks_ + 1) / 2;
  storage_.clear();
  blocks_.clear();
  storage_.reserve(count);
  blocks_.reserve(count);
  row_capacity_.assign(count, 0);
  col_capacity_.assign(count, 0);
  // BlockId order: block_col major, block_row minor (id = br + bc(bc+1)/2)
  for (int bc = 0; bc < num_blocks_; ++bc) {
    const int c0 = bc * block_size_;
    const int cols = std::min(block_size_, size_ - c0);
    const int ccap = cols + (bc > 0 ? 1 : 0);
    for (int br = 0; br <= bc; ++br) {
      const int r0 = br * block_size_;
      const int rows = std::min(block_size_, size_ - r0);
      const int rcap = rows + (br > 0 ? 1 : 0);
      const int id = BlockId(br, bc);
      row_capacity_[id] = rcap;
      col_capacity_[id] = ccap;
      storage_.emplace_back(static_cast<size_t>(rcap) * ccap);
      blocks_.emplace_back(storage_.back().data(), rows, cols, ccap, r0, c0, br, bc);
    }
  }
}

int BlockMatrix::BlockId(int block_row, int block_col) const {
  if (block_row > block_col) std::swap(block_row, block_col);
  return block_row + block_col * (block_col + 1) / 2;
}

Block& BlockMatrix::GetBlock(int block_row, int block_col) { return blocks_.at(BlockId(block_row, block_col)); }

const Block& BlockMatrix::GetBlock(int block_row, int block_col) const {
  return blocks_.at(BlockId(block_row, block_col));
}

namespace {
bool Contains(const Block& b, int row, int col) {
  return b.row0() <= row && row < b.row0() + b.rows() && b.col0() <= col && col < b.col0() + b.cols();
}
}  // namespace

// The tile that holds (row, col), row <= col.  With consistent geometry every
// block row spans one row range and its tiles partition the columns from the
// diagonal on, so two binary searches find it; any other state falls back
// to the first containing tile in storage order.
Block* BlockMatrix::Locate(int row, int col) {
  if (row < 0 || col < 0 || row >= size_ || col >= size_ || blocks_.empty()) return nullptr;
  int lo = 0, hi = num_blocks_ - 1;
  while (lo < hi) {  // last diagonal tile with row0 <= row
    const int mid = (lo + hi + 1) / 2;
    if (blocks_[BlockId(mid, mid)].row0() <= row) lo = mid; else hi = mid - 1;
  }
  const int br = lo;
  int clo = br, chi = num_blocks_ - 1;
  while (clo < chi) {  // last tile of the block row with col0 <= col
    const int mid = (clo + chi + 1) / 2;
    if (blocks_[BlockId(br, mid)].col0() <= col) clo = mid; else chi = mid - 1;
  }
  Block& cand = blocks_[BlockId(br, clo)];
  if (Contains(cand, row, col)) return &cand;
  for (Block& b : blocks_)
    if (Contains(b, row, col)) return &b;
  return nullptr;
}

double& BlockMatrix::operator()(int row, int col) {
  if (row > col) std::swap(row, col);
  Block* b = Locate(row, col);
  if (b == nullptr) throw std::out_of_range("matrix index is outside active block views");
  return (*b)(row - b->row0(), col - b->col0());
}

const double& BlockMatrix::operator()(int row, int col) const {
  return const_cast<BlockMatrix*>(this)->operator()(row, col);
}

BlockColumnLocation BlockMatrix::GlobalColumnToBlockColumn(int block_row, int preferred_block_col,
                                                           int column) const {
  auto holds = [&](int bc) {
    const Block& b = GetBlock(block_row, bc);
    return b.col0() <= column && column < b.col0() + b.cols();
  };
  if (holds(preferred_block_col))
    return {block_row, preferred_block_col, column - GetBlock(block_row, preferred_block_col).col0()};
  for (int bc = preferred_block_col - 1; bc >= 0; --bc)
    if (holds(bc)) return {block_row, bc, column - GetBlock(block_row, bc).col0()};
  for (int bc = preferred_block_col + 1; bc < num_blocks_; ++bc)
    if (holds(bc)) return {block_row, bc, column - GetBlock(block_row, bc).col0()};
  throw std::out_of_range("global column is outside active block row");
}

RegularMatrix BlockMatrix::ToRegular() const {
  RegularMatrix out(size_, size_);
  for (const Block& b : blocks_)
    for (int r = 0; r < b.rows(); ++r)
      for (int c = 0; c < b.cols(); ++c) {
        const int gi = b.row0() + r, gj = b.col0() + c;
        if (gi < 0 || gj < 0 || gi >= size_ || gj >= size_ || gi > gj) continue;
        out(gi, gj) = b(r, c);
        out(gj, gi) = b(r, c);
      }
  return out;
}

RegularMatrix BlockMatrix::ToUpperRegular() const {
  RegularMatrix out(size_, size_);
  for (const Block& b : blocks_)
    for (int r = 0; r < b.rows(); ++r)
      for (int c = 0; c < b.cols(); ++c) {
        const int gi = b.row0() + r, gj = b.col0() + c;
        if (gi < 0 || gj < 0 || gi >= size_ || gj >= size_ || gi > gj) continue;
        out(gi, gj) = b(r, c);
      }
  return out;
}

// New tile (rows x cols at (row0, col0)): cell (i, j) takes the old cell
// (i - row_shift, j - col_shift), zero where that falls outside the old tile.
void BlockMatrix::Reshape(int block_row, int block_col, int rows, int cols, int row_shift,
                          int col_shift, int row0, int col0) {
  const int id = BlockId(block_row, block_col);
  if (rows < 0 || cols < 0) throw std::invalid_argument("block dimensions must be non-negative");
  if (rows > row_capacity_.at(id) || cols > col_capacity_.at(id))
    throw std::logic_error("block resize exceeds preallocated capacity");
  Block& b = blocks_.at(id);
  const int old_rows = b.rows(), old_cols = b.cols(), ld = col_capacity_[id];
  std::vector<double> old(static_cast<size_t>(old_rows) * old_cols);
  for (int i = 0; i < old_rows; ++i)
    for (int j = 0; j < old_cols; ++j) old[static_cast<size_t>(i) * old_cols + j] = b(i, j);
  double* data = storage_[id].data();
  for (int i = 0; i < rows; ++i) {
    const int oi = i - row_shift;
    for (int j = 0; j < cols; ++j) {
      const int oj = j - col_shift;
      const bool inside = oi >= 0 && oi < old_rows && oj >= 0 && oj < old_cols;
      data[static_cast<size_t>(i) * ld + j] = inside ? old[static_cast<size_t>(oi) * old_cols + oj] : 0.0;
    }
  }
  b.Reset(data, rows, cols, ld, row0, col0, block_row, block_col);
}

void BlockMatrix::ExpandBlock(int block_row, int block_col, int col_size) {
  const Block& b = GetBlock(block_row, block_col);
  if (block_row == block_col) {
    // the reference passes (row shift, column shift) = (col_size, 1) here
    Reshape(block_row, block_col, b.rows() + 1, b.cols() + col_size, col_size, 1, b.row0() - 1,
            b.col0() - col_size);
  } else {
    Reshape(block_row, block_col, b.rows() + 1, b.cols(), 1, 0, b.row0() - 1, b.col0());
  }
}

void BlockMatrix::ShrinkBlock(int block_row, int block_col) {
  const Block& b = GetBlock(block_row, block_col);
  if (block_row == block_col) {
    if (b.rows() == 0 || b.cols() == 0) return;
    Reshape(block_row, block_col, b.rows() - 1, b.cols() - 1, 0, 0, b.row0(), b.col0());
  } else {
    if (b.rows() == 0) return;
    Reshape(block_row, block_col, b.rows() - 1, b.cols(), 0, 0, b.row0(), b.col0());
  }
}

void BlockMatrix::AddColumnLeft(int block_row, int block_col, int col_size) {
  const Block& b = GetBlock(block_row, block_col);
  Reshape(block_row, block_col, b.rows(), b.cols() + col_size, 0, col_size, b.row0(),
          b.col0() - col_size);
}

}  // namespace naive_block_ldlt
