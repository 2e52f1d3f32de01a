// RegularMatrix and its helpers (include/regular_matrix.h): host utilities
// with the reference's semantics (src/regular_matrix.cc in
// wentianshu/BlockedBunchKaufmanLDLT); used to check results, never by the
// factorization itself.
#include <cmath>
#include <stdexcept>

#include "regular_matrix.h"

namespace naive_block_ldlt {
namespace {
size_t Elements(int rows, int cols) {
  if (rows < 0 || cols < 0) throw std::invalid_argument("matrix shape must be nonnegative");
  return static_cast<size_t>(rows) * static_cast<size_t>(cols);
}
}  // namespace

RegularMatrix::RegularMatrix(int rows, int cols)
    : rows_(rows), cols_(cols), leading_dimension_(cols), data_(Elements(rows, cols)) {}

RegularMatrix::RegularMatrix(int rows, int cols, const std::vector<double>& values)
    : RegularMatrix(rows, cols) {
  if (values.size() != static_cast<size_t>(rows) * cols)
    throw std::invalid_argument("value count does not match matrix shape");
  for (size_t i = 0; i < values.size(); ++i) data_.data()[i] = values[i];
}

RegularMatrix::RegularMatrix(const RegularMatrix& other) : RegularMatrix(other.rows_, other.cols_) {
  for (size_t i = 0; i < other.data_.size(); ++i) data_.data()[i] = other.data_.data()[i];
}

RegularMatrix& RegularMatrix::operator=(const RegularMatrix& other) {
  if (this == &other) return *this;
  rows_ = other.rows_;
  cols_ = other.cols_;
  leading_dimension_ = other.leading_dimension_;
  data_.Resize(other.data_.size());
  for (size_t i = 0; i < other.data_.size(); ++i) data_.data()[i] = other.data_.data()[i];
  return *this;
}

double& RegularMatrix::operator()(int row, int col) { return data_.data()[row * leading_dimension_ + col]; }

const double& RegularMatrix::operator()(int row, int col) const {
  return data_.data()[row * leading_dimension_ + col];
}

void RegularMatrix::Fill(double value) { data_.Fill(value); }

RegularMatrix RegularMatrix::Identity(int size) {
  RegularMatrix id(size, size);
  for (int i = 0; i < size; ++i) id(i, i) = 1.0;
  return id;
}

double FrobeniusNorm(const RegularMatrix& m) {
  double sum = 0.0;
  for (int i = 0; i < m.Rows(); ++i)
    for (int j = 0; j < m.Cols(); ++j) sum += m(i, j) * m(i, j);
  return std::sqrt(sum);
}

RegularMatrix Multiply(const RegularMatrix& left, const RegularMatrix& right) {
  if (left.Cols() != right.Rows()) throw std::invalid_argument("incompatible matrix multiplication shapes");
  RegularMatrix out(left.Rows(), right.Cols());
  for (int i = 0; i < left.Rows(); ++i)
    for (int k = 0; k < left.Cols(); ++k) {
      const double a = left(i, k);
      for (int j = 0; j < right.Cols(); ++j) out(i, j) += a * right(k, j);
    }
  return out;
}

RegularMatrix Transpose(const RegularMatrix& m) {
  RegularMatrix out(m.Cols(), m.Rows());
  for (int i = 0; i < m.Rows(); ++i)
    for (int j = 0; j < m.Cols(); ++j) out(j, i) = m(i, j);
  return out;
}

RegularMatrix Subtract(const RegularMatrix& left, const RegularMatrix& right) {
  if (left.Rows() != right.Rows() || left.Cols() != right.Cols())
    throw std::invalid_argument("incompatible matrix subtraction shapes");
  RegularMatrix out(left.Rows(), left.Cols());
  for (int i = 0; i < left.Rows(); ++i)
    for (int j = 0; j < left.Cols(); ++j) out(i, j) = left(i, j) - right(i, j);
  return out;
}

}  // namespace naive_block_ldlt
