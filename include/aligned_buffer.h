// Drop-in for the reference's AlignedBuffer (include/aligned_buffer.h in
// wentianshu/BlockedBunchKaufmanLDLT): an owning, zero-initialised, 64-byte
// aligned array of doubles; move-only.
#ifndef NAIVE_BLOCK_LDLT_ALIGNED_BUFFER_H_
#define NAIVE_BLOCK_LDLT_ALIGNED_BUFFER_H_

#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <new>
#include <utility>

namespace naive_block_ldlt {

inline constexpr std::size_t kDefaultAlignment = 64;

class AlignedBuffer {
 public:
  AlignedBuffer() = default;
  explicit AlignedBuffer(std::size_t size) : AlignedBuffer(size, kDefaultAlignment) {}
  AlignedBuffer(std::size_t size, std::size_t alignment) : alignment_(alignment) { Reset(size); }

  AlignedBuffer(const AlignedBuffer&) = delete;
  AlignedBuffer& operator=(const AlignedBuffer&) = delete;
  AlignedBuffer(AlignedBuffer&& other) noexcept { Take(other); }
  AlignedBuffer& operator=(AlignedBuffer&& other) noexcept {
    if (this != &other) {
      Release();
      Take(other);
    }
    return *this;
  }
  ~AlignedBuffer() { Release(); }

  // Reallocates (zero-filled) when the size changes; keeps the data otherwise.
  void Resize(std::size_t size) {
    if (size != size_) {
      Release();
      Reset(size);
    }
  }
  void Fill(double value) {
    for (std::size_t i = 0; i < size_; ++i) data_[i] = value;
  }

  double* data() { return data_; }
  const double* data() const { return data_; }
  std::size_t size() const { return size_; }
  std::size_t alignment() const { return alignment_; }

 private:
  void Reset(std::size_t size) {
    size_ = size;
    data_ = nullptr;
    if (size == 0) return;
    // aligned_alloc wants a size that is a multiple of the alignment
    const std::size_t bytes = (size * sizeof(double) + alignment_ - 1) / alignment_ * alignment_;
    data_ = static_cast<double*>(std::aligned_alloc(alignment_, bytes));
    if (data_ == nullptr) {
      size_ = 0;
      throw std::bad_alloc();
    }
    std::memset(data_, 0, size * sizeof(double));
  }
  void Release() {
    std::free(data_);
    data_ = nullptr;
    size_ = 0;
  }
  void Take(AlignedBuffer& other) {
    data_ = std::exchange(other.data_, nullptr);
    size_ = std::exchange(other.size_, 0);
    alignment_ = other.alignment_;
  }

  double* data_ = nullptr;
  std::size_t size_ = 0;
  std::size_t alignment_ = kDefaultAlignment;
};

}  // namespace naive_block_ldlt

#endif  // NAIVE_BLOCK_LDLT_ALIGNED_BUFFER_H_
