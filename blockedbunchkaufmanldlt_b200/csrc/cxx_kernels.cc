// kernels::ScaleOneByOnePivot / ScaleTwoByTwoPivot / UpdateTrailingBlock
// (include/kernels.h) on host memory: each strided operand is staged to the
// GPU, the C ABI kernel runs there, the destination comes back.
#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

#include "bbk_ldlt.h"
#include "kernels.h"

namespace naive_block_ldlt::kernels {
namespace {

[[noreturn]] void Fail(const char* what) {
  throw std::runtime_error(std::string(what) + ": " + bbk_last_error());
}

void Check(cudaError_t err, const char* what) {
  if (err != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(err));
}

// Device copy of the span [p, p + (count-1)*stride] (element stride >= 0).
class DeviceSpan {
 public:
  DeviceSpan(const double* host, long long count, long long stride, bool upload)
      : host_(const_cast<double*>(host)) {
    if (stride < 0) throw std::invalid_argument("negative strides are not supported");
    elems_ = count > 0 ? (count - 1) * stride + 1 : 0;
    if (elems_ == 0) return;
    Check(cudaMalloc(reinterpret_cast<void**>(&dev_), elems_ * sizeof(double)), "cudaMalloc");
    if (upload) Check(cudaMemcpy(dev_, host_, elems_ * sizeof(double), cudaMemcpyHostToDevice), "upload");
  }
  ~DeviceSpan() { cudaFree(dev_); }
  DeviceSpan(const DeviceSpan&) = delete;
  DeviceSpan& operator=(const DeviceSpan&) = delete;
  double* get() const { return dev_; }
  void Download() {
    if (elems_ == 0) return;
    Check(cudaDeviceSynchronize(), "kernel");
    Check(cudaMemcpy(host_, dev_, elems_ * sizeof(double), cudaMemcpyDeviceToHost), "download");
  }

 private:
  double* host_;
  double* dev_ = nullptr;
  long long elems_ = 0;
};

}  // namespace

void ScaleOneByOnePivot(int count, double pivot, const double* source, int source_stride,
                        double* destination, int destination_stride) {
  if (count <= 0) return;
  DeviceSpan src(source, count, source_stride, true);
  DeviceSpan dst(destination, count, destination_stride, true);
  if (bbk_scale_one_by_one(count, pivot, src.get(), source_stride, dst.get(), destination_stride,
                           nullptr))
    Fail("ScaleOneByOnePivot");
  dst.Download();
}

void ScaleTwoByTwoPivot(int count, double pivot_top_left, double pivot_off_diagonal,
                        double pivot_bottom_right, const double* first_source,
                        int first_source_stride, const double* second_source,
                        int second_source_stride, double* first_destination,
                        int first_destination_stride, double* second_destination,
                        int second_destination_stride) {
  if (count <= 0) return;
  DeviceSpan s1(first_source, count, first_source_stride, true);
  DeviceSpan s2(second_source, count, second_source_stride, true);
  DeviceSpan d1(first_destination, count, first_destination_stride, true);
  DeviceSpan d2(second_destination, count, second_destination_stride, true);
  if (bbk_scale_two_by_two(count, pivot_top_left, pivot_off_diagonal, pivot_bottom_right, s1.get(),
                           first_source_stride, s2.get(), second_source_stride, d1.get(),
                           first_destination_stride, d2.get(), second_destination_stride, nullptr))
    Fail("ScaleTwoByTwoPivot");
  d1.Download();
  d2.Download();
}

void UpdateTrailingBlock(int rows, int cols, int inner_dim, const double* left_panel,
                         int left_panel_stride, const double* workspace_panel,
                         int workspace_panel_stride, double* target, int target_stride) {
  if (rows <= 0 || cols <= 0 || inner_dim <= 0) return;
  // row k of an operand spans stride elements; the last row ends at its width
  const long long lspan = static_cast<long long>(inner_dim - 1) * left_panel_stride + rows;
  const long long wspan = static_cast<long long>(inner_dim - 1) * workspace_panel_stride + cols;
  const long long tspan = static_cast<long long>(rows - 1) * target_stride + cols;
  DeviceSpan l(left_panel, lspan, 1, true);
  DeviceSpan w(workspace_panel, wspan, 1, true);
  DeviceSpan t(target, tspan, 1, true);
  if (bbk_update_trailing_block(rows, cols, inner_dim, l.get(), left_panel_stride, w.get(),
                                workspace_panel_stride, t.get(), target_stride,
                                BBK_UPDATE_FP64_ORDERED, nullptr))
    Fail("UpdateTrailingBlock");
  t.Download();
}

}  // namespace naive_block_ldlt::kernels
