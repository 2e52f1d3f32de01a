// Drop-in for the reference's kernel boundary (include/kernels.h): the same
// three functions on host memory.  Each runs on the GPU through the C ABI
// (bbk_scale_one_by_one, bbk_scale_two_by_two, bbk_update_trailing_block);
// UpdateTrailingBlock uses the reference's summation order, so results are
// bitwise those of the reference's plain-loop build.
#ifndef NAIVE_BLOCK_LDLT_KERNELS_H_
#define NAIVE_BLOCK_LDLT_KERNELS_H_

namespace naive_block_ldlt::kernels {

// destination[i*ds] = source[i*ss] / pivot, or 0 when pivot == 0.
void ScaleOneByOnePivot(int count, double pivot, const double* source, int source_stride,
                        double* destination, int destination_stride);

// [first; second] = inv([[a, b], [b, c]]) [first_source; second_source], or
// zeros when the determinant is 0.
void ScaleTwoByTwoPivot(int count, double pivot_top_left, double pivot_off_diagonal,
                        double pivot_bottom_right, const double* first_source,
                        int first_source_stride, const double* second_source,
                        int second_source_stride, double* first_destination,
                        int first_destination_stride, double* second_destination,
                        int second_destination_stride);

// target[rows x cols] -= left_panel^T * workspace_panel, with left_panel
// inner_dim x rows and workspace_panel inner_dim x cols, row-major.
void UpdateTrailingBlock(int rows, int cols, int inner_dim, const double* left_panel,
                         int left_panel_stride, const double* workspace_panel,
                         int workspace_panel_stride, double* target, int target_stride);

}  // namespace naive_block_ldlt::kernels

#endif  // NAIVE_BLOCK_LDLT_KERNELS_H_
