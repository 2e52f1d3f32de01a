// TEST INFRASTRUCTURE ONLY -- input generators of the reference's own tests,
// restated with the same libstdc++ engines (std::mt19937 and
// std::normal_distribution / std::uniform_int_distribution are
// implementation-specific, so reproducing the reference's inputs needs the
// same C++ standard library, which is why this file is C++ and not C).
#include <random>

#include "bk_oracle.h"

extern "C" {

// tests/block_ldlt_decomposition_test.cc:148-161
void bko_ref_random_symmetric(int n, int seed, double scale, double* out) {
  std::mt19937 generator(seed);
  std::normal_distribution<double> distribution(0.0, 1.0);
  for (int i = 0; i < n; ++i) {
    for (int j = i; j < n; ++j) {
      const double value = scale * distribution(generator);
      out[static_cast<long long>(i) * n + j] = value;
      out[static_cast<long long>(j) * n + i] = value;
    }
  }
}

// tests/block_ldlt_large_stress_test.cc:116-136: blocks in (block_col,
// block_row <= block_col) order, rows then columns, upper entries only.
void bko_ref_random_block_fill(int n, int block_size, int seed, double scale,
                               double* out) {
  std::mt19937 generator(seed);
  std::normal_distribution<double> distribution(0.0, 1.0);
  const int nb = (n + block_size - 1) / block_size;
  for (int bc = 0; bc < nb; ++bc) {
    for (int br = 0; br <= bc; ++br) {
      const int r0 = br * block_size, c0 = bc * block_size;
      const int rows = (n - r0) < block_size ? (n - r0) : block_size;
      const int cols = (n - c0) < block_size ? (n - c0) : block_size;
      for (int r = 0; r < rows; ++r) {
        for (int c = 0; c < cols; ++c) {
          const int gi = r0 + r, gj = c0 + c;
          if (gi > gj) continue;
          const double value = scale * distribution(generator);
          out[static_cast<long long>(gi) * n + gj] = value;
          out[static_cast<long long>(gj) * n + gi] = value;
        }
      }
    }
  }
}

// tests/block_ldlt_large_stress_test.cc:204-218
void bko_ref_residual_samples(int n, int seed, int count, int* rows, int* cols) {
  int k = 0;
  const int fixed[4][2] = {{0, 0}, {0, n - 1}, {n / 2, n / 2}, {n - 1, n - 1}};
  for (int f = 0; f < 4 && k < count; ++f, ++k) {
    rows[k] = fixed[f][0];
    cols[k] = fixed[f][1];
  }
  std::mt19937 generator(seed + 170003);
  std::uniform_int_distribution<int> distribution(0, n - 1);
  while (k < count) {
    rows[k] = distribution(generator);
    cols[k] = distribution(generator);
    ++k;
  }
}

}  // extern "C"
