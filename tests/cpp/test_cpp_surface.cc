// C++ drop-in surface test: the reference's public classes
// (naive_block_ldlt::BlockMatrix, RegularMatrix, kernels::*,
// BlockLdltDecomposition) as implemented by libbbk_b200, checked the way the
// reference's own tests check them (tests/block_ldlt_decomposition_test.cc),
// plus the block geometry after boundary shifts against fixtures produced by
// the reference (tests/golden/ref_geometry.txt).
//
// usage: test_cpp_surface <path to ref_geometry.txt>
#include <cmath>
#include <cstdint>
#include <fstream>
#include <iostream>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "bbk_ldlt.h"
#include "block_ldlt_decomposition.h"
#include "block_matrix.h"
#include "kernels.h"
#include "regular_matrix.h"

using namespace naive_block_ldlt;

namespace {

int g_checks = 0;

void Require(bool ok, const std::string& what) {
  ++g_checks;
  if (!ok) throw std::runtime_error("check failed: " + what);
}

double RelErr(const RegularMatrix& a, const RegularMatrix& b) {
  return FrobeniusNorm(Subtract(a, b)) / std::max(FrobeniusNorm(b), 1.0);
}

RegularMatrix Dense(int n, const std::vector<double>& v) { return RegularMatrix(n, n, v); }

// The reference tests' generator: std::mt19937(seed), N(0,1), filled row by
// row over the upper triangle and mirrored.
RegularMatrix RandomSymmetric(int n, int seed, double scale = 1.0) {
  std::mt19937 gen(seed);
  std::normal_distribution<double> dist(0.0, 1.0);
  RegularMatrix m(n, n);
  for (int i = 0; i < n; ++i)
    for (int j = i; j < n; ++j) {
      const double v = scale * dist(gen);
      m(i, j) = v;
      m(j, i) = v;
    }
  return m;
}

template <typename E, typename F>
bool Throws(F&& f) {
  try {
    f();
  } catch (const E&) {
    return true;
  } catch (...) {
    return false;
  }
  return false;
}

const std::vector<double> kGolden = {6, 12, 3, -6, 12, -8, -13, 4, 3, -13, -1, 1, -6, 4, 1, 6};

void StorageAndIndexing() {
  RegularMatrix m(4, 5);
  Require(reinterpret_cast<std::uintptr_t>(m.Data()) % kDefaultAlignment == 0, "RegularMatrix aligned");
  m(3, 4) = 42.0;
  Require(m.Data()[3 * m.LeadingDimension() + 4] == 42.0, "RegularMatrix row-major");
  BlockMatrix bm(7, 3);
  bm(5, 2) = -3.0;
  Require(bm(2, 5) == -3.0, "BlockMatrix symmetric access");
  Require(reinterpret_cast<std::uintptr_t>(bm.GetBlock(0, 0).Data()) % kDefaultAlignment == 0,
          "BlockMatrix tile aligned");
  Require(bm.num_blocks() == 3 && bm.GetBlock(1, 2).leading_dimension() == 2, "tile geometry");
  Require(Throws<std::invalid_argument>([] { BlockMatrix(0, 2); }), "size 0 rejected");
  Require(Throws<std::invalid_argument>([] { BlockMatrix(4, 0); }), "block size 0 rejected");
  Require(Throws<std::out_of_range>([&] { bm(7, 0); }), "index outside the matrix");
  Require(Throws<std::invalid_argument>([] { BlockMatrix(RegularMatrix(3, 4), 2); }), "non-square rejected");
}

void KernelShapes() {
  double s0[] = {2.0, 4.0, 6.0}, d0[] = {0.0, 0.0, 0.0};
  kernels::ScaleOneByOnePivot(3, 2.0, s0, 1, d0, 1);
  Require(d0[0] == 1.0 && d0[1] == 2.0 && d0[2] == 3.0, "ScaleOneByOnePivot");
  double s1[] = {1.0, 2.0}, s2[] = {3.0, 4.0}, d1[] = {0.0, 0.0}, d2[] = {0.0, 0.0};
  kernels::ScaleTwoByTwoPivot(2, 2.0, 1.0, 3.0, s1, 1, s2, 1, d1, 1, d2, 1);
  Require(std::abs(d1[0]) < 1e-14 && std::abs(d2[0] - 1.0) < 1e-14, "ScaleTwoByTwoPivot");
  // target (2 x 3) -= left^T (2 x 2) ws (2 x 3), strided rows
  double left[] = {1, 2, 0, 3, 4, 0};   // inner 2 x rows 2, stride 3
  double ws[] = {1, 0, 2, 0, 1, 1};     // inner 2 x cols 3, stride 3
  double tgt[] = {10, 10, 10, 10, 10, 10};
  kernels::UpdateTrailingBlock(2, 3, 2, left, 3, ws, 3, tgt, 3);
  // C[i][j] -= sum_k left[k][i] ws[k][j]
  const double want[] = {10 - 1, 10 - 3, 10 - (2 + 3), 10 - 2, 10 - 4, 10 - (4 + 4)};
  for (int i = 0; i < 6; ++i) Require(tgt[i] == want[i], "UpdateTrailingBlock");
}

void GoldenCompactStorage() {
  BlockLdltDecomposition d(BlockMatrix(Dense(4, kGolden), 2));
  d.Factorize();
  const RegularMatrix want = Dense(4, {6.0, 12.0, -0.6875, 0.0, 0.0, -8.0, 0.59375, -0.5, 0.0, 0.0,
                                       8.78125, -0.6263345195729537, 0.0, 0.0, 0.0, 4.555160142348754});
  Require(RelErr(d.CompactFactors().ToUpperRegular(), want) < 1e-10, "golden compact factor");
  Require(d.PivotTypes() == std::vector<int>({2, -2, 1, 1}), "golden pivot types");
  Require(RelErr(d.ReconstructOriginal(), Dense(4, kGolden)) < 1e-10, "golden reconstruction");
  RegularMatrix ldl = Multiply(Multiply(d.LFactor(), d.DFactor()), Transpose(d.LFactor()));
  RegularMatrix back(4, 4);
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) back(d.Permutation()[i], d.Permutation()[j]) = ldl(i, j);
  Require(RelErr(back, Dense(4, kGolden)) < 1e-10, "L and D factors");
}

void FixedAndStateErrors() {
  const std::vector<RegularMatrix> fixed = {
      Dense(4, kGolden), Dense(4, {0, 1, 0, 0, 1, 0, 0, 0, 0, 0, 0, 1, 0, 0, 1, 0}),
      Dense(4, {2, 0, 0, 0, 0, -3, 0, 0, 0, 0, 0, 0, 0, 0, 0, 5})};
  for (const RegularMatrix& m : fixed)
    for (int b = 1; b <= 4; ++b) {
      BlockLdltDecomposition d{BlockMatrix(m, b)};
      Require(Throws<std::logic_error>([&] { d.ReconstructOriginal(); }), "reconstruct before factorize");
      d.Factorize();
      Require(RelErr(d.ReconstructOriginal(), m) < 1e-10, "fixed factorization");
    }
  BlockLdltDecomposition c(BlockMatrix(Dense(4, kGolden), 2),
                           BlockLdltDecomposition::FactorizationMode::kCompactOnly);
  c.Factorize();
  Require(Throws<std::logic_error>([&] { c.ReconstructOriginal(); }), "compact-only reconstruct");
}

void TriangularInput() {
  RegularMatrix up = Dense(4, kGolden), lo = Dense(4, kGolden);
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      if (i > j) up(i, j) = 12345.0;
      if (i < j) lo(i, j) = 12345.0;
    }
  for (int b = 1; b <= 4; ++b) {
    BlockLdltDecomposition du{BlockMatrix(up, b, MatrixTriangle::kUpper)};
    du.Factorize();
    Require(RelErr(du.ReconstructOriginal(), Dense(4, kGolden)) < 1e-10, "upper input");
    BlockLdltDecomposition dl{BlockMatrix(lo, b, MatrixTriangle::kLower)};
    dl.Factorize();
    Require(RelErr(dl.ReconstructOriginal(), Dense(4, kGolden)) < 1e-10, "lower input");
  }
}

void RandomFactorizations() {
  for (int n = 3; n <= 16; ++n)
    for (int b = 1; b <= n; ++b) {
      const RegularMatrix a = RandomSymmetric(n, 10000 * n + 100 * b + 1);
      BlockLdltDecomposition d{BlockMatrix(a, b)};
      d.Factorize();
      Require(RelErr(d.ReconstructOriginal(), a) < 1e-10, "random factorization");
    }
}

void SolveExtension() {
  const int n = 50;
  const RegularMatrix a = RandomSymmetric(n, 4242);
  BlockLdltDecomposition d(BlockMatrix(a, 8), BlockLdltDecomposition::FactorizationMode::kCompactOnly);
  d.Factorize();
  std::vector<double> b(n);
  for (int i = 0; i < n; ++i) b[i] = std::sin(i + 1.0);
  const std::vector<double> x = d.Solve(b);
  double r = 0.0, bn = 0.0;
  for (int i = 0; i < n; ++i) {
    double s = -b[i];
    for (int j = 0; j < n; ++j) s += a(i, j) * x[j];
    r = std::max(r, std::abs(s));
    bn = std::max(bn, std::abs(b[i]));
  }
  Require(r < 1e-12 * std::max(1.0, bn), "Solve residual");
}

// Geometry, permutation, pivots and factor bits against the reference.
void GeometryFixtures(const std::string& path) {
  std::ifstream in(path);
  Require(static_cast<bool>(in), "open " + path);
  int ncase = 0;
  in >> ncase;
  for (int k = 0; k < ncase; ++k) {
    int n = 0, b = 0, seed = 0, nblk = 0;
    in >> n >> b >> seed >> nblk;
    std::vector<int> geo(4 * nblk), perm(n), piv(n);
    for (int& v : geo) in >> v;
    for (int& v : perm) in >> v;
    for (int& v : piv) in >> v;
    RegularMatrix want(n, n), want_ws(n, n);
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) in >> want(i, j);
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) in >> want_ws(i, j);
    BlockLdltDecomposition d(BlockMatrix(RandomSymmetric(n, seed), b),
                             BlockLdltDecomposition::FactorizationMode::kCompactOnly);
    d.SetUpdateMode(BBK_UPDATE_FP64_ORDERED);
    d.Factorize();
    const BlockMatrix& f = d.CompactFactors();
    for (int bc = 0; bc < f.num_blocks(); ++bc)
      for (int br = 0; br <= bc; ++br) {
        const Block& blk = f.GetBlock(br, bc);
        const int* g = &geo[4 * f.BlockId(br, bc)];
        Require(blk.row0() == g[0] && blk.rows() == g[1] && blk.col0() == g[2] && blk.cols() == g[3],
                "block geometry (" + std::to_string(br) + "," + std::to_string(bc) + ") n=" +
                    std::to_string(n));
      }
    Require(d.Permutation() == perm, "permutation vs reference");
    Require(d.PivotTypes() == piv, "pivot types vs reference");
    const RegularMatrix got = f.ToUpperRegular();
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) Require(got(i, j) == want(i, j), "factor bits vs reference");
    // Workspace(): the reference's workspace rows bit for bit outside the
    // diagonal blocks, zero inside them
    const BlockMatrix& w = d.Workspace();
    for (int bc = 0; bc < w.num_blocks(); ++bc)
      for (int br = 0; br <= bc; ++br) {
        const Block& blk = w.GetBlock(br, bc);
        for (int r = 0; r < blk.rows(); ++r)
          for (int c = 0; c < blk.cols(); ++c) {
            const int gi = blk.row0() + r, gj = blk.col0() + c;
            const double expect = br == bc ? 0.0 : want_ws(gi, gj);
            Require(blk(r, c) == expect, "workspace rows vs reference");
          }
      }
  }
}

}  // namespace

int main(int argc, char** argv) {
  try {
    StorageAndIndexing();
    KernelShapes();
    GoldenCompactStorage();
    FixedAndStateErrors();
    TriangularInput();
    RandomFactorizations();
    SolveExtension();
    if (argc > 1) GeometryFixtures(argv[1]);
  } catch (const std::exception& e) {
    std::cerr << "C++ surface test failed: " << e.what() << "\n";
    return 1;
  }
  std::cout << "C++ surface test passed (" << g_checks << " checks)\n";
  return 0;
}
