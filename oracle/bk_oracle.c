/*
 * TEST INFRASTRUCTURE ONLY -- CPU oracle for the blocked Bunch-Kaufman LDL^T
 * hot path (see bk_oracle.h).  Never linked into the product library.
 *
 * Dense restatement of src/block_ldlt_decomposition.cc.  Storage: row-major,
 * upper triangle.  The reference keeps a whole second BlockMatrix of
 * "workspace rows" W; only three parts of it are ever read, and they are kept
 * here explicitly:
 *   - the W rows of the current panel's pivots (buffer `w`, one row per
 *     panel pivot, indexed by global column),
 *   - the candidate column W(i, r), i >= p (buffer `wc`, indexed by i),
 *   - the single entry W(p, r) that CopyCandidateToWorkspace overwrites in
 *     the current row (src/block_ldlt_decomposition.cc:192-193, 212-214),
 *     which later feeds the scaling and the 2x2 D block.
 * Compile with -ffp-contract=off: the reference is built as ISO C++ for
 * baseline x86-64, so every product and sum is rounded separately.
 */
#include "bk_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define IDX(i, j, ld) ((size_t)(i) * (size_t)(ld) + (size_t)(j))

/* src/block_ldlt_decomposition.cc:21-26 */
static double safe_denominator(double v) {
  return fabs(v) <= DBL_EPSILON ? 0.0 : v;
}

/* std::max(a, b) == (a < b) ? b : a, so a NaN candidate never wins. */
static double std_max(double a, double b) { return (a < b) ? b : a; }

static void swap_d(double* x, double* y) {
  double t = *x;
  *x = *y;
  *y = t;
}

/* Symmetric interchange of indices s < r in the upper storage, as far as it
 * matters once row s is about to be overwritten by the pivot's factor row:
 * row s moves to row r, the columns s and r of every earlier row exchange.
 * This is the net effect of SwapOneByOnePivotInMatrix /
 * SwapTwoByTwoPivotInMatrix on factors_ (src/block_ldlt_decomposition.cc:
 * 414-498, 500-587) including the previously factored block rows (:472-491)
 * -- the entries of row s that the reference swaps into place are all
 * rewritten by the subsequent Scale*Pivot call. */
static void symmetric_move(double* a, long long lda, int n, int s, int r,
                           int rows_above) {
  if (s == r) return;
  for (int j = r + 1; j < n; ++j) a[IDX(r, j, lda)] = a[IDX(s, j, lda)];
  for (int j = s + 1; j < r; ++j) a[IDX(j, r, lda)] = a[IDX(s, j, lda)];
  a[IDX(r, r, lda)] = a[IDX(s, s, lda)];
  for (int i = 0; i < rows_above; ++i) swap_d(&a[IDX(i, s, lda)], &a[IDX(i, r, lda)]);
}

/* Every dot product below is accumulated in its own variable, q ascending,
 * starting from 0.0, exactly as the reference's scalar loops do; the loops
 * are only nested with q outermost so the accumulators of a whole row
 * advance together (contiguous, vectorisable loads).  The sequence of
 * roundings each accumulator sees is unchanged, so results are too. */
static int factor_impl(int n, int b, double* a, long long lda, int* perm,
                       int* pivot_types, int* panel_end, int* shifted,
                       int max_panels, double* log, double* w_out) {
  if (n <= 0 || b <= 0 || lda < n || !a || !perm || !pivot_types) return -1;
  const int nb = (n + b - 1) / b;
  double* w = (double*)calloc((size_t)(b + 1) * (size_t)n, sizeof(double));
  double* wc = (double*)calloc((size_t)n, sizeof(double));
  double* acc = (double*)calloc((size_t)n, sizeof(double));
  if (!w || !wc || !acc) {
    free(w);
    free(wc);
    free(acc);
    return -1;
  }
  if (log)
    for (size_t i = 0; i < (size_t)n * BKO_LOG_WORDS; ++i) log[i] = NAN;
  for (int i = 0; i < n; ++i) {
    perm[i] = i;
    pivot_types[i] = 0;
  }

  int k0 = 0; /* first row of the current panel */
  int panels_done = 0;
  for (int panel = 0; panel < nb && panels_done < max_panels; ++panel) {
    /* Nominal end of block `panel`; a shift at the previous boundary made
     * this panel start one column earlier (ExpandBlock, block_matrix.cc:173). */
    const int kend = (panel + 1) * b < n ? (panel + 1) * b : n;
    const int can_shift = panel + 1 < nb;
    int did_shift = 0;
    int p = k0;
    /* FactorPanel, src/block_ldlt_decomposition.cc:80-120 */
    while (p < kend) {
      double* wp = w + (size_t)(p - k0) * n;
      /* CopyCurrentRowToWorkspace + UpdateCurrentRowInWorkspace (:122-162):
       * W[p,j] = A[p,j] - sum_{q<p in panel} U[q,p] W[q,j] */
      for (int j = p; j < n; ++j) acc[j] = 0.0;
      for (int q = k0; q < p; ++q) {
        const double c = a[IDX(q, p, lda)];
        const double* wq = w + (size_t)(q - k0) * n;
        for (int j = p; j < n; ++j) acc[j] += c * wq[j];
      }
      for (int j = p; j < n; ++j) wp[j] = a[IDX(p, j, lda)] - acc[j];
      /* FindCurrentRowMax (:164-182): strict '>' in ascending column order,
       * so the lowest index wins ties and NaN never wins. */
      double omega = 0.0;
      int r = 0;
      for (int j = p + 1; j < n; ++j) {
        const double v = fabs(wp[j]);
        if (v > omega) {
          omega = v;
          r = j;
        }
      }
      const double dpp = wp[p];
      if (log) {
        /* the decision quantities of this step (overwritten if the step is
         * redone after a boundary shift); the runner-up of the row argmax
         * shows how close another column came to being the candidate */
        double second = 0.0;
        for (int j = p + 1; j < n; ++j)
          if (j != r && fabs(wp[j]) > second) second = fabs(wp[j]);
        double* lg = log + (size_t)p * BKO_LOG_WORDS;
        lg[0] = fabs(dpp);
        lg[1] = omega;
        lg[2] = second;
        lg[3] = NAN;
        lg[4] = NAN;
      }
      int kind = 1; /* 1: 1x1 at p; -1: 1x1 after swapping p<->r; 2: 2x2 */
      int have_candidate = 0;
      if (!(fabs(dpp) >= BKO_ALPHA * omega || omega == 0.0)) {
        have_candidate = 1;
        /* CopyCandidateToWorkspace + UpdateCandidateInWorkspace (:184-352):
         * W(i,r) = A(i,r) - sum_q U[q,r] W[q,i] for every active i >= p. */
        for (int i = p; i < n; ++i) acc[i] = 0.0;
        for (int q = k0; q < p; ++q) {
          const double c = a[IDX(q, r, lda)];
          const double* wq = w + (size_t)(q - k0) * n;
          for (int i = p; i < n; ++i) acc[i] += c * wq[i];
        }
        for (int i = p; i < n; ++i) {
          const double aval = i <= r ? a[IDX(i, r, lda)] : a[IDX(r, i, lda)];
          wc[i] = aval - acc[i];
        }
        /* FindCandidateColumnMax (:354-367) */
        double sigma = 0.0;
        for (int i = p; i < n; ++i)
          if (i != r) sigma = std_max(sigma, fabs(wc[i]));
        if (log) {
          log[(size_t)p * BKO_LOG_WORDS + 3] = sigma;
          log[(size_t)p * BKO_LOG_WORDS + 4] = fabs(wc[r]);
        }
        /* SelectPivot (:369-390) */
        if (fabs(dpp) * sigma - BKO_ALPHA * omega * omega >= 0.0) {
          kind = 1;
        } else if (fabs(wc[r]) - BKO_ALPHA * sigma >= 0.0) {
          kind = -1;
        } else {
          kind = 2;
        }
        /* :104-108 -- a 2x2 pivot that would start at the panel's last
         * column moves that column into the next panel instead. */
        if (kind == 2 && p == kend - 1 && can_shift) {
          did_shift = 1;
          break;
        }
      }

      if (kind == 1) {
        /* The candidate copy overwrote W(p,r) with the column version. */
        if (have_candidate) wp[r] = wc[p];
        const double d = wp[p];
        const double den = safe_denominator(d);
        pivot_types[p] = 1;
        for (int j = p + 1; j < n; ++j)
          a[IDX(p, j, lda)] = den == 0.0 ? 0.0 : wp[j] / den;
        a[IDX(p, p, lda)] = d;
        p += 1;
      } else if (kind == -1) {
        /* SwapOneByOnePivot (:392-401) then ScaleOneByOnePivot (:633-656). */
        symmetric_move(a, lda, n, p, r, p);
        for (int q = k0; q < p; ++q)
          swap_d(&w[IDX(q - k0, p, n)], &w[IDX(q - k0, r, n)]);
        for (int j = p + 1; j < n; ++j) wp[j] = (j == r) ? wc[p] : wc[j];
        wp[p] = wc[r];
        { int t = perm[p]; perm[p] = perm[r]; perm[r] = t; }
        const double d = wp[p];
        const double den = safe_denominator(d);
        pivot_types[p] = 1;
        for (int j = p + 1; j < n; ++j)
          a[IDX(p, j, lda)] = den == 0.0 ? 0.0 : wp[j] / den;
        a[IDX(p, p, lda)] = d;
        p += 1;
      } else {
        /* SwapTwoByTwoPivot (:403-412) then ScaleTwoByTwoPivot (:658-704). */
        const int s = p + 1;
        double* ws = w + (size_t)(s - k0) * n;
        const double cur_ps = wp[s];
        symmetric_move(a, lda, n, s, r, p);
        for (int q = k0; q < p; ++q)
          swap_d(&w[IDX(q - k0, s, n)], &w[IDX(q - k0, r, n)]);
        /* Row p: columns s and r exchange; W(p,r) held the candidate value. */
        wp[s] = wc[p];
        if (r != s) wp[r] = cur_ps;
        for (int j = s + 1; j < n; ++j) ws[j] = (j == r) ? wc[s] : wc[j];
        ws[s] = wc[r];
        { int t = perm[s]; perm[s] = perm[r]; perm[r] = t; }

        const double d11 = wp[p], d21 = wp[s], d22 = ws[s];
        const double det = d11 * d22 - d21 * d21;
        const double i11 = d22 / det;
        const double i22 = d11 / det;
        const double i21 = -d21 / det;
        pivot_types[p] = 2;
        pivot_types[s] = -2;
        for (int j = s + 1; j < n; ++j) {
          const double x = wp[j], y = ws[j];
          a[IDX(p, j, lda)] = i11 * x + i21 * y;
          a[IDX(s, j, lda)] = i21 * x + i22 * y;
        }
        a[IDX(p, p, lda)] = d11;
        a[IDX(p, s, lda)] = d21;
        a[IDX(s, s, lda)] = d22;
        p += 2;
      }
    }
    const int e = p; /* first row after this panel */
    if (panel_end) panel_end[panel] = e;
    if (shifted) shifted[panel] = did_shift;
    if (w_out) /* the panel's W rows at the columns the trailing update reads */
      for (int q = k0; q < e; ++q)
        for (int j = e; j < n; ++j) w_out[IDX(q, j, n)] = w[IDX(q - k0, j, n)];

    /* UpdateTrailingBlocks (:706-744) + kernels::UpdateTrailingBlock
     * (kernels.cc:67-91): A[i,j] -= sum_q U[q,i] W[q,j] over the trailing
     * upper triangle, q ascending, sum first then one subtraction. */
    if (e > k0) {
      for (int i = e; i < n; ++i) {
        for (int j = i; j < n; ++j) acc[j] = 0.0;
        for (int q = k0; q < e; ++q) {
          const double c = a[IDX(q, i, lda)];
          const double* wq = w + (size_t)(q - k0) * n;
          for (int j = i; j < n; ++j) acc[j] += c * wq[j];
        }
        double* ai = a + IDX(i, 0, lda);
        for (int j = i; j < n; ++j) ai[j] -= acc[j];
      }
    }
    k0 = e;
    ++panels_done;
  }
  free(w);
  free(wc);
  free(acc);
  return panels_done;
}

int bko_factor(int n, int block_size, double* a, long long lda, int* perm,
               int* pivot_types, int* panel_end, int* shifted) {
  const int r = factor_impl(n, block_size, a, lda, perm, pivot_types,
                            panel_end, shifted, 1 << 30, NULL, NULL);
  return r < 0 ? -1 : 0;
}

int bko_factor_logged(int n, int block_size, double* a, long long lda,
                      int* perm, int* pivot_types, int* panel_end,
                      int* shifted, double* log, double* w_out) {
  const int r = factor_impl(n, block_size, a, lda, perm, pivot_types,
                            panel_end, shifted, 1 << 30, log, w_out);
  return r < 0 ? -1 : 0;
}

int bko_factor_panels(int n, int block_size, double* a, long long lda,
                      int* perm, int* pivot_types, int* panel_end,
                      int* shifted, int max_panels) {
  return factor_impl(n, block_size, a, lda, perm, pivot_types, panel_end,
                     shifted, max_panels, NULL, NULL);
}

void bko_scale_one_by_one(int count, double pivot, const double* source,
                          int source_stride, double* destination,
                          int destination_stride) {
  if (count <= 0) return;
  if (fabs(pivot) == 0.0) {
    for (int i = 0; i < count; ++i) destination[(long)i * destination_stride] = 0.0;
    return;
  }
  for (int i = 0; i < count; ++i)
    destination[(long)i * destination_stride] = source[(long)i * source_stride] / pivot;
}

void bko_scale_two_by_two(int count, double a, double b, double c,
                          const double* first_source, int first_source_stride,
                          const double* second_source,
                          int second_source_stride, double* first_destination,
                          int first_destination_stride,
                          double* second_destination,
                          int second_destination_stride) {
  if (count <= 0) return;
  const double det = a * c - b * b;
  if (fabs(det) == 0.0) {
    for (int i = 0; i < count; ++i) {
      first_destination[(long)i * first_destination_stride] = 0.0;
      second_destination[(long)i * second_destination_stride] = 0.0;
    }
    return;
  }
  for (int i = 0; i < count; ++i) {
    const double x = first_source[(long)i * first_source_stride];
    const double y = second_source[(long)i * second_source_stride];
    first_destination[(long)i * first_destination_stride] = (x * c - y * b) / det;
    second_destination[(long)i * second_destination_stride] = (-x * b + y * a) / det;
  }
}

void bko_update_trailing_block(int rows, int cols, int inner,
                               const double* left, int left_stride,
                               const double* ws, int ws_stride, double* target,
                               int target_stride) {
  if (rows <= 0 || cols <= 0 || inner <= 0) return;
  for (int i = 0; i < rows; ++i) {
    for (int j = 0; j < cols; ++j) {
      double update = 0.0;
      for (int k = 0; k < inner; ++k)
        update += left[(long)k * left_stride + i] * ws[(long)k * ws_stride + j];
      target[(long)i * target_stride + j] -= update;
    }
  }
}

/* L(i,k) for k < i, tests/block_ldlt_large_stress_test.cc:160-172. */
static double l_value(const double* f, long long ldf, const int* pt, int i, int k) {
  if (i == k) return 1.0;
  if (i < k) return 0.0;
  if (pt[k] == 2 && i == k + 1) return 0.0;
  return f[IDX(k, i, ldf)];
}

void bko_solve(int n, const double* f, long long ldf, const int* perm,
               const int* pivot_types, int nrhs, double* b, long long ldb) {
  double* y = (double*)malloc((size_t)n * sizeof(double));
  if (!y) return;
  for (int c = 0; c < nrhs; ++c) {
    double* bc = b + (size_t)c * (size_t)ldb;
    for (int i = 0; i < n; ++i) y[i] = bc[perm[i]];
    /* L z = y */
    for (int i = 0; i < n; ++i) {
      double s = y[i];
      for (int k = 0; k < i; ++k) s -= l_value(f, ldf, pivot_types, i, k) * y[k];
      y[i] = s;
    }
    /* D w = z */
    for (int k = 0; k < n;) {
      if (pivot_types[k] == 2 && k + 1 < n) {
        const double d11 = f[IDX(k, k, ldf)], d21 = f[IDX(k, k + 1, ldf)],
                     d22 = f[IDX(k + 1, k + 1, ldf)];
        const double det = d11 * d22 - d21 * d21;
        const double x = y[k], z = y[k + 1];
        y[k] = (d22 / det) * x + (-d21 / det) * z;
        y[k + 1] = (-d21 / det) * x + (d11 / det) * z;
        k += 2;
      } else {
        const double d = f[IDX(k, k, ldf)];
        y[k] = d == 0.0 ? 0.0 : y[k] / d;
        k += 1;
      }
    }
    /* L^T v = w */
    for (int i = n - 1; i >= 0; --i) {
      double s = y[i];
      for (int k = i + 1; k < n; ++k) s -= l_value(f, ldf, pivot_types, k, i) * y[k];
      y[i] = s;
    }
    for (int i = 0; i < n; ++i) bc[perm[i]] = y[i];
  }
  free(y);
}

void bko_reconstruct(int n, const double* f, long long ldf, const int* perm,
                     const int* pivot_types, double* out) {
  /* M = L D, then (L D L^T)(i,j) = sum_k M(i,k) L(j,k). */
  double* m = (double*)calloc((size_t)n * n, sizeof(double));
  double* l = (double*)calloc((size_t)n * n, sizeof(double));
  if (!m || !l) {
    free(m);
    free(l);
    return;
  }
  for (int i = 0; i < n; ++i)
    for (int k = 0; k <= i; ++k) l[IDX(i, k, n)] = l_value(f, ldf, pivot_types, i, k);
  for (int k = 0; k < n;) {
    if (pivot_types[k] == 2 && k + 1 < n) {
      const double d11 = f[IDX(k, k, ldf)], d21 = f[IDX(k, k + 1, ldf)],
                   d22 = f[IDX(k + 1, k + 1, ldf)];
      for (int i = 0; i < n; ++i) {
        const double x = l[IDX(i, k, n)], y = l[IDX(i, k + 1, n)];
        m[IDX(i, k, n)] = x * d11 + y * d21;
        m[IDX(i, k + 1, n)] = x * d21 + y * d22;
      }
      k += 2;
    } else {
      const double d = f[IDX(k, k, ldf)];
      for (int i = 0; i < n; ++i) m[IDX(i, k, n)] = l[IDX(i, k, n)] * d;
      k += 1;
    }
  }
  for (int i = 0; i < n; ++i) {
    for (int j = 0; j < n; ++j) {
      double s = 0.0;
      const int kmax = (i < j ? j : i) + 1;
      for (int k = 0; k < kmax && k < n; ++k) s += m[IDX(i, k, n)] * l[IDX(j, k, n)];
      out[IDX(perm[i], perm[j], n)] = s;
    }
  }
  free(m);
  free(l);
}

/* tests/block_ldlt_large_stress_test.cc:160-172 (CompactLValue) */
static double compact_l(const double* f, long long ldf, const int* pt, int row, int col) {
  if (row == col) return 1.0;
  if (row < col) return 0.0;
  if (pt[col] == 2 && row == col + 1) return 0.0;
  return f[IDX(col, row, ldf)];
}

double bko_sampled_residual(int n, const double* a, long long lda, const double* f, long long ldf,
                            const int* perm, const int* pt, int count, const int* rows,
                            const int* cols) {
  int* inv = (int*)malloc((size_t)n * sizeof(int));
  if (!inv) return NAN;
  for (int i = 0; i < n; ++i) inv[perm[i]] = i; /* InversePermutation, :196-202 */
  double residual_squared = 0.0, original_squared = 0.0;
  for (int k = 0; k < count; ++k) { /* SampledRelativeResidual, :220-244 */
    const int r = inv[rows[k]], c = inv[cols[k]];
    double value = 0.0; /* ReconstructedPermutedEntry, :174-194 */
    for (int p = 0; p < n; ++p) {
      const double row_left = compact_l(f, ldf, pt, r, p);
      const double col_left = compact_l(f, ldf, pt, c, p);
      value += row_left * f[IDX(p, p, ldf)] * col_left;
      if (pt[p] == 2) {
        const double off = f[IDX(p, p + 1, ldf)];
        const double row_next = compact_l(f, ldf, pt, r, p + 1);
        const double col_next = compact_l(f, ldf, pt, c, p + 1);
        value += off * (row_left * col_next + row_next * col_left);
      }
    }
    const int lo = rows[k] < cols[k] ? rows[k] : cols[k];
    const int hi = rows[k] < cols[k] ? cols[k] : rows[k];
    const double expected = a[IDX(lo, hi, lda)];
    const double difference = value - expected;
    residual_squared += difference * difference;
    original_squared += expected * expected;
  }
  free(inv);
  const double on = sqrt(original_squared);
  return sqrt(residual_squared) / (on < 1.0 ? 1.0 : on);
}
