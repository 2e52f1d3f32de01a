/*
 * TEST INFRASTRUCTURE ONLY -- the CPU oracle for the blocked Bunch-Kaufman
 * LDL^T hot path.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline may load it; the product library never links or calls it.
 *
 * A plain-C restatement of wentianshu/BlockedBunchKaufmanLDLT's algorithm on
 * dense storage.  Matrices are n x n, row-major, leading dimension `lda`;
 * only the upper triangle (i <= j) is read or meaningful, exactly like the
 * reference's BlockMatrix, which stores blocks with block_row <= block_col
 * (src/block_matrix.cc:209-231).
 *
 * Parity is pinned against the reference itself: oracle/Makefile compiles the
 * reference sources into oracle/_ref/libbbk_ref.so and tests/test_oracle.py
 * requires bitwise-equal factors, permutation and pivot types on the
 * reference's own test inputs, plus the reference's golden 4x4 compact factor
 * (tests/block_ldlt_decomposition_test.cc:421-450).
 */
#ifndef BK_ORACLE_H_
#define BK_ORACLE_H_

#ifdef __cplusplus
extern "C" {
#endif

/* Bunch-Kaufman threshold (1 + sqrt(17)) / 8, the literal of
 * src/block_ldlt_decomposition.cc:14. */
#define BKO_ALPHA 0.6403882032022076

/* Factor the upper triangle of `a` in place into the reference's compact
 * storage: D on the diagonal (and on (k,k+1) for a 2x2 pivot), U = L^T in the
 * strict upper triangle.  perm[i] = original index at factored position i;
 * pivot_types[i] in {1, 2, -2}.  panel_end[P] is the first row after panel P
 * (panel P covers [panel_end[P-1], panel_end[P])); shifted[P] is 1 when the
 * last column of panel P moved to panel P+1 because a 2x2 pivot straddled
 * the boundary.  Follows BlockLdltDecomposition::Factorize
 * (src/block_ldlt_decomposition.cc:50-59, 80-120, 122-744) operation by
 * operation, including summation order, so results are bitwise identical.
 * Returns 0, or -1 on bad arguments / allocation failure. */
int bko_factor(int n, int block_size, double* a, long long lda, int* perm,
               int* pivot_types, int* panel_end, int* shifted);

/* Same factorization, also recording the Bunch-Kaufman decision quantities
 * of every pivot step in log[p * BKO_LOG_WORDS + .] for the factored position
 * p where the step's pivot starts (NaN elsewhere, e.g. the second row of a
 * 2x2 pivot):
 *   [0] |W(p,p)|                         the diagonal tested against alpha*omega
 *   [1] omega = max_{j>p} |W(p,j)|       (FindCurrentRowMax, :164-182)
 *   [2] the runner-up of that argmax     (max over j>p, j != r)
 *   [3] sigma = max_{i>=p,i!=r} |W(i,r)| (FindCandidateColumnMax, :354-367;
 *                                         NaN when no candidate was needed)
 *   [4] |W(r,r)|                         (NaN when no candidate was needed)
 * From these, every comparison of FactorPanel (:90-92) and SelectPivot
 * (:369-390) and its margin can be recomputed, so a decision that another
 * summation order could flip (a near-tie) is visible.  `log` may be NULL.
 * w_out (n x n row-major, may be NULL) receives each panel's workspace rows
 * at the columns its trailing update reads (rows of the panel, columns from
 * the panel's end on); nothing else of it is written. */
#define BKO_LOG_WORDS 5
int bko_factor_logged(int n, int block_size, double* a, long long lda,
                      int* perm, int* pivot_types, int* panel_end,
                      int* shifted, double* log, double* w_out);

/* Same factorization, but stops after `max_panels` panels (used to time a
 * bounded sample of a large factorization).  Returns the number of panels
 * processed. */
int bko_factor_panels(int n, int block_size, double* a, long long lda,
                      int* perm, int* pivot_types, int* panel_end,
                      int* shifted, int max_panels);

/* kernels::ScaleOneByOnePivot (src/kernels.cc:11-31). */
void bko_scale_one_by_one(int count, double pivot, const double* source,
                          int source_stride, double* destination,
                          int destination_stride);

/* kernels::ScaleTwoByTwoPivot (src/kernels.cc:33-65). */
void bko_scale_two_by_two(int count, double a, double b, double c,
                          const double* first_source, int first_source_stride,
                          const double* second_source,
                          int second_source_stride, double* first_destination,
                          int first_destination_stride,
                          double* second_destination,
                          int second_destination_stride);

/* kernels::UpdateTrailingBlock (src/kernels.cc:67-91):
 * target[i,j] -= sum_k left[k,i] * ws[k,j], k ascending, sum then subtract. */
void bko_update_trailing_block(int rows, int cols, int inner,
                               const double* left, int left_stride,
                               const double* ws, int ws_stride, double* target,
                               int target_stride);

/* Solve A x = b with the compact factors, nrhs right-hand sides stored
 * column after column (b[k*ldb + i]); x overwrites b.  L and D are read
 * exactly as tests/block_ldlt_large_stress_test.cc:160-194 reads them
 * (CompactLValue / ReconstructedPermutedEntry): L(i,k) = F(k,i) for k < i
 * except L(k+1,k) = 0 inside a 2x2 pivot; D(k,k) = F(k,k) and
 * D(k,k+1) = F(k,k+1) for a 2x2 pivot starting at k.  With P A P^T = L D L^T
 * and (P A P^T)(i,j) = A(perm[i], perm[j]).  A 1x1 pivot equal to zero yields
 * a zero component (the reference zeroes such a column of L); a singular
 * 2x2 pivot divides by zero. */
void bko_solve(int n, const double* f, long long ldf, const int* perm,
               const int* pivot_types, int nrhs, double* b, long long ldb);

/* Dense reconstruction P^T (L D L^T) P into `out` (n x n row-major, full
 * symmetric), the quantity BlockLdltDecomposition::ReconstructOriginal
 * returns (src/block_ldlt_decomposition.cc:61-78). */
void bko_reconstruct(int n, const double* f, long long ldf, const int* perm,
                     const int* pivot_types, double* out);

/* The reference tests' input generators, restated with the same libstdc++
 * engines so that inputs are identical:
 *  - tests/block_ldlt_decomposition_test.cc:148-161 (row by row over the
 *    upper triangle, std::mt19937 + std::normal_distribution(0,1));
 *  - tests/block_ldlt_large_stress_test.cc:116-136 (block by block).
 * Output: full symmetric n x n row-major. */
void bko_ref_random_symmetric(int n, int seed, double scale, double* out);
void bko_ref_random_block_fill(int n, int block_size, int seed, double scale,
                               double* out);

/* The stress test's sampled residual sample set
 * (tests/block_ldlt_large_stress_test.cc:204-218): writes `count` (row, col)
 * pairs into rows/cols. */
void bko_ref_residual_samples(int n, int seed, int count, int* rows, int* cols);

/* The stress test's SampledRelativeResidual (tests/block_ldlt_large_stress_
 * test.cc:160-244): for each sample (rows[k], cols[k]) of the original
 * matrix `a` (upper triangle read), the same entry of P^T L D L^T P from the
 * compact factors (CompactLValue / ReconstructedPermutedEntry, summed over
 * every pivot in order), then sqrt(sum diff^2) / max(sqrt(sum a^2), 1). */
double bko_sampled_residual(int n, const double* a, long long lda, const double* f,
                            long long ldf, const int* perm, const int* pt,
                            int count, const int* rows, const int* cols);

#ifdef __cplusplus
}
#endif

#endif  /* BK_ORACLE_H_ */
