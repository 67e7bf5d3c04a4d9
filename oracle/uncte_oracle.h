/*
 * uncte_oracle.h - CPU FP64 oracle for the uncertaintyTE covariance path.
 *
 * TEST INFRASTRUCTURE ONLY. This library restates, step for step, the
 * reference's CPU algorithm (src/uncertaintyTE/compute.cpp,
 * ScaledSparseMatrix.cpp, ScaledDenseMatrix.cpp) so that the CUDA product
 * path can be checked against it. Only the test suite, the smoke check and
 * the CPU-baseline leg of the benchmark may load it. The product library
 * never links or calls it.
 *
 * Parity pins (checked by tests/test_oracle_golden.py):
 *   - test/EigValues/output.cov  (04_Daliborka, TAYLOR_EXPANSION, end to end)
 *   - test/SparseMatrix/multipl_in_01 -> multipl_out_01  (J^T J, CRS pattern + values)
 *   - test/SparseMatrix/inv_in_01 -> inv_out_01, test/DenseMatrix/inv_in_01 -> inv_out_01
 *     (equilibrated LU inverse)
 */
#pragma once
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int algorithm;            /* 0 SVD_QR_ITERATION, 1 SVD_DEVIDE_AND_CONQUER, 2 TAYLOR_EXPANSION */
    double epsilon;           /* SVD threshold when svd_remove_n == -1 (<0 -> 1e-10) */
    double lambda;            /* TE regulariser; -1 = automatic (compute.cpp:124-125) */
    int num_cams, cam_params, num_points, num_obs;
    int svd_remove_n;         /* SVD: drop this many smallest singular values; -1 = use epsilon */
    int pts2fix[3];
    int has_pts2fix;
    int faithful_point_scan;  /* 1: per point, scan every J row as compute.cpp:393 does */
    int threads;              /* OpenMP + BLAS threads; 0 = leave as is */
    int inverse_route;        /* 0: LU as the reference (ScaledDenseMatrix::inv); 1: Cholesky on the
                                 Jacobi-equilibrated matrix (the CUDA path's route), see below */
    double z_perturb;         /* 0: none. Otherwise every entry of the Schur complement Z is multiplied
                                 by (1 + z_perturb * r), r in [-1, 1) from a fixed hash of (row, col),
                                 symmetric. At z_perturb = 2^-53 this measures how far the results move
                                 under a rounding-level change of Z (cond(Z + lambda*I) * eps): the
                                 floor below which two correct FP64 implementations cannot agree. */
    double z_perturb_terms;   /* 0: none. Otherwise every entry Z_ij of the Schur complement moves by
                                 z_perturb_terms * r * (|U_ij| + |(Y W^T)_ij|), r in [-1, 1) from a fixed
                                 hash of (row, col), symmetric: the rounding error of Z = U - Y W^T at the
                                 size of its terms (what another summation order of the Schur complement
                                 amounts to), where the relative form above stays at the size of the
                                 result and misses the cancellation. */
    int swap_products;        /* 0: Taylor products add * X (the reference's order); 1: X * add. The powers of
                                 X commute, so both are the same series; their rounding differs (another
                                 correct FP64 evaluation, for the parity floor). */
    int skip_dense;           /* timing samples only: 1 skips the dense inverse and the Taylor loop (iZ is
                                 left as Z + lambda*I), so every sparse stage runs at full size but the
                                 outputs are meaningless. 0 for results. */
    int offdiag_nan;          /* 1: every entry of the final iZ outside its cam_params x cam_params diagonal
                                 camera blocks is set to NaN before the camera and point outputs, which
                                 shows what the outputs read (compute.cpp:168-183, 422-441): they are
                                 unchanged, so a solver may form the last Taylor terms on those blocks only.
                                 0 for results. */
} oracle_options;

typedef struct {
    double lambda;
    int fixed_pts[3];
    int te_iterations;
    double cycle_change[20];
    /* true seconds per stage (the reference prints ms/100, compute.cpp:33) */
    double t_fix, t_norm, t_jtj, t_split, t_invv, t_compose_z, t_inv_z, t_te, t_cams, t_pts, t_all;
    int lu_info;
} oracle_stats;

/* Full covariance computation (compute.cpp:458-540). cam_unc: num_cams*45,
 * pt_unc: num_points*6 (caller-initialised, as Uncertainty::init does).
 * dbg_Z / dbg_iZ / dbg_d: optional (may be NULL); TE path only:
 *   dbg_Z  (N*N, column-major) = Schur complement before +lambda*I, N = 9*num_cams
 *   dbg_iZ (N*N)               = final Taylor-series inverse
 *   dbg_d  (N)                 = 1/column-norm of the camera columns
 * Returns 0 on success, <0 on invalid input. */
int oracle_compute(const oracle_options* opt, int nrows, int ncols,
                   const int* rows, const int* cols, const double* vals,
                   double* cam_unc, double* pt_unc, oracle_stats* st,
                   double* dbg_Z, double* dbg_iZ, double* dbg_d);

/* Sparse J^T J exactly as the reference forms it (trn() then operator*):
 * first call with out_cols == NULL returns nnz; second call fills
 * out_rows (ncols+1), out_cols (nnz), out_vals (nnz). Columns ascend per row. */
long oracle_jtj(int nrows, int ncols, const int* rows, const int* cols, const double* vals,
                int* out_rows, int* out_cols, double* out_vals);

/* ScaledDenseMatrix::inv(): row then column 2-norm equilibration, LU with
 * partial pivoting (dgetrf), dgetri, unscale. A is n*n column-major, in place.
 * Returns the LAPACK info. */
int oracle_dense_inv(int n, double* A);

/* Taylor-expansion inverse of a dense N*N column-major Z (compute.cpp:121-166):
 * Z <- Z + lambda*I, X = inv(Z), iZ = X + sum_i lambda^i/(i-1)! X^(i+1).
 * Z is overwritten with iZ. */
int oracle_te_inverse(int n, double* Z, double lambda, oracle_stats* st);

/* Cholesky route of the dense inverse (not in the reference; a second FP64
 * route that measures how far two correct inverses of the same ill-conditioned
 * Z + lambda*I lie apart): E = diag(A)^-1/2, A_s = E A E, dpotrf + dpotri,
 * A^-1 = E A_s^-1 E. A is n*n column-major, in place (both triangles).
 * Returns the LAPACK info. */
int oracle_dense_inv_cholesky(int n, double* A);

/* oracle_te_inverse with the inverse route chosen (0 LU, 1 Cholesky). */
int oracle_te_inverse_route(int n, double* Z, double lambda, int route, oracle_stats* st, int swap_products);

/* One dense product of the Taylor loop (operator*=, ScaledDenseMatrix.cpp:314-353:
 * row and column scaling of A, dgemm, unscaling): C = A * B, all n*n
 * column-major. For timing samples of the dense stage. */
void oracle_gemm(int n, const double* A, const double* B, double* C);

/* Number of BLAS threads used by the oracle after set-up. */
int oracle_set_threads(int threads);

#ifdef __cplusplus
}
#endif
