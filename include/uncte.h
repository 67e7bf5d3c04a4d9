/*
 * uncte.h - C ABI of the B200 (sm_100a) covariance-propagation library
 * (libuncte.so). Plain C types only: pointers, sizes and status codes.
 *
 * Each entry point names the uncertaintyTE interface it replaces (paths are
 * relative to the uncertaintyTE source tree). The C++ drop-in header
 * include/uncertainty.h forwards to these functions.
 *
 * Layout contract (same as the reference): the Jacobian is a Ceres CRS
 * matrix whose columns are [9*numCams camera params | 3*numPoints point
 * params]; every observation is two consecutive rows of 12 entries (9 camera
 * columns then 3 point columns, ascending). Outputs are caller-allocated:
 * cam_unc[numCams*45] (row-major upper triangle of each 9x9 block) and
 * pt_unc[numPoints*6] (00,01,02,11,12,22 of each 3x3 block).
 *
 * All functions are synchronous with respect to the host unless the name
 * ends in _async. Errors are returned, never exit()ed.
 */
#ifndef UNCTE_H
#define UNCTE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define UNC_OK 0
#define UNC_ERR_INVALID_ARG (-1)   /* null pointer, negative size, inconsistent options */
#define UNC_ERR_LAYOUT (-2)        /* Jacobian is not in the 2-row x 12-entry observation layout */
#define UNC_ERR_NO_FIXED_POINTS (-3) /* TAYLOR_EXPANSION needs three fixed points */
#define UNC_ERR_CUDA (-4)          /* CUDA runtime error (message: unc_last_error) */
#define UNC_ERR_OUT_OF_MEMORY (-5) /* device allocation failed / request above the HBM budget */
#define UNC_ERR_SINGULAR (-6)      /* non-positive pivot or non-finite value in the dense inverse */
#define UNC_ERR_UNSUPPORTED (-7)   /* option combination not implemented (message: unc_last_error) */
#define UNC_ERR_TOO_LARGE (-8)     /* size above a documented limit */
#define UNC_ERR_TIMEOUT (-9)       /* unc_server_wait: the request is still running */

/* algorithm selector, same values as include/uncertainty.h:11-13 */
#define UNC_SVD_QR_ITERATION 0
#define UNC_SVD_DEVIDE_AND_CONQUER 1
#define UNC_TAYLOR_EXPANSION 2
/* This library's extension (no counterpart in the reference): the SVD
 * pseudo-inverse of the camera Schur complement Z of the full J^T J (no fixed
 * points) instead of the full J^T J, for scenes whose (9C + 3P)^2 matrix does
 * not fit; point covariances then come from the point stage of the Taylor
 * path. The gauge is the minimum-norm one in camera coordinates. */
#define UNC_SVD_SCHUR 3

/* precision of the dense Taylor-series products */
#define UNC_PRECISION_FP64 0    /* plain FP64 (DMMA) products: the parity path */
#define UNC_PRECISION_MIXED 1   /* int8-sliced tensor-core products, 5 slices (~1e-10 per product) */
#define UNC_PRECISION_MIXED4 2  /* same with 4 slices (~1e-8 per product, faster) */
#define UNC_PRECISION_MIXED3 3  /* same with 3 slices (~1e-6 per product) */

/* How the Taylor series of teInverse (compute.cpp:141-160) is evaluated; both
 * give the reference's polynomial, coefficients and stop decisions.
 * POWERS: from X^2, X^3, X^4, X^8, X^12 (X^16 past 15 iterations): the stop
 * rule's max|X^(i+1)| is the largest diagonal entry of the SPD power, a column
 * dot product of two lower powers, and the sum is formed in blocks of four
 * coefficients (8 products for up to 15 iterations). SEQUENTIAL: one product
 * per iteration, the reference's order. */
#define UNC_TAYLOR_POWERS 0
#define UNC_TAYLOR_SEQUENTIAL 1

typedef struct unc_context unc_context;

/* Mirrors cov::Options (src/uncertaintyTE/uncertainty.h:52-71) as plain C. */
typedef struct {
    int algorithm;      /* UNC_SVD_QR_ITERATION / UNC_SVD_DEVIDE_AND_CONQUER / UNC_TAYLOR_EXPANSION */
    double epsilon;     /* SVD: singular-value threshold when svd_remove_n == -1 */
    double lambda;      /* TE regulariser, -1 = automatic 10^(-1.2653 log10 N - 2.9415) */
    int num_cams, cam_params, num_points, num_obs;
    int svd_remove_n;   /* SVD: number of smallest singular values dropped (-1 = use epsilon) */
    int max_iter_te;    /* unused by the reference (-1); kept for layout parity */
    int pts2fix[3];     /* fixed point ids (TE); only the first two are sorted, as the reference does */
    int has_pts2fix;    /* 0 = no fixed points given */
    int precision;      /* UNC_PRECISION_FP64 / _MIXED / _MIXED4 / _MIXED3 */
    int taylor_eval;    /* UNC_TAYLOR_POWERS (0, default) / UNC_TAYLOR_SEQUENTIAL */
} unc_options;

/* Mirrors cov::Statistic (src/uncertaintyTE/uncertainty.h:73-82). Times are
 * true seconds measured with CUDA events (the reference prints ms/100). */
typedef struct {
    double time_create_j, time_fix_j, time_norm_j, time_multiply_jj, time_split_jj, time_inv_v,
        time_compose_z, time_inv_z, time_te, time_pts_unc, time_all;
    double lambda;
    int fixed_pts[3];
    int te_iterations;        /* == cycle_change.size() in the reference */
    double cycle_change[20];
    long long device_bytes;   /* device workspace used by the call */
} unc_statistic;

/* Fill *opt with the reference's defaults: TAYLOR_EXPANSION, epsilon 1e-10,
 * lambda -1, svd_remove_n -1, max_iter_te -1, 9 camera parameters
 * (cov::Options::Options(numCams, camParams, numPoints, numObs),
 * src/uncertaintyTE/uncertainty.h:62-63). */
void unc_options_init(unc_options* opt, int num_cams, int cam_params, int num_points, int num_obs);

/* A context owns a CUDA device, a stream and a growable device workspace
 * that is reused across calls. Not thread-safe: one context per thread. */
int unc_context_create(int device, unc_context** ctx);
int unc_context_destroy(unc_context* ctx);

/* computeCovariances(options, statistic, jacobian, camUnc, ptUnc)
 * (src/uncertaintyTE/compute.h:92-97, compute.cpp:458-540).
 * Host pointers in and out; ctx may be NULL (a temporary context on device 0
 * is created and destroyed). stat may be NULL. Arrays in ordinary (pageable)
 * host memory of 8 MB or more are copied through a 64 MB pinned ring that the
 * context allocates at its first such copy and frees when it is destroyed;
 * pinned or registered arrays are copied directly. */
int unc_compute(unc_context* ctx, const unc_options* opt, int num_rows, int num_cols,
                const int* rows, const int* cols, const double* values, double* cam_unc,
                double* pt_unc, unc_statistic* stat);

/* Same computation with every array already in device memory (inputs
 * resident in HBM). stream: a cudaStream_t or NULL for the context's stream.
 * pt_unc follows the reference's zeroing rule (compute.cpp:511): entries
 * [0, 6*(numPoints-3)) are cleared and fixed points beyond that keep their
 * previous contents. Returns after the results are written. */
int unc_compute_device(unc_context* ctx, const unc_options* opt, int num_rows, int num_cols,
                       const int* d_rows, const int* d_cols, const double* d_values,
                       double* d_cam_unc, double* d_pt_unc, unc_statistic* stat, void* stream);

/* Profiling of the dense Taylor-series products: when enabled, every
 * N x N x N product of the Taylor loop is bracketed by CUDA events on the
 * stream it runs on. unc_context_profile returns the number of products, their
 * summed device time (s) and their algorithmic flops since the last reset.
 * The powers of the symmetric inverse are symmetric, so a product computes
 * its lower triangle only: N^2 (N + 1) flops (the reference spends 2 N^3). */
int unc_context_set_profiling(unc_context* ctx, int enable);
int unc_context_profile(unc_context* ctx, long long* launches, double* seconds, double* flops,
                        int reset);
/* Mixed modes: the int8 multiply-adds x 2 those products issued (tile padding
 * included; each product with its own slice count). Read it before a reset. */
int unc_context_profile_int8(unc_context* ctx, double* int8_ops);

/* Device bytes unc_compute_device would use for this problem (admission). */
long long unc_workspace_bytes(const unc_options* opt, int num_rows, int num_cols);

/* The Jacobian of the reprojection residuals built on the GPU from the scene,
 * replacing Ceres Evaluate (src/uncertaintyTE/JacobianComposer.cpp:123-166,
 * src/matlab/matlabInterface.cpp:182-200) for the SnavelyReprojectionError
 * camera (snavely_reprojection_error.h:309-350, unit parameter weights):
 * cams 9 per camera [angle-axis, centre, f, k1, k2], points 3 per point,
 * observation camera / point ids. Writes the reference CRS layout (rows
 * 2 num_obs + 1, cols / values 24 per observation: 9 camera then 3 point
 * columns per row), all device pointers; synchronous. */
int unc_jacobian_device(int num_cams, int num_points, int num_obs, const double* d_cams, const double* d_points,
                        const int* d_obs_cam, const int* d_obs_pt, int* d_rows, int* d_cols, double* d_values,
                        void* stream);
/* computeCovariances from the scene on host arrays (opt->num_obs
 * observations): only cameras, points and observation ids cross PCIe, the
 * Jacobian is built on the device (unc_jacobian_device), then the same
 * pipeline as unc_compute. */
int unc_compute_scene(unc_context* ctx, const unc_options* opt, const double* cams, const double* points,
                      const int* obs_cam, const int* obs_pt, double* cam_unc, double* pt_unc, unc_statistic* st);

/* Eigen-decompositions of many small covariance blocks (the Uncertainty
 * accessors, src/uncertaintyTE/uncertainty.cpp:74-183), one warp per block:
 * packed upper triangles of block_params x block_params blocks (45 values for
 * 9 camera parameters, 6 for points), sub-block [sub_offset, sub_offset +
 * sub_dim) of each (the camera centre: 3, 3). Eigenvalues descending
 * (sub_dim per block); eigenvectors (optional, NULL to skip) as columns in the
 * same order, sub_dim x sub_dim per block, column-major. _device: device
 * pointers; the other form takes host arrays. block_params <= 9. */
int unc_block_eigen_device(const double* d_packed, int num_blocks, int block_params, int sub_offset, int sub_dim,
                           double* d_values, double* d_vectors, void* stream);
int unc_block_eigen(const double* packed, int num_blocks, int block_params, int sub_offset, int sub_dim,
                    double* values, double* vectors);

/* ---- .jacob input (src/uncertaintyTE/JacobianIO.cpp:32-63) ----
 * Header of a text .jacob file or of its binary form (this library's: a
 * 64-byte header starting "UNCJACB1", then the three arrays as stored in
 * memory). The text body is parsed by all host threads. Errors:
 * UNC_ERR_INVALID_ARG with unc_last_error(). */
typedef struct {
    double lambda;
    int num_cams, cam_params, num_points, num_obs;
    int pts2fix[3];     /* -1 -1 -1: none */
    int num_rows, num_cols;
    long long nnz;
    int binary;         /* 1: the binary form */
} unc_jacob_header;
int unc_jacob_read_header(const char* path, unc_jacob_header* header);
/* rows: num_rows + 1, cols / values: nnz (caller-allocated). */
int unc_jacob_read(const char* path, const unc_jacob_header* header, int* rows, int* cols, double* values);
int unc_jacob_write_binary(const char* path, const unc_jacob_header* header, const int* rows, const int* cols,
                           const double* values);

/* Device bytes one unc_compute call needs for this Jacobian (host arrays):
 * the workspace with the input copies, the Schur pair list (counted from the
 * point columns of the rows) and the int8 slices of the mixed modes. -1 for
 * invalid options. No counterpart in the reference (admission control). */
long long unc_request_bytes(const unc_options* opt, int num_rows, int num_cols, const int* rows,
                            const int* cols);

/* Device buffers a context keeps between calls: their size, and a release
 * (the next call allocates again). No counterpart in the reference. */
long long unc_context_device_bytes(const unc_context* ctx);
int unc_context_release(unc_context* ctx);
/* Run the context's work on the device's highest-priority stream (high != 0)
 * or a default-priority one: latency-sensitive small requests next to large
 * ones. No counterpart in the reference. */
int unc_context_set_priority(unc_context* ctx, int high);

/* ---- Request server: many reconstructions on one GPU (no counterpart in the
 * reference, which computes one reconstruction per call and is not
 * re-entrant, src/uncertaintyTE/compute.cpp:461-468).
 * max_inflight worker threads, each with its own context (stream and reused
 * workspace), run requests concurrently; a request starts when a worker is
 * free and its unc_request_bytes fit in max_device_bytes (<= 0: 90 % of the
 * free device memory at creation) next to the running requests and the
 * workspaces idle workers hold (each worker keeps one for single requests and
 * one for packs of small requests; idle ones are freed when that makes room).
 * The host arrays of
 * a request (Jacobian in, covariances out) must stay valid until
 * unc_server_wait has returned its result. Results do not depend on what else
 * runs. Thread-safe. */
typedef struct unc_server unc_server;
int unc_server_create(int device, long long max_device_bytes, int max_inflight, unc_server** out);
/* Queue one computeCovariances; *id identifies it. UNC_ERR_OUT_OF_MEMORY when
 * the request alone exceeds the budget; option errors as unc_compute. */
int unc_server_submit(unc_server* srv, const unc_options* opt, int num_rows, int num_cols, const int* rows,
                      const int* cols, const double* values, double* cam_unc, double* pt_unc, long long* id);
/* Wait up to timeout_s seconds (< 0: no limit) for request id; UNC_OK when it
 * finished (its own status in *status, statistics, submit-to-finish latency and
 * queueing time in seconds), UNC_ERR_TIMEOUT when it still runs. A finished
 * request is collected once. */
int unc_server_wait(unc_server* srv, long long id, double timeout_s, int* status, unc_statistic* st,
                    double* latency_s, double* queue_s);
/* Finish every queued and running request, then stop the workers. */
int unc_server_destroy(unc_server* srv);

/* ---- Batches: many reconstructions in one grouped launch sequence. No
 * counterpart in the reference, whose computeCovariances
 * (src/uncertaintyTE/compute.cpp:458-540) solves one reconstruction per call
 * and is not re-entrant; unc_batch_compute is that call over num_scenes scenes
 * at once. The inputs of all scenes go to the device in one copy; the sparse
 * stages of the scenes run as parallel branches, the dense stage is grouped
 * (one persistent tile-task kernel inverts every scene's Schur complement,
 * each step of the Taylor series is one launch over all scenes); the
 * sequence of a batch shape (sizes, fixed points, lambda) is captured in a
 * CUDA graph the second time it is seen and replayed after. The product tile
 * width is chosen by timing the candidates on the first batch of a size class.
 * Each scene's result is bitwise the one unc_compute gives for it alone.
 * Scenes outside the grouped path (the SVD algorithms, UNC_PRECISION_FP64,
 * UNC_TAYLOR_SEQUENTIAL, 9 * num_cams above 3584, Jacobians not in the
 * 24-entries-per-observation layout) are computed with unc_compute in the
 * same call.
 * Per scene i: opts[i], the host CRS arrays and the host outputs as for
 * unc_compute; status[i] receives the scene's own status code; stats (NULL or
 * num_scenes entries) the statistics (time_all: the whole batch's time). The
 * call returns UNC_OK unless the batch itself could not run. A batch object is
 * not thread-safe. */
typedef struct unc_batch unc_batch;
int unc_batch_create(int device, unc_batch** out);
int unc_batch_destroy(unc_batch* batch);
int unc_batch_compute(unc_batch* batch, int num_scenes, const unc_options* opts, const int* num_rows,
                      const int* num_cols, const int* const* rows, const int* const* cols,
                      const double* const* values, double* const* cam_unc, double* const* pt_unc, int* status,
                      unc_statistic* stats);
/* Times of the last unc_batch_compute (seconds): the input copy, the device
 * work of the grouped scenes, the output copy; how many scenes were grouped
 * and the product tile width used. */
int unc_batch_last_timing(const unc_batch* batch, double* h2d_s, double* device_s, double* d2h_s,
                          int* grouped_scenes, int* tile_n);
/* Device bytes a batch object keeps between calls, and their release (the
 * next call allocates again). */
long long unc_batch_device_bytes(const unc_batch* batch);
int unc_batch_release(unc_batch* batch);
/* Product tile width of the 5-slice grouped products: 0 (default) picks 64 or
 * 96 by a cost model of the tiles on the SMs; 64 or 96 force it. Results do
 * not depend on it (bitwise). */
int unc_batch_set_tile_width(unc_batch* batch, int tile_n);

/* SDM::inv (src/uncertaintyTE/ScaledDenseMatrix.cpp:232-279) for a
 * symmetric positive-definite n x n matrix in device memory (column-major,
 * leading dimension lda >= n, lda even): inverted in place on the GPU
 * (equilibration, Cholesky with L^-1 formed on the way, then L^-T L^-1; for
 * n <= 3584 as 64 x 64 tile tasks in one persistent kernel, above by
 * recursion on halves). Scratch is allocated per call. */
int unc_dense_inverse_device(double* d_A, int n, int lda, void* stream);

/* The pseudo-inverse step of svdInverse (src/uncertaintyTE/compute.cpp:200-245)
 * for a symmetric positive semi-definite n x n matrix in device memory
 * (column-major, ld >= n, ld even), in place: the remove_n smallest singular
 * values are dropped (remove_n in 0..31), or with remove_n == -1 every
 * singular value <= epsilon (at most 20 of them). Only the dropped
 * eigenvectors are computed (subspace iteration on the shifted inverse), the
 * rest follows from one Cholesky inverse of the matrix with those directions
 * lifted and a two-sided projection. UNC_ERR_SINGULAR when a kept eigenvalue is
 * not positive. Scratch (4 n x ld matrices) is allocated per call. */
int unc_pinv_psd_device(double* d_M, int n, int ld, int remove_n, double epsilon, void* stream);

/* The SPD inverse of unc_dense_inverse_device (its recursive form), for callers that cannot
 * let a library allocate device memory (their device memory is reserved by
 * their own pool allocator, or cudaMalloc/cudaFree would stall a latency-
 * critical loop). No counterpart in the reference. It allocates nothing: its
 * scratch is a fixed __device__ array of about 6.3 MB held by every device the
 * library is loaded on, so n and lda are limited to 512 (UNC_ERR_TOO_LARGE
 * beyond). All calls on a device share that array; calls that overlap on the
 * GPU race. The first call on a device looks up the array's address (again
 * after a device reset); make it before any stream capture. Synchronous, like
 * unc_dense_inverse_device. */
int unc_dense_inverse_noalloc(double* d_A, int n, int lda, void* stream);

/* Diagnostics of the tile-task form of unc_dense_inverse_device (n <= 3584):
 * the same inverse with the dependency waits limited to poll_limit polls each
 * (1..2^22; the regular calls use 2^22) and, when skip_task >= 0, that task
 * (an index of the unc_spd_task_list order) left out of the schedule. Every
 * wait of the persistent kernel is bounded: a wait that runs out raises an
 * abort flag that all CTAs check, the launch drains and the call returns
 * UNC_ERR_CUDA ("bounded device wait ... ran out") instead of hanging, and the
 * device stays usable. A schedule with a task left out cannot complete, which
 * is how a test makes a wait run out. No counterpart in the reference. */
int unc_spd_inverse_tasks_bounded(double* d_A, int n, int lda, long long poll_limit, int skip_task, void* stream);

/* The order in which the tile-task form of unc_dense_inverse_device (n <= 3584)
 * runs its 64 x 64 tile tasks; no counterpart in the reference (its inverse is
 * LAPACK's). For tools that check or draw the schedule. Returns the number of
 * tasks (UNC_ERR_INVALID_ARG outside 1..3584); when out is non-NULL and
 * capacity is at least that number, out receives 4 ints per task: the kind
 * (0 diagonal factorisation with its fused update and next solve, 1 triangular
 * solve, 2 trailing update, 3 inverse accumulation, 4 inverse finish, 5 product
 * accumulation) and the tile indices i, j, k. Host only; needs no GPU. */
int unc_spd_task_list(int n, int* out, int capacity);

/* SSM J^T J (trn() then operator*, ScaledSparseMatrix.cpp:384-388,517-539)
 * computed by the GPU block-assembly kernels and returned as host CRS in the
 * reference's pattern. Observations may have 12-entry rows (camera + point)
 * or 9-entry rows (camera only). First call with out_cols == NULL returns
 * the nnz in *nnz; the second call fills out_rows (num_cols+1), out_cols,
 * out_vals. num_cams/cam_params describe the camera column block. */
int unc_jtj_crs(int num_rows, int num_cols, const int* rows, const int* cols, const double* values,
                int num_cams, int cam_params, long long* nnz, int* out_rows, int* out_cols,
                double* out_vals);

/* C = alpha * A * B + beta * C on the library's FP64 tensor-core GEMM (the
 * dense products of the Taylor series, ScaledDenseMatrix.cpp:314-353). All
 * matrices column-major in device memory; lda/ldb/ldc even; rows past M (A)
 * and K (B) up to the next even row must be readable and finite. */
int unc_gemm_f64_device(int M, int N, int K, double alpha, const double* d_A, int lda,
                        const double* d_B, int ldb, double beta, double* d_C, int ldc, void* stream);

/* C = P * X for symmetric n x n FP64 matrices P and X (column-major, leading
 * dimension ld) on the tensor cores: both operands are split into `slices`
 * (3..5) 7-bit integer slices with power-of-two row scales, the slice
 * products run as tcgen05 int8 GEMMs with exact int32 accumulation, and the
 * levels are combined in FP64 (relative error about 2^(-7 slices) of the row
 * and column maxima). The mixed-precision Taylor products use this kernel.
 * Scratch is allocated per call. */
int unc_gemm_mixed_device(int n, const double* d_P, const double* d_X, int ld, double* d_C, int slices,
                          void* stream);
/* A = T^T T (n x n, column-major, leading dimension ld for both) for a lower
 * triangular T (zero above the diagonal) on the tensor cores: the columns of
 * T split into 7 int8 slices, lower 128 x 64 tiles whose k loops start at the
 * tile's first nonzero row, the result written in both triangles (per term an
 * error of about 2^-50 of the two columns' maxima, zero-mean). The last product of the mixed
 * modes' SPD inverse above N = 3584 (A^{-1} = L^{-T} L^{-1}). Scratch is
 * allocated per call. */
int unc_gram_lower_mixed_device(int n, const double* d_T, int ld, double* d_A, void* stream);

/* Human-readable name of a status code, and the last error message of the
 * calling thread (empty when none). */
const char* unc_status_string(int status);
const char* unc_last_error(void);

/* Number of this library's kernels launched since load (diagnostics). */
long long unc_kernel_launches(void);

#ifdef __cplusplus
}
#endif
#endif /* UNCTE_H */
