// internal.h - shared declarations of the uncertaintyTE B200 kernels.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/uncte.h"

namespace unc {

// Device-side error bits (accumulated with atomicOr into a device int).
enum : int {
    ERRBIT_LAYOUT = 1,      // observation rows not 12 entries / columns out of range
    ERRBIT_SINGULAR = 2,    // non-positive or non-finite pivot
    ERRBIT_NONFINITE = 4,   // NaN / Inf produced
    ERRBIT_SORT_CAP = 8,    // a segment was too long to sort (order left nondeterministic)
    ERRBIT_TIMEOUT = 16,    // a bounded device wait ran out (tensor-core pipeline)
    ERRBIT_SCHUR_CAP = 32,  // an observation has more Schur partners than one chunk holds (Z incomplete)
};

constexpr int kCamParams = 9;
constexpr int kObsVals = 24;  // one observation = 2 rows x (9 camera + 3 point) values

// Round a leading dimension up so every column starts 64-byte aligned.
inline int ld_of(int n) { return (n + 7) & ~7; }

extern thread_local std::string g_last_error;

// Streaming multiprocessors of the current device (queried once per device;
// 148 on a B200, fewer on a partitioned GPU).
int device_sms();

// Runs f() (returning true on success) until it succeeds once per device
// (ordinal < 64) for one call site, from any thread: per-function CUDA
// attributes are per device, and several host threads (one per context) may
// launch the same kernels concurrently. prepare_kernels() runs every such site
// when a context is created, outside any stream capture.
template <class F>
void once_per_device(std::atomic<unsigned long long>& done, F&& f) {
    int dev = 0;
    cudaGetDevice(&dev);
    const unsigned long long bit = 1ULL << (dev & 63);
    if (done.load(std::memory_order_acquire) & bit) return;
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    if (done.load(std::memory_order_relaxed) & bit) return;
    if (f()) done.fetch_or(bit, std::memory_order_release);
}
// Per-device set-up of the kernels' shared-memory attributes (current device).
void prepare_assembly_kernels();
void prepare_dense_kernels();
void prepare_mixed_kernels();

// Bump allocator over one device allocation; every piece 256-byte aligned.
// With base == nullptr it only measures the total size.
struct Carver {
    char* base;
    size_t off = 0;
    template <class T>
    T* take(size_t n) {
        off = (off + 255) & ~size_t(255);
        T* p = reinterpret_cast<T*>(base ? base + off : nullptr);
        off += n * sizeof(T);
        return p;
    }
};
extern long long g_launches;
extern thread_local long long g_thread_launches;
inline void count_launch(int n = 1) {
    __atomic_add_fetch(&g_launches, n, __ATOMIC_RELAXED);
    g_thread_launches += n;
}

// ---------------- assembly.cu ----------------
struct SceneDev {
    int num_cams, num_points, num_obs;  // num_obs = num_rows / 2
    long nnz;                           // entries of cols / values
    int fix[3];
    int has_fix;
    const int* rows;      // CRS rowptr
    const int* cols;      // CRS column ids
    const double* J;      // observation blocks, 24 doubles each: [row0: c0..c8 p0..p2 | row1: ...]
    int* obs_cam;         // per observation camera id (-1 = dropped)
    int* obs_pt;          // per observation point id (-1 = dropped: fixed point or no point)
    int* cam_ptr;         // num_cams + 1
    int* cam_obs;         // observation ids grouped by camera (ascending within a camera)
    int* pt_ptr;          // num_points + 1
    int* pt_obs;          // observation ids grouped by point (ascending within a point)
    int* cursor;          // scratch: max(num_cams, num_points) + 1 ints
    int* scan_tmp;        // scratch for the scan
    double* s_cam;        // 9*num_cams column norms of J (camera columns)
    double* s_pt;         // 3*num_points column norms (point columns)
    double* Vraw;         // 6*num_points upper triangle of the unscaled point block J_p^T J_p
    double* iVs;          // 6*num_points upper triangle of the inverse of the scaled point block
    double* Ws;           // 27*num_obs scaled W_o = (J_c^T J_p)/(s s), 9x3 row-major
    double* Ys;           // 27*num_obs Y_o = W_o * iV_p, 9x3 row-major
    double* cam_part;     // 45 * camera_tile_slots(): per-tile partial sums of the camera blocks
    double* Ucam;         // 81*num_cams scaled camera blocks U (9 x 9, column-major)
    int* err;             // device error bits
};

void launch_validate_obs(const SceneDev& s, cudaStream_t st);
// Camera observations are processed in tiles of 256; slots = C + num_obs/256 + 1.
size_t camera_tile_slots(int num_cams, int num_obs);
void launch_build_index(SceneDev& s, cudaStream_t st);
// U blocks (scaled) into s.Ucam, column norms into s.s_cam.
void launch_camera_blocks(const SceneDev& s, cudaStream_t st);
void launch_point_blocks(const SceneDev& s, cudaStream_t st);
void launch_obs_blocks(const SceneDev& s, cudaStream_t st);
// The Schur complement Z = U - W V^-1 W^T (schur.cu) over a zeroed Z: the
// diagonal blocks from s.Ucam, every co-visible camera-pair block written in
// both triangles, bitwise symmetric. UNC_ERR_TOO_LARGE above kSchurMaxCams.
constexpr int kSchurMaxCams = 5120;  // above the dense path's limit (9 C <= 46000)
int launch_schur_columns(const SceneDev& s, double* Z, int ldz, cudaStream_t st);
size_t schur_columns_smem(int num_cams);
void prepare_schur_columns();  // kernel attributes (before any stream capture)
// Generic 9/12-entry-row repack for the J^T J export (camera-only rows allowed).
void launch_repack_generic(int num_obs, int cam_off, const int* rows, const int* cols,
                           const double* vals, double* J, int* obs_cam, int* obs_pt, int* err,
                           cudaStream_t st);
void launch_unscaled_blocks(const SceneDev& s, double* U, double* W, cudaStream_t st);
void exclusive_scan(const int* in, int* out, int n, int* tmp, cudaStream_t st);
size_t scan_tmp_ints(int n);

// ---------------- dense.cu ----------------
// C = alpha*A*B + beta*C, column-major, FP64 on DMMA. If amax != nullptr the
// epilogue folds max|C| into *amax (bit pattern of a non-negative double).
void gemm_f64(int M, int N, int K, double alpha, const double* A, int lda, const double* B,
              int ldb, double beta, double* C, int ldc, unsigned long long* amax, cudaStream_t st);
// General form: lower_only skips output tiles strictly above the diagonal
// (symmetric results; mirror afterwards with launch_mirror_lower).
// trans_b: B(k, n) is read from B[n + k * ldb] (the transpose of a column-major matrix).
void gemm_f64_ex(int M, int N, int K, double alpha, const double* A, int lda, const double* B, int ldb,
                 double beta, double* C, int ldc, unsigned long long* amax, bool lower_only, cudaStream_t st,
                 bool trans_b = false);
// Mode bits of gemm_f64_mode. The k-range bits restrict the k loop of the
// output tile at (m0, n0) when an operand is triangular (terms outside the
// range are zero): KLO_M k >= m0, KLO_N k >= n0, KHI_M k < m0 + 128,
// KHI_N k < n0 + 128 (tile size 128 x 128).
enum : int {
    GEMM_LOWER = 1,
    GEMM_TRANS_B = 2,
    GEMM_KLO_M = 4,
    GEMM_KLO_N = 8,
    GEMM_KHI_M = 16,
    GEMM_KHI_N = 32,
    GEMM_MIRROR = 64,  // symmetric C: write the lower triangle at (i, j) and (j, i), nothing above it directly
    GEMM_SHORT_ACC = 128,  // partial sums over k = 8 from zero, added with ordinary FP64 additions (the
                           // products that feed Cholesky pivots: see k_gemm_f64)
};
// ws (ws_doubles): optional scratch that enables split-K for outputs with
// fewer tiles than SMs (partials summed in a fixed order by a second kernel).
// skip: optional device flag; when it is non-zero the kernels return at once
// (the Taylor loop launches all its iterations and stops on the device).
void gemm_f64_mode(int M, int N, int K, double alpha, const double* A, int lda, const double* B, int ldb,
                   double beta, double* C, int ldc, unsigned long long* amax, int mode, cudaStream_t st,
                   double* ws = nullptr, size_t ws_doubles = 0, const int* skip = nullptr);
void launch_mirror_lower(double* Z, int n, int ld, cudaStream_t st, const int* skip = nullptr);
// Same, skipping output tiles strictly above the diagonal (symmetric updates).
void gemm_f64_tri(int M, int N, int K, double alpha, const double* A, int lda, const double* B, int ldb,
                  double beta, double* C, int ldc, cudaStream_t st);
// In-place inverse of an SPD matrix (n x n, lda): recursive Cholesky that
// forms T = L^{-1} directly (64 x 64 leaves, GEMM merges), then A^{-1} = T^T T.
// T, W, Tt: n x lda scratch matrices, all finite, T zero on entry; small:
// chol_small_doubles(n) doubles (unused by the recursive form, kept for the
// workspace layout). Sets ERRBIT_SINGULAR in err.
size_t chol_small_doubles(int n);
void chol_inverse(double* A, int n, int lda, double* T, double* W, double* Tt, double* small, int* err,
                  cudaStream_t st);
// The recursion of chol_inverse alone: T = L^{-1} (lower triangle; T zero on
// entry), A overwritten; ws: n x lda doubles of split-K scratch.
void chol_lower_inverse(double* A, int n, int lda, double* T, double* W, double* ws, int* err, cudaStream_t st);
// A <- A + lambda*I and symmetric Jacobi equilibration: A_s = E A E, E = diag(A_ii)^-1/2.
void launch_shift_equilibrate(double* A, int n, int lda, double lambda, double* e, int* err,
                              cudaStream_t st);
// X <- E X E (undo equilibration), also copies into Y if Y != nullptr.
void launch_unequilibrate(double* X, int n, int lda, const double* e, double* Y, cudaStream_t st);
// X = diag(e) S diag(e) from a separate source S, Y (optional) = X.
void launch_unequilibrate_from(const double* S, double* X, int n, int lda, const double* e, double* Y,
                               cudaStream_t st);

// ---------------- dag.cu ----------------
// SPD inverse as 64 x 64 tile tasks in one persistent kernel, for n <= 3584:
// A (lower triangle) is overwritten by L, T receives L^{-1} (lower tiles) and
// O = A^{-1} (both triangles). state: spd_task_state_ints(n) ints.
// spd_tasks_prepare uploads the task list of this size once per device (call it
// outside stream capture).
bool spd_tasks_apply(int n);
size_t spd_task_state_ints(int n);
int spd_tasks_prepare(int n);
// max_ctas bounds the persistent grid (at most one CTA per SM is used anyway);
// the task order and every tile's update order do not depend on it, so neither
// do the results.
// poll_limit (> 0): polls of one dependency before a wait gives up (default
// and maximum 2^22); skip_task >= 0 leaves that task out of the schedule, which
// can then not complete: only for tests of the bounded waits.
int chol_inverse_tasks(double* A, int n, int lda, double* T, double* O, int* state, int* err, cudaStream_t st,
                       int max_ctas = 148, long long poll_limit = 0, int skip_task = -1);
// One matrix of a grouped tile-task inverse: A (lower triangle) becomes L, T
// receives L^{-1}, O = A^{-1}; state: spd_task_state_ints(n) zeroed ints; err:
// the matrix's error word.
struct SpdTaskMatrix {
    double *A, *T, *O;
    long ld;
    int n, ntri;
    int* state;
    int* err;
};
// The interleaved task list of matrices of sizes ns (each <= 3584): every
// matrix's own order kept, merged by fractional position so that all matrices
// progress together; task.x = type + 8 * matrix index.
std::vector<int4> spd_tasks_grouped_list(const std::vector<int>& ns);
// Shared-memory attributes of the tile-task kernels (current device; call it
// outside any stream capture).
void prepare_task_kernels();
// One persistent launch over the list (d_mats / d_tasks in device memory; ctl:
// 2 ints, zeroed by the caller in stream order, as is every matrix's state).
int chol_inverse_tasks_grouped(const SpdTaskMatrix* d_mats, const int4* d_tasks, int ntasks, int* ctl,
                               cudaStream_t st, int max_ctas, long long poll_limit = 0);
// per context: the largest grid of the tile-task inverse (148 unless set)
void context_set_task_ctas(unc_context* c, int max_ctas);
// Y <- Y + k*X  (N x N, column-major)
void launch_axpy(double* Y, const double* X, double k, int n, int ld, cudaStream_t st);

// Device-side control of the Taylor loop (compute.cpp:141-160): the stop rule
// runs on the device so that the host never waits inside the loop.
struct TeState {
    int done;               // the loop has stopped: later iteration kernels return at once
    int bad;                // a power was not finite
    int iters;              // iterations performed
    double old_change;      // previous |k * max|add||
    double coef;            // k of the current iteration (read by the axpy)
    double change[20];      // cycle_change record
    // blocked-power evaluation (powers.cu): the series' coefficients c[0] = 1,
    // c[i] = k_i for the performed iterations, 0 after; skip[0]: X^16 is not
    // needed, skip[q] (q = 1..4): the block X^(4q) G_q is zero
    double c[20];
    int skip[8];
};
// One thread: change = |k * max(amax, DBL_MIN)|; stop when change < 1e-5 or
// change > old_change, else record it and publish k for the axpy.
void launch_te_decide(TeState* s, const unsigned long long* amax, double k, cudaStream_t st);
// Reset the state (not done, no iteration, old change = DBL_MAX).
void launch_te_init(TeState* s, cudaStream_t st);
// ---------------- powers.cu ----------------
// The Taylor series iZ = X + sum_{i=1..m} k_i X^(i+1) (compute.cpp:141-160)
// evaluated from the powers X^2, X^3, X^4, X^8, X^12 (X^16 when m >= 15):
// the stop rule's max|X^j| is the largest diagonal entry of the SPD power X^j,
// the dot product of columns of two lower powers; the sum is formed in blocks
// iZ = G_0 + X^4 G_1 + X^8 G_2 + X^12 G_3 + X^16 G_4, G_q = sum_r c_(4q+r) X^(r+1).
// 8 products for m <= 15 instead of m + 1.
struct PowerSet {
    double* M[7];  // X, X^2, X^3, X^4, X^8, X^12, X^16
    double *iZ, *G;
    int n;
    long ld;
    unsigned long long* dmax;  // 21 words: max diag of X^j, j = 0..20 (bits of a non-negative double)
    TeState* te;
};
// Slices of the int8-sliced products of the blocked-power evaluation (mixed
// modes with S slices). Product q: 0..5 = X^2, X^3, X^4, X^8, X^12, X^16;
// 6..9 = X^4 G_1, X^8 G_2, X^12 G_3, X^16 G_4 (counts kept for the int8
// product entry points; the solves form these four on the camera blocks in
// FP64, launch_taylor_blocks). Z is positive semi-definite,
// so the eigenvalues of X = (Z + lambda I)^-1 are at most 1/lambda and the
// series term lambda^i / (i-1)! X^(i+1) = X (lambda X)^i / (i-1)! has norm at
// most ||X|| / (i-1)! (32-bit factorial). G_2 (terms 8..11) therefore adds at
// most 2.3e-4 ||X||, G_3 3e-8 and G_4 1e-8 (the factorial wraps there): their
// products keep the absolute error of the full-slice ones with 2 and 3 slices
// (7 bits each) fewer. X^8, X^12 and X^16 feed only those blocks and the stop
// rule's diagonal maxima (relative error ~2^-28 with one slice fewer). The
// digits are rounded greedily, so the first k slices of an operand are its
// k-slice form: the same slice buffers serve every count.
inline int power_product_slices(int q, int S) {
    const int drop = (q >= 3 && q <= 5) ? 1 : (q == 7 ? 2 : (q >= 8 ? 3 : 0));
    return S - drop < 2 ? (S < 2 ? S : 2) : S - drop;
}
// k[i - 1] = lambda^i / factorial(i - 1), i = 1..19 (host values)
struct TaylorCoefs {
    double k[19];
};
// The powers' diagonal maxima for j in [jlo, jhi] (2..16 or 17..20), unless *skip.
void launch_power_diag(const PowerSet& ps, int jlo, int jhi, const int* skip, cudaStream_t st);
// The stop rule over iterations [ilo, ihi] from the diagonal maxima (a
// non-finite one marks the state bad); the coefficients c[i] of the performed
// iterations; after ilo..15 the X^16 skip word, after ..19 the block skip words.
void launch_power_decide(TeState* te, const unsigned long long* dmax, const TaylorCoefs& k, int ilo, int ihi,
                         cudaStream_t st);
// out = c[4q] X + c[4q+1] X^2 + c[4q+2] X^3 + c[4q+3] X^4 (q = 0: into iZ), unless skipped.
void launch_power_combine(const PowerSet& ps, int q, double* out, const int* skip, cudaStream_t st);
// The 9 x 9 camera blocks of iZ += X^(4q) G_q, q = 1..4 (skipped blocks left out);
// grouped: over the cameras of every set (d_blk_cols: the sets' column offsets).
void launch_taylor_blocks(const PowerSet& ps, cudaStream_t st);
void launch_taylor_blocks_grouped(const PowerSet* d_sets, int nsets, const long* d_blk_cols, long nblk_cols,
                                  cudaStream_t st);
// Grouped forms over many matrices (a batch): one block per column (diag) or
// per 256 elements (combine) of set m with blk[m] <= b < blk[m + 1].
void launch_power_diag_grouped(const PowerSet* d_sets, int nsets, const long* d_blk_cols, long nblk, int jlo,
                               int jhi, bool skip_if_done_early, cudaStream_t st);
// d_k: 19 coefficients per set (set-major)
void launch_power_decide_grouped(const PowerSet* d_sets, int nsets, const double* d_k, int ilo, int ihi,
                                 cudaStream_t st);
void launch_power_combine_grouped(const PowerSet* d_sets, int nsets, const long* d_blk_elems, long nblk, int q,
                                  cudaStream_t st);

// Grouped dense-stage kernels over many matrices (a batch). Element-wise
// launches: block b belongs to job m with blk[m] <= b < blk[m + 1] (blk: njobs
// + 1 longs; 256 threads per block over the job's rows, or n^2 elements).
struct DenseJob {
    double *Z, *iZ, *add, *e;  // Z (in: Schur complement, out: X), iZ (T, then X), add (O = inverse)
    long ld;
    int n;
    double lambda;
    int* err;
    TeState* te;
    const unsigned long long* amax;
};
// Z += lambda I and the symmetric equilibration of every job (as launch_shift_equilibrate).
void launch_shift_equilibrate_grouped(const DenseJob* d_jobs, int njobs, const long* d_blk_rows, long nblk_rows,
                                      const long* d_blk_elems, long nblk_elems, cudaStream_t st);
// Z = E add E, iZ = Z for every job (as launch_unequilibrate_from(add, Z, ..., iZ)).
void launch_unequilibrate_grouped(const DenseJob* d_jobs, int njobs, const long* d_blk_elems, long nblk_elems,
                                  cudaStream_t st);
void launch_te_init_grouped(const DenseJob* d_jobs, int njobs, cudaStream_t st);
// the stop rule of every job with its coefficient d_k[m]
void launch_te_decide_grouped(const DenseJob* d_jobs, int njobs, const double* d_k, cudaStream_t st);
// Y <- Y + s->coef * X unless s->done.
void launch_axpy_te(double* Y, const double* X, const TeState* s, int n, int ld, cudaStream_t st);
void launch_zero(double* p, size_t n, cudaStream_t st);
// Camera output (a+b/2 quirk) and the unscaled 9x9 camera covariance blocks.
void launch_camera_output(const double* iZ, int ldz, const double* s_cam, int num_cams,
                          double* cam_unc, double* sig, cudaStream_t st);

// ---------------- mixed.cu ----------------
// A symmetric FP64 operand sliced into `slices` int8 planes for the tcgen05
// (kind::i8) products, with its TMA descriptor and per-row exponents.
struct MixedOperand {
    CUtensorMap map;
    int8_t* buf;   // slices x rows x kp bytes, zero padding
    int* exps;     // n row exponents
    int n, slices, rows, kp;
};
int mixed_tile_n(int slices, int n);
// int8 multiply-adds x 2 that one lower-triangle product of n x n operands
// issues with `slices` slices (tile padding included).
double mixed_issued_ops(int n, int slices);
size_t mixed_slice_bytes(int n, int slices);
// Prepare the operand over buf/exps (as_b: box rows of the B operand). False
// when the driver's tensor-map encoder is unavailable.
bool mixed_plan(MixedOperand& op, int8_t* buf, int* exps, int n, int slices, bool as_b);
struct TeState;
// Operand planning with an explicit output tile width nt (the B boxes' rows):
// rows padded for both the 128-row A boxes and nt; the slice bytes for it.
bool mixed_plan_nt(MixedOperand& op, int8_t* buf, int* exps, int n, int slices, bool as_b, int nt);
size_t mixed_slice_bytes_nt(int n, int slices, int nt);
// The same sliced operand used with its first `slices` slices only (the digits
// are greedy, so they are the operand's representation with fewer slices):
// same buffer and plane stride; as_b: a B map with that slice count's tile
// width. *ok: false when the tensor map could not be encoded.
MixedOperand mixed_fewer_slices(const MixedOperand& op, int slices, bool as_b, bool* ok);
// Grouped forms for a batch of matrices (arguments in device memory).
struct MixedSliceJob {  // k_slice_rows of one matrix
    const double* A;
    long lda;
    int n, S;
    int8_t* out;
    int rows_pad, kp;
    int* exps;
    double* Y;            // optional Taylor update Y += te->coef * A
    const TeState* te;
    const int* skip;      // optional: return when *skip != 0
};
struct MixedGemmJob {  // one lower-triangle symmetric product C = P X (mirrored)
    const CUtensorMap* tA;  // 64-byte aligned maps in device memory
    const CUtensorMap* tB;
    int n, kp, rowsA, rowsB;
    const int* eA;
    const int* eB;
    double* C;
    long ldc;
    unsigned long long* amax;
    int* err;
    const int* skip;
    int accumulate;  // C += P X
};
// block b of the launch slices row b - row_start[m] of job m (row_start: njobs + 1 ints)
void mixed_slice_grouped(const MixedSliceJob* d_jobs, int njobs, const int* d_row_start, int total_rows,
                         cudaStream_t st);
// the lower-triangle 128 x nt tiles of an n x n product, as (job, m0, n0, 0)
void mixed_lower_tiles(int job, int n, int nt, std::vector<int4>& out);
// tile width of a grouped product over scenes of sizes ns: 128 for up to 4
// slices; for 5, 64 or 96 by the single-scene cost model over all the tiles
int mixed_group_tile_n(int slices, const std::vector<int>& ns);
// A = T^T T (lower tiles, mirrored) for lower-triangular n x n T from
// kGramSlices int8 slices of T's columns; buf holds mixed_gram_bytes(n) bytes
// whose padding is zero, exps n + 64 ints. false: tensor-map encoding failed.
constexpr int kGramSlices = 7;
size_t mixed_gram_bytes(int n);
bool mixed_gram_lower_tri(const double* T, int n, int ld, int8_t* buf, int* exps, double* A, int lda, int* err,
                          cudaStream_t st);
void mixed_gemm_grouped(int slices, int nt, const MixedGemmJob* d_jobs, const int4* d_tiles, int ntiles,
                        cudaStream_t st);
// Y, te (optional): Y += te->coef * A while A is sliced, unless te->done.
void mixed_slice(const double* A, int lda, MixedOperand& op, cudaStream_t st, const int* skip = nullptr,
                 double* Y = nullptr, const TeState* te = nullptr);
// C = P * X from the slices of P (a) and X (b); lower_only: tiles on/below the
// diagonal; mirror: the result's lower triangle is also written transposed
// into the upper one (a symmetric product needs no separate mirror pass).
// accumulate: C += P X (C symmetric, with mirror) instead of C = P X.
void mixed_gemm(const MixedOperand& a, const MixedOperand& b, double* C, int ldc, unsigned long long* amax,
                bool lower_only, int* err, cudaStream_t st, const int* skip = nullptr, bool mirror = false,
                bool accumulate = false);

// ---------------- svd.cu ----------------
// Scratch of the PSD pseudo-inverse (n x ld matrices and p x n blocks).
struct PinvBuffers {
    double *G, *T, *W, *Tt;        // shifted inverse, Cholesky-inverse scratch
    double *X, *Y, *MX, *MX2;      // n x 32 subspace blocks
    double *H, *Wr, *S;            // 32 x 32
    double *theta, *res, *e;
    int* err;
    unsigned long long* dmax;
};
struct PinvInfo {
    int iterations, removed;
    double shift, residual, lambda_removed_max, lambda_kept_min;
};
size_t pinv_carve(char* base, int n, int ld, PinvBuffers& b);
// In place: M (n x ld, symmetric PSD) <- its pseudo-inverse without the
// remove_n smallest |eigenvalues| (remove_n >= 0) or without those with
// |eigenvalue| <= eps (remove_n == -1). Synchronises the stream.
int pinv_psd(double* M, int n, int ld, int remove_n, double eps, const PinvBuffers& b, cudaStream_t sm,
             PinvInfo* info);
// SVD_QR_ITERATION / SVD_DEVIDE_AND_CONQUER of computeCovariances; ev: 6 events.
size_t svd_workspace_bytes(int C, int P, int nobs, bool host_io, long long nnz, int nrows);
int svd_pipeline(char* ws, const unc_options* o, int num_rows, long long nnz, const int* rows, const int* cols,
                 const double* vals, double* cam_unc, double* pt_unc, bool host_io, unc_statistic* st,
                 cudaEvent_t* ev, cudaStream_t sm);

// ---------------- jacobian.cu ----------------
// Analytic reprojection Jacobian of a scene in the reference CRS layout
// (rows: 2 * num_obs + 1, cols / vals: 24 per observation).
int launch_scene_jacobian(int num_cams, int num_points, int num_obs, const double* cams, const double* pts,
                          const int* obs_cam, const int* obs_pt, int* rows, int* cols, double* vals, int* err,
                          cudaStream_t st);

// ---------------- points.cu ----------------
void launch_point_cov(const SceneDev& s, const double* sig, double* pt_unc, cudaStream_t st);

}  // namespace unc
