// svd.cu - the SVD algorithms of computeCovariances on the GPU (svdInverse,
// compute.cpp:185-249): the pseudo-inverse of the full, unscaled, unfixed
// J^T J with its smallest singular values removed, then the camera output with
// the reference's (a + b/2) expression and no column scaling (compute.cpp:247,
// removeScaleJ4Z with d = NULL) and the 3x3 point blocks of the same matrix.
//
// M = J^T J is symmetric positive semi-definite, so its SVD is its eigen-
// decomposition and U diag(f) V^T is the sum over the kept eigenpairs of
// v v^T / lambda (a tiny negative eigenvalue comes back from LAPACK's SVD as
// sigma = |lambda| with u = -v, which gives the same term). The removed set is
// the svd_remove_n smallest |lambda| (compute.cpp:222-229) or every
// |lambda| <= epsilon (compute.cpp:230-240).
//
// Only the removed eigenvectors V_R are computed, not the whole spectrum:
//   1. G = (M + s I)^{-1}, s = 1e-13 max_i M_ii, by the Cholesky inverse of
//      dense.cu (equilibrated); the removed directions are G's dominant ones.
//   2. Subspace iteration on G with p = removed + 8 vectors: Y = G X,
//      Gram-Schmidt (twice), Rayleigh-Ritz with M (p x p cyclic Jacobi), until
//      the Ritz residuals of the removed vectors stop shrinking.
//   3. B = M + c V_R V_R^T with c the smallest kept Ritz value: SPD when every
//      kept eigenvalue is positive, with the removed directions lifted.
//   4. pinv(M) = P B^{-1} P with P = I - V_R V_R^T (two-sided projection: the
//      result has exactly V_R as its null space, like an eigen-decomposition).
// The answer is limited by the conditioning of M (lambda_max / smallest kept
// lambda), like the reference's own LAPACK SVD.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/uncte.h"
#include "internal.h"

namespace unc {

namespace {

constexpr int kMaxBlock = 32;  // largest subspace block (the p x p kernels run in one warp)

#define SVD_CK(call)                                                                              \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) {                                                                  \
            g_last_error = std::string(#call) + ": " + cudaGetErrorString(e_);                    \
            return e_ == cudaErrorMemoryAllocation ? UNC_ERR_OUT_OF_MEMORY : UNC_ERR_CUDA;        \
        }                                                                                         \
    } while (0)

int svd_fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

// Sum over the block (blockDim.x a multiple of 32, at most 1024) in a fixed
// order; red: 33 doubles of shared memory.
__device__ double block_sum(double v, double* red) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    if (w == 0) {
        v = l < nw ? red[l] : 0.0;
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
        if (l == 0) red[32] = v;
    }
    __syncthreads();
    return red[32];
}

// splitmix64 (Steele, Lea, Flood 2014): deterministic start vectors.
__device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
    x += 0x9e3779b97f4a7c15ULL;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
    return x ^ (x >> 31);
}

__device__ __forceinline__ double uniform_pm1(unsigned long long seed, int j, int r) {
    const unsigned long long h = mix64(seed ^ mix64(((unsigned long long)(unsigned)j << 32) | (unsigned)r));
    return (double)(h >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

// ---- dense J^T J from the unscaled blocks --------------------------------
// Camera diagonal blocks: U row-major 9 x 9 per camera.
__global__ void k_dense_cam(const double* __restrict__ U, int C, double* M, long ld) {
    const int c = blockIdx.x, e = threadIdx.x;
    if (c >= C || e >= 81) return;
    const int i = e / 9, j = e - 9 * i;
    M[(9L * c + i) + (9L * c + j) * ld] = U[81L * c + e];
}

// Point diagonal blocks from the upper triangle (00 01 02 11 12 22).
__global__ void k_dense_pt(const double* __restrict__ Vraw, int P, long b0, double* M, long ld) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P) return;
    const double* v = Vraw + 6L * p;
    const double a[3][3] = {{v[0], v[1], v[2]}, {v[1], v[3], v[4]}, {v[2], v[4], v[5]}};
    const long r = b0 + 3L * p;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) M[(r + i) + (r + j) * ld] = a[i][j];
}

// Camera-point blocks: one thread per point walks its observations in order,
// so a camera seeing the point twice is summed deterministically; the thread
// owns the point's three columns (upper right) and three rows (lower left).
__global__ void k_dense_w(const double* __restrict__ W, const int* __restrict__ obs_cam,
                          const int* __restrict__ pt_ptr, const int* __restrict__ pt_obs, int P, long b0,
                          double* M, long ld) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P) return;
    const long r = b0 + 3L * p;
    for (int q = pt_ptr[p]; q < pt_ptr[p + 1]; ++q) {
        const int o = pt_obs[q], c = obs_cam[o];
        if (c < 0) continue;
        const double* w = W + 27L * o;
        for (int i = 0; i < 9; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const double v = w[3 * i + j];
                M[(9L * c + i) + (r + j) * ld] += v;
                M[(r + j) + (9L * c + i) * ld] += v;
            }
    }
}

// max_i |M_ii| as the bit pattern of a non-negative double (NaN counts as +inf).
__global__ void k_diag_absmax(const double* __restrict__ M, int n, long ld, unsigned long long* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0.0;
    if (i < n) {
        v = fabs(M[i + i * ld]);
        if (!(v <= DBL_MAX)) v = __longlong_as_double(0x7ff0000000000000LL);
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, d));
    if ((threadIdx.x & 31) == 0 && v > 0.0) atomicMax(out, (unsigned long long)__double_as_longlong(v));
}

__global__ void k_fill_random(double* X, int n, long ld, int p, unsigned long long seed) {
    const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (idx >= (long)n * p) return;
    const int j = (int)(idx / n), r = (int)(idx - (long)j * n);
    X[r + j * ld] = uniform_pm1(seed, j, r);
}

// G(i, j) = sum_r A(r, i) B(r, j): one CTA per entry, fixed-order reduction.
__global__ void __launch_bounds__(256) k_gram(const double* __restrict__ A, long lda, const double* __restrict__ B,
                                              long ldb, int n, double* G, int ldg) {
    __shared__ double red[33];
    const int i = blockIdx.x, j = blockIdx.y;
    const double* a = A + i * lda;
    const double* b = B + j * ldb;
    double s = 0.0;
    for (int r = threadIdx.x; r < n; r += blockDim.x) s += a[r] * b[r];
    s = block_sum(s, red);
    if (threadIdx.x == 0) G[i + j * ldg] = s;
}

// Orthonormalise the p columns of Y in place: Gram-Schmidt run twice per
// column (the second pass restores orthogonality lost to cancellation). A
// column that vanishes (dependent on the earlier ones) restarts from a random
// vector (status bit 1); if that fails three times status bit 2 is set. Each
// thread owns a fixed set of rows, so threads only meet in the reductions.
__global__ void __launch_bounds__(1024) k_orthonormalize(double* Y, int n, long ld, int p, unsigned long long seed,
                                                         int* status) {
    __shared__ double red[33];
    const int t = threadIdx.x, nt = blockDim.x;
    for (int j = 0; j < p; ++j) {
        double* y = Y + j * ld;
        bool done = false;
        for (int attempt = 0; attempt < 3 && !done; ++attempt) {
            double s0 = 0.0;
            for (int r = t; r < n; r += nt) s0 += y[r] * y[r];
            const double n0 = sqrt(block_sum(s0, red));
            for (int pass = 0; pass < 2; ++pass)
                for (int i = 0; i < j; ++i) {
                    const double* q = Y + i * ld;
                    double d = 0.0;
                    for (int r = t; r < n; r += nt) d += q[r] * y[r];
                    d = block_sum(d, red);
                    for (int r = t; r < n; r += nt) y[r] -= d * q[r];
                }
            double s1 = 0.0;
            for (int r = t; r < n; r += nt) s1 += y[r] * y[r];
            const double n1 = sqrt(block_sum(s1, red));
            if (n1 > 0.0 && n1 > 1e-10 * n0) {
                const double inv = 1.0 / n1;
                for (int r = t; r < n; r += nt) y[r] *= inv;
                done = true;
            } else {
                if (t == 0) atomicOr(status, 1);
                for (int r = t; r < n; r += nt) y[r] = uniform_pm1(seed + 7919ULL * (attempt + 1), j, r);
            }
        }
        if (!done && t == 0) atomicOr(status, 2);
    }
}

// Eigen-decomposition of the symmetric p x p matrix H (p <= 32) by cyclic
// Jacobi rotations in one warp (lane = row). Outputs ascending eigenvalues
// theta and the matching orthonormal eigenvectors as the columns of Wr.
// Rotation: t = sgn(th) / (|th| + sqrt(th^2 + 1)), th = (a_bb - a_aa) / (2 a_ab),
// c = 1 / sqrt(t^2 + 1), s = t c (Golub & Van Loan, symmetric Schur 2 x 2);
// off-diagonal entries below 1e-17 sqrt(|a_aa a_bb|) are left alone.
__global__ void __launch_bounds__(32) k_small_jacobi(const double* __restrict__ H, int ldh, int p, double* theta,
                                                     double* Wr, int ldw) {
    __shared__ double A[kMaxBlock][kMaxBlock + 1], V[kMaxBlock][kMaxBlock + 1];
    const int l = threadIdx.x;
    for (int c = 0; c < p; ++c)
        if (l < p) {
            A[l][c] = 0.5 * (H[l + c * ldh] + H[c + l * ldh]);
            V[l][c] = (l == c) ? 1.0 : 0.0;
        }
    __syncwarp();
    for (int sweep = 0; sweep < 60; ++sweep) {
        double off = 0.0, dg = 0.0;
        if (l < p) {
            for (int c = 0; c < l; ++c) off += A[l][c] * A[l][c];
            dg = A[l][l] * A[l][l];
        }
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) {
            off += __shfl_xor_sync(0xffffffffu, off, d);
            dg += __shfl_xor_sync(0xffffffffu, dg, d);
        }
        if (off <= 1e-30 * dg) break;
        for (int a = 0; a < p - 1; ++a)
            for (int b = a + 1; b < p; ++b) {
                const double apq = A[a][b], aa = A[a][a], bb = A[b][b];
                if (apq == 0.0 || fabs(apq) <= 1e-17 * sqrt(fabs(aa * bb))) continue;
                const double th = (bb - aa) / (2.0 * apq);
                const double t = fabs(th) > 1e100 ? 0.5 / th
                                                  : (th >= 0.0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                __syncwarp();
                if (l < p) {
                    const double x = A[l][a], y = A[l][b];
                    A[l][a] = c * x - s * y;
                    A[l][b] = s * x + c * y;
                    const double vx = V[l][a], vy = V[l][b];
                    V[l][a] = c * vx - s * vy;
                    V[l][b] = s * vx + c * vy;
                }
                __syncwarp();
                if (l < p) {
                    const double x = A[a][l], y = A[b][l];
                    A[a][l] = c * x - s * y;
                    A[b][l] = s * x + c * y;
                }
                __syncwarp();
            }
    }
    if (l < p) {
        const double w = A[l][l];
        int rank = 0;
        for (int i = 0; i < p; ++i) {
            const double u = A[i][i];
            rank += (u < w) || (u == w && i < l);
        }
        theta[rank] = w;
        for (int r = 0; r < p; ++r) Wr[r + rank * ldw] = V[r][l];
    }
}

// res_j = || MX(:, j) - theta_j X(:, j) ||
__global__ void __launch_bounds__(256) k_resid(const double* __restrict__ MX, const double* __restrict__ X, long ld,
                                               int n, const double* __restrict__ theta, double* res) {
    __shared__ double red[33];
    const int j = blockIdx.x;
    double s = 0.0;
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
        const double d = MX[r + j * ld] - theta[j] * X[r + j * ld];
        s += d * d;
    }
    s = block_sum(s, red);
    if (threadIdx.x == 0) res[j] = sqrt(s);
}

// Upper triangle (00 01 02 11 12 22) of every 3 x 3 point block on the diagonal.
__global__ void k_point_diag_out(const double* __restrict__ P, long ld, long b0, int num_points, double* pt_unc) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= num_points) return;
    const long r = b0 + 3L * p;
    double* o = pt_unc + 6L * p;
    o[0] = P[r + r * ld];
    o[1] = P[r + (r + 1) * ld];
    o[2] = P[r + (r + 2) * ld];
    o[3] = P[(r + 1) + (r + 1) * ld];
    o[4] = P[(r + 1) + (r + 2) * ld];
    o[5] = P[(r + 2) + (r + 2) * ld];
}

int read_err(const int* d_err, int* h, cudaStream_t sm) {
    SVD_CK(cudaMemcpyAsync(h, d_err, sizeof(int), cudaMemcpyDeviceToHost, sm));
    SVD_CK(cudaStreamSynchronize(sm));
    return UNC_OK;
}

// In-place SPD inverse with equilibration (the inverse of the Taylor path).
int spd_inverse(double* A, int n, int ld, const PinvBuffers& b, cudaStream_t sm) {
    const size_t mat = (size_t)n * ld;
    SVD_CK(cudaMemsetAsync(b.T, 0, sizeof(double) * mat, sm));
    SVD_CK(cudaMemsetAsync(b.err, 0, sizeof(int), sm));
    launch_shift_equilibrate(A, n, ld, 0.0, b.e, b.err, sm);
    chol_inverse(A, n, ld, b.T, b.W, b.Tt, nullptr, b.err, sm);
    launch_unequilibrate(A, n, ld, b.e, nullptr, sm);
    int e = 0;
    if (int rc = read_err(b.err, &e, sm)) return rc;
    if (e & (ERRBIT_SINGULAR | ERRBIT_NONFINITE)) return svd_fail(UNC_ERR_SINGULAR, "matrix is not positive definite");
    return UNC_OK;
}

}  // namespace

size_t pinv_carve(char* base, int n, int ld, PinvBuffers& b) {
    Carver c{base};
    const size_t mat = (size_t)n * ld, blk = (size_t)ld * kMaxBlock;
    b.G = c.take<double>(mat);
    b.T = c.take<double>(mat);
    b.W = c.take<double>(mat);
    b.Tt = c.take<double>(mat);
    b.X = c.take<double>(blk);
    b.Y = c.take<double>(blk);
    b.MX = c.take<double>(blk);
    b.MX2 = c.take<double>(blk);
    b.H = c.take<double>(kMaxBlock * kMaxBlock);
    b.Wr = c.take<double>(kMaxBlock * kMaxBlock);
    b.S = c.take<double>(kMaxBlock * kMaxBlock);
    b.theta = c.take<double>(kMaxBlock);
    b.res = c.take<double>(kMaxBlock);
    b.e = c.take<double>((size_t)n + 64);
    b.err = c.take<int>(4);
    b.dmax = c.take<unsigned long long>(1);
    return c.off + 256;
}

int pinv_psd(double* M, int n, int ld, int remove_n, double eps, const PinvBuffers& b, cudaStream_t sm,
             PinvInfo* info) {
    PinvInfo loc{};
    PinvInfo& inf = info ? *info : loc;
    inf = PinvInfo{};
    if (n <= 0 || ld < n || (ld & 1)) return svd_fail(UNC_ERR_INVALID_ARG, "bad matrix arguments");
    if (remove_n > kMaxBlock - 1)
        return svd_fail(UNC_ERR_UNSUPPORTED, "at most 31 singular values can be removed");
    const size_t mat = (size_t)n * ld, blk = (size_t)ld * kMaxBlock;
    // every scratch matrix starts finite (the GEMM reads padding rows in pairs)
    SVD_CK(cudaMemsetAsync(b.W, 0, sizeof(double) * mat, sm));
    SVD_CK(cudaMemsetAsync(b.Tt, 0, sizeof(double) * mat, sm));
    SVD_CK(cudaMemsetAsync(b.X, 0, sizeof(double) * blk, sm));
    SVD_CK(cudaMemsetAsync(b.Y, 0, sizeof(double) * blk, sm));
    SVD_CK(cudaMemsetAsync(b.MX, 0, sizeof(double) * blk, sm));
    SVD_CK(cudaMemsetAsync(b.MX2, 0, sizeof(double) * blk, sm));
    SVD_CK(cudaMemsetAsync(b.H, 0, sizeof(double) * kMaxBlock * kMaxBlock, sm));
    SVD_CK(cudaMemsetAsync(b.Wr, 0, sizeof(double) * kMaxBlock * kMaxBlock, sm));
    SVD_CK(cudaMemsetAsync(b.S, 0, sizeof(double) * kMaxBlock * kMaxBlock, sm));
    SVD_CK(cudaMemsetAsync(b.dmax, 0, sizeof(unsigned long long), sm));

    if (remove_n == 0) {  // nothing removed: the plain inverse
        inf.removed = 0;
        return spd_inverse(M, n, ld, b, sm);
    }
    k_diag_absmax<<<(n + 255) / 256, 256, 0, sm>>>(M, n, ld, b.dmax);
    count_launch();
    unsigned long long dbits = 0;
    SVD_CK(cudaMemcpyAsync(&dbits, b.dmax, 8, cudaMemcpyDeviceToHost, sm));
    SVD_CK(cudaStreamSynchronize(sm));
    double dmax;
    memcpy(&dmax, &dbits, 8);
    if (!(dmax <= DBL_MAX)) return svd_fail(UNC_ERR_SINGULAR, "non-finite diagonal");
    if (dmax == 0.0 || (remove_n > 0 && remove_n >= n)) {  // everything removed
        SVD_CK(cudaMemsetAsync(M, 0, sizeof(double) * mat, sm));
        inf.removed = n;
        return UNC_OK;
    }

    // 1. G = (M + s I)^{-1}; a shift too small for FP64 Cholesky is raised
    double s = 1e-13 * dmax;
    bool ok = false;
    for (int attempt = 0; attempt < 4 && !ok; ++attempt) {
        SVD_CK(cudaMemcpyAsync(b.G, M, sizeof(double) * mat, cudaMemcpyDeviceToDevice, sm));
        SVD_CK(cudaMemsetAsync(b.T, 0, sizeof(double) * mat, sm));
        SVD_CK(cudaMemsetAsync(b.err, 0, sizeof(int), sm));
        launch_shift_equilibrate(b.G, n, ld, s, b.e, b.err, sm);
        chol_inverse(b.G, n, ld, b.T, b.W, b.Tt, nullptr, b.err, sm);
        launch_unequilibrate(b.G, n, ld, b.e, nullptr, sm);
        int e = 0;
        if (int rc = read_err(b.err, &e, sm)) return rc;
        ok = !(e & (ERRBIT_SINGULAR | ERRBIT_NONFINITE));
        if (!ok) s *= 100.0;
    }
    if (!ok) return svd_fail(UNC_ERR_SINGULAR, "shifted J^T J is not positive definite (not a PSD matrix)");
    inf.shift = s;

    // 2. subspace iteration
    const int p = std::min(remove_n > 0 ? remove_n + 8 : 24, std::min(n, kMaxBlock));
    {
        const long tot = (long)n * p;
        k_fill_random<<<(unsigned)((tot + 255) / 256), 256, 0, sm>>>(b.X, n, ld, p, 0x5eedULL);
        count_launch();
    }
    std::vector<double> th(p), rs(p);
    double best = DBL_MAX;
    int stall = 0, it = 0, kk = 0;
    SVD_CK(cudaMemsetAsync(b.err, 0, sizeof(int) * 2, sm));
    for (it = 0; it < 60; ++it) {
        gemm_f64(n, p, n, 1.0, b.G, ld, b.X, ld, 0.0, b.Y, ld, nullptr, sm);  // Y = G X
        k_orthonormalize<<<1, 1024, 0, sm>>>(b.Y, n, ld, p, 0x9e37ULL + (unsigned long long)it, b.err + 1);
        count_launch();
        gemm_f64(n, p, n, 1.0, M, ld, b.Y, ld, 0.0, b.MX, ld, nullptr, sm);  // M Q
        k_gram<<<dim3(p, p), 256, 0, sm>>>(b.Y, ld, b.MX, ld, n, b.H, kMaxBlock);  // Q^T M Q
        k_small_jacobi<<<1, 32, 0, sm>>>(b.H, kMaxBlock, p, b.theta, b.Wr, kMaxBlock);
        gemm_f64(n, p, p, 1.0, b.Y, ld, b.Wr, kMaxBlock, 0.0, b.X, ld, nullptr, sm);     // Ritz vectors
        gemm_f64(n, p, p, 1.0, b.MX, ld, b.Wr, kMaxBlock, 0.0, b.MX2, ld, nullptr, sm);  // M X
        k_resid<<<p, 256, 0, sm>>>(b.MX2, b.X, ld, n, b.theta, b.res);
        count_launch(3);
        SVD_CK(cudaMemcpyAsync(th.data(), b.theta, sizeof(double) * p, cudaMemcpyDeviceToHost, sm));
        SVD_CK(cudaMemcpyAsync(rs.data(), b.res, sizeof(double) * p, cudaMemcpyDeviceToHost, sm));
        SVD_CK(cudaStreamSynchronize(sm));
        if (remove_n > 0) {
            kk = remove_n;
        } else {
            kk = 0;
            for (int j = 0; j < p; ++j) kk += fabs(th[j]) <= eps;
        }
        double conv = 0.0;
        for (int j = 0; j < std::max(kk, 1); ++j) conv = std::max(conv, rs[j]);
        if (!(conv <= DBL_MAX)) return svd_fail(UNC_ERR_SINGULAR, "non-finite Ritz residual");
        inf.residual = conv;
        // stop once the residuals of the removed vectors no longer shrink
        if (conv < 0.5 * best) {
            best = conv;
            stall = 0;
        } else {
            ++stall;
        }
        if (conv == 0.0 || stall >= 3) {
            ++it;
            break;
        }
    }
    inf.iterations = it;
    int ostat = 0;
    SVD_CK(cudaMemcpyAsync(&ostat, b.err + 1, sizeof(int), cudaMemcpyDeviceToHost, sm));
    SVD_CK(cudaStreamSynchronize(sm));
    if (ostat & 2) return svd_fail(UNC_ERR_SINGULAR, "subspace iteration lost rank");
    if (remove_n < 0 && kk > p - 4)
        return svd_fail(UNC_ERR_UNSUPPORTED, "more than 20 singular values at or below epsilon");
    inf.removed = kk;
    if (kk == 0) return spd_inverse(M, n, ld, b, sm);
    if (kk >= n) {
        SVD_CK(cudaMemsetAsync(M, 0, sizeof(double) * mat, sm));
        return UNC_OK;
    }
    const double c = th[kk];
    inf.lambda_removed_max = th[kk - 1];
    inf.lambda_kept_min = c;
    // a kept eigenvalue at the rounding level of M (below 8 eps max_i M_ii)
    // means more null directions than are removed: the result would be noise.
    // Nearly-null but resolvable spectra (04_Daliborka: kept eigenvalues from
    // 8.9e-6 with lambda_max 7.7e8) pass, ill-conditioned like the reference.
    if (!(c > 8.0 * DBL_EPSILON * dmax))
        return svd_fail(UNC_ERR_SINGULAR, "the matrix has more (near-)null directions than are removed");

    // 3. B = M + c V_R V_R^T, inverted in place
    gemm_f64_mode(n, n, kk, c, b.X, ld, b.X, ld, 1.0, M, ld, nullptr, GEMM_TRANS_B, sm);
    if (int rc = spd_inverse(M, n, ld, b, sm)) return rc;

    // 4. P B^{-1} P = B^{-1} - Z V^T - V Z^T + V (V^T Z) V^T, Z = B^{-1} V
    gemm_f64(n, kk, n, 1.0, M, ld, b.X, ld, 0.0, b.Y, ld, nullptr, sm);
    k_gram<<<dim3(kk, kk), 256, 0, sm>>>(b.X, ld, b.Y, ld, n, b.S, kMaxBlock);
    count_launch();
    gemm_f64_mode(n, n, kk, -1.0, b.Y, ld, b.X, ld, 1.0, M, ld, nullptr, GEMM_TRANS_B, sm);
    gemm_f64_mode(n, n, kk, -1.0, b.X, ld, b.Y, ld, 1.0, M, ld, nullptr, GEMM_TRANS_B, sm);
    gemm_f64(n, kk, kk, 1.0, b.X, ld, b.S, kMaxBlock, 0.0, b.MX, ld, nullptr, sm);
    gemm_f64_mode(n, n, kk, 1.0, b.MX, ld, b.X, ld, 1.0, M, ld, nullptr, GEMM_TRANS_B, sm);
    SVD_CK(cudaGetLastError());
    return UNC_OK;
}

// ---------------------------------------------------------------------------
// The SVD algorithms of computeCovariances
// ---------------------------------------------------------------------------
namespace {
struct SvdLayout {
    int *rows, *cols;
    double* vals;
    double *cam_out, *pt_out;
    SceneDev s;
    double *U, *Wb, *M;
    PinvBuffers pb;
};

size_t svd_carve(char* base, int C, int P, int nobs, bool host_io, long long nnz, int nrows, SvdLayout& L) {
    Carver c{base};
    memset(&L, 0, sizeof(L));
    if (host_io) {
        L.rows = c.take<int>((size_t)nrows + 1);
        L.cols = c.take<int>((size_t)nnz);
        L.vals = c.take<double>((size_t)nnz);
        L.cam_out = c.take<double>((size_t)C * 45);
        L.pt_out = c.take<double>((size_t)P * 6);
    }
    SceneDev& s = L.s;
    s.obs_cam = c.take<int>(nobs);
    s.obs_pt = c.take<int>(nobs);
    s.cam_ptr = c.take<int>((size_t)C + 1);
    s.cam_obs = c.take<int>(nobs);
    s.pt_ptr = c.take<int>((size_t)P + 1);
    s.pt_obs = c.take<int>(nobs);
    s.cursor = c.take<int>((size_t)C + P + 1);
    s.scan_tmp = c.take<int>(scan_tmp_ints(std::max(C, P)));
    s.s_pt = c.take<double>((size_t)P * 3);
    s.Vraw = c.take<double>((size_t)P * 6);
    s.iVs = c.take<double>((size_t)P * 6);
    s.err = c.take<int>(4);
    L.U = c.take<double>((size_t)C * 81);
    L.Wb = c.take<double>((size_t)nobs * 27);
    const int n = 9 * C + 3 * P, ld = ld_of(n);
    L.M = c.take<double>((size_t)n * ld);
    size_t used = c.off;
    size_t pin = pinv_carve(base ? base + ((used + 255) & ~size_t(255)) : nullptr, n, ld, L.pb);
    return ((used + 255) & ~size_t(255)) + pin;
}

float ev_s(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    return ms * 1e-3f;
}
}  // namespace

size_t svd_workspace_bytes(int C, int P, int nobs, bool host_io, long long nnz, int nrows) {
    SvdLayout L;
    return svd_carve(nullptr, C, P, nobs, host_io, nnz, nrows, L);
}

int svd_pipeline(char* ws, const unc_options* o, int num_rows, long long nnz, const int* rows, const int* cols,
                 const double* vals, double* cam_unc, double* pt_unc, bool host_io, unc_statistic* st,
                 cudaEvent_t* ev, cudaStream_t sm) {
    const int C = o->num_cams, P = o->num_points, nobs = num_rows / 2;
    const int n = 9 * C + 3 * P, ld = ld_of(n);
    SvdLayout L;
    svd_carve(ws, C, P, nobs, host_io, nnz, num_rows, L);
    const int* d_rows = rows;
    const int* d_cols = cols;
    const double* d_vals = vals;
    double* d_cam = cam_unc;
    double* d_pt = pt_unc;
    SVD_CK(cudaEventRecord(ev[0], sm));
    if (host_io) {
        SVD_CK(cudaMemcpyAsync(L.rows, rows, sizeof(int) * ((size_t)num_rows + 1), cudaMemcpyHostToDevice, sm));
        SVD_CK(cudaMemcpyAsync(L.cols, cols, sizeof(int) * (size_t)nnz, cudaMemcpyHostToDevice, sm));
        SVD_CK(cudaMemcpyAsync(L.vals, vals, sizeof(double) * (size_t)nnz, cudaMemcpyHostToDevice, sm));
        d_rows = L.rows;
        d_cols = L.cols;
        d_vals = L.vals;
        d_cam = L.cam_out;
        d_pt = L.pt_out;
    }
    SceneDev& s = L.s;
    s.nnz = (long)nnz;
    s.num_cams = C;
    s.num_points = P;
    s.num_obs = nobs;
    s.rows = d_rows;
    s.cols = d_cols;
    s.J = d_vals;
    s.has_fix = 0;  // the SVD algorithms keep every point (no fixPts, compute.cpp:483-495)
    SVD_CK(cudaMemsetAsync(s.err, 0, 16, sm));
    SVD_CK(cudaEventRecord(ev[1], sm));
    launch_validate_obs(s, sm);
    launch_build_index(s, sm);
    SVD_CK(cudaEventRecord(ev[2], sm));
    // dense J^T J, unscaled (compute.cpp:189-199)
    SVD_CK(cudaMemsetAsync(L.M, 0, sizeof(double) * (size_t)n * ld, sm));
    launch_point_blocks(s, sm);
    launch_unscaled_blocks(s, L.U, L.Wb, sm);
    const long b0 = 9L * C;
    k_dense_cam<<<C, 96, 0, sm>>>(L.U, C, L.M, ld);
    if (P > 0) {
        k_dense_pt<<<(P + 127) / 128, 128, 0, sm>>>(s.Vraw, P, b0, L.M, ld);
        k_dense_w<<<(P + 127) / 128, 128, 0, sm>>>(L.Wb, s.obs_cam, s.pt_ptr, s.pt_obs, P, b0, L.M, ld);
    }
    count_launch(P > 0 ? 3 : 1);
    int err = 0;
    SVD_CK(cudaMemcpyAsync(&err, s.err, sizeof(int), cudaMemcpyDeviceToHost, sm));
    SVD_CK(cudaEventRecord(ev[3], sm));
    SVD_CK(cudaStreamSynchronize(sm));
    if (err & ERRBIT_LAYOUT)
        return svd_fail(UNC_ERR_LAYOUT, "Jacobian rows are not in the 2 x (9 camera + 3 point) observation layout");
    // pseudo-inverse (compute.cpp:200-245)
    PinvInfo info{};
    const int remove_n = o->svd_remove_n;  // -1: remove singular values <= epsilon
    const double eps = o->epsilon < 0 ? 1e-10 : o->epsilon;
    if (remove_n < -1) return svd_fail(UNC_ERR_INVALID_ARG, "svd_remove_n must be -1 or >= 0");
    if (int rc = pinv_psd(L.M, n, ld, remove_n, eps, L.pb, sm, &info)) return rc;
    SVD_CK(cudaEventRecord(ev[4], sm));
    // outputs: camera blocks with the (a + b/2) expression and d = NULL
    // (compute.cpp:247), point blocks of the same matrix
    launch_camera_output(L.M, ld, nullptr, C, d_cam, nullptr, sm);
    if (P > 0) {
        k_point_diag_out<<<(P + 127) / 128, 128, 0, sm>>>(L.M, ld, b0, P, d_pt);
        count_launch();
    }
    SVD_CK(cudaEventRecord(ev[5], sm));
    if (host_io) {
        SVD_CK(cudaMemcpyAsync(cam_unc, L.cam_out, sizeof(double) * 45 * (size_t)C, cudaMemcpyDeviceToHost, sm));
        SVD_CK(cudaMemcpyAsync(pt_unc, L.pt_out, sizeof(double) * 6 * (size_t)P, cudaMemcpyDeviceToHost, sm));
    }
    SVD_CK(cudaStreamSynchronize(sm));
    SVD_CK(cudaGetLastError());
    if (st) {
        st->time_create_j = ev_s(ev[0], ev[1]);
        st->time_fix_j = 0;
        st->time_norm_j = ev_s(ev[1], ev[2]);
        st->time_multiply_jj = ev_s(ev[2], ev[3]);
        st->time_inv_z = ev_s(ev[3], ev[4]);
        st->time_pts_unc = ev_s(ev[4], ev[5]);
        st->time_all = ev_s(ev[0], ev[5]);
        st->te_iterations = info.iterations;  // SVD algorithms: subspace iterations
        st->lambda = 0;
        st->fixed_pts[0] = st->fixed_pts[1] = st->fixed_pts[2] = -1;
    }
    return UNC_OK;
}

}  // namespace unc

using namespace unc;

extern "C" int unc_pinv_psd_device(double* d_M, int n, int ld, int remove_n, double epsilon, void* stream) {
    g_last_error.clear();
    if (!d_M || n <= 0 || ld < n || (ld & 1)) return svd_fail(UNC_ERR_INVALID_ARG, "bad matrix arguments");
    if (remove_n < -1) return svd_fail(UNC_ERR_INVALID_ARG, "remove_n must be -1 or >= 0");
    cudaStream_t sm = (cudaStream_t)stream;
    PinvBuffers b;
    const size_t bytes = pinv_carve(nullptr, n, ld, b);
    char* ws = nullptr;
    SVD_CK(cudaMalloc(&ws, bytes));
    pinv_carve(ws, n, ld, b);
    int rc = pinv_psd(d_M, n, ld, remove_n, epsilon < 0 ? 1e-10 : epsilon, b, sm, nullptr);
    cudaStreamSynchronize(sm);
    cudaFree(ws);
    return rc;
}
