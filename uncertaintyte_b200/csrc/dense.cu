// dense.cu - FP64 dense kernels for the inverse of the camera Schur
// complement (sm_100a):
//   * gemm_f64      : C = alpha*A*B + beta*C on DMMA (mma.sync m8n8k4 f64),
//                     4-stage cp.async pipeline, optional fused max|C| for the
//                     Taylor stop rule (ScaledDenseMatrix.cpp:207-216,314-353).
//   * gj_inverse    : blocked Gauss-Jordan inverse of an SPD matrix; every
//                     panel step is a rank-nb update on gemm_f64
//                     (replaces dgetrf+dgetri in SDM::inv, ScaledDenseMatrix.cpp:232-279).
//   * shift/equilibrate, un-equilibrate, axpy (iZupdate, compute.cpp:64-71),
//     camera output with the reference's (a + b/2) quirk (compute.cpp:168-183).
#include "internal.h"

namespace unc {

// ------------------------------------------------------------------------
// GEMM
// ------------------------------------------------------------------------
namespace {
constexpr int BM = 128, BN = 128, BK = 16, STAGES = 4;
constexpr int LDA_S = BM + 8;   // As[k][m]: 136 doubles per k row (conflict-free fragment reads)
constexpr int LDB_S = BK + 4;   // Bs[n][k]: 20 doubles per n row
constexpr int A_STAGE = BK * LDA_S;
constexpr int B_STAGE = BN * LDB_S;
constexpr int GEMM_THREADS = 256;
constexpr size_t GEMM_SMEM = sizeof(double) * (size_t)STAGES * (A_STAGE + B_STAGE);

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool pred) {
    unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    int sz = pred ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}
}  // namespace

// Tile loader: A tile (BM rows x BK cols of column-major A), B tile (BK rows
// x BN cols of column-major B). Out-of-range chunks are zero-filled. Rows
// past M (or K for B) inside the allocation are read as 16-byte pairs; the
// buffers keep their padding rows at zero so those reads are inert.
__device__ __forceinline__ void load_tiles(double* As, double* Bs, const double* __restrict__ A,
                                           long lda, const double* __restrict__ B, long ldb, int M,
                                           int N, int K, int m0, int n0, int k0, int tid) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        int idx = tid + q * GEMM_THREADS;  // 0..1023
        int k = idx >> 6, m2 = (idx & 63) * 2;
        bool p = (m0 + m2 < M) && (k0 + k < K);
        const double* src = p ? A + (m0 + m2) + (long)(k0 + k) * lda : A;
        cp_async16(As + k * LDA_S + m2, src, p);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        int idx = tid + q * GEMM_THREADS;
        int n = idx >> 3, k2 = (idx & 7) * 2;
        bool p = (n0 + n < N) && (k0 + k2 < K);
        const double* src = p ? B + (k0 + k2) + (long)(n0 + n) * ldb : B;
        cp_async16(Bs + n * LDB_S + k2, src, p);
    }
}

__global__ void __launch_bounds__(GEMM_THREADS, 1)
    k_gemm_f64(int M, int N, int K, double alpha, const double* __restrict__ A, long lda,
               const double* __restrict__ B, long ldb, double beta, double* C, long ldc,
               unsigned long long* amax, int lower_only) {
    // lower_only: tiles strictly above the diagonal of C are skipped (SYRK-style update)
    if (lower_only && (int)(blockIdx.x * BN) > (int)(blockIdx.y * BM) + BM - 1) return;
    extern __shared__ __align__(16) double smem[];
    double* As = smem;
    double* Bs = smem + STAGES * A_STAGE;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = (warp & 3) * 32, wn = (warp >> 2) * 64;
    const int g = lane >> 2, t = lane & 3;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int KT = (K + BK - 1) / BK;

    double acc[4][8][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
        if (s < KT) load_tiles(As + s * A_STAGE, Bs + s * B_STAGE, A, lda, B, ldb, M, N, K, m0, n0, s * BK, tid);
        cp_async_commit();
    }
    for (int kt = 0; kt < KT; ++kt) {
        cp_async_wait<STAGES - 2>();
        __syncthreads();
        int pf = kt + STAGES - 1;
        if (pf < KT) {
            int ps = pf % STAGES;
            load_tiles(As + ps * A_STAGE, Bs + ps * B_STAGE, A, lda, B, ldb, M, N, K, m0, n0, pf * BK, tid);
        }
        cp_async_commit();
        const double* as = As + (kt % STAGES) * A_STAGE;
        const double* bs = Bs + (kt % STAGES) * B_STAGE;
#pragma unroll
        for (int kk = 0; kk < BK; kk += 4) {
            double af[4], bf[8];
#pragma unroll
            for (int i = 0; i < 4; ++i) af[i] = as[(kk + t) * LDA_S + wm + i * 8 + g];
#pragma unroll
            for (int j = 0; j < 8; ++j) bf[j] = bs[(wn + j * 8 + g) * LDB_S + kk + t];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) dmma(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
        }
    }
    cp_async_wait<0>();

    double mx = 0.0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        int row = m0 + wm + i * 8 + g;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                int col = n0 + wn + j * 8 + t * 2 + h;
                if (row < M && col < N) {
                    double* c = C + row + (long)col * ldc;
                    double v = alpha * acc[i][j][h];
                    if (beta != 0.0) v += beta * *c;
                    *c = v;
                    double av = fabs(v);
                    mx = fmax(mx, av <= 1.7976931348623157e308 ? av : __longlong_as_double(0x7ff0000000000000LL));
                }
            }
        }
    }
    if (amax) {
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, d));
        if (lane == 0) atomicMax(amax, (unsigned long long)__double_as_longlong(mx));
    }
}

void gemm_f64(int M, int N, int K, double alpha, const double* A, int lda, const double* B,
              int ldb, double beta, double* C, int ldc, unsigned long long* amax, cudaStream_t st) {
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_gemm_f64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GEMM_SMEM);
        attr = true;
    }
    if (M <= 0 || N <= 0) return;
    dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM);
    k_gemm_f64<<<grid, GEMM_THREADS, GEMM_SMEM, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, amax, 0);
    count_launch();
}

void gemm_f64_tri(int M, int N, int K, double alpha, const double* A, int lda, const double* B, int ldb,
                  double beta, double* C, int ldc, cudaStream_t st) {
    gemm_f64(0, 0, 0, 0, nullptr, 0, nullptr, 0, 0, nullptr, 0, nullptr, st);  // sets the smem attribute
    if (M <= 0 || N <= 0) return;
    dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM);
    k_gemm_f64<<<grid, GEMM_THREADS, GEMM_SMEM, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc,
                                                      nullptr, 1);
    count_launch();
}

// ------------------------------------------------------------------------
// SPD inverse: blocked Cholesky A = L L^T, T = L^{-1}, A^{-1} = T^T T
// ------------------------------------------------------------------------
constexpr int NB = 64;                       // panel width
constexpr int SQ_SMEM = (int)(sizeof(double) * 2 * NB * (NB + 1));

size_t chol_small_doubles(int n) { return (size_t)NB * NB + (size_t)NB * (n + 8) + 64; }

// Unblocked Cholesky of the kb x kb diagonal block at (k0, k0) in shared
// memory (lower triangle read), written back as L_kk; its inverse (lower)
// goes to Linv (64 x 64, ld 64). One CTA.
__global__ void __launch_bounds__(256) k_chol_diag(double* A, long lda, int k0, int kb, double* Linv,
                                                   int* err) {
    extern __shared__ double sm_[];
    double(*a)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(sm_);
    double(*x)[NB + 1] = a + NB;  // x[i][c]: column c of the inverse
    const int tid = threadIdx.x;
    for (int e = tid; e < kb * kb; e += blockDim.x) {
        int r = e % kb, c = e / kb;
        a[r][c] = r >= c ? A[(k0 + r) + (long)(k0 + c) * lda] : 0.0;
    }
    __syncthreads();
    for (int p = 0; p < kb; ++p) {
        if (tid == 0) {
            double d = a[p][p];
            if (!(d > 0.0 && d <= 1.7976931348623157e308)) atomicOr(err, ERRBIT_SINGULAR);
            a[p][p] = sqrt(d);
        }
        __syncthreads();
        double lp = a[p][p];
        for (int i = p + 1 + tid; i < kb; i += blockDim.x) a[i][p] /= lp;
        __syncthreads();
        const int m = kb - p - 1;  // trailing size
        for (int e = tid; e < m * m; e += blockDim.x) {
            int i = p + 1 + e % m, j = p + 1 + e / m;
            if (j <= i) a[i][j] -= a[i][p] * a[j][p];
        }
        __syncthreads();
    }
    for (int e = tid; e < kb * kb; e += blockDim.x) {
        int r = e % kb, c = e / kb;
        if (r >= c) A[(k0 + r) + (long)(k0 + c) * lda] = a[r][c];
    }
    // forward substitution, one thread per column of the inverse
    if (tid < kb) {
        const int c = tid;
        for (int i = 0; i < c; ++i) x[i][c] = 0.0;
        x[c][c] = 1.0 / a[c][c];
        for (int i = c + 1; i < kb; ++i) {
            double s = 0.0;
            for (int j = c; j < i; ++j) s += a[i][j] * x[j][c];
            x[i][c] = -s / a[i][i];
        }
    }
    __syncthreads();
    for (int e = tid; e < kb * kb; e += blockDim.x) {
        int r = e % kb, c = e / kb;
        Linv[r + (long)c * NB] = x[r][c];
    }
}

// Panel: L_ik = A_ik * Linv_kk^T for the 64-row chunk starting at i0 (rows
// below the pivot block); written into A and transposed into R (R[q + i*NB] =
// L(i, k0+q)) as the B operand of the trailing update.
__global__ void __launch_bounds__(256) k_chol_panel(double* A, long lda, int n, int k0, int kb, int i0,
                                                    const double* __restrict__ Linv, double* R) {
    extern __shared__ double sm_[];
    double(*sp)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(sm_);  // sp[q][r] = Linv(q, r)
    double(*sx)[NB + 1] = sp + NB;                                   // sx[i][r] = A(row, k0 + r)
    const int tid = threadIdx.x;
    const int r0 = i0 + blockIdx.x * NB;
    const int rn = min(NB, n - r0);
    if (rn <= 0) return;
    for (int e = tid; e < kb * kb; e += blockDim.x) {
        int q = e % kb, r = e / kb;
        sp[q][r] = Linv[q + (long)r * NB];
    }
    for (int e = tid; e < rn * kb; e += blockDim.x) {
        int i = e % rn, r = e / rn;
        sx[i][r] = A[(r0 + i) + (long)(k0 + r) * lda];
    }
    __syncthreads();
    for (int e = tid; e < rn * kb; e += blockDim.x) {
        int i = e % rn, q = e / rn;
        double s = 0.0;
        for (int r = 0; r <= q; ++r) s += sx[i][r] * sp[q][r];
        A[(r0 + i) + (long)(k0 + q) * lda] = s;
        R[q + (long)(r0 + i) * NB] = s;
    }
}

// Inverse of every 64 x 64 diagonal block of the lower-triangular L (the
// leaves of the recursive triangular inverse). One CTA per block.
__global__ void __launch_bounds__(256) k_trtri_leaves(const double* __restrict__ L, long lda, int n,
                                                      double* T, long ldt) {
    extern __shared__ double sm_[];
    double(*a)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(sm_);
    double(*x)[NB + 1] = a + NB;
    const int b0 = blockIdx.x * NB, bs = min(NB, n - b0);
    const int tid = threadIdx.x;
    for (int e = tid; e < bs * bs; e += blockDim.x) {
        int r = e % bs, c = e / bs;
        a[r][c] = r >= c ? L[(b0 + r) + (long)(b0 + c) * lda] : 0.0;
    }
    __syncthreads();
    if (tid < bs) {
        const int c = tid;
        for (int i = 0; i < c; ++i) x[i][c] = 0.0;
        x[c][c] = 1.0 / a[c][c];
        for (int i = c + 1; i < bs; ++i) {
            double s = 0.0;
            for (int j = c; j < i; ++j) s += a[i][j] * x[j][c];
            x[i][c] = -s / a[i][i];
        }
    }
    __syncthreads();
    for (int e = tid; e < bs * bs; e += blockDim.x) {
        int r = e % bs, c = e / bs;
        T[(b0 + r) + (long)(b0 + c) * ldt] = x[r][c];
    }
}

// Tt = T^T (n x n), 32 x 32 tiles through shared memory.
__global__ void k_transpose(const double* __restrict__ T, long ldt, int n, double* Tt, long ldo) {
    __shared__ double t[32][33];
    int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += 8) {
        int i = by + r, j = bx + threadIdx.x;
        if (i < n && j < n) t[r][threadIdx.x] = T[i + (long)j * ldt];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += 8) {
        int j = bx + r, i = by + threadIdx.x;  // out(j, i) = T(i, j)
        if (i < n && j < n) Tt[j + (long)i * ldo] = t[threadIdx.x][r];
    }
}

namespace {
void set_smem_attr() {
    static bool done = false;
    if (done) return;
    cudaFuncSetAttribute(k_chol_diag, cudaFuncAttributeMaxDynamicSharedMemorySize, SQ_SMEM);
    cudaFuncSetAttribute(k_chol_panel, cudaFuncAttributeMaxDynamicSharedMemorySize, SQ_SMEM);
    cudaFuncSetAttribute(k_trtri_leaves, cudaFuncAttributeMaxDynamicSharedMemorySize, SQ_SMEM);
    done = true;
}

// T[r0:r1, r0:r1] = inverse of L[r0:r1, r0:r1] given the inverted leaves:
// T21 = -T22 * (L21 * T11), split at a multiple of 64.
void trtri_merge(const double* L, int lda, double* T, int ldt, double* W, int ldw, int r0, int r1,
                 cudaStream_t st) {
    if (r1 - r0 <= NB) return;
    int half = (r1 - r0) / 2;
    int m = r0 + ((half + NB - 1) / NB) * NB;
    if (m >= r1) m = r1 - NB;
    trtri_merge(L, lda, T, ldt, W, ldw, r0, m, st);
    trtri_merge(L, lda, T, ldt, W, ldw, m, r1, st);
    const int m2 = r1 - m, m1 = m - r0;
    gemm_f64(m2, m1, m1, 1.0, L + m + (long)r0 * lda, lda, T + r0 + (long)r0 * ldt, ldt, 0.0, W, ldw,
             nullptr, st);
    gemm_f64(m2, m1, m2, -1.0, T + m + (long)m * ldt, ldt, W, ldw, 0.0, T + m + (long)r0 * ldt, ldt,
             nullptr, st);
}
}  // namespace

void chol_inverse(double* A, int n, int lda, double* T, double* W, double* Tt, double* small, int* err,
                  cudaStream_t st) {
    set_smem_attr();
    double* Linv = small;
    double* R = small + NB * NB;
    // 1. blocked right-looking Cholesky (lower triangle of A becomes L)
    for (int k0 = 0; k0 < n; k0 += NB) {
        const int kb = min(NB, n - k0), k1 = k0 + kb;
        k_chol_diag<<<1, 256, SQ_SMEM, st>>>(A, lda, k0, kb, Linv, err);
        count_launch();
        if (k1 < n) {
            const int rows = n - k1;
            k_chol_panel<<<(rows + NB - 1) / NB, 256, SQ_SMEM, st>>>(A, lda, n, k0, kb, k1, Linv, R);
            count_launch();
            gemm_f64_tri(rows, rows, kb, -1.0, A + k1 + (long)k0 * lda, lda, R + (long)k1 * NB, NB, 1.0,
                         A + k1 + (long)k1 * lda, lda, st);
        }
    }
    // 2. T = L^{-1}: leaves, then recursive merges
    k_trtri_leaves<<<(n + NB - 1) / NB, 256, SQ_SMEM, st>>>(A, lda, n, T, lda);
    count_launch();
    trtri_merge(A, lda, T, lda, W, lda, 0, n, st);
    // 3. A^{-1} = T^T T
    dim3 g((n + 31) / 32, (n + 31) / 32);
    k_transpose<<<g, dim3(32, 8), 0, st>>>(T, lda, n, Tt, lda);
    count_launch();
    gemm_f64(n, n, n, 1.0, Tt, lda, T, lda, 0.0, A, lda, nullptr, st);
}

// ------------------------------------------------------------------------
// elementwise helpers
// ------------------------------------------------------------------------
__global__ void k_shift_diag_scale(double* A, int n, long lda, double lambda, double* e, int* err) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double d = A[i + i * lda] + lambda;
    A[i + i * lda] = d;
    if (!(d > 0.0 && isfinite(d))) {
        atomicOr(err, ERRBIT_SINGULAR);
        e[i] = 1.0;
    } else {
        e[i] = 1.0 / sqrt(d);
    }
}

__global__ void k_scale_sym(double* A, int n, long lda, const double* __restrict__ e,
                            double* Y, long ldy) {
    long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
    long total = (long)n * n;
    if (idx >= total) return;
    int c = (int)(idx / n), r = (int)(idx - (long)c * n);
    double v = A[r + c * lda] * e[r] * e[c];
    A[r + c * lda] = v;
    if (Y) Y[r + c * ldy] = v;
}

void launch_shift_equilibrate(double* A, int n, int lda, double lambda, double* e, int* err,
                              cudaStream_t st) {
    k_shift_diag_scale<<<(n + 255) / 256, 256, 0, st>>>(A, n, lda, lambda, e, err);
    long total = (long)n * n;
    k_scale_sym<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(A, n, lda, e, nullptr, 0);
    count_launch(2);
}

void launch_unequilibrate(double* X, int n, int lda, const double* e, double* Y, cudaStream_t st) {
    long total = (long)n * n;
    k_scale_sym<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(X, n, lda, e, Y, lda);
    count_launch();
}

__global__ void k_axpy(double* Y, const double* __restrict__ X, double k, int n, long ld) {
    long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
    long total = (long)n * n;
    if (idx >= total) return;
    int c = (int)(idx / n), r = (int)(idx - (long)c * n);
    long o = r + c * ld;
    Y[o] = Y[o] + k * X[o];
}

void launch_axpy(double* Y, const double* X, double k, int n, int ld, cudaStream_t st) {
    long total = (long)n * n;
    k_axpy<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(Y, X, k, n, ld);
    count_launch();
}

void launch_zero(double* p, size_t n, cudaStream_t st) { cudaMemsetAsync(p, 0, n * sizeof(double), st); }

// Camera output: for camera c and j <= k in its block,
//   camUnc = (iZ(j,k) + iZ(k,j)/2) * d_j * d_k,  d = 1/s   (compute.cpp:176)
// plus the unscaled 9x9 covariance used by the point stage (compute.cpp:435):
//   sig(j,k) = iZ(j,k) * d_j * d_k.
__global__ void k_camera_output(const double* __restrict__ iZ, long ldz,
                                const double* __restrict__ s_cam, int num_cams, double* cam_unc,
                                double* sig) {
    int c = blockIdx.x;
    int e = threadIdx.x;  // 0..80
    if (c >= num_cams || e >= 81) return;
    int j = e / 9, k = e - j * 9;
    long r = 9L * c + j, q = 9L * c + k;
    double dj = 1.0 / s_cam[r], dk = 1.0 / s_cam[q];
    double a = iZ[r + q * ldz], b = iZ[q + r * ldz];
    sig[81L * c + e] = a * dj * dk;
    if (k >= j) {
        int t = j * 9 - (j * (j - 1)) / 2 + (k - j);
        cam_unc[45L * c + t] = (a + b / 2) * dj * dk;
    }
}

void launch_camera_output(const double* iZ, int ldz, const double* s_cam, int num_cams,
                          double* cam_unc, double* sig, cudaStream_t st) {
    if (num_cams == 0) return;
    k_camera_output<<<num_cams, 96, 0, st>>>(iZ, ldz, s_cam, num_cams, cam_unc, sig);
    count_launch();
}

}  // namespace unc
