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
               unsigned long long* amax) {
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
    k_gemm_f64<<<grid, GEMM_THREADS, GEMM_SMEM, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, amax);
    count_launch();
}

// ------------------------------------------------------------------------
// Blocked Gauss-Jordan inverse (SPD, no pivoting)
// ------------------------------------------------------------------------
constexpr int GJ_NB = 64;

size_t gj_workspace_doubles(int n) {
    // P (nb x nb), Cbuf (ld_of(n) x nb), Rbuf (nb x n, ld = nb)
    return (size_t)GJ_NB * GJ_NB + (size_t)ld_of(n) * GJ_NB + (size_t)GJ_NB * (n + 8) + 64;
}

// In-place Gauss-Jordan inverse of the kb x kb diagonal block (kb <= 64) in
// shared memory; one CTA. Writes the inverse to P (kb x kb, ld GJ_NB).
__global__ void __launch_bounds__(256) k_gj_diag(double* A, long lda, int k0, int kb, double* P,
                                                 int* err) {
    __shared__ double a[GJ_NB][GJ_NB + 1];  // a[row][col]
    __shared__ double fcol[GJ_NB];
    const int tid = threadIdx.x;
    for (int e = tid; e < kb * kb; e += blockDim.x) {
        int r = e % kb, c = e / kb;
        a[r][c] = A[(k0 + r) + (long)(k0 + c) * lda];
    }
    __syncthreads();
    for (int p = 0; p < kb; ++p) {
        double piv = a[p][p];
        if (tid == 0 && !(piv > 0.0 && isfinite(piv))) atomicOr(err, ERRBIT_SINGULAR);
        __syncthreads();
        // save column p (rows != p) and scale row p
        for (int i = tid; i < kb; i += blockDim.x) fcol[i] = a[i][p];
        __syncthreads();
        double ip = 1.0 / piv;
        for (int j = tid; j < kb; j += blockDim.x) a[p][j] = (j == p ? 1.0 : a[p][j]) * ip;
        __syncthreads();
        for (int e = tid; e < kb * kb; e += blockDim.x) {
            int i = e % kb, j = e / kb;
            if (i == p) continue;
            double v = (j == p ? 0.0 : a[i][j]);
            a[i][j] = v - fcol[i] * a[p][j];
        }
        __syncthreads();
    }
    for (int e = tid; e < kb * kb; e += blockDim.x) {
        int r = e % kb, c = e / kb;
        P[r + (long)c * GJ_NB] = a[r][c];
    }
}

// Row panel: R(:, j) = P * A(k rows, j) for j outside the pivot block (0
// inside), written back into A's pivot rows. Column panel: Cb(i, :) = A(i, k
// cols) for i outside the pivot block (0 inside), A(i, k cols) = -Cb(i,:) P.
// Pivot block: A_kk = P. blockIdx.y = 0 -> row panel, 1 -> column panel.
__global__ void __launch_bounds__(256) k_gj_panels(double* A, long lda, int n, int k0, int kb,
                                                   const double* __restrict__ P, double* Cb,
                                                   long ldc, double* R) {
    extern __shared__ double gj_smem[];
    double(*sp)[GJ_NB + 1] = reinterpret_cast<double(*)[GJ_NB + 1]>(gj_smem);  // sp[r][c] = P(r, c)
    double(*sx)[GJ_NB + 1] = sp + GJ_NB;                                        // chunk
    const int tid = threadIdx.x;
    for (int e = tid; e < kb * kb; e += blockDim.x) {
        int r = e % kb, c = e / kb;
        sp[r][c] = P[r + (long)c * GJ_NB];
    }
    const int c0 = blockIdx.x * GJ_NB;  // chunk start (columns for the row panel, rows for the column panel)
    const int cn = min(GJ_NB, n - c0);
    if (cn <= 0) return;
    if (blockIdx.y == 0) {
        // sx[r][j] = A(k0 + r, c0 + j)
        for (int e = tid; e < kb * cn; e += blockDim.x) {
            int r = e % kb, j = e / kb;
            sx[r][j] = A[(k0 + r) + (long)(c0 + j) * lda];
        }
        __syncthreads();
        for (int e = tid; e < kb * cn; e += blockDim.x) {
            int r = e % kb, j = e / kb;
            int col = c0 + j;
            double v;
            if (col >= k0 && col < k0 + kb) {
                v = 0.0;
                A[(k0 + r) + (long)col * lda] = sp[r][col - k0];  // A_kk = P
            } else {
                double s = 0.0;
                for (int q = 0; q < kb; ++q) s += sp[r][q] * sx[q][j];
                v = s;
                A[(k0 + r) + (long)col * lda] = s;
            }
            R[r + (long)col * GJ_NB] = v;
        }
    } else {
        // sx[i][q] = A(c0 + i, k0 + q)
        for (int e = tid; e < cn * kb; e += blockDim.x) {
            int i = e % cn, q = e / cn;
            sx[i][q] = A[(c0 + i) + (long)(k0 + q) * lda];
        }
        __syncthreads();
        for (int e = tid; e < cn * kb; e += blockDim.x) {
            int i = e % cn, q = e / cn;
            int row = c0 + i;
            if (row >= k0 && row < k0 + kb) {
                Cb[row + (long)q * ldc] = 0.0;
            } else {
                double s = 0.0;
                for (int r = 0; r < kb; ++r) s += sx[i][r] * sp[r][q];
                Cb[row + (long)q * ldc] = sx[i][q];
                A[row + (long)(k0 + q) * lda] = -s;
            }
        }
    }
}

void gj_inverse(double* A, int n, int lda, double* ws, int* err, cudaStream_t st) {
    double* P = ws;
    double* Cb = P + GJ_NB * GJ_NB;
    const int ldc = ld_of(n);
    double* R = Cb + (size_t)ldc * GJ_NB;
    cudaMemsetAsync(Cb, 0, sizeof(double) * ((size_t)ldc * GJ_NB + (size_t)GJ_NB * (n + 8)), st);
    const int nchunks = (n + GJ_NB - 1) / GJ_NB;
    const int panel_smem = (int)(sizeof(double) * 2 * GJ_NB * (GJ_NB + 1));
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_gj_panels, cudaFuncAttributeMaxDynamicSharedMemorySize, panel_smem);
        attr = true;
    }
    for (int k0 = 0; k0 < n; k0 += GJ_NB) {
        int kb = n - k0 < GJ_NB ? n - k0 : GJ_NB;
        k_gj_diag<<<1, 256, 0, st>>>(A, lda, k0, kb, P, err);
        k_gj_panels<<<dim3(nchunks, 2), 256, panel_smem, st>>>(A, lda, n, k0, kb, P, Cb, ldc, R);
        count_launch(2);
        // A -= Cb * R  (rank-kb update; pivot rows/cols receive zero updates)
        gemm_f64(n, n, kb, -1.0, Cb, ldc, R, GJ_NB, 1.0, A, lda, nullptr, st);
    }
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
