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
constexpr int B_STAGE = BN * LDB_S;  // >= BK * LDA_S (layout of a transposed B tile)
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
template <bool kTransB>
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
    if (kTransB) {
        // B(k, n) = B[n + k * ldb]: tile stored Bs[k][n] like A
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            int idx = tid + q * GEMM_THREADS;
            int k = idx >> 6, n2 = (idx & 63) * 2;
            bool p = (n0 + n2 < N) && (k0 + k < K);
            const double* src = p ? B + (n0 + n2) + (long)(k0 + k) * ldb : B;
            cp_async16(Bs + k * LDA_S + n2, src, p);
        }
    } else {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            int idx = tid + q * GEMM_THREADS;
            int n = idx >> 3, k2 = (idx & 7) * 2;
            bool p = (n0 + n < N) && (k0 + k2 < K);
            const double* src = p ? B + (k0 + k2) + (long)(n0 + n) * ldb : B;
            cp_async16(Bs + n * LDB_S + k2, src, p);
        }
    }
}

template <bool kTransB>
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
        if (s < KT) load_tiles<kTransB>(As + s * A_STAGE, Bs + s * B_STAGE, A, lda, B, ldb, M, N, K, m0, n0, s * BK, tid);
        cp_async_commit();
    }
    for (int kt = 0; kt < KT; ++kt) {
        cp_async_wait<STAGES - 2>();
        __syncthreads();
        int pf = kt + STAGES - 1;
        if (pf < KT) {
            int ps = pf % STAGES;
            load_tiles<kTransB>(As + ps * A_STAGE, Bs + ps * B_STAGE, A, lda, B, ldb, M, N, K, m0, n0, pf * BK, tid);
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
            for (int j = 0; j < 8; ++j)
                bf[j] = kTransB ? bs[(kk + t) * LDA_S + wn + j * 8 + g] : bs[(wn + j * 8 + g) * LDB_S + kk + t];
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

void gemm_f64_ex(int M, int N, int K, double alpha, const double* A, int lda, const double* B, int ldb,
                 double beta, double* C, int ldc, unsigned long long* amax, bool lower_only, cudaStream_t st,
                 bool trans_b) {
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_gemm_f64<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GEMM_SMEM);
        cudaFuncSetAttribute(k_gemm_f64<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GEMM_SMEM);
        attr = true;
    }
    if (M <= 0 || N <= 0) return;
    dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM);
    if (trans_b)
        k_gemm_f64<true><<<grid, GEMM_THREADS, GEMM_SMEM, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc,
                                                                amax, lower_only ? 1 : 0);
    else
        k_gemm_f64<false><<<grid, GEMM_THREADS, GEMM_SMEM, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc,
                                                                 amax, lower_only ? 1 : 0);
    count_launch();
}

void gemm_f64(int M, int N, int K, double alpha, const double* A, int lda, const double* B, int ldb,
              double beta, double* C, int ldc, unsigned long long* amax, cudaStream_t st) {
    gemm_f64_ex(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, amax, false, st, false);
}

void gemm_f64_tri(int M, int N, int K, double alpha, const double* A, int lda, const double* B, int ldb,
                  double beta, double* C, int ldc, cudaStream_t st) {
    gemm_f64_ex(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, nullptr, true, st, false);
}

// Copy the strict lower triangle onto the upper one (32 x 32 tiles).
__global__ void k_mirror_lower(double* Z, int n, long ld) {
    __shared__ double t[32][33];
    const int bi = blockIdx.y, bj = blockIdx.x;  // tile row, tile col of the source (lower) tile
    if (bj > bi) return;
    for (int r = threadIdx.y; r < 32; r += 8) {
        int i = bi * 32 + r, j = bj * 32 + threadIdx.x;
        t[r][threadIdx.x] = (i < n && j < n) ? Z[i + (long)j * ld] : 0.0;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += 8) {
        int j = bj * 32 + r, i = bi * 32 + threadIdx.x;  // target (j, i) = source (i, j), i > j
        if (i < n && j < n && i > j) Z[j + (long)i * ld] = t[threadIdx.x][r];
    }
}

void launch_mirror_lower(double* Z, int n, int ld, cudaStream_t st) {
    if (n == 0) return;
    dim3 g((n + 31) / 32, (n + 31) / 32);
    k_mirror_lower<<<g, dim3(32, 8), 0, st>>>(Z, n, ld);
    count_launch();
}

// ------------------------------------------------------------------------
// SPD inverse: blocked Cholesky A = L L^T, T = L^{-1}, A^{-1} = T^T T
// ------------------------------------------------------------------------
constexpr int NB = 64;                       // panel width

size_t chol_small_doubles(int n) { (void)n; return (size_t)NB * NB + 64; }

// Cholesky of the kb x kb (kb <= 64) diagonal block at (k0, k0) and the
// inverse of its factor in one CTA of 1024 threads. Thread t owns the
// lower-triangle elements e = t and e = t + 1024 (row-major packing of the
// 2080 elements of a 64 x 64 lower triangle) in registers, both of L and of
// T = L^{-1}. Every elimination step publishes one column (and one row of T)
// through shared memory and costs two barriers; the pivot scale rsqrt(d) is
// applied on the fly, so no extra pass is needed.
// Writes L_kk into A (lower), T_kk into the diagonal block of T, and T_kk^T
// into LinvT (64 x 64, column-major: LinvT[k + 64 q] = T_kk(q, k)), the B
// operand of the panel solve L_ik = A_ik T_kk^T.
constexpr int kTri = NB * (NB + 1) / 2;  // 2080

__device__ __forceinline__ void tri_rc(int e, int& i, int& j) {
    // e = i (i + 1) / 2 + j, 0 <= j <= i
    int r = (int)((sqrtf(8.0f * (float)e + 1.0f) - 1.0f) * 0.5f);
    while ((r + 1) * (r + 2) / 2 <= e) ++r;
    while (r * (r + 1) / 2 > e) --r;
    i = r;
    j = e - r * (r + 1) / 2;
}

__global__ void __launch_bounds__(1024) k_chol_diag(double* A, long lda, int k0, int kb, double* T, long ldt,
                                                    double* LinvT, int* err) {
    __shared__ double colv[NB], rowt[NB], ilv[NB];
    const int tid = threadIdx.x;
    constexpr int E = (kTri + 1023) / 1024;  // 3 elements for the first threads, 2 for the rest
    int ii[E], jj[E];
    bool v[E];
    double a[E], t[E];
#pragma unroll
    for (int k = 0; k < E; ++k) {
        const int e = tid + 1024 * k;
        if (e < kTri) {
            tri_rc(e, ii[k], jj[k]);
        } else {
            ii[k] = jj[k] = 0;
        }
        v[k] = e < kTri && ii[k] < kb;
        a[k] = v[k] ? A[(k0 + ii[k]) + (long)(k0 + jj[k]) * lda] : 0.0;
    }
    for (int p = 0; p < kb; ++p) {
#pragma unroll
        for (int k = 0; k < E; ++k)
            if (v[k] && jj[k] == p) colv[ii[k]] = a[k];
        __syncthreads();
        const double d = colv[p];
        const double r = rsqrt(d);
        if (tid == 0) {
            ilv[p] = r;
            if (!(d > 0.0 && d <= 1.7976931348623157e308)) atomicOr(err, ERRBIT_SINGULAR);
        }
#pragma unroll
        for (int k = 0; k < E; ++k) {
            if (!v[k]) continue;
            if (jj[k] == p) a[k] = (ii[k] == p) ? d * r : a[k] * r;
            else if (jj[k] > p) a[k] -= (colv[ii[k]] * r) * (colv[jj[k]] * r);
        }
        __syncthreads();
    }
    // T = L^{-1}: forward elimination on [L | I]
#pragma unroll
    for (int k = 0; k < E; ++k) t[k] = (v[k] && ii[k] == jj[k]) ? 1.0 : 0.0;
    for (int p = 0; p < kb; ++p) {
        const double r = ilv[p];
#pragma unroll
        for (int k = 0; k < E; ++k) {
            if (!v[k]) continue;
            if (ii[k] == p) {
                t[k] *= r;
                rowt[jj[k]] = t[k];
            } else if (jj[k] == p && ii[k] > p) {
                colv[ii[k]] = a[k];
            }
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < E; ++k)
            if (v[k] && ii[k] > p && jj[k] <= p) t[k] -= colv[ii[k]] * rowt[jj[k]];
        __syncthreads();
    }
    for (int e = tid; e < NB * NB; e += 1024) LinvT[e] = 0.0;
    __syncthreads();
#pragma unroll
    for (int k = 0; k < E; ++k) {
        if (!v[k]) continue;
        const int i = ii[k], j = jj[k];
        A[(k0 + i) + (long)(k0 + j) * lda] = a[k];
        T[(k0 + i) + (long)(k0 + j) * ldt] = t[k];
        if (i != j) T[(k0 + j) + (long)(k0 + i) * ldt] = 0.0;
        LinvT[j + (long)i * NB] = t[k];  // LinvT(k = j, q = i) = T(i, j)
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
    double* LinvT = small;
    // 1. blocked right-looking Cholesky (lower triangle of A becomes L); the
    //    diagonal blocks of T = L^{-1} are produced on the way
    for (int k0 = 0; k0 < n; k0 += NB) {
        const int kb = min(NB, n - k0), k1 = k0 + kb;
        k_chol_diag<<<1, 1024, 0, st>>>(A, lda, k0, kb, T, lda, LinvT, err);
        count_launch();
        if (k1 < n) {
            const int rows = n - k1;
            double* P = A + k1 + (long)k0 * lda;  // panel below the pivot block
            // L_ik = A_ik T_kk^T, in place (each CTA owns its rows and all 64 columns)
            gemm_f64_ex(rows, kb, kb, 1.0, P, lda, LinvT, NB, 0.0, P, lda, nullptr, false, st, false);
            // A22 -= L_ik L_ik^T, lower tiles; B = panel^T read in place
            gemm_f64_ex(rows, rows, kb, -1.0, P, lda, P, lda, 1.0, A + k1 + (long)k1 * lda, lda, nullptr, true,
                        st, true);
        }
    }
    // 2. T = L^{-1}: recursive merges above the inverted diagonal blocks
    trtri_merge(A, lda, T, lda, W, lda, 0, n, st);
    // 3. A^{-1} = T^T T (symmetric: lower-triangle tiles, then mirror)
    dim3 g((n + 31) / 32, (n + 31) / 32);
    k_transpose<<<g, dim3(32, 8), 0, st>>>(T, lda, n, Tt, lda);
    count_launch();
    gemm_f64_ex(n, n, n, 1.0, Tt, lda, T, lda, 0.0, A, lda, nullptr, true, st, false);
    launch_mirror_lower(A, n, lda, st);
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
