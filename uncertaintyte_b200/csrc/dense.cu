// dense.cu - FP64 dense kernels for the inverse of the camera Schur
// complement (sm_100a):
//   * gemm_f64      : C = alpha*A*B + beta*C on DMMA (mma.sync m8n8k4 f64),
//                     3-stage cp.async pipeline of 32-deep K tiles, optional fused max|C| for the
//                     Taylor stop rule (ScaledDenseMatrix.cpp:207-216,314-353),
//                     lower-tile and triangular-operand (k range per tile) modes.
//   * chol_inverse  : SPD inverse by recursive Cholesky that forms T = L^{-1}
//                     on the way, then A^{-1} = T^T T; every step is a GEMM
//                     (replaces dgetrf+dgetri in SDM::inv, ScaledDenseMatrix.cpp:232-279).
//   * shift/equilibrate, un-equilibrate, axpy (iZupdate, compute.cpp:64-71),
//     camera output with the reference's (a + b/2) quirk (compute.cpp:168-183).
#include <algorithm>

#include "chol_leaf.cuh"
#include "internal.h"

namespace unc {

// ------------------------------------------------------------------------
// GEMM
// ------------------------------------------------------------------------
namespace {
constexpr int BK = 32, STAGES = 3, GEMM_THREADS = 256;  // 32-deep K stages: half the barriers of 16
constexpr int LDB_S = BK + 4;  // Bs[n][k]: 36 doubles per n row (8 mod 32 banks: conflict-free fragment reads)

// Output tile BM x BN computed by 8 warps of WM x WN (FM x FN fragments of
// the 8 x 8 DMMA result). Shared-memory rows of A (and of the transposed B)
// are padded by 4 doubles: a fragment read takes rows kk + t (t = 0..3) at 8
// doubles apart in bank space (row pitch = 8 mod 32 banks), so each half-warp
// hits 16 distinct bank pairs; cp.async rows stay 16-byte aligned.
template <int BM_, int BN_, int WM_, int WN_>
struct GemmCfg {
    static constexpr int BM = BM_, BN = BN_, WM = WM_, WN = WN_;
    static constexpr int WARPS_M = BM / WM;
    static_assert((BM / WM) * (BN / WN) == GEMM_THREADS / 32, "8 warps per CTA");
    static constexpr int FM = WM / 8, FN = WN / 8;
    static constexpr int LDA_S = BM + 4;   // As[k][m]
    static constexpr int LDBT_S = BN + 4;  // Bs[k][n] (transposed B)
    static_assert((2 * LDA_S) % 32 == 8 && (2 * LDBT_S) % 32 == 8, "conflict-free fragment rows");
    static constexpr int A_STAGE = BK * LDA_S;
    static constexpr int B_STAGE = (BN * LDB_S > BK * LDBT_S) ? BN * LDB_S : BK * LDBT_S;
    static constexpr size_t SMEM = sizeof(double) * (size_t)STAGES * (A_STAGE + B_STAGE);
    static constexpr int A_CHUNKS = BM * BK / 2 / GEMM_THREADS;  // 16-byte copies per thread
    static constexpr int B_CHUNKS = BN * BK / 2 / GEMM_THREADS;
};
using CfgBig = GemmCfg<128, 128, 32, 64>;   // 1 CTA per SM (212 KB shared)
using CfgSmall = GemmCfg<64, 64, 16, 32>;   // small outputs: 4x the CTAs (108 KB shared, 2 per SM)

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

// Accumulation. By default the products accumulate in the MMA's own C
// operand over the whole k range. With GEMM_SHORT_ACC they accumulate there
// over two 8 x 8 x 4 steps only (k = 8), starting from zero, and those partial
// sums are added to the running sums with ordinary FP64 additions (IEEE
// round to nearest): accumulating in the C operand over the thousands of
// steps of a long dot product carried a one-sided rounding into the SPD
// inverse's Cholesky pivots (the last ones are ~lambda, formed by cancellation
// from O(1) entries, and set the inverse's largest, gauge, components), so the
// products that feed pivots (L21 = A21 T11^T and A22 -= L21 L21^T) take it.
__device__ __forceinline__ void dmma0(double& t0, double& t1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%4,%4};\n"
                 : "=d"(t0), "=d"(t1)
                 : "d"(a), "d"(b), "d"(0.0));
}
__device__ __forceinline__ void dmma_acc(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}
}  // namespace

// Tile loader: A tile (BM rows x BK cols of column-major A), B tile (BK rows
// x BN cols of column-major B). Out-of-range chunks are zero-filled. Rows
// past M (or K for B) inside the allocation are read as 16-byte pairs; the
// values there only meet zero-filled partners or land in unstored rows, so
// they must merely be finite.
template <class Cfg, bool kTransB>
__device__ __forceinline__ void load_tiles(double* As, double* Bs, const double* __restrict__ A,
                                           long lda, const double* __restrict__ B, long ldb, int M,
                                           int N, int K, int m0, int n0, int k0, int tid) {
    constexpr int AH = Cfg::BM / 2, BH = Cfg::BN / 2;
#pragma unroll
    for (int q = 0; q < Cfg::A_CHUNKS; ++q) {
        int idx = tid + q * GEMM_THREADS;
        int k = idx / AH, m2 = (idx % AH) * 2;
        bool p = (m0 + m2 < M) && (k0 + k < K);
        const double* src = p ? A + (m0 + m2) + (long)(k0 + k) * lda : A;
        cp_async16(As + k * Cfg::LDA_S + m2, src, p);
    }
    if (kTransB) {
        // B(k, n) = B[n + k * ldb]: tile stored Bs[k][n] like A
#pragma unroll
        for (int q = 0; q < Cfg::B_CHUNKS; ++q) {
            int idx = tid + q * GEMM_THREADS;
            int k = idx / BH, n2 = (idx % BH) * 2;
            bool p = (n0 + n2 < N) && (k0 + k < K);
            const double* src = p ? B + (n0 + n2) + (long)(k0 + k) * ldb : B;
            cp_async16(Bs + k * Cfg::LDBT_S + n2, src, p);
        }
    } else {
#pragma unroll
        for (int q = 0; q < Cfg::B_CHUNKS; ++q) {
            int idx = tid + q * GEMM_THREADS;
            int n = idx / (BK / 2), k2 = (idx % (BK / 2)) * 2;
            bool p = (n0 + n < N) && (k0 + k2 < K);
            const double* src = p ? B + (k0 + k2) + (long)(n0 + n) * ldb : B;
            cp_async16(Bs + n * LDB_S + k2, src, p);
        }
    }
}

template <class Cfg, bool kTransB, bool kShortAcc>
__global__ void __launch_bounds__(GEMM_THREADS, (Cfg::BM == 128 ? 1 : 2))
    k_gemm_f64(int M, int N, int K, double alpha, const double* __restrict__ A, long lda,
               const double* __restrict__ B, long ldb, double beta, double* C, long ldc,
               unsigned long long* amax, int mode, double* part, const int* skip) {
    constexpr int BM = Cfg::BM, BN = Cfg::BN, FM = Cfg::FM, FN = Cfg::FN;
    if (skip && *skip) return;
    // GEMM_LOWER: tiles strictly above the diagonal of C are skipped (SYRK-style update)
    if ((mode & GEMM_LOWER) && (int)(blockIdx.x * BN) > (int)(blockIdx.y * BM) + BM - 1) return;
    extern __shared__ __align__(16) double smem[];
    double* As = smem;
    double* Bs = smem + STAGES * Cfg::A_STAGE;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = (warp % Cfg::WARPS_M) * Cfg::WM, wn = (warp / Cfg::WARPS_M) * Cfg::WN;
    const int g = lane >> 2, t = lane & 3;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const bool wact = (m0 + wm < M) && (n0 + wn < N);
    // triangular operands: the k range of this tile outside which a product term is zero
    int kbeg = 0, kend = K;
    if (mode & GEMM_KLO_M) kbeg = max(kbeg, m0);
    if (mode & GEMM_KLO_N) kbeg = max(kbeg, n0);
    if (mode & GEMM_KHI_M) kend = min(kend, m0 + BM);
    if (mode & GEMM_KHI_N) kend = min(kend, n0 + BN);
    int kt0 = kbeg / BK;
    int KT = kend > kbeg ? (kend + BK - 1) / BK - kt0 : 0;  // k tiles of this output tile
    if (gridDim.z > 1) {  // split-K: a contiguous share of the k tiles, partial sums to part
        const int chunk = (KT + gridDim.z - 1) / gridDim.z;
        const int b0 = min(KT, (int)blockIdx.z * chunk);
        KT = min(KT, b0 + chunk) - b0;
        kt0 += b0;
    }

    double acc[FM][FN][2];
#pragma unroll
    for (int i = 0; i < FM; ++i)
#pragma unroll
        for (int j = 0; j < FN; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
        if (s < KT)
            load_tiles<Cfg, kTransB>(As + s * Cfg::A_STAGE, Bs + s * Cfg::B_STAGE, A, lda, B, ldb, M, N, K, m0,
                                     n0, (kt0 + s) * BK, tid);
        cp_async_commit();
    }
    for (int kt = 0; kt < KT; ++kt) {
        cp_async_wait<STAGES - 2>();
        __syncthreads();
        int pf = kt + STAGES - 1;
        if (pf < KT) {
            int ps = pf % STAGES;
            load_tiles<Cfg, kTransB>(As + ps * Cfg::A_STAGE, Bs + ps * Cfg::B_STAGE, A, lda, B, ldb, M, N, K,
                                     m0, n0, (kt0 + pf) * BK, tid);
        }
        cp_async_commit();
        const double* as = As + (kt % STAGES) * Cfg::A_STAGE;
        const double* bs = Bs + (kt % STAGES) * Cfg::B_STAGE;
        if (!wact) continue;  // this warp's sub-tile lies outside C
        if (kShortAcc) {
#pragma unroll 1
            for (int kk = 0; kk < BK; kk += 8) {  // two 4-deep steps: a partial sum from zero, then added
                double af[2][FM], bf[2][FN];
#pragma unroll
                for (int h = 0; h < 2; ++h) {
#pragma unroll
                    for (int i = 0; i < FM; ++i) af[h][i] = as[(kk + 4 * h + t) * Cfg::LDA_S + wm + i * 8 + g];
#pragma unroll
                    for (int j = 0; j < FN; ++j)
                        bf[h][j] = kTransB ? bs[(kk + 4 * h + t) * Cfg::LDBT_S + wn + j * 8 + g]
                                           : bs[(wn + j * 8 + g) * LDB_S + kk + 4 * h + t];
                }
                constexpr int FH = FN >= 8 ? FN / 2 : FN;  // fragments per group (register pressure)
#pragma unroll
                for (int i = 0; i < FM; ++i)  // FH partial sums at a time, then added
#pragma unroll
                    for (int j0 = 0; j0 < FN; j0 += FH) {
                        double p[FH][2];
#pragma unroll
                        for (int j = 0; j < FH; ++j) dmma0(p[j][0], p[j][1], af[0][i], bf[0][j0 + j]);
#pragma unroll
                        for (int j = 0; j < FH; ++j) dmma_acc(p[j][0], p[j][1], af[1][i], bf[1][j0 + j]);
#pragma unroll
                        for (int j = 0; j < FH; ++j) {
                            acc[i][j0 + j][0] += p[j][0];
                            acc[i][j0 + j][1] += p[j][1];
                        }
                    }
            }
        } else {
#pragma unroll
            for (int kk = 0; kk < BK; kk += 4) {
                double af[FM], bf[FN];
#pragma unroll
                for (int i = 0; i < FM; ++i) af[i] = as[(kk + t) * Cfg::LDA_S + wm + i * 8 + g];
#pragma unroll
                for (int j = 0; j < FN; ++j)
                    bf[j] = kTransB ? bs[(kk + t) * Cfg::LDBT_S + wn + j * 8 + g]
                                    : bs[(wn + j * 8 + g) * LDB_S + kk + t];
#pragma unroll
                for (int i = 0; i < FM; ++i)
#pragma unroll
                    for (int j = 0; j < FN; ++j) dmma_acc(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
            }
        }
    }
    cp_async_wait<0>();

    if (part) {  // raw partial tile of split blockIdx.z (M x N slab, leading dimension M)
        double* P = part + (size_t)blockIdx.z * M * N;
#pragma unroll
        for (int i = 0; i < FM; ++i) {
            int row = m0 + wm + i * 8 + g;
#pragma unroll
            for (int j = 0; j < FN; ++j)
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    int col = n0 + wn + j * 8 + t * 2 + h;
                    if (row < M && col < N) P[row + (size_t)col * M] = acc[i][j][h];
                }
        }
        return;
    }

    double mx = 0.0;
#pragma unroll
    for (int i = 0; i < FM; ++i) {
        int row = m0 + wm + i * 8 + g;
#pragma unroll
        for (int j = 0; j < FN; ++j) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                int col = n0 + wn + j * 8 + t * 2 + h;
                if (row < M && col < N && (!(mode & GEMM_MIRROR) || row >= col)) {
                    double* c = C + row + (long)col * ldc;
                    double v = alpha * acc[i][j][h];
                    if (beta != 0.0) v += beta * *c;
                    *c = v;
                    if ((mode & GEMM_MIRROR) && row > col) C[col + (long)row * ldc] = v;
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

// C = alpha * sum_s part[s] + beta * C over the tiles the GEMM computed
// (tile size bm x bn), the splits summed in a fixed order (deterministic),
// max|C| folded into amax.
__global__ void k_splitk_reduce(int M, int N, int splits, const double* __restrict__ part, double alpha,
                                double beta, double* C, long ldc, unsigned long long* amax, int mode, int bm,
                                int bn, const int* skip) {
    if (skip && *skip) return;
    const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
    double mx = 0.0;
    if (idx < (long)M * N) {
        const int col = (int)(idx / M), row = (int)(idx - (long)col * M);
        if (!((mode & GEMM_LOWER) && (col / bn) * bn > (row / bm) * bm + bm - 1) &&
            !((mode & GEMM_MIRROR) && row < col)) {
            double v = 0.0;
            for (int s = 0; s < splits; ++s) v += part[(size_t)s * M * N + idx];
            double* c = C + row + (long)col * ldc;
            v *= alpha;
            if (beta != 0.0) v += beta * *c;
            *c = v;
            if ((mode & GEMM_MIRROR) && row > col) C[col + (long)row * ldc] = v;
            const double av = fabs(v);
            mx = av <= 1.7976931348623157e308 ? av : __longlong_as_double(0x7ff0000000000000LL);
        }
    }
    if (amax) {
        const int lane = threadIdx.x & 31;
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, d));
        if (lane == 0 && mx > 0.0) atomicMax(amax, (unsigned long long)__double_as_longlong(mx));
    }
}

namespace {
template <class Cfg>
int active_tiles(dim3 grid, int mode) {
    if (!(mode & GEMM_LOWER)) return (int)(grid.x * grid.y);
    int tiles = 0;
    for (unsigned by = 0; by < grid.y; ++by)
        for (unsigned bx = 0; bx < grid.x; ++bx) tiles += (int)(bx * Cfg::BN) <= (int)(by * Cfg::BM) + Cfg::BM - 1;
    return tiles;
}

template <class Cfg>
void gemm_attr() {
    static std::atomic<unsigned long long> attr{0};
    once_per_device(attr, [] {
        return cudaFuncSetAttribute(k_gemm_f64<Cfg, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)Cfg::SMEM) == cudaSuccess &&
               cudaFuncSetAttribute(k_gemm_f64<Cfg, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)Cfg::SMEM) == cudaSuccess &&
               cudaFuncSetAttribute(k_gemm_f64<Cfg, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)Cfg::SMEM) == cudaSuccess &&
               cudaFuncSetAttribute(k_gemm_f64<Cfg, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)Cfg::SMEM) == cudaSuccess;
    });
}

template <class Cfg>
void launch_gemm(int M, int N, int K, double alpha, const double* A, int lda, const double* B, int ldb, double beta,
                 double* C, int ldc, unsigned long long* amax, int mode, cudaStream_t st, double* ws,
                 size_t ws_doubles, const int* skip) {
    gemm_attr<Cfg>();
    dim3 grid((N + Cfg::BN - 1) / Cfg::BN, (M + Cfg::BM - 1) / Cfg::BM);
    // split-K when the output has too few tiles to fill the SMs: each split
    // keeps at least kMinSplitTiles k tiles, the partial slabs fit in ws
    const int tiles = active_tiles<Cfg>(grid, mode);
    constexpr int kSMs = 148, kMinSplitTiles = 3, kMaxSplits = 16;
    const int slots = kSMs * (Cfg::BM == 128 ? 1 : 2);
    int splits = 1;
    const int kt = (K + BK - 1) / BK;
    if (ws && tiles > 0 && tiles < slots && kt >= 2 * kMinSplitTiles) {
        splits = std::min(std::min(slots / tiles, kt / kMinSplitTiles), kMaxSplits);
        const size_t slab = (size_t)M * N;
        while (splits > 1 && (size_t)splits * slab > ws_doubles) --splits;
    }
    double* part = splits > 1 ? ws : nullptr;
    grid.z = splits;
    const bool tb = (mode & GEMM_TRANS_B) != 0, sa = (mode & GEMM_SHORT_ACC) != 0;
    auto kern = tb ? (sa ? k_gemm_f64<Cfg, true, true> : k_gemm_f64<Cfg, true, false>)
                   : (sa ? k_gemm_f64<Cfg, false, true> : k_gemm_f64<Cfg, false, false>);
    kern<<<grid, GEMM_THREADS, Cfg::SMEM, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, amax, mode, part,
                                                skip);
    count_launch();
    if (part) {
        const long total = (long)M * N;
        k_splitk_reduce<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(M, N, splits, part, alpha, beta, C, ldc,
                                                                          amax, mode, Cfg::BM, Cfg::BN, skip);
        count_launch();
    }
}
}  // namespace

void gemm_f64_mode(int M, int N, int K, double alpha, const double* A, int lda, const double* B, int ldb,
                   double beta, double* C, int ldc, unsigned long long* amax, int mode, cudaStream_t st,
                   double* ws, size_t ws_doubles, const int* skip) {
    if (M <= 0 || N <= 0) return;
    // 64 x 64 tiles when 128 x 128 tiles would leave most SMs idle
    const dim3 g128((N + 127) / 128, (M + 127) / 128);
    if (active_tiles<CfgBig>(g128, mode) * 4 <= 148)
        launch_gemm<CfgSmall>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, amax, mode, st, ws, ws_doubles, skip);
    else
        launch_gemm<CfgBig>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, amax, mode, st, ws, ws_doubles, skip);
}

void gemm_f64_ex(int M, int N, int K, double alpha, const double* A, int lda, const double* B, int ldb,
                 double beta, double* C, int ldc, unsigned long long* amax, bool lower_only, cudaStream_t st,
                 bool trans_b) {
    gemm_f64_mode(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, amax,
                  (lower_only ? GEMM_LOWER : 0) | (trans_b ? GEMM_TRANS_B : 0), st);
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
__global__ void k_mirror_lower(double* Z, int n, long ld, const int* skip) {
    if (skip && *skip) return;
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

void launch_mirror_lower(double* Z, int n, int ld, cudaStream_t st, const int* skip) {
    if (n == 0) return;
    dim3 g((n + 31) / 32, (n + 31) / 32);
    k_mirror_lower<<<g, dim3(32, 8), 0, st>>>(Z, n, ld, skip);
    count_launch();
}

// ------------------------------------------------------------------------
// SPD inverse: recursive Cholesky A = L L^T that forms T = L^{-1} on the
// way, then A^{-1} = T^T T
// ------------------------------------------------------------------------
size_t chol_small_doubles(int n) { (void)n; return (size_t)NB * NB + 64; }

__global__ void __launch_bounds__(LEAF_THREADS) k_chol_leaf(const double* __restrict__ A, long lda, int k0,
                                                            int kb, double* T, long ldt, int* err) {
    extern __shared__ __align__(16) double lsm[];
    chol_leaf_tile(A, lda, k0, kb, T, ldt, err, lsm);
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

void prepare_dense_kernels() {
    gemm_attr<CfgBig>();
    gemm_attr<CfgSmall>();
    static std::atomic<unsigned long long> attr{0};
    once_per_device(attr, [] {
        return cudaFuncSetAttribute(k_chol_leaf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LEAF_SMEM) ==
               cudaSuccess;
    });
}

namespace {

// Factor A[r0:r1, r0:r1] (already updated by the earlier panels) and write
// T[r0:r1, r0:r1] = L^{-1}. With the split [r0, m) [m, r1):
//   L21 = A21 T11^T                 (into W; T11^T upper triangular)
//   A22 -= L21 L21^T                (lower tiles)
//   X   = L21 T11                   (into the A21 slot; T11 lower triangular)
//   recurse on A22 -> T22
//   T21 = -T22 X                    (T22 lower triangular)
// Every product is a GEMM whose k loop skips the zero triangle of its
// triangular operand, so the whole recursion costs n^3 / 3 + n^3 / 3 flops.
void chol_rec(double* A, int lda, double* T, double* W, double* ws, size_t wsd, int r0, int r1, int* err,
              cudaStream_t st) {
    const int n = r1 - r0;
    if (n <= NB) {
        prepare_dense_kernels();
        k_chol_leaf<<<1, LEAF_THREADS, LEAF_SMEM, st>>>(A, lda, r0, n, T, lda, err);
        count_launch();
        return;
    }
    int m = r0 + ((n / 2 + NB - 1) / NB) * NB;
    if (m >= r1) m = r1 - NB;
    const int h1 = m - r0, h2 = r1 - m;
    chol_rec(A, lda, T, W, ws, wsd, r0, m, err, st);
    double* A21 = A + m + (long)r0 * lda;
    const double* T11 = T + r0 + (long)r0 * lda;
    gemm_f64_mode(h2, h1, h1, 1.0, A21, lda, T11, lda, 0.0, W, lda, nullptr,
                  GEMM_TRANS_B | GEMM_KHI_N | GEMM_SHORT_ACC, st, ws, wsd);
    gemm_f64_mode(h2, h2, h1, -1.0, W, lda, W, lda, 1.0, A + m + (long)m * lda, lda, nullptr,
                  GEMM_TRANS_B | GEMM_LOWER | GEMM_SHORT_ACC, st, ws, wsd);
    gemm_f64_mode(h2, h1, h1, 1.0, W, lda, T11, lda, 0.0, A21, lda, nullptr, GEMM_KLO_N, st, ws, wsd);
    chol_rec(A, lda, T, W, ws, wsd, m, r1, err, st);
    gemm_f64_mode(h2, h1, h2, -1.0, T + m + (long)m * lda, lda, A21, lda, 0.0, T + m + (long)r0 * lda, lda,
                  nullptr, GEMM_KHI_M, st, ws, wsd);
}
}  // namespace

void chol_lower_inverse(double* A, int n, int lda, double* T, double* W, double* ws, int* err, cudaStream_t st) {
    chol_rec(A, lda, T, W, ws, (size_t)n * lda, 0, n, err, st);
}

void chol_inverse(double* A, int n, int lda, double* T, double* W, double* Tt, double* small, int* err,
                  cudaStream_t st) {
    (void)small;
    // Tt is free until the final product: split-K partial sums of the recursion
    chol_lower_inverse(A, n, lda, T, W, Tt, err, st);
    // A^{-1} = T^T T: lower tiles, k >= the tile's first row (T lower triangular), then mirror
    dim3 g((n + 31) / 32, (n + 31) / 32);
    k_transpose<<<g, dim3(32, 8), 0, st>>>(T, lda, n, Tt, lda);
    count_launch();
    gemm_f64_mode(n, n, n, 1.0, Tt, lda, T, lda, 0.0, A, lda, nullptr, GEMM_LOWER | GEMM_KLO_M, st);
    launch_mirror_lower(A, n, lda, st);
}

// ------------------------------------------------------------------------
// elementwise helpers
// ------------------------------------------------------------------------
__device__ __forceinline__ void shift_diag_one(double* A, int i, long lda, double lambda, double* e, int* err) {
    double d = A[i + i * lda] + lambda;
    A[i + i * lda] = d;
    if (!(d > 0.0 && isfinite(d))) {
        atomicOr(err, ERRBIT_SINGULAR);
        e[i] = 1.0;
    } else {
        e[i] = 1.0 / sqrt(d);
    }
}

__global__ void k_shift_diag_scale(double* A, int n, long lda, double lambda, double* e, int* err) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    shift_diag_one(A, i, lda, lambda, e, err);
}

// element idx of a column-major n x n matrix: A <- A e_r e_c (and Y = the same)
__device__ __forceinline__ void scale_sym_one(double* A, long idx, int n, long lda, const double* __restrict__ e,
                                              double* Y, long ldy) {
    int c = (int)(idx / n), r = (int)(idx - (long)c * n);
    double v = A[r + c * lda] * e[r] * e[c];
    A[r + c * lda] = v;
    if (Y) Y[r + c * ldy] = v;
}

__global__ void k_scale_sym(double* A, int n, long lda, const double* __restrict__ e,
                            double* Y, long ldy) {
    long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
    long total = (long)n * n;
    if (idx >= total) return;
    scale_sym_one(A, idx, n, lda, e, Y, ldy);
}

void launch_shift_equilibrate(double* A, int n, int lda, double lambda, double* e, int* err,
                              cudaStream_t st) {
    k_shift_diag_scale<<<(n + 255) / 256, 256, 0, st>>>(A, n, lda, lambda, e, err);
    long total = (long)n * n;
    k_scale_sym<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(A, n, lda, e, nullptr, 0);
    count_launch(2);
}

__device__ __forceinline__ void scale_sym_from_one(const double* __restrict__ S, double* A, long idx, int n,
                                                   long lda, const double* __restrict__ e, double* Y, long ldy) {
    int c = (int)(idx / n), r = (int)(idx - (long)c * n);
    double v = S[r + c * lda] * e[r] * e[c];
    A[r + c * lda] = v;
    if (Y) Y[r + c * ldy] = v;
}

__global__ void k_scale_sym_from(const double* __restrict__ S, double* A, int n, long lda,
                                 const double* __restrict__ e, double* Y, long ldy) {
    long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
    long total = (long)n * n;
    if (idx >= total) return;
    scale_sym_from_one(S, A, idx, n, lda, e, Y, ldy);
}

void launch_unequilibrate_from(const double* S, double* X, int n, int lda, const double* e, double* Y,
                               cudaStream_t st) {
    long total = (long)n * n;
    k_scale_sym_from<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(S, X, n, lda, e, Y, lda);
    count_launch();
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

__device__ __forceinline__ void te_decide_one(TeState* s, const unsigned long long* amax_bits, double k) {
    if (s->done) return;
    double amax = __longlong_as_double((long long)*amax_bits);
    amax = fmax(amax, 2.2250738585072014e-308);  // absMax starts at DBL_MIN (ScaledDenseMatrix.cpp:208)
    if (!(amax <= 1.7976931348623157e308)) s->bad = 1;
    const double change = fabs(k * amax);
    if (change < 1e-5 || change > s->old_change) {  // compute.cpp:150-152
        s->done = 1;
        return;
    }
    s->old_change = change;
    if (s->iters < 20) s->change[s->iters] = change;
    s->iters += 1;
    s->coef = k;
}

__global__ void k_te_decide(TeState* s, const unsigned long long* amax_bits, double k) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    te_decide_one(s, amax_bits, k);
}

__device__ __forceinline__ void te_init_one(TeState* s) {
    s->done = 0;
    s->bad = 0;
    s->iters = 0;
    s->old_change = 1.7976931348623157e308;  // DBL_MAX (compute.cpp:140)
    s->coef = 0.0;
    for (int i = 0; i < 20; ++i) s->change[i] = 0.0;
    for (int i = 0; i < 20; ++i) s->c[i] = 0.0;
    for (int i = 0; i < 8; ++i) s->skip[i] = 0;
}

__global__ void k_te_init(TeState* s) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    te_init_one(s);
}

// ---- grouped forms over the dense stages of many matrices (a batch) ----
// Block b of an element-wise launch belongs to job m with blk[m] <= b < blk[m + 1].
__device__ __forceinline__ int job_of_block(const long* __restrict__ blk, int njobs, long b) {
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (blk[mid] <= b) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__global__ void k_shift_diag_scale_grouped(const DenseJob* __restrict__ jobs, int njobs, const long* __restrict__ blk) {
    const int m = job_of_block(blk, njobs, blockIdx.x);
    const DenseJob& j = jobs[m];
    const long i = (blockIdx.x - blk[m]) * (long)blockDim.x + threadIdx.x;
    if (i < j.n) shift_diag_one(j.Z, (int)i, j.ld, j.lambda, j.e, j.err);
}

__global__ void k_scale_sym_grouped(const DenseJob* __restrict__ jobs, int njobs, const long* __restrict__ blk) {
    const int m = job_of_block(blk, njobs, blockIdx.x);
    const DenseJob& j = jobs[m];
    const long idx = (blockIdx.x - blk[m]) * (long)blockDim.x + threadIdx.x;
    if (idx < (long)j.n * j.n) scale_sym_one(j.Z, idx, j.n, j.ld, j.e, nullptr, 0);
}

__global__ void k_unequilibrate_grouped(const DenseJob* __restrict__ jobs, int njobs, const long* __restrict__ blk) {
    const int m = job_of_block(blk, njobs, blockIdx.x);
    const DenseJob& j = jobs[m];
    const long idx = (blockIdx.x - blk[m]) * (long)blockDim.x + threadIdx.x;
    if (idx < (long)j.n * j.n) scale_sym_from_one(j.add, j.Z, idx, j.n, j.ld, j.e, j.iZ, j.ld);
}

__global__ void k_te_init_grouped(const DenseJob* __restrict__ jobs, int njobs) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m < njobs) te_init_one(jobs[m].te);
}

__global__ void k_te_decide_grouped(const DenseJob* __restrict__ jobs, int njobs, const double* __restrict__ k) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m < njobs) te_decide_one(jobs[m].te, jobs[m].amax, k[m]);
}

void launch_shift_equilibrate_grouped(const DenseJob* d_jobs, int njobs, const long* d_blk_rows, long nblk_rows,
                                      const long* d_blk_elems, long nblk_elems, cudaStream_t st) {
    if (njobs <= 0) return;
    k_shift_diag_scale_grouped<<<(unsigned)nblk_rows, 256, 0, st>>>(d_jobs, njobs, d_blk_rows);
    k_scale_sym_grouped<<<(unsigned)nblk_elems, 256, 0, st>>>(d_jobs, njobs, d_blk_elems);
    count_launch(2);
}

void launch_unequilibrate_grouped(const DenseJob* d_jobs, int njobs, const long* d_blk_elems, long nblk_elems,
                                  cudaStream_t st) {
    if (njobs <= 0) return;
    k_unequilibrate_grouped<<<(unsigned)nblk_elems, 256, 0, st>>>(d_jobs, njobs, d_blk_elems);
    count_launch();
}

void launch_te_init_grouped(const DenseJob* d_jobs, int njobs, cudaStream_t st) {
    if (njobs <= 0) return;
    k_te_init_grouped<<<(njobs + 127) / 128, 128, 0, st>>>(d_jobs, njobs);
    count_launch();
}

void launch_te_decide_grouped(const DenseJob* d_jobs, int njobs, const double* d_k, cudaStream_t st) {
    if (njobs <= 0) return;
    k_te_decide_grouped<<<(njobs + 127) / 128, 128, 0, st>>>(d_jobs, njobs, d_k);
    count_launch();
}

void launch_te_init(TeState* s, cudaStream_t st) {
    k_te_init<<<1, 32, 0, st>>>(s);
    count_launch();
}

void launch_te_decide(TeState* s, const unsigned long long* amax, double k, cudaStream_t st) {
    k_te_decide<<<1, 32, 0, st>>>(s, amax, k);
    count_launch();
}

__global__ void k_axpy_te(double* Y, const double* __restrict__ X, const TeState* s, int n, long ld) {
    if (s->done) return;
    const double k = s->coef;
    long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
    long total = (long)n * n;
    if (idx >= total) return;
    int c = (int)(idx / n), r = (int)(idx - (long)c * n);
    long o = r + c * ld;
    Y[o] = Y[o] + k * X[o];
}

void launch_axpy_te(double* Y, const double* X, const TeState* s, int n, int ld, cudaStream_t st) {
    long total = (long)n * n;
    k_axpy_te<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(Y, X, s, n, ld);
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
    // s_cam == nullptr: no column scaling (the SVD path, removeScaleJ4Z with d = NULL)
    double dj = s_cam ? 1.0 / s_cam[r] : 1.0, dk = s_cam ? 1.0 / s_cam[q] : 1.0;
    double a = iZ[r + q * ldz], b = iZ[q + r * ldz];
    if (sig) sig[81L * c + e] = a * dj * dk;
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
