// mixed.cu - mixed-precision Taylor-series products on the sm_100a tensor
// cores (tcgen05, kind::i8), fed by TMA, accumulated in TMEM.
//
// A dense FP64 product C = P * X of symmetric operands is evaluated from
// 7-bit integer slices of the operands (the Ozaki splitting):
//
//   row r of P:  P[r, :] = 2^e_r * (sum_{s=1..S} P_s[r, :] 2^(-7 s) + tail),  P_s int8
//   row c of X:  X[c, :] = 2^f_c * (sum_{t=1..S} X_t[c, :] 2^(-7 t) + tail)
//   C[r, c]     = 2^(e_r + f_c) * sum_{L=2..S+1} 2^(-7 L) * sum_{s+t=L} (P_s X_t^T)[r, c]
//
// The digits are rounded to nearest (|digit| <= 64, row scale chosen so that
// |P[r, k]| 2^-e_r < 1/2): the tails are zero-mean, so their contributions
// partly cancel over K instead of adding up with one sign as truncated digits
// do. Each slice product is an int8 GEMM with exact int32 accumulation
// ((L-1) K 64^2 < 2^31 for K < 10^5); products of the same level L share one
// TMEM accumulator, and the FP64 epilogue combines the levels. The error is
// about 2^(-7 S) relative to the row/column maxima: S = 5 gives ~1e-10 on the
// Taylor products of the reference scenes, S = 4 ~1e-8. Both operands are
// symmetric, so their columns are their rows and the column-major FP64
// matrices are read as K-major operands.
//
// Kernel layout: 128 threads. Warp 0 lane 0 issues the TMA loads of the S
// slices of both operands per 64-byte K block (3-stage mbarrier pipeline);
// warp 1 lane 0 issues the tcgen05.mma (M = 128, N = up to 256, K = 32 bytes:
// one A slice against several adjacent B slices) and commits each stage back
// to the producer; all four warps then read the
// accumulators with tcgen05.ld and write FP64. Every mbarrier wait has an
// iteration limit after which the kernel records ERRBIT_TIMEOUT and unwinds
// (TMEM is always freed).
#include <algorithm>
#include <functional>
#include <queue>
#include <vector>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "internal.h"

namespace unc {

namespace mp {

constexpr int BM = 128;         // tile rows (TMEM lanes)
constexpr int BKB = 64;         // K bytes per pipeline stage (SWIZZLE_64B rows)
constexpr int STAGES = 3;
constexpr int THREADS = 128;
constexpr long kSpinLimit = 1L << 26;

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// bounded wait for the completion of phase `parity`; false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
    const unsigned a = smem_u32(bar);
    for (long it = 0; it < kSpinLimit; ++it) {
        unsigned ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::
            "r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// K-major shared-memory matrix descriptor, 64-byte swizzle: rows of 64 bytes,
// 8-row groups 512 bytes apart (SBO), version 1 (sm_100).
__device__ __forceinline__ uint64_t desc_sw64(const void* p) {
    const uint64_t addr = smem_u32(p);
    return ((addr >> 4) & 0x3FFFull) | (1ull << 16) | ((uint64_t)(512 >> 4) << 32) | (1ull << 46) |
           (4ull << 61);
}

// instruction descriptor: kind::i8, signed A/B, S32 accumulate, K-major, M=128, N=n
__host__ __device__ constexpr uint32_t idesc_i8(int n) {
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, bool acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc ? 1u : 0u));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// 16 consecutive 32-bit TMEM columns of this warp's 32 lanes; the values may
// be used only after tmem_wait_ld.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, int (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }

// After tmem_wait_ld: ties the 16 registers to this point of the program, so
// that no use of them is scheduled before the wait.
__device__ __forceinline__ void tmem_fence_regs(int (&r)[16]) {
    asm volatile("" : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]),
                 "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]),
                 "+r"(r[14]), "+r"(r[15]));
}

template <int NT, int S>
struct Shape {
    static constexpr int A_BOX = BM * BKB;                 // bytes of one A slice box
    static constexpr int B_BOX = NT * BKB;                 // bytes of one B slice box
    static constexpr int STAGE = S * (A_BOX + B_BOX);
    static constexpr int LEVELS = S;                       // L = 2 .. S+1
    static constexpr int GROUP = 256 / NT;                 // B slices per MMA (N <= 256)
    static constexpr int TMEM_COLS = LEVELS * NT <= 256 ? (LEVELS * NT <= 128 ? 128 : 256) : 512;
    // three pipeline stages where they fit in the 227 KB of shared memory, else two
    static constexpr int NSTAGE = STAGES * STAGE + 1280 <= 232448 ? STAGES : 2;
    static constexpr int SMEM = NSTAGE * STAGE + 1024 /*align*/ + 256 /*barriers*/;
    static_assert(SMEM <= 232448, "one CTA's shared memory is at most 227 KB");
    static_assert(LEVELS * NT <= 512, "TMEM holds at most 512 accumulator columns");
};

}  // namespace mp

using namespace mp;

// Slice rows of a symmetric FP64 matrix (row j = column j, contiguous) into S
// int8 planes out[s][j][k] (pitch kp bytes, plane stride rows_pad * kp) of
// round-to-nearest digits in [-64, 64], and the row exponents e[j] with
// max_k |A[j,k]| 2^-e < 1/2. One CTA per row.
// 2^e exactly (bit pattern for normal exponents): v * pow2(e) == ldexp(v, e)
__device__ __forceinline__ double pow2(int e) {
    return (e >= -1022 && e <= 1023) ? __longlong_as_double((long long)(e + 1023) << 52) : ldexp(1.0, e);
}

// Y (optional): Y += te->coef * A on the way (the Taylor update iZ += k add of
// the power being sliced, compute.cpp:64-71), unless te->done.
// Row j of one matrix, all 256 threads of the block (red: 8 shared doubles).
__device__ __forceinline__ void slice_row(int j, const double* __restrict__ A, long lda, int n, int S,
                                          int8_t* __restrict__ out, int rows_pad, int kp, int* __restrict__ exps,
                                          double* Y, const TeState* te, double* red) {
    const double* col = A + (long)j * lda;
    double m = 0.0;
    for (int k = threadIdx.x; k < n; k += 256) m = fmax(m, fabs(col[k]));
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, d));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < 8 ? red[threadIdx.x] : 0.0;
#pragma unroll
        for (int d = 4; d > 0; d >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, d));
        if (threadIdx.x == 0) red[0] = v;
    }
    __syncthreads();
    int e = 0;
    if (red[0] > 0.0 && red[0] <= 1.7976931348623157e308) frexp(red[0], &e);  // max * 2^-e in [0.5, 1)
    e += 1;                                                                     // max * 2^-e in [0.25, 0.5)
    if (threadIdx.x == 0) exps[j] = e;
    if (Y) {
        const double c = te->coef;
        double* y = Y + (long)j * lda;
        for (int k = threadIdx.x; k < n; k += 256) y[k] += c * col[k];
    }
    const double sc = pow2(-e);
    const size_t plane = (size_t)rows_pad * kp;
    int8_t* row = out + (size_t)j * kp;
    for (int k0 = 4 * threadIdx.x; k0 < n; k0 += 4 * 256) {
        double v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) v[u] = (k0 + u < n) ? col[k0 + u] * sc : 0.0;
        for (int s = 0; s < S; ++s) {
            char4 q;
            signed char qs[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                v[u] *= 128.0;
                const double t = rint(v[u]);  // |v| <= 64 before, |v - t| <= 1/2 after
                v[u] -= t;
                qs[u] = (signed char)(int)t;
            }
            q.x = qs[0];
            q.y = qs[1];
            q.z = qs[2];
            q.w = qs[3];
            if (k0 + 3 < n) {
                *reinterpret_cast<char4*>(row + s * plane + k0) = q;
            } else {
                for (int u = 0; u < 4 && k0 + u < n; ++u) row[s * plane + k0 + u] = qs[u];
            }
        }
    }
}

__global__ void __launch_bounds__(256) k_slice_rows(const double* __restrict__ A, long lda, int n, int S,
                                                   int8_t* __restrict__ out, int rows_pad, int kp,
                                                   int* __restrict__ exps, const int* skip, double* Y,
                                                   const TeState* te) {
    if (skip && *skip) return;
    __shared__ double red[8];
    slice_row(blockIdx.x, A, lda, n, S, out, rows_pad, kp, exps, Y, te, red);
}

// The same over the rows of many matrices (a batch): block b slices row
// b - row_start[m] of matrix m, row_start[m] <= b < row_start[m + 1].
__global__ void __launch_bounds__(256) k_slice_rows_grouped(const MixedSliceJob* __restrict__ jobs, int njobs,
                                                           const int* __restrict__ row_start) {
    int lo = 0, hi = njobs - 1;
    const int b = blockIdx.x;
    while (lo < hi) {  // the last m with row_start[m] <= b
        const int mid = (lo + hi + 1) >> 1;
        if (row_start[mid] <= b) lo = mid; else hi = mid - 1;
    }
    const MixedSliceJob& jb = jobs[lo];
    if (jb.skip && *jb.skip) return;
    __shared__ double red[8];
    slice_row(b - row_start[lo], jb.A, jb.lda, jb.n, jb.S, jb.out, jb.rows_pad, jb.kp, jb.exps, jb.Y, jb.te, red);
}

// One 128 x NT output tile at (m0, n0): TMA producer, MMA issuer, epilogue.
// tA / tB: the operands' tensor maps (kernel parameters, or 64-byte aligned
// maps in global memory written before the launch: maps_in_global).
template <int NT, int S>
__device__ __forceinline__ void ozaki_tile(const CUtensorMap* tA, const CUtensorMap* tB, int m0, int n0, int M, int N,
                                           int kp, int rowsA, int rowsB, const int* __restrict__ eA,
                                           const int* __restrict__ eB, double* C, long ldc,
                                           unsigned long long* amax, int* err, int mirror, bool maps_in_global,
                                           int accumulate, int klo = 0) {
    using Sh = Shape<NT, S>;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(base + Sh::NSTAGE * Sh::STAGE);
    uint64_t* empty = full + Sh::NSTAGE;
    uint64_t* done = empty + Sh::NSTAGE;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tmem_slot)),
                     "r"(Sh::TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    if (tid == 32) {
        for (int s = 0; s < Sh::NSTAGE; ++s) {
            mbar_init(full + s, 1);
            mbar_init(empty + s, 1);
        }
        mbar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    const int KT = kp / BKB;
    // klo: both operands are the columns of one lower-triangular matrix T (C = T^T T),
    // column r being zero above row r, so no term of this tile has k < max(m0, n0)
    const int kt0 = klo ? (m0 > n0 ? m0 : n0) / BKB : 0;
    const int kt1 = KT;

    if (warp == 0) {
      if (lane == 0) {
        // TMA producer
        if (maps_in_global) {  // maps written to global memory by the host: acquire them for the TMA unit
            asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;\n" ::"l"(tA) : "memory");
            asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;\n" ::"l"(tB) : "memory");
        }
        bool ok = true;
        int issued = 0;
        for (int kt = kt0; kt < kt1 && ok; ++kt) {
            const int i = kt - kt0;  // pipeline step
            const int s = i % Sh::NSTAGE;
            const unsigned ph = (unsigned)(i / Sh::NSTAGE) & 1u;
            if (i >= Sh::NSTAGE && !mbar_wait(empty + s, ph ^ 1u)) {
                atomicOr(err, ERRBIT_TIMEOUT);
                ok = false;
                break;
            }
            uint8_t* st = base + s * Sh::STAGE;
            mbar_expect_tx(full + s, Sh::STAGE);
            for (int q = 0; q < S; ++q) tma_load_2d(st + q * Sh::A_BOX, tA, kt * BKB, q * rowsA + m0, full + s);
            for (int q = 0; q < S; ++q)
                tma_load_2d(st + S * Sh::A_BOX + q * Sh::B_BOX, tB, kt * BKB, q * rowsB + n0, full + s);
            issued = i + 1;
        }
        // no copy may be in flight when the CTA exits
        for (int i = issued - Sh::NSTAGE < 0 ? 0 : issued - Sh::NSTAGE; i < issued; ++i)
            if (!mbar_wait(full + i % Sh::NSTAGE, (unsigned)(i / Sh::NSTAGE) & 1u)) atomicOr(err, ERRBIT_TIMEOUT);
      }
      __syncwarp();
    } else if (warp == 1) {
      if (lane == 0) {
        // MMA issuer
        for (int i = 0; i < kt1 - kt0; ++i) {
            const int s = i % Sh::NSTAGE;
            if (!mbar_wait(full + s, (unsigned)(i / Sh::NSTAGE) & 1u)) {
                atomicOr(err, ERRBIT_TIMEOUT);
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const uint8_t* st = base + s * Sh::STAGE;
#pragma unroll
            for (int kk = 0; kk < BKB / 32; ++kk) {
                // A slice sa meets B slices 1 .. S+1-sa, whose levels sa-1 .. S-1 are adjacent
                // accumulators: consecutive B boxes form one taller operand, so one MMA of
                // N = g * NT (<= 256) covers g of them and A is read once per group.
#pragma unroll
                for (int sa = 1; sa <= S; ++sa) {
                    const uint64_t a = desc_sw64(st + (sa - 1) * Sh::A_BOX + kk * 32);
#pragma unroll
                    for (int sb0 = 1; sb0 <= S + 1 - sa; sb0 += Sh::GROUP) {
                        const int g = (S + 1 - sa - sb0 + 1) < Sh::GROUP ? (S + 1 - sa - sb0 + 1) : Sh::GROUP;
                        const int l = sa + sb0 - 2;
                        const uint64_t b = desc_sw64(st + S * Sh::A_BOX + (sb0 - 1) * Sh::B_BOX + kk * 32);
                        // the first A slice of the first K step opens every level
                        mma_i8(tmem + (uint32_t)(l * NT), a, b, idesc_i8(g * NT), i > 0 || kk > 0 || sa > 1);
                    }
                }
            }
            mma_commit(empty + s);  // stage free once these MMAs completed
        }
        mma_commit(done);
      }
      __syncwarp();
    }
    // epilogue: every warp reads its 32 TMEM lanes (tile rows)
    const bool ok = __all_sync(0xffffffffu, mbar_wait(done, 0));  // warp-uniform
    if (!ok && lane == 0) atomicOr(err, ERRBIT_TIMEOUT);
    __syncwarp();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const int row = m0 + warp * 32 + lane;
    const int er = row < M ? eA[row] : 0;
    double mx = 0.0;
    if (ok) {
        for (int c0 = 0; c0 < NT; c0 += 16) {
            // all levels' accumulators of these 16 columns in one round trip
            int r[S][16];
#pragma unroll
            for (int l = 0; l < S; ++l) tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(l * NT + c0), r[l]);
            // accumulate: the previous values of C, loaded together before any store of
            // this chunk (reads are of the lower triangle, mirrored stores go above it)
            double prev[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int col = n0 + c0 + j;
                prev[j] = accumulate && row < M && col < N && (!mirror || row >= col) ? C[row + (long)col * ldc] : 0.0;
            }
            tmem_wait_ld();
#pragma unroll
            for (int l = 0; l < S; ++l) tmem_fence_regs(r[l]);
            double v[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) v[j] = 0.0;
#pragma unroll
            for (int l = S - 1; l >= 0; --l) {  // small levels first
                const double w = ldexp(1.0, -7 * (l + 2));
#pragma unroll
                for (int j = 0; j < 16; ++j) v[j] += (double)r[l][j] * w;
            }
            if (row < M) {
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int col = n0 + c0 + j;
                    if (col < N) {
                        double x = v[j] * pow2(er + eB[col]);
                        // mirror: the lower triangle is written at (row, col) and at
                        // (col, row); nothing above the diagonal is written directly
                        // accumulate: C += P X (C symmetric: its lower element is read)
                        if (accumulate && (!mirror || row >= col)) x += prev[j];
                        if (!mirror || row >= col) {
                            C[row + (long)col * ldc] = x;
                            const double ax = fabs(x);
                            mx = fmax(mx, ax <= 1.7976931348623157e308 ? ax
                                                                       : __longlong_as_double(0x7ff0000000000000LL));
                        }
                        if (mirror && row > col) C[col + (long)row * ldc] = x;
                    }
                }
            }
        }
    }
    if (amax) {
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, d));
        if (lane == 0) atomicMax(amax, (unsigned long long)__double_as_longlong(mx));
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(Sh::TMEM_COLS));
}

// Lower-triangle tile t of an n x n product in grouped order: row blocks in
// groups of gm, each group walked column by column (the rows of a column whose
// lower tiles reach it), so that the CTAs running together share the B tiles
// of a few columns and the A tiles of gm row blocks in L2 instead of streaming
// B once per row block. O(columns) integer steps per CTA.
__device__ __forceinline__ void grouped_lower_tile(int t, int n, int nt, int gm, int& by, int& bx) {
    const int by_n = (n + BM - 1) / BM, bx_n = (n + nt - 1) / nt;
    by = bx = 0;
    for (int r0 = 0; r0 < by_n; r0 += gm) {
        const int r1 = min(r0 + gm, by_n) - 1;
        const int cols = min((r1 * BM + BM - 1) / nt + 1, bx_n);
        for (int c = 0; c < cols; ++c) {
            const int need = c * nt - (BM - 1);  // by * BM + BM - 1 >= c * nt
            const int lo = max(r0, need > 0 ? (need + BM - 1) / BM : 0);
            const int cnt = r1 - lo + 1;
            if (t < cnt) {
                by = lo + t;
                bx = c;
                return;
            }
            t -= cnt;
        }
    }
}

template <int NT, int S>
__global__ void __launch_bounds__(THREADS, 1)
    k_ozaki_gemm(const __grid_constant__ CUtensorMap tA, const __grid_constant__ CUtensorMap tB, int M, int N,
                 int kp, int rowsA, int rowsB, const int* __restrict__ eA, const int* __restrict__ eB, double* C,
                 long ldc, unsigned long long* amax, int lower_only, int* err, const int* skip, int mirror,
                 int accumulate, int group_m, int klo) {
    if (skip && *skip) return;
    int m0, n0;
    if (group_m > 0) {  // 1-D grid over exactly the lower tiles, grouped order
        __shared__ int s_tile[2];
        if (threadIdx.x == 0) grouped_lower_tile(blockIdx.x, N, NT, group_m, s_tile[0], s_tile[1]);
        __syncthreads();
        m0 = s_tile[0] * BM;
        n0 = s_tile[1] * NT;
    } else {
        m0 = blockIdx.y * BM;
        n0 = blockIdx.x * NT;
        if (lower_only && n0 > m0 + BM - 1) return;
    }
    ozaki_tile<NT, S>(&tA, &tB, m0, n0, M, N, kp, rowsA, rowsB, eA, eB, C, ldc, amax, err, mirror, false,
                      accumulate, klo);
}

// The products of many matrices (a batch) in one launch: CTA b computes tile
// tiles[b] = (job, m0, n0) of jobs[job] (lower-triangle tiles only; the result
// mirrored). The per-element arithmetic is that of k_ozaki_gemm for any tile
// width, so a batch gives the bytes of one launch per matrix.
template <int NT, int S>
__global__ void __launch_bounds__(THREADS, 1)
    k_ozaki_gemm_grouped(const MixedGemmJob* __restrict__ jobs, const int4* __restrict__ tiles) {
    const int4 t = tiles[blockIdx.x];
    const MixedGemmJob& j = jobs[t.x];
    if (j.skip && *j.skip) return;
    ozaki_tile<NT, S>(j.tA, j.tB, t.y, t.z, j.n, j.n, j.kp, j.rowsA, j.rowsB, j.eA, j.eB, j.C, j.ldc, j.amax, j.err,
                      1, true, j.accumulate);
}

// ------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------
namespace {
PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
    // a driver entry point: the same for every device; resolved once, thread-safe
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        cudaDriverEntryPointQueryResult q;
        void* p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        return (PFN_cuTensorMapEncodeTiled_v12000) nullptr;
    }();
    return fn;
}

// 2-D map over `rows` rows of `kp` int8 (row pitch kp bytes), box = box_rows x 64 bytes, 64-byte swizzle
bool make_map(CUtensorMap* map, const int8_t* base, int rows, int kp, int box_rows) {
    auto enc = get_encode();
    if (!enc) return false;
    cuuint64_t dims[2] = {(cuuint64_t)kp, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)kp};
    cuuint32_t box[2] = {(cuuint32_t)BKB, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<int8_t*>(base), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

template <int NT, int S>
void set_attr_once() {
    static std::atomic<unsigned long long> done{0};
    once_per_device(done, [] {
        return cudaFuncSetAttribute(k_ozaki_gemm<NT, S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    Shape<NT, S>::SMEM) == cudaSuccess;
    });
}
}  // namespace

template <int NT, int S>
void set_attr_grouped_once() {
    static std::atomic<unsigned long long> done{0};
    once_per_device(done, [] {
        return cudaFuncSetAttribute(k_ozaki_gemm_grouped<NT, S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    Shape<NT, S>::SMEM) == cudaSuccess;
    });
}

void prepare_mixed_kernels() {
    set_attr_once<128, 4>();
    set_attr_once<64, 5>();
    set_attr_once<96, 5>();
    set_attr_once<128, 3>();
    set_attr_once<128, 2>();
    set_attr_once<64, kGramSlices>();
    set_attr_grouped_once<128, 4>();
    set_attr_grouped_once<64, 5>();
    set_attr_grouped_once<96, 5>();
    set_attr_grouped_once<128, 3>();
    set_attr_grouped_once<128, 2>();
}

// Output tile width: slices * tile_n <= 512 TMEM columns, so 128 for up to 4
// slices and 96 for 5. For 5 slices a 64-wide tile is taken when it needs
// fewer tile-waves on the 148 SMs: the lower-triangle tile count of an n x n
// product is what fills the machine at moderate n (n = 1800: 164 tiles of
// 128 x 96 take two waves, the second 16 tiles deep; 239 tiles of 128 x 64
// also take two, each 2/3 as long). Cost model: waves x (tile_n + 16), the
// 16 standing for the per-tile prologue and epilogue.
static int lower_tiles(int n, int nt) {
    int tiles = 0;
    const int by_n = (n + BM - 1) / BM, bx_n = (n + nt - 1) / nt;
    for (int by = 0; by < by_n; ++by) {
        const int last = (by * BM + BM - 1) / nt;  // last tile column on or below the diagonal
        tiles += (last + 1 < bx_n ? last + 1 : bx_n);
    }
    return tiles;
}

int mixed_tile_n(int slices, int n) {
    if (slices <= 4) return 128;
    constexpr int kSMs = 148;
    const long w96 = (lower_tiles(n, 96) + kSMs - 1) / kSMs, w64 = (lower_tiles(n, 64) + kSMs - 1) / kSMs;
    return w64 * (64 + 16) < w96 * (96 + 16) ? 64 : 96;
}

double mixed_issued_ops(int n, int slices) {
    const int nt = mixed_tile_n(slices, n);
    const double kp = (double)(((n + BKB - 1) / BKB) * BKB);
    return 2.0 * (slices * (slices + 1) / 2) * (double)lower_tiles(n, nt) * BM * nt * kp;
}

static int mixed_rows(int n, int slices) {
    const int nt = mixed_tile_n(slices, n);
    const int ra = ((n + BM - 1) / BM) * BM, rb = ((n + nt - 1) / nt) * nt;
    return ra > rb ? ra : rb;
}

size_t mixed_slice_bytes(int n, int slices) {
    const int kp = ((n + BKB - 1) / BKB) * BKB;
    return (size_t)slices * (size_t)mixed_rows(n, slices) * kp;
}

bool mixed_plan(MixedOperand& op, int8_t* buf, int* exps, int n, int slices, bool as_b) {
    const int nt = mixed_tile_n(slices, n);
    op.n = n;
    op.slices = slices;
    op.kp = ((n + BKB - 1) / BKB) * BKB;
    op.rows = mixed_rows(n, slices);
    op.buf = buf;
    op.exps = exps;
    return make_map(&op.map, buf, op.rows * slices, op.kp, as_b ? nt : BM);
}

static int mixed_rows_nt(int n, int nt) {
    const int ra = ((n + BM - 1) / BM) * BM, rb = ((n + nt - 1) / nt) * nt;
    return ra > rb ? ra : rb;
}

size_t mixed_slice_bytes_nt(int n, int slices, int nt) {
    const int kp = ((n + BKB - 1) / BKB) * BKB;
    return (size_t)slices * (size_t)mixed_rows_nt(n, nt) * kp;
}

bool mixed_plan_nt(MixedOperand& op, int8_t* buf, int* exps, int n, int slices, bool as_b, int nt) {
    op.n = n;
    op.slices = slices;
    op.kp = ((n + BKB - 1) / BKB) * BKB;
    op.rows = mixed_rows_nt(n, nt);
    op.buf = buf;
    op.exps = exps;
    return make_map(&op.map, buf, op.rows * slices, op.kp, as_b ? nt : BM);
}

MixedOperand mixed_fewer_slices(const MixedOperand& op, int slices, bool as_b, bool* ok) {
    MixedOperand r = op;
    r.slices = slices;
    if (as_b) *ok = make_map(&r.map, op.buf, op.rows * op.slices, op.kp, mixed_tile_n(slices, op.n));
    else *ok = true;  // A boxes are 128 rows whatever the slice count
    return r;
}

void mixed_slice_grouped(const MixedSliceJob* d_jobs, int njobs, const int* d_row_start, int total_rows,
                         cudaStream_t st) {
    if (total_rows <= 0) return;
    k_slice_rows_grouped<<<total_rows, 256, 0, st>>>(d_jobs, njobs, d_row_start);
    count_launch();
}

void mixed_lower_tiles(int job, int n, int nt, std::vector<int4>& out) {
    const int by_n = (n + BM - 1) / BM, bx_n = (n + nt - 1) / nt;
    for (int by = 0; by < by_n; ++by) {
        const int last = (by * BM + BM - 1) / nt;
        for (int bx = 0; bx <= last && bx < bx_n; ++bx) out.push_back(make_int4(job, by * BM, bx * nt, 0));
    }
}

// The single-scene cost model over a group's tiles: each tile costs its
// K-steps x (tile_n + 16); tiles go, longest first (the grouped launch's
// order), to whichever of the 148 SMs frees first; the width with the
// shorter makespan wins (ties: 96, fewer tiles).
int mixed_group_tile_n(int slices, const std::vector<int>& ns) {
    if (slices <= 4) return 128;
    constexpr int kSMs = 148;
    double span_of[2] = {0, 0};
    const int widths[2] = {96, 64};
    for (int w = 0; w < 2; ++w) {
        const int nt = widths[w];
        std::vector<double> cost;
        for (int n : ns) {
            const double c = (double)((n + BKB - 1) / BKB) * (nt + 16);
            cost.insert(cost.end(), (size_t)lower_tiles(n, nt), c);
        }
        std::sort(cost.begin(), cost.end(), std::greater<double>());
        std::priority_queue<double, std::vector<double>, std::greater<double>> sm;
        for (int i = 0; i < kSMs; ++i) sm.push(0.0);
        double span = 0;
        for (double c : cost) {
            const double t = sm.top() + c;
            sm.pop();
            sm.push(t);
            span = std::max(span, t);
        }
        span_of[w] = span;
    }
    return span_of[1] < span_of[0] ? 64 : 96;
}

void mixed_gemm_grouped(int slices, int nt, const MixedGemmJob* d_jobs, const int4* d_tiles, int ntiles,
                        cudaStream_t st) {
    if (ntiles <= 0) return;
    if (slices == 5 && nt == 64) {
        k_ozaki_gemm_grouped<64, 5><<<ntiles, THREADS, Shape<64, 5>::SMEM, st>>>(d_jobs, d_tiles);
    } else if (slices == 5) {
        k_ozaki_gemm_grouped<96, 5><<<ntiles, THREADS, Shape<96, 5>::SMEM, st>>>(d_jobs, d_tiles);
    } else if (slices == 4) {
        k_ozaki_gemm_grouped<128, 4><<<ntiles, THREADS, Shape<128, 4>::SMEM, st>>>(d_jobs, d_tiles);
    } else if (slices == 3) {
        k_ozaki_gemm_grouped<128, 3><<<ntiles, THREADS, Shape<128, 3>::SMEM, st>>>(d_jobs, d_tiles);
    } else {
        k_ozaki_gemm_grouped<128, 2><<<ntiles, THREADS, Shape<128, 2>::SMEM, st>>>(d_jobs, d_tiles);
    }
    count_launch();
}

void mixed_slice(const double* A, int lda, MixedOperand& op, cudaStream_t st, const int* skip, double* Y,
                 const TeState* te) {
    k_slice_rows<<<op.n, 256, 0, st>>>(A, lda, op.n, op.slices, op.buf, op.rows, op.kp, op.exps, skip, Y, te);
    count_launch();
}

// Row blocks per group of the grouped tile order: used when one operand's
// slices exceed about 3/4 of L2 (the B operand would be re-streamed from HBM
// for every row block); small products keep the 2-D grid.
static int group_rows_for(int n, int slices) {
    const double b_bytes = (double)slices * n * (double)n;
    return b_bytes > 96.0 * (1 << 20) ? 8 : 0;
}

template <int NT, int S>
static void launch_ozaki(const MixedOperand& a, const MixedOperand& b, double* C, int ldc, unsigned long long* amax,
                         bool lower_only, int* err, cudaStream_t st, const int* skip, bool mirror, bool accumulate,
                         bool klo = false) {
    set_attr_once<NT, S>();
    const int n = a.n;
    const int gm = lower_only ? group_rows_for(n, S) : 0;
    dim3 grid = gm > 0 ? dim3((unsigned)lower_tiles(n, NT), 1) : dim3((n + NT - 1) / NT, (n + BM - 1) / BM);
    k_ozaki_gemm<NT, S><<<grid, THREADS, Shape<NT, S>::SMEM, st>>>(a.map, b.map, n, n, a.kp, a.rows, b.rows, a.exps,
                                                                   b.exps, C, ldc, amax, lower_only ? 1 : 0, err,
                                                                   skip, mirror ? 1 : 0, accumulate ? 1 : 0, gm,
                                                                   klo ? 1 : 0);
}

void mixed_gemm(const MixedOperand& a, const MixedOperand& b, double* C, int ldc, unsigned long long* amax,
                bool lower_only, int* err, cudaStream_t st, const int* skip, bool mirror, bool accumulate) {
    const int n = a.n;
    if (a.slices == 4)
        launch_ozaki<128, 4>(a, b, C, ldc, amax, lower_only, err, st, skip, mirror, accumulate);
    else if (a.slices == 5 && mixed_tile_n(5, n) == 64)
        launch_ozaki<64, 5>(a, b, C, ldc, amax, lower_only, err, st, skip, mirror, accumulate);
    else if (a.slices == 5)
        launch_ozaki<96, 5>(a, b, C, ldc, amax, lower_only, err, st, skip, mirror, accumulate);
    else if (a.slices == 3)
        launch_ozaki<128, 3>(a, b, C, ldc, amax, lower_only, err, st, skip, mirror, accumulate);
    else
        launch_ozaki<128, 2>(a, b, C, ldc, amax, lower_only, err, st, skip, mirror, accumulate);
    count_launch();
}


size_t mixed_gram_bytes(int n) {
    return (mixed_slice_bytes_nt(n, kGramSlices, 64) + 255) & ~size_t(255);
}

// A = T^T T for lower-triangular T (the last product of the SPD inverse,
// A^{-1} = L^{-T} L^{-1}): the columns of T sliced into kGramSlices int8
// planes, lower 128 x 64 tiles, each tile's K loop from max(m0, n0) (the rows
// above are zero in both of its columns), the result mirrored. buf: the
// slice planes (mixed_gram_bytes(n)); its K and row padding must be zero.
bool mixed_gram_lower_tri(const double* T, int n, int ld, int8_t* buf, int* exps, double* A, int lda, int* err,
                          cudaStream_t st) {
    MixedOperand a, b;
    if (!mixed_plan_nt(a, buf, exps, n, kGramSlices, false, 64) || !mixed_plan_nt(b, buf, exps, n, kGramSlices, true, 64))
        return false;
    mixed_slice(T, ld, a, st);
    launch_ozaki<64, kGramSlices>(a, b, A, lda, nullptr, true, err, st, nullptr, true, false, true);
    count_launch();
    return true;
}

}  // namespace unc
