// powers.cu - the Taylor series of teInverse (compute.cpp:141-160) evaluated
// from a few powers of X instead of one product per iteration.
//
// The reference forms add = X^(i+1) by one product per iteration, stops when
// change = |k_i max|add|| falls below 1e-5 or grows (k_i = lambda^i / (i-1)!,
// the 32-bit factorial of compute.cpp:57-62), and sums iZ = X + sum_i k_i add_i.
// Here:
//   * X is SPD, so every power X^j is SPD and its largest |entry| is its
//     largest diagonal entry; diag(X^(a+b))_c is the dot product of column c
//     of X^a and of X^b. From X, X^2, X^3, X^4, X^8, X^12 (and X^16) every
//     j = 2..20 is such a pair, so the stop rule runs on the device from
//     O(N^2) column dot products;
//   * the sum is taken in blocks of four coefficients,
//       iZ = G_0 + X^4 G_1 + X^8 G_2 + X^12 G_3 + X^16 G_4,
//       G_q = c_4q X + c_(4q+1) X^2 + c_(4q+2) X^3 + c_(4q+3) X^4,
//     with c_0 = 1, c_i = k_i for the performed iterations and 0 after; the
//     blocks whose coefficients are all zero are skipped on the device.
// Products: X^2, X^3, X^4, X^8, X^12 (X^16 past 15 iterations): 5 for the
// 12..15 iterations of the reference scenes, instead of 13..16. The block
// terms X^(4q) G_q are formed on the 9 x 9 camera blocks of iZ only, the only
// part of iZ read afterwards (k_taylor_blocks: 81 N multiply-adds per camera
// and block instead of a full product). The polynomial, its coefficients and
// the stop decisions are the reference's;
// the results differ from the one-product-per-iteration order at the
// rounding level. Every kernel here has a fixed summation order, so the
// results are bitwise repeatable.
#include <cfloat>

#include "internal.h"

namespace unc {
namespace {

// diag(X^j) = dot of the columns of slots slot_a(j), slot_b(j): slots 0..3 =
// X..X^4, 4 = X^8, 5 = X^12, 6 = X^16 (j = 2..20)
__host__ __device__ constexpr int slot_a(int j) {
    return j == 2 || j == 3 ? 0 : (j == 4 ? 1 : (j <= 8 ? j - 5 : (j - 9) % 4));
}
__host__ __device__ constexpr int slot_b(int j) {
    return j == 2 ? 0 : (j <= 4 ? 1 : (j <= 8 ? 3 : (j <= 12 ? 4 : (j <= 16 ? 5 : 6))));
}
static_assert(slot_a(2) == 0 && slot_b(2) == 0 && slot_a(3) == 0 && slot_b(3) == 1 && slot_a(4) == 1 &&
                  slot_b(4) == 1 && slot_a(5) == 0 && slot_b(5) == 3 && slot_a(8) == 3 && slot_a(9) == 0 &&
                  slot_b(9) == 4 && slot_a(16) == 3 && slot_b(16) == 5 && slot_a(20) == 3 && slot_b(20) == 6,
              "power pairs");

constexpr int kDiagThreads = 256;

// The diagonal entries c of X^j, j in [JLO, JHI], into dmax (max over c of the
// non-negative values; a non-finite value becomes +inf). One block per column.
template <int JLO, int JHI>
__device__ __forceinline__ void power_diag_column(const PowerSet& ps, int c, double (*red)[JHI - JLO + 1]) {
    constexpr int NJ = JHI - JLO + 1;
    const long off = (long)c * ps.ld;
    double acc[NJ];
#pragma unroll
    for (int q = 0; q < NJ; ++q) acc[q] = 0.0;
    for (int r = threadIdx.x; r < ps.n; r += kDiagThreads) {
        double v[7];
#pragma unroll
        for (int s = 0; s < 7; ++s) {
            bool used = false;
#pragma unroll
            for (int j = JLO; j <= JHI; ++j) used |= (slot_a(j) == s) | (slot_b(j) == s);
            v[s] = used ? ps.M[s][off + r] : 0.0;
        }
#pragma unroll
        for (int j = JLO; j <= JHI; ++j) acc[j - JLO] += v[slot_a(j)] * v[slot_b(j)];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NJ; ++q) {
        double a = acc[q];
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) a += __shfl_xor_sync(0xffffffffu, a, d);
        if (lane == 0) red[warp][q] = a;
    }
    __syncthreads();
    if (threadIdx.x < NJ) {
        double t = 0.0;
#pragma unroll
        for (int w = 0; w < kDiagThreads / 32; ++w) t += red[w][threadIdx.x];
        const double v = (t <= DBL_MAX) ? fmax(t, 0.0) : __longlong_as_double(0x7ff0000000000000LL);  // NaN -> inf
        atomicMax(ps.dmax + JLO + threadIdx.x, (unsigned long long)__double_as_longlong(v));
    }
}

template <int JLO, int JHI>
__global__ void __launch_bounds__(kDiagThreads) k_power_diag(PowerSet ps, const int* skip) {
    if (skip && *skip) return;
    __shared__ double red[kDiagThreads / 32][JHI - JLO + 1];
    power_diag_column<JLO, JHI>(ps, blockIdx.x, red);
}

__device__ __forceinline__ int set_of_block(const long* __restrict__ blk, int nsets, long b) {
    int lo = 0, hi = nsets - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (blk[mid] <= b) lo = mid; else hi = mid - 1;
    }
    return lo;
}

template <int JLO, int JHI>
__global__ void __launch_bounds__(kDiagThreads) k_power_diag_grouped(const PowerSet* __restrict__ sets, int nsets,
                                                                      const long* __restrict__ blk, int skip_done) {
    const int m = set_of_block(blk, nsets, blockIdx.x);
    const PowerSet ps = sets[m];
    if (skip_done && ps.te->skip[0]) return;
    __shared__ double red[kDiagThreads / 32][JHI - JLO + 1];
    power_diag_column<JLO, JHI>(ps, (int)(blockIdx.x - blk[m]), red);
}

// The reference's stop rule (compute.cpp:145-155) over iterations ilo..ihi.
__device__ __forceinline__ void power_decide_one(TeState* s, const unsigned long long* dmax, const double* k, int ilo,
                                                 int ihi) {
    if (ilo == 1) s->c[0] = 1.0;
    for (int i = ilo; i <= ihi && !s->done; ++i) {
        double amax = __longlong_as_double((long long)dmax[i + 1]);
        amax = fmax(amax, 2.2250738585072014e-308);  // absMax starts at DBL_MIN (ScaledDenseMatrix.cpp:208)
        if (!(amax <= 1.7976931348623157e308)) s->bad = 1;
        const double change = fabs(k[i - 1] * amax);
        if (change < 1e-5 || change > s->old_change) {  // compute.cpp:150-152
            s->done = 1;
            break;
        }
        s->old_change = change;
        if (s->iters < 20) s->change[s->iters] = change;
        s->iters += 1;
        s->c[i] = k[i - 1];
    }
    if (ihi == 15) s->skip[0] = s->done;  // X^16 is needed only past iteration 15
    if (ihi == 19)
        for (int q = 1; q <= 4; ++q) s->skip[q] = s->iters < 4 * q;
}

__global__ void k_power_decide(TeState* s, const unsigned long long* dmax, TaylorCoefs k, int ilo, int ihi) {
    if (threadIdx.x == 0 && blockIdx.x == 0) power_decide_one(s, dmax, k.k, ilo, ihi);
}

__global__ void k_power_decide_grouped(const PowerSet* __restrict__ sets, int nsets, const double* __restrict__ k,
                                       int ilo, int ihi) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m < nsets) power_decide_one(sets[m].te, sets[m].dmax, k + 19L * m, ilo, ihi);
}

// out(idx) = c[4q] X + c[4q+1] X^2 + c[4q+2] X^3 + c[4q+3] X^4 (element idx of the n x n matrix)
__device__ __forceinline__ void power_combine_one(const PowerSet& ps, int q, double* out, long idx) {
    const int col = (int)(idx / ps.n), r = (int)(idx - (long)col * ps.n);
    const long o = r + col * ps.ld;
    const double* c = ps.te->c + 4 * q;
    double v = c[0] * ps.M[0][o];
    v += c[1] * ps.M[1][o];
    v += c[2] * ps.M[2][o];
    v += c[3] * ps.M[3][o];
    out[o] = v;
}

__global__ void k_power_combine(PowerSet ps, int q, double* out, const int* skip) {
    if (skip && *skip) return;
    const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (idx < (long)ps.n * ps.n) power_combine_one(ps, q, out, idx);
}

__global__ void k_power_combine_grouped(const PowerSet* __restrict__ sets, int nsets, const long* __restrict__ blk,
                                        int q) {
    const int m = set_of_block(blk, nsets, blockIdx.x);
    const PowerSet& ps = sets[m];
    if (q > 0 && ps.te->skip[q]) return;
    const long idx = (blockIdx.x - blk[m]) * (long)blockDim.x + threadIdx.x;
    if (idx < (long)ps.n * ps.n) power_combine_one(ps, q, q == 0 ? ps.iZ : ps.G, idx);
}

// The camera blocks of iZ += X^(4q) G_q, q = 1..4 (blocks whose skip word is
// set left out). Only the 9 x 9 diagonal camera blocks of iZ are read after
// the series (the camera output, compute.cpp:168-183, and the point stage's
// block-diagonal camera covariance, compute.cpp:422-441), so these products
// are formed on those blocks only: element (r, c) of camera block b, r >= c,
// is sum_k G_q(k, r) X^(4q)(k, c) with G_q(k, r) = c_4q X + c_(4q+1) X^2 +
// c_(4q+2) X^3 + c_(4q+3) X^4 at (k, r) (G_q and the powers are symmetric,
// so their columns are their rows), added to iZ(r, c) in the order q = 1..4
// and written at (r, c) and (c, r). One CTA per camera; each thread sums a
// fixed stride of k, the partial sums are added in a fixed tree and warp
// order, so the result is bitwise repeatable.
constexpr int kBlkThreads = 128;
constexpr int kBlkPairs = 45;  // lower triangle of a 9 x 9 block

__device__ __forceinline__ void taylor_camera_block(const PowerSet& ps, int cam, double (*red)[kBlkPairs],
                                                    double* val) {
    const long ld = ps.ld;
    const int n = ps.n, c0 = 9 * cam, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid < kBlkPairs) {  // iZ holds G_0 here
        int r = 0, s = tid;
        while (s > r) s -= ++r;  // tid = r (r + 1) / 2 + s, s <= r
        val[tid] = ps.iZ[(c0 + r) + (long)(c0 + s) * ld];
    }
    for (int q = 1; q <= 4; ++q) {
        if (ps.te->skip[q]) continue;  // the same word for every thread of the CTA
        const double* cq = ps.te->c + 4 * q;
        const double k0 = cq[0], k1 = cq[1], k2 = cq[2], k3 = cq[3];
        const double* P = ps.M[q + 2];  // X^4, X^8, X^12, X^16
        double acc[kBlkPairs];
#pragma unroll
        for (int p = 0; p < kBlkPairs; ++p) acc[p] = 0.0;
        for (int k = tid; k < n; k += kBlkThreads) {
            double g[9], x[9];
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                const long o = k + (long)(c0 + i) * ld;
                double v = k0 * ps.M[0][o];
                v += k1 * ps.M[1][o];
                v += k2 * ps.M[2][o];
                v += k3 * ps.M[3][o];
                g[i] = v;
                x[i] = P[o];
            }
#pragma unroll
            for (int r = 0, p = 0; r < 9; ++r)
#pragma unroll
                for (int s = 0; s <= r; ++s, ++p) acc[p] = fma(g[r], x[s], acc[p]);
        }
#pragma unroll
        for (int p = 0; p < kBlkPairs; ++p) {
            double a = acc[p];
#pragma unroll
            for (int d = 16; d > 0; d >>= 1) a += __shfl_xor_sync(0xffffffffu, a, d);
            if (lane == 0) red[warp][p] = a;
        }
        __syncthreads();
        if (tid < kBlkPairs) {
            double t = red[0][tid];
#pragma unroll
            for (int w = 1; w < kBlkThreads / 32; ++w) t += red[w][tid];
            val[tid] += t;
        }
        __syncthreads();  // red is reused by the next block
    }
    if (tid < kBlkPairs) {
        int r = 0, s = tid;
        while (s > r) s -= ++r;
        ps.iZ[(c0 + r) + (long)(c0 + s) * ld] = val[tid];
        ps.iZ[(c0 + s) + (long)(c0 + r) * ld] = val[tid];
    }
}

__global__ void __launch_bounds__(kBlkThreads) k_taylor_blocks(PowerSet ps) {
    __shared__ double red[kBlkThreads / 32][kBlkPairs];
    __shared__ double val[kBlkPairs];
    taylor_camera_block(ps, blockIdx.x, red, val);
}

// The same over the cameras of many sets: blk holds the sets' column offsets
// (multiples of 9), so set m owns the cameras [blk[m] / 9, blk[m + 1] / 9).
__global__ void __launch_bounds__(kBlkThreads) k_taylor_blocks_grouped(const PowerSet* __restrict__ sets, int nsets,
                                                                       const long* __restrict__ blk) {
    const int m = set_of_block(blk, nsets, 9L * blockIdx.x);
    __shared__ double red[kBlkThreads / 32][kBlkPairs];
    __shared__ double val[kBlkPairs];
    taylor_camera_block(sets[m], (int)(blockIdx.x - blk[m] / 9), red, val);
}

}  // namespace

void launch_taylor_blocks(const PowerSet& ps, cudaStream_t st) {
    k_taylor_blocks<<<ps.n / 9, kBlkThreads, 0, st>>>(ps);
    count_launch();
}

void launch_taylor_blocks_grouped(const PowerSet* d_sets, int nsets, const long* d_blk_cols, long nblk_cols,
                                  cudaStream_t st) {
    if (nsets <= 0 || nblk_cols < 9) return;
    k_taylor_blocks_grouped<<<(unsigned)(nblk_cols / 9), kBlkThreads, 0, st>>>(d_sets, nsets, d_blk_cols);
    count_launch();
}

void launch_power_diag(const PowerSet& ps, int jlo, int jhi, const int* skip, cudaStream_t st) {
    if (jlo == 2 && jhi == 16) {
        k_power_diag<2, 16><<<ps.n, kDiagThreads, 0, st>>>(ps, skip);
    } else {
        k_power_diag<17, 20><<<ps.n, kDiagThreads, 0, st>>>(ps, skip);
    }
    count_launch();
}

void launch_power_decide(TeState* te, const unsigned long long* dmax, const TaylorCoefs& k, int ilo, int ihi,
                         cudaStream_t st) {
    k_power_decide<<<1, 32, 0, st>>>(te, dmax, k, ilo, ihi);
    count_launch();
}

void launch_power_combine(const PowerSet& ps, int q, double* out, const int* skip, cudaStream_t st) {
    const long total = (long)ps.n * ps.n;
    k_power_combine<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(ps, q, out, skip);
    count_launch();
}

void launch_power_diag_grouped(const PowerSet* d_sets, int nsets, const long* d_blk_cols, long nblk, int jlo,
                               int jhi, bool skip_if_done_early, cudaStream_t st) {
    if (nsets <= 0) return;
    if (jlo == 2 && jhi == 16) {
        k_power_diag_grouped<2, 16><<<(unsigned)nblk, kDiagThreads, 0, st>>>(d_sets, nsets, d_blk_cols,
                                                                             skip_if_done_early ? 1 : 0);
    } else {
        k_power_diag_grouped<17, 20><<<(unsigned)nblk, kDiagThreads, 0, st>>>(d_sets, nsets, d_blk_cols,
                                                                              skip_if_done_early ? 1 : 0);
    }
    count_launch();
}

void launch_power_decide_grouped(const PowerSet* d_sets, int nsets, const double* d_k, int ilo, int ihi,
                                 cudaStream_t st) {
    if (nsets <= 0) return;
    k_power_decide_grouped<<<(nsets + 127) / 128, 128, 0, st>>>(d_sets, nsets, d_k, ilo, ihi);
    count_launch();
}

void launch_power_combine_grouped(const PowerSet* d_sets, int nsets, const long* d_blk_elems, long nblk, int q,
                                  cudaStream_t st) {
    if (nsets <= 0) return;
    k_power_combine_grouped<<<(unsigned)nblk, 256, 0, st>>>(d_sets, nsets, d_blk_elems, q);
    count_launch();
}

}  // namespace unc
