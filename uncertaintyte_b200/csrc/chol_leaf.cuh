// chol_leaf.cuh - the 64 x 64 Cholesky + inverse leaf shared by the recursive
// SPD inverse (dense.cu) and the tile-task inverse (dag.cu).
#pragma once
#include "internal.h"

namespace unc {

constexpr int NB = 64;  // leaf size

// Leaf: Cholesky of the kb x kb (kb <= 64) diagonal block of A at (k0, k0)
// and T_kk = L_kk^{-1}, written as a full kb x kb block of T (zeros above the
// diagonal). One CTA of 512 threads; the block (S) and its inverse (Ts) sit in
// shared memory, padded to 64 x 64 with an identity tail (the factor and
// inverse of blockdiag(A, I) are blockdiag(L, I) and blockdiag(L^-1, I), so
// every step has fixed shapes). Four 16-column panels:
//  (A) warp 0 factors the 16 x 16 diagonal block in registers (lane = row,
//      column p broadcast by shuffle; the pivot check is folded into a flag so
//      that the dependent chain carries no branch), 1 / L(p, p) kept in rinv;
//  (B) the rows below solve x L_qq^T = A_iq by forward substitution, one
//      thread per row;
//  (C) the trailing lower triangle takes the rank-16 update in 2 x 2 register
//      tiles.
// Then T = L^{-1} from the diagonal inverses D_q = L_qq^{-1} (D_0..D_2 are
// formed beside the last panel's factorisation): T_{q+1,q} = -D_{q+1} L_{q+1,q}
// D_q for the two 16-row pairs, then T21 = -T1 (L21 T0) for the 32-row halves.
// Intermediate products are kept transposed in the unused upper blocks of Ts,
// and only the lower triangle is written out.
// Non-positive or non-finite pivots set ERRBIT_SINGULAR.
constexpr int LEAF_THREADS = 512;
constexpr int LEAF_LD = NB + 1;
constexpr int LEAF_PW = 16;
constexpr size_t LEAF_SMEM = sizeof(double) * (2 * NB * LEAF_LD + NB);

// lane = column of D_q = L_qq^{-1} (lanes 16..31 idle)
__device__ __forceinline__ void diag_inverse(const double* S, double* Ts, const double* rinv, int c0, int lane) {
    double t[LEAF_PW];
#pragma unroll
    for (int r = 0; r < LEAF_PW; ++r) {
        double s0 = (r == lane) ? 1.0 : 0.0, s1 = 0.0;
#pragma unroll
        for (int k = 0; k < r; ++k) {
            const double v = S[(c0 + r) * LEAF_LD + c0 + k] * t[k];
            if (k & 1) s1 -= v; else s0 -= v;
        }
        t[r] = (r >= lane) ? (s0 + s1) * rinv[c0 + r] : 0.0;
    }
    if (lane < LEAF_PW) {
#pragma unroll
        for (int r = 0; r < LEAF_PW; ++r) Ts[(c0 + r) * LEAF_LD + c0 + lane] = t[r];
    }
}

// X = L_{b+1,b} D_b (16 x 16, b0 = 16 b), stored transposed in the upper block: Ts(b0 + j, b0 + 16 + i)
__device__ __forceinline__ void pair_x(const double* S, double* Ts, int b0, int e) {
    const int i = e >> 4, j = e & 15;
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < LEAF_PW; ++k) s = fma(S[(b0 + 16 + i) * LEAF_LD + b0 + k], Ts[(b0 + k) * LEAF_LD + b0 + j], s);
    Ts[(b0 + j) * LEAF_LD + b0 + 16 + i] = s;
}
// T_{b+1,b} = -D_{b+1} X
__device__ __forceinline__ void pair_t(double* Ts, int b0, int e) {
    const int i = e >> 4, j = e & 15;
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < LEAF_PW; ++k) s = fma(Ts[(b0 + 16 + i) * LEAF_LD + b0 + 16 + k], Ts[(b0 + j) * LEAF_LD + b0 + 16 + k], s);
    Ts[(b0 + 16 + i) * LEAF_LD + b0 + j] = -s;
}

// Load phase: the kb x kb diagonal block of A at (k0, k0) into S (lower
// triangle; the upper one zero; identity tail) and Ts cleared. A is read
// through L2 only (ld.global.cg), so that a persistent caller never sees a
// stale L1 line of a tile another CTA rewrote. The caller synchronises.
__device__ __forceinline__ void chol_leaf_load(const double* A, long lda, int k0, int kb, double* lsm) {
    double* S = lsm;
    double* Ts = lsm + NB * LEAF_LD;
    const int tid = threadIdx.x;
    constexpr int kPer = NB * NB / LEAF_THREADS;
    double v[kPer];
    const int i = tid & (NB - 1);
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
        const int j = (tid >> 6) + u * (LEAF_THREADS / NB);
        v[u] = (i < kb && j < kb) ? (j <= i ? __ldcg(A + (k0 + i) + (long)(k0 + j) * lda) : 0.0) : (i == j ? 1.0 : 0.0);
    }
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
        const int j = (tid >> 6) + u * (LEAF_THREADS / NB);
        S[i * LEAF_LD + j] = v[u];
        Ts[i * LEAF_LD + j] = 0.0;
    }
}

// Factorisation of the block in S (after chol_leaf_load and a barrier), T_kk
// written to T at (k0, k0). One 512-thread CTA, lsm: LEAF_SMEM bytes.
__device__ __forceinline__ void chol_leaf_factor(int k0, int kb, double* T, long ldt, int* err, double* lsm) {
    double* S = lsm;
    double* Ts = lsm + NB * LEAF_LD;
    double* rinv = Ts + NB * LEAF_LD;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int q = 0; q < NB / LEAF_PW; ++q) {
        const int c0 = q * LEAF_PW;
        if (warp == 0) {  // (A) Cholesky of the diagonal block in registers, lane = row
            double a[LEAF_PW];
#pragma unroll
            for (int j = 0; j < LEAF_PW; ++j) a[j] = (lane < LEAF_PW && j <= lane) ? S[(c0 + lane) * LEAF_LD + c0 + j] : 0.0;
            bool bad = false;
#pragma unroll
            for (int p = 0; p < LEAF_PW; ++p) {
                const double d = __shfl_sync(0xffffffffu, a[p], p);
                const double r = rsqrt(d);
                if (lane == p) rinv[c0 + p] = r;
                bad |= !(d > 0.0 && d <= 1.7976931348623157e308);
                a[p] = (lane == p) ? d * r : a[p] * r;
                const double lp = a[p];
#pragma unroll
                for (int j = p + 1; j < LEAF_PW; ++j) {
                    const double ljp = __shfl_sync(0xffffffffu, lp, j);
                    a[j] = fma(-lp, ljp, a[j]);
                }
            }
            if (lane == 0 && bad) atomicOr(err, ERRBIT_SINGULAR);
            if (lane < LEAF_PW) {
#pragma unroll
                for (int j = 0; j < LEAF_PW; ++j)
                    if (j <= lane) S[(c0 + lane) * LEAF_LD + c0 + j] = a[j];
            }
        } else if (q == NB / LEAF_PW - 1 && warp < NB / LEAF_PW) {
            diag_inverse(S, Ts, rinv, (warp - 1) * LEAF_PW, lane);  // D_0 .. D_2 beside the last factorisation
        }
        __syncthreads();
        const int r0 = c0 + LEAF_PW, m = NB - r0;
        if (m == 0) break;
        // (B) rows below: forward substitution x L_qq^T = A_iq, one thread per row
        if (tid < m) {
            double* row = S + (r0 + tid) * LEAF_LD + c0;
            double x[LEAF_PW];
#pragma unroll
            for (int j = 0; j < LEAF_PW; ++j) {
                double s = row[j];
#pragma unroll
                for (int k = 0; k < j; ++k) s = fma(-x[k], S[(c0 + j) * LEAF_LD + c0 + k], s);
                x[j] = s * rinv[c0 + j];
            }
#pragma unroll
            for (int j = 0; j < LEAF_PW; ++j) row[j] = x[j];
        }
        __syncthreads();
        // (C) trailing update, lower 2 x 2 tiles: S(i, j) -= sum_k L(i, c0 + k) L(j, c0 + k)
        {
            const int mt = m / 2, ntile = mt * (mt + 1) / 2;
            if (tid < ntile) {
                int ti = (int)((sqrtf(8.0f * tid + 1.0f) - 1.0f) * 0.5f);
                while (ti * (ti + 1) / 2 > tid) --ti;
                while ((ti + 1) * (ti + 2) / 2 <= tid) ++ti;
                const int tj = tid - ti * (ti + 1) / 2;
                const int i0 = r0 + 2 * ti, j0 = r0 + 2 * tj;
                const double* a0 = S + i0 * LEAF_LD + c0;
                const double* a1 = a0 + LEAF_LD;
                const double* b0 = S + j0 * LEAF_LD + c0;
                const double* b1 = b0 + LEAF_LD;
                double c00 = 0.0, c01 = 0.0, c10 = 0.0, c11 = 0.0;
#pragma unroll
                for (int k = 0; k < LEAF_PW; ++k) {
                    const double x0 = a0[k], x1 = a1[k], y0 = b0[k], y1 = b1[k];
                    c00 = fma(x0, y0, c00);
                    c01 = fma(x0, y1, c01);
                    c10 = fma(x1, y0, c10);
                    c11 = fma(x1, y1, c11);
                }
                double* z = S + i0 * LEAF_LD + j0;
                z[0] -= c00;
                z[1] -= c01;
                z[LEAF_LD] -= c10;
                z[LEAF_LD + 1] -= c11;
            }
        }
        __syncthreads();
    }
    // T = L^{-1} from the four D_q: 16-level pairs, then the 32-level block. Intermediate
    // products sit transposed in the (unused) upper blocks of Ts.
    if (warp == 0)
        diag_inverse(S, Ts, rinv, 48, lane);
    else if (warp < 9)
        pair_x(S, Ts, 0, tid - 32);
    __syncthreads();
    if (tid < 256)
        pair_t(Ts, 0, tid);
    else
        pair_x(S, Ts, 32, tid - 256);
    __syncthreads();
    if (tid < 256) pair_t(Ts, 32, tid);
    {  // X = L21 T0 (32 x 32), stored transposed: Ts(j, 32 + i)
        const int j = tid & 31, i0 = 2 * (tid >> 5);
        double s0 = 0.0, s1 = 0.0;
#pragma unroll 8
        for (int k = 0; k < 32; ++k) {
            const double t = k >= j ? Ts[k * LEAF_LD + j] : 0.0;  // the upper block holds X of the first pair
            s0 = fma(S[(32 + i0) * LEAF_LD + k], t, s0);
            s1 = fma(S[(33 + i0) * LEAF_LD + k], t, s1);
        }
        Ts[j * LEAF_LD + 32 + i0] = s0;
        Ts[j * LEAF_LD + 33 + i0] = s1;
    }
    __syncthreads();
    {  // T21 = -T1 X
        const int j = tid & 31, i0 = 2 * (tid >> 5);
        double s0 = 0.0, s1 = 0.0;
#pragma unroll 4
        for (int k = 0; k < i0 + 2; ++k) {
            const double x = Ts[j * LEAF_LD + 32 + k];
            s0 = fma(Ts[(32 + i0) * LEAF_LD + 32 + k], x, s0);
            s1 = fma(Ts[(33 + i0) * LEAF_LD + 32 + k], x, s1);
        }
        Ts[(32 + i0) * LEAF_LD + j] = -s0;
        Ts[(33 + i0) * LEAF_LD + j] = -s1;
    }
    __syncthreads();
    {
        const int i = tid & (NB - 1);
#pragma unroll
        for (int u = 0; u < NB * NB / LEAF_THREADS; ++u) {
            const int j = (tid >> 6) + u * (LEAF_THREADS / NB);
            if (i < kb && j < kb) T[(k0 + i) + (long)(k0 + j) * ldt] = i >= j ? Ts[i * LEAF_LD + j] : 0.0;
        }
    }
}

// The whole leaf: load, barrier, factorisation.
__device__ __forceinline__ void chol_leaf_tile(const double* A, long lda, int k0, int kb, double* T, long ldt,
                                               int* err, double* lsm) {
    chol_leaf_load(A, lda, k0, kb, lsm);
    __syncthreads();
    chol_leaf_factor(k0, kb, T, ldt, err, lsm);
}

}  // namespace unc
