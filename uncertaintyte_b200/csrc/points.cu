// points.cu - fused point-covariance kernel (sm_100a).
//
// Replaces the per-point loop of uncertaintyTE (compute.cpp:517-527 with
// findCams2Point :370-380, composeCams2PointJacobian :382-420,
// composeCamCovariances :422-441, fillPtUnc2OutArray :443-455):
//
//   Sigma_pt = pinv(A) * B * Sigma * B^T * pinv(A)^T
//
// with A = stacked 2x3 point Jacobians (unscaled), B = [J_cam,o | -I2] per
// observation and Sigma = blockdiag(Sigma_cam(o), I2), Sigma_cam the unscaled
// 9x9 diagonal block of the inverse (block-diagonal: the reference drops
// cross-camera terms). With pinv(A) = D^+ A^T, D = A^T A, this is exactly
//
//   Sigma_pt = D^+ + D^+ (sum_o W_o^T Sigma_cam(o) W_o) D^+,   W_o = J_cam,o^T A_o
//
// evaluated per point in FP64 registers: no 2n x 11n matrices, no O(P*obs)
// scan (the reference rescans every Jacobian row per point, :393).
#include "internal.h"

namespace unc {

// Pseudo-inverse of a symmetric PSD 3x3 (a00 a01 a02 a11 a12 a22) through a
// cyclic Jacobi eigen-decomposition. Eigenvalues below 64*eps*max are
// dropped (rank-deficient D when a point has a single observation).
__device__ void sym3_pinv(const double in[6], double out[3][3]) {
    double a[3][3] = {{in[0], in[1], in[2]}, {in[1], in[3], in[4]}, {in[2], in[4], in[5]}};
    double v[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int sweep = 0; sweep < 12; ++sweep) {
        double off = fabs(a[0][1]) + fabs(a[0][2]) + fabs(a[1][2]);
        double dia = fabs(a[0][0]) + fabs(a[1][1]) + fabs(a[2][2]);
        if (off <= 1e-300 || off < dia * 1e-18) break;
#pragma unroll
        for (int pq = 0; pq < 3; ++pq) {
            const int p = pq == 2 ? 1 : 0, q = pq == 0 ? 1 : 2;
            double apq = a[p][q];
            if (apq == 0.0) continue;
            double theta = (a[q][q] - a[p][p]) / (2.0 * apq);
            double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
            double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                double akp = a[k][p], akq = a[k][q];
                a[k][p] = c * akp - s * akq;
                a[k][q] = s * akp + c * akq;
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                double apk = a[p][k], aqk = a[q][k];
                a[p][k] = c * apk - s * aqk;
                a[q][k] = s * apk + c * aqk;
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                double vkp = v[k][p], vkq = v[k][q];
                v[k][p] = c * vkp - s * vkq;
                v[k][q] = s * vkp + c * vkq;
            }
        }
    }
    double w[3] = {a[0][0], a[1][1], a[2][2]};
    double wmax = fmax(fabs(w[0]), fmax(fabs(w[1]), fabs(w[2])));
    double iw[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) iw[k] = (w[k] > 64.0 * 2.220446049250313e-16 * wmax) ? 1.0 / w[k] : 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            out[i][j] = v[i][0] * v[j][0] * iw[0] + v[i][1] * v[j][1] * iw[1] + v[i][2] * v[j][2] * iw[2];
}

// Four threads per point: thread q of the quad sums observations b + q,
// b + q + 4, ... of the point into its S; the quad then adds its four partial
// S in a fixed butterfly order (bitwise repeatable) and thread 0 finishes.
constexpr int kPointLanes = 4;
__global__ void __launch_bounds__(128) k_point_cov(int num_points, int3 fix, int has_fix,
                                                   const double* __restrict__ J,
                                                   const int* __restrict__ pt_ptr,
                                                   const int* __restrict__ pt_obs,
                                                   const int* __restrict__ obs_cam,
                                                   const double* __restrict__ Vraw,
                                                   const double* __restrict__ sig,
                                                   double* __restrict__ pt_unc) {
    const int gt = blockIdx.x * blockDim.x + threadIdx.x;
    const int p = gt / kPointLanes, q = gt % kPointLanes;
    const unsigned quad = 0xfu << (threadIdx.x & 28);
    if (p >= num_points) return;  // whole quads leave together
    if (has_fix && (p == fix.x || p == fix.y || p == fix.z)) return;  // fixed points are skipped
    double* out = pt_unc + 6L * p;
    const int b = pt_ptr[p], e = pt_ptr[p + 1];
    if (b == e) {  // pinv of an empty A: zero covariance
        if (q == 0) out[0] = out[1] = out[2] = out[3] = out[4] = out[5] = 0.0;
        return;
    }
    double S[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int i = b + q; i < e; i += kPointLanes) {
        int o = pt_obs[i];
        const double* r = J + 24L * o;
        const double2* qv = reinterpret_cast<const double2*>(r);
        double v[24];
#pragma unroll
        for (int k = 0; k < 12; ++k) {
            double2 x = __ldg(qv + k);
            v[2 * k] = x.x;
            v[2 * k + 1] = x.y;
        }
        // W = Jc^T Jp (9x3)
        double W[9][3];
#pragma unroll
        for (int j = 0; j < 9; ++j)
#pragma unroll
            for (int k = 0; k < 3; ++k) W[j][k] = v[j] * v[9 + k] + v[12 + j] * v[21 + k];
        const double* sg = sig + 81L * obs_cam[o];
        // S += W^T Sig W  (Sig row-major 9x9: sg[9*j + k] = Sigma(j, k))
#pragma unroll
        for (int j = 0; j < 9; ++j) {
            double t0 = 0, t1 = 0, t2 = 0;  // (Sig W)(j, :)
#pragma unroll
            for (int k = 0; k < 9; ++k) {
                double s = __ldg(sg + 9 * j + k);
                t0 += s * W[k][0];
                t1 += s * W[k][1];
                t2 += s * W[k][2];
            }
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                S[a][0] += W[j][a] * t0;
                S[a][1] += W[j][a] * t1;
                S[a][2] += W[j][a] * t2;
            }
        }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            S[a][c] += __shfl_xor_sync(quad, S[a][c], 1);
            S[a][c] += __shfl_xor_sync(quad, S[a][c], 2);
        }
    if (q != 0) return;
    double Dp[3][3];
    sym3_pinv(Vraw + 6L * p, Dp);
    // Sigma_pt = D^+ + D^+ S D^+
    double T[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) T[i][j] = S[i][0] * Dp[0][j] + S[i][1] * Dp[1][j] + S[i][2] * Dp[2][j];
    double R[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            R[i][j] = Dp[i][j] + Dp[i][0] * T[0][j] + Dp[i][1] * T[1][j] + Dp[i][2] * T[2][j];
    out[0] = R[0][0];
    out[1] = R[0][1];
    out[2] = R[0][2];
    out[3] = R[1][1];
    out[4] = R[1][2];
    out[5] = R[2][2];
}

void launch_point_cov(const SceneDev& s, const double* sig, double* pt_unc, cudaStream_t st) {
    if (s.num_points == 0) return;
    int3 fix = make_int3(s.fix[0], s.fix[1], s.fix[2]);
    const long threads = (long)s.num_points * kPointLanes;
    k_point_cov<<<(unsigned)((threads + 127) / 128), 128, 0, st>>>(s.num_points, fix, s.has_fix, s.J,
                                                            s.pt_ptr, s.pt_obs, s.obs_cam, s.Vraw,
                                                            sig, pt_unc);
    count_launch();
}

}  // namespace unc
