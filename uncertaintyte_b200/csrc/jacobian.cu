// jacobian.cu - the Jacobian of the reprojection residuals built on the GPU
// from the scene (cameras, points, observations), in the reference's CRS
// layout, so that a reconstruction never has to travel as a text .jacob or as
// 288 bytes per observation over PCIe.
//
// Camera model (SnavelyReprojectionError, snavely_reprojection_error.h:309-350,
// with unit parameter weights): camera = [angle-axis w (3), centre C (3), focal
// f, k1, k2]; p = R(w) (X - C); x = p / p_z; d = 1 + k1 r^2 + k2 r^4 (r^2 = |x|^2);
// predicted = f d x. The reference differentiates this with Ceres autodiff
// (JacobianComposer.cpp:123-166); here the derivatives are analytic:
//   du/dp = f [d I + 2 g x x^T] [I | -x] / p_z,  g = k1 + 2 k2 r^2
//   du/dX = du/dp R,  du/dC = -du/dX
//   du/dw = -du/dp R [X - C]_x J_r(w),  J_r = I - a [w]_x + b [w]_x^2,
//           a = (1 - cos t) / t^2, b = (t - sin t) / t^3, t = |w|
//   du/df = d x,  du/dk1 = f r^2 x,  du/dk2 = f r^4 x.
// Output rows 2o, 2o+1 of observation o hold 12 entries each: the camera's
// 9 columns (9c .. 9c+8) then the point's 3 (9C + 3p ..), ascending, the
// layout the reference's .jacob files and compute.cpp:256-261 use.
#include <cmath>

#include "../../include/uncte.h"
#include "internal.h"

namespace unc {
namespace {

__device__ __forceinline__ void skew(const double v[3], double W[3][3]) {
    W[0][0] = 0.0;   W[0][1] = -v[2]; W[0][2] = v[1];
    W[1][0] = v[2];  W[1][1] = 0.0;   W[1][2] = -v[0];
    W[2][0] = -v[1]; W[2][1] = v[0];  W[2][2] = 0.0;
}

__global__ void k_scene_jacobian(int num_cams, int num_points, int num_obs, const double* __restrict__ cams,
                                 const double* __restrict__ pts, const int* __restrict__ obs_cam,
                                 const int* __restrict__ obs_pt, int* __restrict__ rows, int* __restrict__ cols,
                                 double* __restrict__ vals, int* err) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o == 0) rows[2L * num_obs] = 24 * num_obs;
    if (o >= num_obs) return;
    rows[2L * o] = 24 * o;
    rows[2L * o + 1] = 24 * o + 12;
    const int c = obs_cam[o], q = obs_pt[o];
    int* cc = cols + 24L * o;
    double* vv = vals + 24L * o;
    if (c < 0 || c >= num_cams || q < 0 || q >= num_points) {
        atomicOr(err, ERRBIT_LAYOUT);
        for (int k = 0; k < 24; ++k) {
            cc[k] = 0;
            vv[k] = 0.0;
        }
        return;
    }
    const double* cam = cams + 9L * c;
    const double w[3] = {cam[0], cam[1], cam[2]};
    const double pC[3] = {pts[3L * q] - cam[3], pts[3L * q + 1] - cam[4], pts[3L * q + 2] - cam[5]};
    const double f = cam[6], k1 = cam[7], k2 = cam[8];
    // R(w) by Rodrigues' formula; first order below |w| = 1e-6
    double W[3][3], W2[3][3], R[3][3];
    skew(w, W);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) W2[i][j] = W[i][0] * W[0][j] + W[i][1] * W[1][j] + W[i][2] * W[2][j];
    const double t2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
    const double t = sqrt(t2);
    double sA, cA, a, bb;  // R = I + sA W + cA W^2 ; J_r = I - a W + bb W^2
    if (t < 1e-6) {
        sA = 1.0;
        cA = 0.5;
        a = 0.5;
        bb = 1.0 / 6.0;
    } else {
        double st, ct;
        sincos(t, &st, &ct);
        sA = st / t;
        cA = (1.0 - ct) / t2;
        a = cA;
        bb = (t - st) / (t2 * t);
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) R[i][j] = (i == j ? 1.0 : 0.0) + sA * W[i][j] + cA * W2[i][j];
    double p[3];
    for (int i = 0; i < 3; ++i) p[i] = R[i][0] * pC[0] + R[i][1] * pC[1] + R[i][2] * pC[2];
    const double z = p[2], xp = p[0] / z, yp = p[1] / z;
    const double r2 = xp * xp + yp * yp;
    const double d = 1.0 + k1 * r2 + k2 * r2 * r2;
    const double g = k1 + 2.0 * k2 * r2;
    const double M00 = f * (d + 2.0 * xp * xp * g), M01 = f * 2.0 * xp * yp * g, M11 = f * (d + 2.0 * yp * yp * g);
    // du/dp = M Q, Q = [[1/z, 0, -p0/z^2], [0, 1/z, -p1/z^2]]
    const double iz = 1.0 / z, q02 = -p[0] * iz * iz, q12 = -p[1] * iz * iz;
    double D[2][3];
    D[0][0] = M00 * iz;
    D[0][1] = M01 * iz;
    D[0][2] = M00 * q02 + M01 * q12;
    D[1][0] = M01 * iz;
    D[1][1] = M11 * iz;
    D[1][2] = M01 * q02 + M11 * q12;
    double Jp[2][3];
    for (int r = 0; r < 2; ++r)
        for (int j = 0; j < 3; ++j) Jp[r][j] = D[r][0] * R[0][j] + D[r][1] * R[1][j] + D[r][2] * R[2][j];
    // du/dw = -Jp [pC]_x J_r
    double P[3][3], Jr[3][3], PJ[3][3];
    skew(pC, P);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Jr[i][j] = (i == j ? 1.0 : 0.0) - a * W[i][j] + bb * W2[i][j];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) PJ[i][j] = P[i][0] * Jr[0][j] + P[i][1] * Jr[1][j] + P[i][2] * Jr[2][j];
    const double xy[2] = {xp, yp};
    for (int r = 0; r < 2; ++r) {
        double* row = vv + 12 * r;
        int* cr = cc + 12 * r;
        for (int j = 0; j < 3; ++j) row[j] = -(Jp[r][0] * PJ[0][j] + Jp[r][1] * PJ[1][j] + Jp[r][2] * PJ[2][j]);
        for (int j = 0; j < 3; ++j) row[3 + j] = -Jp[r][j];
        row[6] = xy[r] * d;
        row[7] = f * xy[r] * r2;
        row[8] = f * xy[r] * r2 * r2;
        for (int j = 0; j < 3; ++j) row[9 + j] = Jp[r][j];
        for (int k = 0; k < 9; ++k) cr[k] = 9 * c + k;
        for (int k = 0; k < 3; ++k) cr[9 + k] = 9 * num_cams + 3 * q + k;
    }
}

}  // namespace

int launch_scene_jacobian(int num_cams, int num_points, int num_obs, const double* cams, const double* pts,
                          const int* obs_cam, const int* obs_pt, int* rows, int* cols, double* vals, int* err,
                          cudaStream_t st) {
    k_scene_jacobian<<<(num_obs + 127) / 128 + (num_obs == 0), 128, 0, st>>>(
        num_cams, num_points, num_obs, cams, pts, obs_cam, obs_pt, rows, cols, vals, err);
    count_launch();
    return cudaGetLastError() == cudaSuccess ? UNC_OK : UNC_ERR_CUDA;
}

}  // namespace unc

using namespace unc;

extern "C" int unc_jacobian_device(int num_cams, int num_points, int num_obs, const double* d_cams,
                                   const double* d_points, const int* d_obs_cam, const int* d_obs_pt, int* d_rows,
                                   int* d_cols, double* d_values, void* stream) {
    g_last_error.clear();
    if (num_cams <= 0 || num_points < 0 || num_obs < 0 || !d_cams || (num_points && !d_points) ||
        (num_obs && (!d_obs_cam || !d_obs_pt || !d_cols || !d_values)) || !d_rows) {
        g_last_error = "unc_jacobian_device: bad arguments";
        return UNC_ERR_INVALID_ARG;
    }
    cudaStream_t sm = (cudaStream_t)stream;
    int* err = nullptr;
    if (cudaMallocAsync((void**)&err, sizeof(int), sm) != cudaSuccess) return UNC_ERR_OUT_OF_MEMORY;
    cudaMemsetAsync(err, 0, sizeof(int), sm);
    int rc = launch_scene_jacobian(num_cams, num_points, num_obs, d_cams, d_points, d_obs_cam, d_obs_pt, d_rows,
                                   d_cols, d_values, err, sm);
    int h = 0;
    cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, sm);
    cudaFreeAsync(err, sm);
    cudaError_t e = cudaStreamSynchronize(sm);
    if (rc != UNC_OK || e != cudaSuccess) {
        g_last_error = std::string("unc_jacobian_device: ") + cudaGetErrorString(e);
        return UNC_ERR_CUDA;
    }
    if (h & ERRBIT_LAYOUT) {
        g_last_error = "unc_jacobian_device: camera or point id out of range";
        return UNC_ERR_INVALID_ARG;
    }
    return UNC_OK;
}
