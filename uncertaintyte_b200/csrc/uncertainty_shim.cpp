// uncertainty_shim.cpp - the C++ drop-in entry points of include/uncertainty.h,
// forwarding to the C ABI of uncte.h (all compute on the GPU).
//
// Mirrors src/uncertaintyTE/uncertainty.cpp:20-186 and the dispatch of
// computeCovariances (compute.cpp:458-540).
#include "uncertainty.h"

#include <algorithm>
#include <cstring>

#include "uncte.h"

namespace {

struct CtxHolder {
    unc_context* ctx = nullptr;
    ~CtxHolder() { unc_context_destroy(ctx); }
};

unc_context* thread_context() {
    static thread_local CtxHolder h;
    if (!h.ctx) {
        int rc = unc_context_create(0, &h.ctx);
        if (rc != UNC_OK) throw cov::Error(rc, std::string("uncertainty: ") + unc_last_error());
    }
    return h.ctx;
}

double dist3(const double* a, const double* b) {
    double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
    return std::sqrt(dx * dx + dy * dy + dz * dz);
}

}  // namespace

namespace cov {

void Uncertainty::init(const Options& options) {
    _camParams = options._camParams;
    _numCams = options._numCams;
    _numPoints = options._numPoints;
    _nbCovarianceValuePerCam = (std::size_t)(0.5 * options._camParams * (options._camParams + 1));
    _camerasUnc.resize(options._numCams * _nbCovarianceValuePerCam);
    _pointsUnc.resize(options._numPoints * 6);
}

const std::vector<double> Uncertainty::getCamerasUncRaw() const { return _camerasUnc; }

const std::vector<double> Uncertainty::getCameraUncMatrix(int id) const {
    std::vector<double> m(_camParams * _camParams);
    std::size_t t = 0;
    for (std::size_t i = 0; i < _camParams; i++)
        for (std::size_t j = i; j < _camParams; j++) {
            double v = _camerasUnc[t + id * _nbCovarianceValuePerCam];
            m[i * _camParams + j] = v;
            m[i + j * _camParams] = v;
            t++;
        }
    return m;
}

const std::vector<double> Uncertainty::getCamerasUncMatrices() const {
    std::vector<double> out;
    out.reserve(_numCams * _camParams * _camParams);
    for (std::size_t k = 0; k < _numCams; k++) {
        std::vector<double> m = getCameraUncMatrix((int)k);
        out.insert(out.end(), m.begin(), m.end());
    }
    return out;
}

// eigen-decompositions of all blocks in one GPU call (uncertainty.cpp:74-115)
const std::vector<double> Uncertainty::getCamerasUncEigenValues() const {
    std::vector<double> out(_numCams * _camParams);
    int rc = unc_block_eigen(_camerasUnc.data(), (int)_numCams, (int)_camParams, 0, (int)_camParams, out.data(),
                             nullptr);
    if (rc != UNC_OK) throw Error(rc, std::string("getCamerasUncEigenValues: ") + unc_last_error());
    return out;
}

const std::vector<double> Uncertainty::getCamerasCentersUncEigVec() const {
    std::vector<double> vals(_numCams * 3), out(_numCams * 9);
    int rc = unc_block_eigen(_camerasUnc.data(), (int)_numCams, (int)_camParams, 3, 3, vals.data(), out.data());
    if (rc != UNC_OK) throw Error(rc, std::string("getCamerasCentersUncEigVec: ") + unc_last_error());
    return out;
}

const std::vector<double> Uncertainty::getPointsUncRaw() const { return _pointsUnc; }

const std::vector<double> Uncertainty::getPointUncMatrix(int id) const {
    const double* p = _pointsUnc.data() + 6 * (std::size_t)id;
    return {p[0], p[1], p[2], p[1], p[3], p[4], p[2], p[4], p[5]};
}

const std::vector<double> Uncertainty::getPointsUncMatrices() const {
    std::vector<double> out;
    out.reserve(_numPoints * 9);
    for (std::size_t k = 0; k < _numPoints; k++) {
        std::vector<double> m = getPointUncMatrix((int)k);
        out.insert(out.end(), m.begin(), m.end());
    }
    return out;
}

// eigen-decompositions of all point blocks in one GPU call (uncertainty.cpp:146-183)
const std::vector<double> Uncertainty::getPointsUncEigenValues() const {
    std::vector<double> out(_numPoints * 3);
    int rc = unc_block_eigen(_pointsUnc.data(), (int)_numPoints, 3, 0, 3, out.data(), nullptr);
    if (rc != UNC_OK) throw Error(rc, std::string("getPointsUncEigenValues: ") + unc_last_error());
    return out;
}

const std::vector<double> Uncertainty::getPointsUncEigVectors() const {
    std::vector<double> vals(_numPoints * 3), out(_numPoints * 9);
    int rc = unc_block_eigen(_pointsUnc.data(), (int)_numPoints, 3, 0, 3, vals.data(), out.data());
    if (rc != UNC_OK) throw Error(rc, std::string("getPointsUncEigVectors: ") + unc_last_error());
    return out;
}

void findPts2Fix(Options& opt, int N, const double* pts) {
    if (N < 3 || !pts) throw Error(UNC_ERR_INVALID_ARG, "findPts2Fix: need at least 3 points");
    double cen[3] = {0, 0, 0};
    for (int i = 0; i < N; ++i)
        for (int k = 0; k < 3; ++k) cen[k] += pts[3 * i + k] / N;
    auto argmax = [&](auto score, int ex0, int ex1) {
        int best = -1;
        double bs = -1;
        for (int i = 0; i < N; ++i) {
            if (i == ex0 || i == ex1) continue;
            double s = score(i);
            if (s > bs) {
                bs = s;
                best = i;
            }
        }
        return best;
    };
    int a = argmax([&](int i) { return dist3(pts + 3 * i, cen); }, -1, -1);
    int b = argmax([&](int i) { return dist3(pts + 3 * i, pts + 3 * a); }, a, -1);
    int c = argmax([&](int i) { return dist3(pts + 3 * i, pts + 3 * a) + dist3(pts + 3 * i, pts + 3 * b); }, a, b);
    for (int round = 0; round < 16; ++round) {  // local improvement of the perimeter
        int a2 = argmax([&](int i) { return dist3(pts + 3 * i, pts + 3 * b) + dist3(pts + 3 * i, pts + 3 * c); }, b, c);
        int b2 = argmax([&](int i) { return dist3(pts + 3 * i, pts + 3 * a2) + dist3(pts + 3 * i, pts + 3 * c); }, a2, c);
        int c2 = argmax([&](int i) { return dist3(pts + 3 * i, pts + 3 * a2) + dist3(pts + 3 * i, pts + 3 * b2); }, a2, b2);
        bool same = a2 == a && b2 == b && c2 == c;
        a = a2;
        b = b2;
        c = c2;
        if (same) break;
    }
    int t[3] = {a, b, c};
    std::sort(t, t + 3);
    opt.setPts2Fix(t[0], t[1], t[2]);
}

}  // namespace cov

void computeCovariances(cov::Options& options, cov::Statistic& statistic, ceres::CRSMatrix& jacobian,
                        double* camUnc, double* ptUnc) {
    if (camUnc == NULL || ptUnc == NULL) return;  // compute.cpp:459
    unc_options o;
    unc_options_init(&o, options._numCams, options._camParams, options._numPoints, options._numObs);
    o.algorithm = (int)options._algorithm;
    o.epsilon = options._epsilon;
    o.lambda = options._lambda;
    o.svd_remove_n = options._svdRemoveN;
    o.max_iter_te = options._maxIterTE;
    o.precision = (int)options._precision;
    if (options._pts2fix) {
        o.has_pts2fix = 1;
        for (int i = 0; i < 3; ++i) o.pts2fix[i] = options._pts2fix[i];
    }
    unc_statistic st;
    int rc = unc_compute(thread_context(), &o, jacobian.num_rows, jacobian.num_cols,
                         jacobian.rows.data(), jacobian.cols.data(), jacobian.values.data(), camUnc,
                         ptUnc, &st);
    if (rc != UNC_OK)
        throw cov::Error(rc, std::string("computeCovariances: ") + unc_status_string(rc) + ": " + unc_last_error());
    statistic.timeCreateJ = st.time_create_j;
    statistic.timeFixJ = st.time_fix_j;
    statistic.timeNormJ = st.time_norm_j;
    statistic.timeMultiplyJJ = st.time_multiply_jj;
    statistic.timeSplitJJ = st.time_split_jj;
    statistic.timeInvV = st.time_inv_v;
    statistic.timeComposeZ = st.time_compose_z;
    statistic.timeInvZ = st.time_inv_z;
    statistic.timeTE = st.time_te;
    statistic.timePtsUnc = st.time_pts_unc;
    statistic.timeAll = st.time_all;
    statistic.lambda = st.lambda;
    if (o.algorithm == UNC_TAYLOR_EXPANSION) {
        if (!statistic.fixedPts) statistic.fixedPts = static_cast<int*>(malloc(3 * sizeof(int)));
        for (int i = 0; i < 3; ++i) statistic.fixedPts[i] = st.fixed_pts[i];
    }
    statistic.cycle_change.assign(st.cycle_change, st.cycle_change + st.te_iterations);
}

void getCovariances(cov::Options& options, cov::Statistic& statistic, ceres::CRSMatrix& jacobian,
                    double* h_camUnc, double* h_ptUnc) {
    computeCovariances(options, statistic, jacobian, h_camUnc, h_ptUnc);
}

void getCovariances(cov::Options& options, cov::Statistic& statistic, ceres::CRSMatrix& jacobian,
                    double* points3D, cov::Uncertainty& uncertainties) {
    cov::findPts2Fix(options, options._numPoints, points3D);
    uncertainties.init(options);
    computeCovariances(options, statistic, jacobian, uncertainties._camerasUnc.data(),
                       uncertainties._pointsUnc.data());
}
