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

// symmetric eigen-decomposition (cyclic Jacobi), n <= 16, row-major in/out
void sym_eig(int n, std::vector<double> a, std::vector<double>& w, std::vector<double>& v) {
    v.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) v[(size_t)i * n + i] = 1.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0, dia = 0;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j)
                (i == j ? dia : off) += std::fabs(a[(size_t)i * n + j]);
        if (off <= 1e-300 || off < dia * 1e-17) break;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                double apq = a[(size_t)p * n + q];
                if (apq == 0) continue;
                double theta = (a[(size_t)q * n + q] - a[(size_t)p * n + p]) / (2 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1));
                double c = 1 / std::sqrt(t * t + 1), s = t * c;
                for (int k = 0; k < n; ++k) {
                    double akp = a[(size_t)k * n + p], akq = a[(size_t)k * n + q];
                    a[(size_t)k * n + p] = c * akp - s * akq;
                    a[(size_t)k * n + q] = s * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {
                    double apk = a[(size_t)p * n + k], aqk = a[(size_t)q * n + k];
                    a[(size_t)p * n + k] = c * apk - s * aqk;
                    a[(size_t)q * n + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < n; ++k) {
                    double vkp = v[(size_t)k * n + p], vkq = v[(size_t)k * n + q];
                    v[(size_t)k * n + p] = c * vkp - s * vkq;
                    v[(size_t)k * n + q] = s * vkp + c * vkq;
                }
            }
    }
    w.resize(n);
    for (int i = 0; i < n; ++i) w[i] = a[(size_t)i * n + i];
}

// eigenvalues sorted descending with their eigenvectors (columns)
void sorted_eig(int n, const std::vector<double>& m, std::vector<double>& w, std::vector<double>& vec) {
    std::vector<double> wv, vv;
    sym_eig(n, m, wv, vv);
    std::vector<int> idx(n);
    for (int i = 0; i < n; ++i) idx[i] = i;
    std::sort(idx.begin(), idx.end(), [&](int a, int b) { return wv[a] > wv[b]; });
    w.resize(n);
    vec.resize((size_t)n * n);
    for (int c = 0; c < n; ++c) {
        w[c] = wv[idx[c]];
        for (int r = 0; r < n; ++r) vec[(size_t)r * n + c] = vv[(size_t)r * n + idx[c]];
    }
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

const std::vector<double> Uncertainty::getCamerasUncEigenValues() const {
    std::vector<double> out;
    for (std::size_t i = 0; i < _numCams; i++) {
        std::vector<double> w, v;
        sorted_eig((int)_camParams, getCameraUncMatrix((int)i), w, v);
        out.insert(out.end(), w.begin(), w.end());
    }
    return out;
}

const std::vector<double> Uncertainty::getCamerasCentersUncEigVec() const {
    std::vector<double> out;
    for (std::size_t i = 0; i < _numCams; i++) {
        std::vector<double> m = getCameraUncMatrix((int)i), b(9), w, v;
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) b[r * 3 + c] = m[(3 + r) * _camParams + (3 + c)];
        sorted_eig(3, b, w, v);
        for (int c = 0; c < 3; ++c)
            for (int r = 0; r < 3; ++r) out.push_back(v[r * 3 + c]);
    }
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

const std::vector<double> Uncertainty::getPointsUncEigenValues() const {
    std::vector<double> out;
    for (std::size_t i = 0; i < _numPoints; i++) {
        std::vector<double> w, v;
        sorted_eig(3, getPointUncMatrix((int)i), w, v);
        out.insert(out.end(), w.begin(), w.end());
    }
    return out;
}

const std::vector<double> Uncertainty::getPointsUncEigVectors() const {
    std::vector<double> out;
    for (std::size_t i = 0; i < _numPoints; i++) {
        std::vector<double> w, v;
        sorted_eig(3, getPointUncMatrix((int)i), w, v);
        for (int c = 0; c < 3; ++c)
            for (int r = 0; r < 3; ++r) out.push_back(v[r * 3 + c]);
    }
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
