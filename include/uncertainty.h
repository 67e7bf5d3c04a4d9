/*
 * uncertainty.h - drop-in C++ interface of the B200 covariance library.
 *
 * Source-compatible with uncertaintyTE's public header
 * (src/uncertaintyTE/uncertainty.h:24-158 and include/uncertainty.h:11-62):
 * the same cov::Options / cov::Statistic / cov::Uncertainty types (same field
 * order; new fields are appended), the same getCovariances overloads and
 * computeCovariances (src/uncertaintyTE/compute.h:92-97). Link against
 * libuncte.so instead of the reference library; all compute runs on the GPU
 * through the C ABI in uncte.h.
 *
 * Differences a caller can observe:
 *   - errors throw cov::Error (status code + message) instead of exit(1);
 *   - getCovariances(..., points3D, ...) picks the fixed points
 *     deterministically (the reference samples 100k random triples);
 *   - Options::_debug does not dump matrices;
 *   - times in Statistic are true seconds (the reference stores ms/100);
 *   - getCamerasCentersUncEigVec / getPointsUncEigVectors return the
 *     eigenvectors in descending eigenvalue order, the order of the eigenvalue
 *     accessors (the reference returns them in Eigen::EigenSolver's unspecified
 *     order, uncertainty.cpp:92-115,164-183); each vector's sign is arbitrary in
 *     both.
 */
#pragma once
#include <cmath>
#include <cstdlib>
#include <iostream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#if defined(UNC_WITH_CERES)
#include "ceres/ceres.h"
#else
namespace ceres {
/* Layout-compatible stand-in for ceres::CRSMatrix (only these fields are
 * used: compute.cpp:474, JacobianIO.cpp:50-60). Define UNC_WITH_CERES to use
 * the real Ceres type instead. */
struct CRSMatrix {
    CRSMatrix() : num_cols(0), num_rows(0) {}
    int num_cols;
    int num_rows;
    std::vector<int> cols;
    std::vector<int> rows;
    std::vector<double> values;
};
}  // namespace ceres
#endif

#define SVD_QR_ITERATION 0
#define SVD_DEVIDE_AND_CONQUER 1
#define TAYLOR_EXPANSION 2

namespace cov {

enum EAlgorithm {
    eAlgorithmSvdQrIteration = 0,
    eAlgorithmSvdDeviceAndconquer = 1,
    eAlgorithmSvdTaylorExpansion = 2,
    /* extension: SVD pseudo-inverse of the camera Schur complement (UNC_SVD_SCHUR) */
    eAlgorithmSvdSchur = 3
};

/* precision of the dense Taylor-series products (new; appended field) */
enum EPrecision { ePrecisionFP64 = 0, ePrecisionMixed = 1 };

inline std::string EAlgorithm_enumToString(EAlgorithm alg) {
    switch (alg) {
        case eAlgorithmSvdQrIteration: return "SVD_QR_ITERATION";
        case eAlgorithmSvdDeviceAndconquer: return "SVD_DEVIDE_AND_CONQUER";
        case eAlgorithmSvdTaylorExpansion: return "TAYLOR_EXPANSION";
        case eAlgorithmSvdSchur: return "SVD_SCHUR";
        default: return "not defined";
    }
}

inline EAlgorithm EAlgorithm_stringToEnum(const std::string& algorithm) {
    if (algorithm == "SVD_QR_ITERATION") return eAlgorithmSvdQrIteration;
    if (algorithm == "SVD_DEVIDE_AND_CONQUER") return eAlgorithmSvdDeviceAndconquer;
    if (algorithm == "TAYLOR_EXPANSION") return eAlgorithmSvdTaylorExpansion;
    if (algorithm == "SVD_SCHUR") return eAlgorithmSvdSchur;
    throw std::runtime_error(std::string("Unrecognized algorithm: ") + algorithm);
}

struct Options {
   public:
    double _epsilon, _lambda;
    EAlgorithm _algorithm;
    int _numCams, _camParams, _numPoints, _numObs, _svdRemoveN, _maxIterTE;
    int* _pts2fix = NULL; /* malloc'ed: released with free() as the reference does */
    bool _debug = false;
    EPrecision _precision = ePrecisionFP64;

    Options()
        : _epsilon(1e-10), _lambda(-1), _algorithm(eAlgorithmSvdTaylorExpansion), _numCams(0),
          _camParams(9), _numPoints(0), _numObs(0), _svdRemoveN(-1), _maxIterTE(-1) {}
    Options(int numCams, int camParams, int numPoints, int numObs)
        : _epsilon(1e-10), _lambda(-1), _algorithm(eAlgorithmSvdTaylorExpansion), _numCams(numCams),
          _camParams(camParams), _numPoints(numPoints), _numObs(numObs), _svdRemoveN(-1),
          _maxIterTE(-1) {}
    Options(EAlgorithm algorithm, double eps_or_lamb, int numCams, int camParams, int numPoints,
            int numObs)
        : _epsilon(eps_or_lamb), _lambda(eps_or_lamb), _algorithm(algorithm), _numCams(numCams),
          _camParams(camParams), _numPoints(numPoints), _numObs(numObs), _svdRemoveN(-1),
          _maxIterTE(-1) {}
    Options(const Options&) = delete;
    Options& operator=(const Options&) = delete;
    ~Options() { free(_pts2fix); }
    /* set the three fixed points (copied into a malloc'ed array) */
    void setPts2Fix(int a, int b, int c) {
        if (!_pts2fix) _pts2fix = static_cast<int*>(malloc(3 * sizeof(int)));
        _pts2fix[0] = a;
        _pts2fix[1] = b;
        _pts2fix[2] = c;
    }
};

struct Statistic {
    double timeCreateJ = 0, timeFixJ = 0, timeNormJ = 0, timeMultiplyJJ = 0, timeSplitJJ = 0,
           timeInvV = 0, timeComposeZ = 0, timeInvZ = 0, timeTE = 0, timePtsUnc = 0, timeAll = 0;
    double lambda = 0;
    int* fixedPts = NULL; /* malloc'ed */
    std::vector<double> cycle_change;

    Statistic() = default;
    Statistic(const Statistic&) = delete;
    Statistic& operator=(const Statistic&) = delete;
    ~Statistic() { free(fixedPts); }
};

struct Uncertainty {
    std::size_t _camParams = 0;
    std::size_t _numCams = 0;
    std::size_t _numPoints = 0;
    std::size_t _nbCovarianceValuePerCam = 0;
    std::vector<double> _camerasUnc;
    std::vector<double> _pointsUnc;

    /* uncertainty.cpp:36-44 */
    void init(const Options& options);
    /* upper triangle, p(p+1)/2 values per camera (uncertainty.cpp:46) */
    const std::vector<double> getCamerasUncRaw() const;
    /* full p x p matrix of one camera (uncertainty.cpp:48-61) */
    const std::vector<double> getCameraUncMatrix(int id) const;
    const std::vector<double> getCamerasUncMatrices() const;
    /* eigenvalues of each camera block, descending (uncertainty.cpp:74-90) */
    const std::vector<double> getCamerasUncEigenValues() const;
    /* eigenvectors of the 3x3 camera-centre block (uncertainty.cpp:92-115), column by
     * column in descending eigenvalue order */
    const std::vector<double> getCamerasCentersUncEigVec() const;
    const std::vector<double> getPointsUncRaw() const;
    const std::vector<double> getPointUncMatrix(int id) const;
    const std::vector<double> getPointsUncMatrices() const;
    const std::vector<double> getPointsUncEigenValues() const;
    const std::vector<double> getPointsUncEigVectors() const;
};

/* Thrown by the entry points below on failure (the reference exit()s). */
class Error : public std::runtime_error {
   public:
    Error(int status, const std::string& msg) : std::runtime_error(msg), status(status) {}
    int status;
};

/* Deterministic fixed-point choice: the three points spanning the
 * (locally) largest-perimeter triangle, sorted ascending. Replaces the random
 * sampling of JacobianComposer::findPts2Fix (JacobianComposer.cpp:63-83). */
void findPts2Fix(Options& opt, int N, const double* points3D);

}  // namespace cov

/* include/uncertainty.h:55-62 (legacy 5-argument form) */
void getCovariances(cov::Options& options, cov::Statistic& statistic, ceres::CRSMatrix& jacobian,
                    double* h_camUnc, double* h_ptUnc);

/* src/uncertaintyTE/uncertainty.h:153-158, uncertainty.cpp:20-30 */
void getCovariances(cov::Options& options, cov::Statistic& statistic, ceres::CRSMatrix& jacobian,
                    double* points3D, cov::Uncertainty& uncertainties);

/* src/uncertaintyTE/compute.h:92-97 */
void computeCovariances(cov::Options& options, cov::Statistic& statistic, ceres::CRSMatrix& jacobian,
                        double* camUnc, double* ptUnc);
