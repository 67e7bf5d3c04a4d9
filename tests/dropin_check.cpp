// dropin_check.cpp - a small caller of the C++ drop-in interface
// (include/uncertainty.h), compiled and run by tests/test_gpu_dropin.py the way
// an uncertaintyTE user would: same types, same entry points, libuncte.so in
// place of the reference library.
//
//   dropin_check <in.jacob> <out prefix> [points.bin]
//   dropin_check --accessors <num_cams> <num_points> <packed.bin> <out.bin>
//
// Writes, as raw little-endian doubles / ints:
//   <prefix>.compute.bin  computeCovariances (compute.h:92-97): cams then points
//   <prefix>.get5.bin     getCovariances, legacy 5-argument form (include/uncertainty.h:55-62)
//   <prefix>.stats.txt    lambda, iterations, fixed points and the cycle changes of the first call
// and with points.bin (3 doubles per point):
//   <prefix>.unc.bin      getCovariances(..., points3D, Uncertainty&) (uncertainty.cpp:20-30)
//                         called twice: both fixed-point triples (6 ints as doubles), then the
//                         second call's cams, points, camera eigenvalues, point eigenvalues,
//                         camera-centre eigenvectors and point eigenvectors (accessors).
// The --accessors form fills an Uncertainty from packed upper triangles (45 per
// camera, then 6 per point, as a .cov file lists them) and writes the results
// of getCameraUncMatrix(4), getPointUncMatrix(142), getCamerasUncMatrices,
// getPointsUncMatrices, getCamerasUncEigenValues and getPointsUncEigenValues
// (uncertainty.cpp:46-183), as the reference's accessor test calls them.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <vector>

#include "uncertainty.h"
#include "uncte.h"

namespace {

bool load(const char* path, cov::Options& opt, ceres::CRSMatrix& J) {
    unc_jacob_header h;
    if (unc_jacob_read_header(path, &h) != UNC_OK) return false;
    opt._algorithm = cov::eAlgorithmSvdTaylorExpansion;  // JacobianIO.cpp:40-43
    opt._epsilon = 1e-10;
    opt._svdRemoveN = 7;
    opt._lambda = h.lambda;
    opt._numCams = h.num_cams;
    opt._camParams = h.cam_params;
    opt._numPoints = h.num_points;
    opt._numObs = h.num_obs;
    if (h.pts2fix[0] >= 0) opt.setPts2Fix(h.pts2fix[0], h.pts2fix[1], h.pts2fix[2]);
    J.num_rows = h.num_rows;
    J.num_cols = h.num_cols;
    J.rows.resize((size_t)h.num_rows + 1);
    J.cols.resize((size_t)h.nnz);
    J.values.resize((size_t)h.nnz);
    return unc_jacob_read(path, &h, J.rows.data(), J.cols.data(), J.values.data()) == UNC_OK;
}

void put(std::ofstream& f, const std::vector<double>& v) {
    f.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * sizeof(double)));
}

}  // namespace

int accessors(int argc, char** argv) {
    if (argc < 6) return 1;
    cov::Uncertainty u;
    u._camParams = 9;
    u._numCams = (std::size_t)std::atoi(argv[2]);
    u._numPoints = (std::size_t)std::atoi(argv[3]);
    u._nbCovarianceValuePerCam = 45;
    std::ifstream in(argv[4], std::ios::binary);
    u._camerasUnc.resize(u._numCams * 45);
    u._pointsUnc.resize(u._numPoints * 6);
    in.read(reinterpret_cast<char*>(u._camerasUnc.data()), (std::streamsize)(u._camerasUnc.size() * 8));
    in.read(reinterpret_cast<char*>(u._pointsUnc.data()), (std::streamsize)(u._pointsUnc.size() * 8));
    if (!in) return 1;
    std::ofstream f(argv[5], std::ios::binary);
    put(f, u.getCameraUncMatrix(4));
    put(f, u.getPointUncMatrix(142));
    put(f, u.getCamerasUncMatrices());
    put(f, u.getPointsUncMatrices());
    put(f, u.getCamerasUncEigenValues());
    put(f, u.getPointsUncEigenValues());
    return 0;
}

int main(int argc, char** argv) {
    if (argc > 1 && std::string(argv[1]) == "--accessors") {
        try {
            return accessors(argc, argv);
        } catch (const cov::Error& e) {
            std::cerr << "cov::Error " << e.status << ": " << e.what() << "\n";
            return 2;
        }
    }
    if (argc < 3) {
        std::cerr << "usage: dropin_check <in.jacob> <out prefix> [points.bin]\n";
        return 1;
    }
    const std::string prefix = argv[2];
    try {
        {
            cov::Options opt;
            cov::Statistic stat;
            ceres::CRSMatrix J;
            if (!load(argv[1], opt, J)) {
                std::cerr << "cannot read " << argv[1] << ": " << unc_last_error() << "\n";
                return 1;
            }
            cov::Uncertainty u;
            u.init(opt);
            computeCovariances(opt, stat, J, u._camerasUnc.data(), u._pointsUnc.data());
            std::ofstream f(prefix + ".compute.bin", std::ios::binary);
            put(f, u._camerasUnc);
            put(f, u._pointsUnc);
            std::ofstream s(prefix + ".stats.txt");
            s.precision(17);
            s << stat.lambda << " " << stat.cycle_change.size() << " " << stat.fixedPts[0] << " "
              << stat.fixedPts[1] << " " << stat.fixedPts[2];
            for (double c : stat.cycle_change) s << " " << c;
            s << "\n";
        }
        {
            cov::Options opt;
            cov::Statistic stat;
            ceres::CRSMatrix J;
            if (!load(argv[1], opt, J)) return 1;
            std::vector<double> cam((size_t)opt._numCams * 45), pt((size_t)opt._numPoints * 6);
            getCovariances(opt, stat, J, cam.data(), pt.data());
            std::ofstream f(prefix + ".get5.bin", std::ios::binary);
            put(f, cam);
            put(f, pt);
        }
        if (argc > 3) {
            std::ifstream pf(argv[3], std::ios::binary);
            std::vector<double> pts;
            double x;
            while (pf.read(reinterpret_cast<char*>(&x), sizeof(double))) pts.push_back(x);
            std::vector<double> fixed;
            cov::Uncertainty u;
            for (int call = 0; call < 2; ++call) {
                cov::Options opt;
                cov::Statistic stat;
                ceres::CRSMatrix J;
                if (!load(argv[1], opt, J)) return 1;
                if ((size_t)opt._numPoints * 3 != pts.size()) {
                    std::cerr << "points.bin does not match the Jacobian\n";
                    return 1;
                }
                u = cov::Uncertainty();
                getCovariances(opt, stat, J, pts.data(), u);
                for (int k = 0; k < 3; ++k) fixed.push_back(opt._pts2fix[k]);
            }
            std::ofstream f(prefix + ".unc.bin", std::ios::binary);
            put(f, fixed);
            put(f, u.getCamerasUncRaw());
            put(f, u.getPointsUncRaw());
            put(f, u.getCamerasUncEigenValues());
            put(f, u.getPointsUncEigenValues());
            put(f, u.getCamerasCentersUncEigVec());
            put(f, u.getPointsUncEigVectors());
        }
    } catch (const cov::Error& e) {
        std::cerr << "cov::Error " << e.status << ": " << e.what() << "\n";
        return 2;
    }
    return 0;
}
