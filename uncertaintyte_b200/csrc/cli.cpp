// cli.cpp - the `uncertainty` command-line tool on the GPU library.
//
// Same flags as the reference CLI (src/software/main_uncertainty.cpp:35-52):
//   -in=<file.jacob> -in_form=JACOBIAN -out=<file.cov> [-alg=...] [-debug]
// Like the reference, a .jacob input runs TAYLOR_EXPANSION whatever -alg says
// (JacobianIO.cpp:25); -force_alg makes -alg effective. -precision=FP64|MIXED
// selects the Taylor-product precision. COLMAP / ALICEVISION scene inputs are
// not supported (the Jacobian is the input of this library).
#include <chrono>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "uncertainty.h"
#include "uncte.h"

namespace {

// JacobianIO::loadJacobian (JacobianIO.cpp:32-63) through the library's
// parser: text (all host threads) or this library's binary form.
bool load_jacob(const std::string& path, cov::Options& opt, ceres::CRSMatrix& J) {
    unc_jacob_header h;
    if (unc_jacob_read_header(path.c_str(), &h) != UNC_OK) {
        std::cerr << "\n" << unc_last_error() << "\n";
        return false;
    }
    opt._algorithm = cov::eAlgorithmSvdTaylorExpansion;
    opt._epsilon = 1e-10;
    opt._svdRemoveN = 7;
    opt._maxIterTE = -1;
    opt._lambda = h.lambda;
    opt._numCams = h.num_cams;
    opt._camParams = h.cam_params;
    opt._numPoints = h.num_points;
    opt._numObs = h.num_obs;
    if (h.pts2fix[0] >= 0 && h.pts2fix[1] >= 0 && h.pts2fix[2] >= 0)
        opt.setPts2Fix(h.pts2fix[0], h.pts2fix[1], h.pts2fix[2]);
    J.num_rows = h.num_rows;
    J.num_cols = h.num_cols;
    J.rows.resize((size_t)h.num_rows + 1);
    J.cols.resize((size_t)h.nnz);
    J.values.resize((size_t)h.nnz);
    if (unc_jacob_read(path.c_str(), &h, J.rows.data(), J.cols.data(), J.values.data()) != UNC_OK) {
        std::cerr << "\n" << unc_last_error() << "\n";
        return false;
    }
    return true;
}

// -write_binary=<path>: the same Jacobian in this library's binary form
bool save_binary(const std::string& path, const cov::Options& opt, const ceres::CRSMatrix& J) {
    unc_jacob_header h{};
    h.lambda = opt._lambda;
    h.num_cams = opt._numCams;
    h.cam_params = opt._camParams;
    h.num_points = opt._numPoints;
    h.num_obs = opt._numObs;
    for (int i = 0; i < 3; ++i) h.pts2fix[i] = opt._pts2fix ? opt._pts2fix[i] : -1;
    h.num_rows = J.num_rows;
    h.num_cols = J.num_cols;
    h.nnz = (long long)J.values.size();
    h.binary = 1;
    return unc_jacob_write_binary(path.c_str(), &h, J.rows.data(), J.cols.data(), J.values.data()) == UNC_OK;
}

// saveResults (IO.cpp:15-60); times are true seconds.
void save_cov(const std::string& path, cov::Options& o, cov::Statistic& s, int per_cam,
              const std::vector<double>& cam, const std::vector<double>& pt) {
    std::ofstream f(path);
    f << "# ---- Covariance v0.1 ----\n";
    f << "# Number of cameras: " << o._numCams << "\n";
    f << "# Number of camera parameters: " << o._camParams << "\n";
    f << "# Number of points in 3D: " << o._numPoints << "\n";
    f << "# Number of observations: " << o._numObs << "\n";
    f << "# Used algorithm: " << cov::EAlgorithm_enumToString(o._algorithm) << "\n";
    if (o._algorithm == cov::eAlgorithmSvdTaylorExpansion) {
        if (s.fixedPts) f << "# Fixed points: " << s.fixedPts[0] << ", " << s.fixedPts[1] << ", " << s.fixedPts[2] << "\n";
        f << "# Used lambda: " << s.lambda << "\n";
        f << "# Loading jacobian time: " << s.timeCreateJ << "s\n";
        f << "# Normalization of jacobian time: " << s.timeNormJ << "s\n";
        f << "# Compose information matrix time: " << s.timeMultiplyJJ << "s\n";
        f << "# Split infromation matrix time: " << s.timeSplitJJ << "s\n";
        f << "# Inverse V time: " << s.timeInvV << "s\n";
        f << "# Compose Z time: " << s.timeComposeZ << "s\n";
        f << "# Inverse Z time: " << s.timeInvZ << "s\n";
        f << "# Taylor expansion time: " << s.timeTE << "s\n";
        f << "# Point uncertainty time: " << s.timePtsUnc << "s\n";
        f << "# TE number of iterations: " << s.cycle_change.size() << "\n";
        f << "# TE cycle change: ";
        for (double c : s.cycle_change) f << c << " ";
        f << "\n";
    }
    f << "# Time of the algorithm: " << s.timeAll << "s\n";
    f << "# -----------------------\n";
    for (int i = 0; i < o._numCams; ++i) {
        for (int j = 0; j < per_cam; ++j) f << cam[(size_t)i * per_cam + j] << " ";
        f << "\n";
    }
    for (int i = 0; i < o._numPoints; ++i) {
        for (int j = 0; j < 6; ++j) f << pt[(size_t)i * 6 + j] << " ";
        f << "\n";
    }
}

std::string flag(int argc, char** argv, const std::string& name, const std::string& def) {
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        for (const std::string pre : {"--", "-"}) {
            std::string k = pre + name + "=";
            if (a.rfind(k, 0) == 0) return a.substr(k.size());
            if (a == pre + name && i + 1 < argc) return argv[i + 1];
        }
    }
    return def;
}

bool has_flag(int argc, char** argv, const std::string& name) {
    for (int i = 1; i < argc; ++i)
        if (std::string(argv[i]) == "-" + name || std::string(argv[i]) == "--" + name) return true;
    return false;
}

}  // namespace

int main(int argc, char** argv) {
    std::string in = flag(argc, argv, "in", "."), out = flag(argc, argv, "out", "out.cov");
    std::string form = flag(argc, argv, "in_form", "JACOBIAN"), alg = flag(argc, argv, "alg", "TAYLOR_EXPANSION");
    std::string prec = flag(argc, argv, "precision", "FP64");
    if (form != "JACOBIAN") {
        std::cerr << "only -in_form=JACOBIAN is supported\n";
        return 1;
    }
    cov::Options opt;
    cov::Statistic stat;
    ceres::CRSMatrix J;
    if (!load_jacob(in, opt, J)) {
        std::cerr << "cannot read " << in << "\n";
        return 1;
    }
    const std::string bin = flag(argc, argv, "write_binary", "");
    if (!bin.empty()) {
        if (!save_binary(bin, opt, J)) {
            std::cerr << "cannot write " << bin << ": " << unc_last_error() << "\n";
            return 1;
        }
        std::cout << "wrote " << bin << "\n";
        return 0;
    }
    if (has_flag(argc, argv, "force_alg")) opt._algorithm = cov::EAlgorithm_stringToEnum(alg);
    opt._precision = prec == "MIXED" ? cov::ePrecisionMixed : cov::ePrecisionFP64;
    cov::Uncertainty unc;
    unc.init(opt);
    try {
        computeCovariances(opt, stat, J, unc._camerasUnc.data(), unc._pointsUnc.data());
    } catch (const cov::Error& e) {
        std::cerr << e.what() << "\n";
        return 2;
    }
    std::cout << "------ " << cov::EAlgorithm_enumToString(opt._algorithm) << " ------\n"
              << "lambda " << stat.lambda << ", TE iterations " << stat.cycle_change.size()
              << ", total " << stat.timeAll << " s\n";
    save_cov(out, opt, stat, (int)unc._nbCovarianceValuePerCam, unc._camerasUnc, unc._pointsUnc);
    return 0;
}
