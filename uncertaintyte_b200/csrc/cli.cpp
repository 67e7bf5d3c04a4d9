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

namespace {

bool read_file(const std::string& path, std::string& out) {
    std::ifstream f(path, std::ios::binary);
    if (!f.good()) return false;
    std::ostringstream ss;
    ss << f.rdbuf();
    out = ss.str();
    return true;
}

// JacobianIO::loadJacobian (JacobianIO.cpp:32-63) with a fast tokenizer;
// '#' starts a comment (the documented template carries some).
bool load_jacob(const std::string& path, cov::Options& opt, ceres::CRSMatrix& J) {
    std::string text;
    if (!read_file(path, text)) {
        std::cerr << "\nThe input file doesn't exist.\n";
        return false;
    }
    for (size_t i = 0; i < text.size(); ++i)
        if (text[i] == '#')
            while (i < text.size() && text[i] != '\n') text[i++] = ' ';
    const char* p = text.c_str();
    char* end = nullptr;
    auto num = [&](double& v) {
        v = strtod(p, &end);
        if (end == p) return false;
        p = end;
        return true;
    };
    double h[11];
    for (double& v : h)
        if (!num(v)) return false;
    opt._algorithm = cov::eAlgorithmSvdTaylorExpansion;
    opt._epsilon = 1e-10;
    opt._svdRemoveN = 7;
    opt._maxIterTE = -1;
    opt._lambda = h[0];
    opt._numCams = (int)h[1];
    opt._camParams = (int)h[2];
    opt._numPoints = (int)h[3];
    opt._numObs = (int)h[4];
    if (h[5] >= 0 && h[6] >= 0 && h[7] >= 0) opt.setPts2Fix((int)h[5], (int)h[6], (int)h[7]);
    J.num_rows = (int)h[8];
    J.num_cols = (int)h[9];
    long nnz = (long)h[10];
    J.rows.resize((size_t)J.num_rows + 1);
    J.cols.resize(nnz);
    J.values.resize(nnz);
    for (auto& r : J.rows) {
        long v = strtol(p, &end, 10);
        if (end == p) return false;
        p = end;
        r = (int)v;
    }
    for (auto& c : J.cols) {
        long v = strtol(p, &end, 10);
        if (end == p) return false;
        p = end;
        c = (int)v;
    }
    for (auto& v : J.values)
        if (!num(v)) return false;
    return true;
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
