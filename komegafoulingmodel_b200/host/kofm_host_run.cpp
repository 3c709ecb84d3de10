// kofm_host_run - runs the reference's step loop through the host classes.
//
//   kofm_host_run <dir> <nsteps>
//
// <dir>/params.txt   "key value" lines: nX XsizeFull nY tau Fval MuVal
//                    kOmega (0/1) [maxTurbVisc krylovDim relTol absTol]
//                    [thermal (0/1) tempRelTol tempAbsTol]
// <dir>/ntype.bin    int16 node flags (XsizeFull * nY)
// <dir>/wallD.bin    FP64 wall distance (k-omega only)
// <dir>/dX.bin       FP64 link fractions, 4 planes E,W,N,S (optional; 1)
// <dir>/lbf.bin, lbkappa.bin, lbomega.bin   restart files (Array::savebin)
// <dir>/temp.bin     FP64 temperature (thermal only; Tinitial when absent)
// <dir>/ibbArr.bin, ibbDistArr.bin   interpolated bounce-back links (int32
//                    link index, FP64 wall fraction; optional)
// <dir>/walls.bin    instead of the geometry files above: FP64 wall heights
//                    per column, [2][nX] (bottom, top) or [4][nX] (+ the
//                    unfouled walls); the geometry is built on the device
// <dir>/walls_moved.bin  (with walls.bin, same layout) the walls after they
//                    moved: applied by clVariablesLB::update after `moveAt`
//                    steps (params.txt)
//
// Loads the restart files, advances nsteps of clProblem::step (Solve_no_TR),
// writes the restart files of the final state to <dir>/out/ and prints one
// JSON line with the reductions of clProblem's step loop.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <string>
#include <sys/stat.h>

#include "kofm_host.hpp"

using namespace kofm::host;

static std::map<std::string, std::string> read_params(const std::string& path) {
    std::map<std::string, std::string> m;
    std::ifstream s(path);
    std::string k, v;
    while (s >> k >> v) m[k] = v;
    return m;
}

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s <dir> <nsteps>\n", argv[0]);
        return 2;
    }
    const std::string dir = argv[1];
    const int nsteps = std::atoi(argv[2]);
    try {
        auto m = read_params(dir + "/params.txt");
        auto get = [&](const char* key, const std::string& def) {
            auto it = m.find(key);
            return it == m.end() ? def : it->second;
        };
        Params p;
        p.nX = std::stoi(get("nX", "256"));
        p.XsizeFull = std::stoi(get("XsizeFull", get("nX", "256")));
        p.nY = std::stoi(get("nY", "64"));
        p.tau = std::stod(get("tau", "1.25"));
        p.Fval = std::stod(get("Fval", "0"));
        p.MuVal = std::stod(get("MuVal", "0.1"));
        p.kOmegaSolverFlag = std::stoi(get("kOmega", "0")) != 0;
        p.maxTurbVisc = std::stod(get("maxTurbVisc", "10"));
        p.krylovDim = std::stoi(get("krylovDim", "10"));
        p.relTol = std::stod(get("relTol", "1e-4"));
        p.absTol = std::stod(get("absTol", "1e-7"));
        p.thermalSolverFlag = std::stoi(get("thermal", "0")) != 0;
        p.tempMaxRelTol = std::stod(get("tempRelTol", "1e-4"));
        p.tempMaxAbsTol = std::stod(get("tempAbsTol", "1e-7"));

        clVariablesLB vlb(p);
        const size_t n = vlb.fullSize();
        const size_t nx = (size_t)p.nX;
        // wall heights [2][nX] or [4][nX]
        auto load_walls = [&](const std::string& path, std::vector<double>* w[4]) -> bool {
            std::ifstream s(path, std::ios::binary | std::ios::ate);
            if (!s) return false;
            const size_t nd = (size_t)s.tellg() / sizeof(double);
            if (nd != 2 * nx && nd != 4 * nx) throw Error(path + ": size", KOFM_ERR_LOADING_PARAMS);
            s.seekg(0);
            for (size_t k = 0; k < 4; ++k) {
                w[k]->clear();
                if (k * nx >= nd) continue;
                w[k]->resize(nx);
                s.read(reinterpret_cast<char*>(w[k]->data()), (std::streamsize)(nx * sizeof(double)));
            }
            return true;
        };
        std::vector<double>* wv[4] = {&vlb.yBot, &vlb.yTop, &vlb.yBot0, &vlb.yTop0};
        const bool walls = load_walls(dir + "/walls.bin", wv);
        const int moveAt = std::stoi(get("moveAt", "-1"));
        if (!walls) {
        vlb.nType.resize(n);
        {
            std::ifstream s(dir + "/ntype.bin", std::ios::binary);
            s.read(reinterpret_cast<char*>(vlb.nType.data()), (std::streamsize)(n * sizeof(int16_t)));
            if (s.gcount() != (std::streamsize)(n * sizeof(int16_t)))
                throw Error("ntype.bin", KOFM_ERR_LOADING_PARAMS);
        }
        if (p.kOmegaSolverFlag || p.thermalSolverFlag) {
            vlb.dXArr.resize(4 * n);
            if (!loadBin(dir + "/dX.bin", vlb.dXArr.data(), 4 * n)) vlb.dXArr.clear();
        }
        if (p.kOmegaSolverFlag) {
            vlb.WallD.resize(n);
            if (!loadBin(dir + "/wallD.bin", vlb.WallD.data(), n)) vlb.WallD.clear();
        }
        {
            std::ifstream s(dir + "/ibbArr.bin", std::ios::binary | std::ios::ate);
            if (s) {
                const size_t nb = (size_t)s.tellg() / sizeof(int32_t);
                s.seekg(0);
                vlb.ibbArr.resize(nb);
                s.read(reinterpret_cast<char*>(vlb.ibbArr.data()), (std::streamsize)(nb * sizeof(int32_t)));
                vlb.ibbDistArr.resize(nb);
                if (!loadBin(dir + "/ibbDistArr.bin", vlb.ibbDistArr.data(), nb))
                    throw Error("ibbDistArr.bin", KOFM_ERR_LOADING_PARAMS);
            }
        }
        }
        if (!vlb.loadRestartFiles(dir)) throw Error("restart files in " + dir, KOFM_ERR_LOADING_PARAMS);
        vlb.ini();
        clVariablesFD vfd(vlb);
        if (p.thermalSolverFlag) {
            vfd.loadRestartFiles(dir);
            vfd.ini();
        }
        clProblem prob(vlb, &vfd);
        for (int t = 0; t < nsteps; ++t) {
            if (walls && t == moveAt) {
                if (!load_walls(dir + "/walls_moved.bin", wv)) throw Error("walls_moved.bin", KOFM_ERR_LOADING_PARAMS);
                vlb.update();
            }
            prob.step();
        }
        const std::string out = dir + "/out";
        mkdir(out.c_str(), 0755);
        vlb.saveRestartFiles(out);
        if (p.thermalSolverFlag) vfd.saveRestartFiles(out);
        const double rho = vlb.sumRo.reduceSingle();
        std::printf("{\"steps\": %d, \"sum_rho\": %.17g, \"umean\": %.17g", nsteps, rho, vlb.calcUmean());
        if (p.kOmegaSolverFlag)
            std::printf(", \"sum_k\": %.17g, \"sum_omega\": %.17g, \"min_k\": %.17g, \"min_omega\": %.17g, "
                        "\"steps_per_lb\": %d, \"omega_iters\": %d, \"k_iters\": %d",
                        vlb.kOmegaClass.sumKappa.reduceSingle(), vlb.kOmegaClass.sumOmega.reduceSingle(),
                        vlb.kOmegaClass.minKappa.reduceSingle(), vlb.kOmegaClass.minOmega.reduceSingle(),
                        vlb.kOmegaClass.stepsPerLB, vlb.kOmegaClass.lastOmegaIters,
                        vlb.kOmegaClass.lastKappaIters);
        if (p.thermalSolverFlag)
            std::printf(", \"sum_temp\": %.17g, \"temp_steps_per_lb\": %d, \"temp_iters\": %d",
                        vfd.calcAverageT(), vfd.stepsPerLB, vfd.lastIters);
        std::printf("}\n");
    } catch (const Error& e) {
        std::fprintf(stderr, "kofm_host_run: %s\n", e.what());
        return 1;
    }
    return 0;
}
