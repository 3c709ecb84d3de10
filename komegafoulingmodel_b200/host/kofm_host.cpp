// kofm_host.cpp - the host classes of kofm_host.hpp over the C ABI.
#include "kofm_host.hpp"

#include <cstdio>
#include <fstream>

namespace kofm {
namespace host {

Error::Error(const std::string& what, int st)
    : std::runtime_error(what + ": " + kofm_error_string(st)), status(st) {}

void check(const char* what, int st) {
    if (st != KOFM_OK) throw Error(what, st);
}

namespace {
// D2Q9 order of the reference (Heading.cl): C, E, W, N, S, NE, SW, SE, NW
constexpr int CX[9] = {0, 1, -1, 0, 0, 1, -1, 1, -1};
constexpr int CY[9] = {0, 0, 0, 1, -1, 1, -1, -1, 1};

// one-dimensional factor of the product-form equilibrium
double phi(int c, double u) {
    return c == 0 ? 2.0 / 3.0 - u * u : 0.5 * (1.0 / 3.0 + c * u + u * u);
}
}  // namespace

bool saveBin(const std::string& path, const double* data, size_t n) {
    std::ofstream s(path, std::ios::binary | std::ios::trunc);
    if (!s) return false;
    s.write(reinterpret_cast<const char*>(data), (std::streamsize)(n * sizeof(double)));
    return (bool)s;
}

bool loadBin(const std::string& path, double* data, size_t n) {
    std::ifstream s(path, std::ios::binary);
    if (!s) return false;
    s.read(reinterpret_cast<char*>(data), (std::streamsize)(n * sizeof(double)));
    return s.gcount() == (std::streamsize)(n * sizeof(double));
}

double Reducer::reduceSingle() const {
    double out = 0.0;
    check("Reducer::reduceSingle", kofm_reduce(*ctx_, field_, op_, &out));
    return out;
}

// ---- kOmega ---------------------------------------------------------------------
kOmega::kOmega(clVariablesLB& lb)
    : sumKappa(&lb.ctx, KOFM_FIELD_K, KOFM_OP_SUM),
      sumOmega(&lb.ctx, KOFM_FIELD_OMEGA, KOFM_OP_SUM),
      minKappa(&lb.ctx, KOFM_FIELD_K, KOFM_OP_MIN),
      minOmega(&lb.ctx, KOFM_FIELD_OMEGA, KOFM_OP_MIN),
      lb_(lb) {}

void kOmega::setInitialValues(const double* kappa, const double* omega, const double* nut) {
    const size_t n = lb_.fullSize();
    Kappa_array.assign(kappa, kappa + n);
    Omega_array.assign(omega, omega + n);
    if (nut) Nut_array.assign(nut, nut + n);
    else Nut_array.clear();
}

void kOmega::Solve() {
    check("kOmega::Solve", kofm_komega_update(lb_.ctx));
    kofm_stats st;
    check("kOmega::Solve stats", kofm_get_stats(lb_.ctx, &st));
    stepsPerLB = st.steps_per_lb;
    timeSinceTimeStepChange = st.time_since_change;
    timeStep = st.dt;
    lastOmegaIters = st.omega_iters;
    lastKappaIters = st.k_iters;
}

void kOmega::saveRestartFiles(const std::string& dir) const {
    const size_t n = lb_.fullSize();
    if (!saveBin(dir + "/lbkappa.bin", Kappa_array.data(), n) ||
        !saveBin(dir + "/lbomega.bin", Omega_array.data(), n))
        throw Error("kOmega::saveRestartFiles " + dir, KOFM_ERR_INVALID_ARG);
}

bool kOmega::loadRestartFiles(const std::string& dir) {
    const size_t n = lb_.fullSize();
    Kappa_array.resize(n);
    Omega_array.resize(n);
    return loadBin(dir + "/lbkappa.bin", Kappa_array.data(), n) &&
           loadBin(dir + "/lbomega.bin", Omega_array.data(), n);
}

// ---- clVariablesLB ----------------------------------------------------------------
clVariablesLB::clVariablesLB(const Params& prm)
    : p(prm),
      kOmegaClass(*this),
      sumUx(&ctx, KOFM_FIELD_UX, KOFM_OP_SUM),
      sumUy(&ctx, KOFM_FIELD_UY, KOFM_OP_SUM),
      sumRo(&ctx, KOFM_FIELD_RHO, KOFM_OP_SUM) {
    kOmegaClass.kOmegaSolverFlag = p.kOmegaSolverFlag;
}

clVariablesLB::~clVariablesLB() {
    if (ctx) kofm_destroy(ctx);
}

void clVariablesLB::calcFeqVals(double* Feq_vals, double rho_val, double ux, double uy) {
    for (int i = 0; i < 9; ++i) Feq_vals[i] = rho_val * phi(CX[i], ux) * phi(CY[i], uy);
}

void clVariablesLB::iniDists() {
    const size_t n = fullSize();
    double w[9];
    calcFeqVals(w, 1.0, 0.0, 0.0);
    FA.assign(9 * n, 0.0);
    for (int i = 0; i < 9; ++i)
        for (size_t g = 0; g < n; ++g) FA[i * n + g] = w[i];
}

void clVariablesLB::iniDistsFromVel(const double* ux, const double* uy) {
    const size_t n = fullSize();
    FA.assign(9 * n, 0.0);
    double f[9];
    for (size_t g = 0; g < n; ++g) {
        calcFeqVals(f, 1.0, ux ? ux[g] : 0.0, uy ? uy[g] : 0.0);
        for (int i = 0; i < 9; ++i) FA[i * n + g] = f[i];
    }
}

// kofm_set_walls with this object's walls, then the geometry back into nType,
// WallD, dXArr and the interpolated-link lists
static void set_walls_and_fetch(clVariablesLB& lb) {
    const size_t nx = (size_t)lb.p.nX, n = lb.fullSize();
    if (lb.yBot.size() != nx || lb.yTop.size() != nx ||
        (!lb.yBot0.empty() && lb.yBot0.size() != nx) || (!lb.yTop0.empty() && lb.yTop0.size() != nx))
        throw Error("clVariablesLB: wall heights need one value per column", KOFM_ERR_INVALID_ARG);
    check("clVariablesLB (kofm_set_walls)",
          kofm_set_walls(lb.ctx, lb.yBot.data(), lb.yTop.data(), lb.yBot0.empty() ? nullptr : lb.yBot0.data(),
                         lb.yTop0.empty() ? nullptr : lb.yTop0.data(), lb.minDxDist, lb.wallDSearchRad, 0));
    int32_t nl = 0;
    check("kofm_get_geometry", kofm_get_geometry(lb.ctx, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, 0, &nl));
    lb.nType.resize(n);
    lb.dXArr.resize(4 * n);
    lb.ibbArr.resize((size_t)nl);
    lb.ibbDistArr.resize((size_t)nl);
    if (lb.p.kOmegaSolverFlag) lb.WallD.resize(n);
    check("kofm_get_geometry",
          kofm_get_geometry(lb.ctx, lb.nType.data(), lb.p.kOmegaSolverFlag ? lb.WallD.data() : nullptr,
                            lb.dXArr.data(), nullptr, lb.ibbArr.data(), lb.ibbDistArr.data(), nl, &nl));
}

void clVariablesLB::update() {
    if (!ctx) throw Error("clVariablesLB::update before ini", KOFM_ERR_STATE);
    set_walls_and_fetch(*this);
}

void clVariablesLB::ini() {
    const size_t n = fullSize();
    const bool walls = !yBot.empty();
    if (!walls && nType.size() != n) throw Error("clVariablesLB::ini: nType size", KOFM_ERR_INVALID_ARG);
    kofm_desc d;
    check("kofm_desc_default", kofm_desc_default(&d));
    d.nx = p.nX;
    d.nx_full = p.XsizeFull;
    d.ny = p.nY;
    d.use_komega = p.kOmegaSolverFlag ? 1 : 0;
    d.tau = p.tau;
    d.fterm = p.Fval;
    d.mu = p.MuVal;
    d.max_turb_visc = p.maxTurbVisc;
    d.storage = p.storage;
    d.device = p.device;
    d.komega_max_iters = p.maxIters;
    d.krylov_dim = p.krylovDim;
    d.komega_rel_tol = p.relTol;
    d.komega_abs_tol = p.absTol;
    d.komega_dt = p.dTlb;
    d.use_thermal = p.thermalSolverFlag ? 1 : 0;
    d.thermal_every = p.tfdSteps;
    d.pr_number = p.PrNum;
    d.pr_turb_number = p.PrTurbNum;
    d.alpha_foul = p.AlphaFoul;
    d.t_in = p.ROE_INX;
    d.thermal_max_iters = p.tempMaxIters;
    d.thermal_rel_tol = p.tempMaxRelTol;
    d.thermal_abs_tol = p.tempMaxAbsTol;
    d.thermal_dt = (double)p.tfdSteps;  // dTtfd (clProblem.cpp:510)
    if (ctx) {
        kofm_destroy(ctx);
        ctx = nullptr;
    }
    check("clVariablesLB::ini (kofm_create)", kofm_create(&d, &ctx));
    const bool ko = p.kOmegaSolverFlag;
    const bool th = p.thermalSolverFlag;
    if (walls) {
        set_walls_and_fetch(*this);
    } else {
        if (ko && WallD.size() != n)
            throw Error("clVariablesLB::ini: WallD missing", KOFM_ERR_INITIALIZING_KOMEGA);
        // link fractions default to whole links (dXArr = 1, no wall cut)
        if ((ko || th) && dXArr.size() != 4 * n) dXArr.assign(4 * n, 1.0);
        check("clVariablesLB::ini (geometry)",
              kofm_set_geometry(ctx, nType.data(), ko && !WallD.empty() ? WallD.data() : nullptr,
                                (ko || th) && !dXArr.empty() ? dXArr.data() : nullptr,
                                ibbArr.empty() ? nullptr : ibbArr.data(),
                                ibbDistArr.empty() ? nullptr : ibbDistArr.data(),
                                (int32_t)ibbArr.size()));
    }
    if (FA.size() != 9 * n) iniDists();
    kOmega& K = kOmegaClass;
    if (ko && (K.Kappa_array.size() != n || K.Omega_array.size() != n))
        throw Error("clVariablesLB::ini: k-omega initial values missing", KOFM_ERR_INITIALIZING_KOMEGA);
    if (ko && K.Sxy_array.size() != 3 * n) K.Sxy_array.assign(3 * n, 0.0);
    check("clVariablesLB::ini (state)",
          kofm_set_state(ctx, FA.data(), ko ? K.Kappa_array.data() : nullptr,
                         ko ? K.Omega_array.data() : nullptr,
                         ko && K.Nut_array.size() == n ? K.Nut_array.data() : nullptr,
                         ko ? K.Sxy_array.data() : nullptr));
    alter = 0;
    TimeN = 0;
}

void clVariablesLB::Solve(int option) {
    check("clVariablesLB::Solve (collide)",
          kofm_lb_step(ctx, p.kOmegaSolverFlag ? (option | KOFM_OPTION_SAVE_MACRO_FIELDS) : option));
    alter ^= 1;
    if (kOmegaClass.kOmegaSolverFlag) kOmegaClass.Solve();
    else check("clVariablesLB::Solve (finish)", kofm_sync(ctx));
    ++TimeN;
}

double clVariablesLB::calcUmean() const { return sumUx.reduceSingle() / sumRo.reduceSingle(); }

void clVariablesLB::getInitialFlow(int nsteps, int printEvery) {
    for (int t = 1; t <= nsteps; ++t) {
        Solve(KOFM_OPTION_SAVE_MACRO_FIELDS);
        if (printEvery > 0 && t % printEvery == 0) {
            const double rho = sumRo.reduceSingle();
            const double ux = sumUx.reduceSingle() / rho;
            if (kOmegaClass.kOmegaSolverFlag) {
                std::printf("Time = %d, Umean = %g, K = %g, Omega = %g\n", t, ux,
                            kOmegaClass.sumKappa.reduceSingle() / rho,
                            kOmegaClass.sumOmega.reduceSingle() / rho);
                const double kmin = kOmegaClass.minKappa.reduceSingle();
                const double omin = kOmegaClass.minOmega.reduceSingle();
                if (omin < 0.) std::printf("warning: omega contains negative values of %g\n", omin);
                if (kmin < 0.) std::printf("warning: kappa contains negative values of %g\n", kmin);
            } else {
                std::printf("Time = %d, Umean = %g\n", t, ux);
            }
        }
    }
}

void clVariablesLB::downloadState() {
    const size_t n = fullSize();
    FA.resize(9 * n);
    kOmega& K = kOmegaClass;
    if (p.kOmegaSolverFlag) {
        K.Kappa_array.resize(n);
        K.Omega_array.resize(n);
        K.Nut_array.resize(n);
    }
    check("clVariablesLB::downloadState",
          kofm_get_state(ctx, FA.data(), p.kOmegaSolverFlag ? K.Kappa_array.data() : nullptr,
                         p.kOmegaSolverFlag ? K.Omega_array.data() : nullptr,
                         p.kOmegaSolverFlag ? K.Nut_array.data() : nullptr, nullptr));
}

void clVariablesLB::saveRestartFiles(const std::string& dir) {
    downloadState();
    if (!saveBin(dir + "/lbf.bin", FA.data(), FA.size()))
        throw Error("clVariablesLB::saveRestartFiles " + dir, KOFM_ERR_INVALID_ARG);
    if (kOmegaClass.kOmegaSolverFlag) kOmegaClass.saveRestartFiles(dir);
}

bool clVariablesLB::loadRestartFiles(const std::string& dir) {
    const size_t n = fullSize();
    FA.resize(9 * n);
    if (!loadBin(dir + "/lbf.bin", FA.data(), FA.size())) return false;
    if (kOmegaClass.kOmegaSolverFlag && !kOmegaClass.loadRestartFiles(dir)) return false;
    return true;
}

// ---- clProblem ----------------------------------------------------------------
void clProblem::step() {
    // collide + IBB, then kOmega::Solve (which ends with the queue drained)
    const long long timeN = vlb_.TimeN;
    vlb_.Solve(KOFM_OPTION_SAVE_MACRO_FIELDS);
    if (vfd_ && vfd_->thermalSolverFlag && timeN % vlb_.p.tfdSteps == 0) vfd_->Solve();
}

clVariablesFD::clVariablesFD(clVariablesLB& vlb)
    : thermalSolverFlag(vlb.p.thermalSolverFlag), sumTemp(&vlb.ctx, KOFM_FIELD_TEMP, KOFM_OP_SUM), lb_(vlb) {}

void clVariablesFD::ini() {
    if (!thermalSolverFlag) return;
    if (!lb_.ctx) throw Error("clVariablesFD::ini: clVariablesLB::ini first", KOFM_ERR_STATE);
    const size_t n = lb_.fullSize();
    if (tempArray.size() != n) tempArray.assign(n, lb_.p.ROE0);
    if (!dXArr0.empty()) {
        if (dXArr0.size() != 4 * n) throw Error("clVariablesFD::ini: dXArr0 size", KOFM_ERR_INVALID_ARG);
        check("clVariablesFD::ini (dXArr0)", kofm_set_thermal_geometry(lb_.ctx, dXArr0.data()));
    }
    check("clVariablesFD::ini (temperature)", kofm_set_temperature(lb_.ctx, tempArray.data()));
}

void clVariablesFD::Solve() {
    check("clVariablesFD::Solve", kofm_thermal_update(lb_.ctx));
    kofm_stats st;
    check("kofm_get_stats", kofm_get_stats(lb_.ctx, &st));
    stepsPerLB = st.thermal_steps_per_lb;
    timeSinceTimeStepChange = st.thermal_time_since_change;
    timeStep = st.thermal_dt;
    lastIters = st.thermal_iters;
}

void clVariablesFD::saveRestartFiles(const std::string& dir) {
    const size_t n = lb_.fullSize();
    tempArray.resize(n);
    check("kofm_get_temperature", kofm_get_temperature(lb_.ctx, tempArray.data()));
    if (!saveBin(dir + "/temp.bin", tempArray.data(), n))
        throw Error("clVariablesFD::saveRestartFiles", KOFM_ERR_MEMORY_COPY);
}

bool clVariablesFD::loadRestartFiles(const std::string& dir) {
    const size_t n = lb_.fullSize();
    std::vector<double> t(n);
    if (!loadBin(dir + "/temp.bin", t.data(), n)) return false;
    tempArray.swap(t);
    return true;
}

}  // namespace host
}  // namespace kofm
