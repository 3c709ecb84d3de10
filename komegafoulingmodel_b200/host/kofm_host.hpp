// kofm_host.hpp - host classes with the reference's method surface for the
// LB / k-omega step, driving the B200 library through the C ABI (kofm.h).
//
//   clVariablesLB   <- clVariablesLB (clVariablesLB.h:249-441)
//   kOmega          <- kOmega (kOmega.h:222-340)
//   Reducer         <- Reducer<double,double>::reduceSingle (Reducer.h:240-278)
//   clProblem::step <- Solve_no_TR (LBLS.cpp:185-205) as called by the
//                      clProblem step loop (clProblem.cpp:104-108)
//
// The classes keep the reference's method names and call order; what the
// reference did with OpenCL buffers and kernel objects is one kofm context
// (one CUDA stream, which plays LBQUEUE).  Host arrays use the reference's
// padded FP64 layout: index i + XsizeFull*j (+ XsizeFull*nY*dir).  Errors
// throw kofm::host::Error carrying the library status instead of exit().
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "kofm.h"

namespace kofm {
namespace host {

struct Error : std::runtime_error {
    int status;
    Error(const std::string& what, int st);
};

// Throws Error if st != KOFM_OK.
void check(const char* what, int st);

// The parameters of the path that the reference reads from its YAML files
// (clVariablesLB::loadParams, kOmega::loadParams, clProblem.cpp:337-405).
struct Params {
    int nX = 256;                // channel length (p.nX)
    int XsizeFull = 256;         // padded row length (p.XsizeFull)
    int nY = 64;                 // p.nY
    double tau = 1.25;           // relaxation RATE of the collision (tau0)
    double Fval = 0.0;           // body force (FTERM_VAL)
    double MuVal = 0.1;          // laminar viscosity (MU_NUMBER)
    double maxTurbVisc = 10.0;   // MAX_TURB_VISC
    bool kOmegaSolverFlag = false;
    int krylovDim = 10;          // GMRES_KRYLOV_DIM_SIZE
    int maxIters = 1000;         // KOMEGA_MAX_ITERS
    double relTol = 1.0e-4;      // KOMEGA_MAX_REL_TOL
    double absTol = 1.0e-7;      // KOMEGA_MAX_ABS_TOL
    double dTlb = 1.0;           // p.dTlb
    // thermal solver (clVariablesFD::loadParams, clVariablesFD.cpp:444-493)
    bool thermalSolverFlag = false;  // "Thermal Solver"
    int tfdSteps = 1;                // "LB Steps Per T" (LB_STEPS_PER_FD)
    double PrNum = 0.708;            // "Pr Number"
    double PrTurbNum = 0.9;          // PR_TURB_NUMBER
    double AlphaFoul = 0.0;          // LB_ALPHA_FOUL (fouling-layer diffusivity)
    double ROE0 = 0.5;               // "Tinitial" (TFD_INI_TEMP)
    double ROE_INX = 2.0;            // "Tinlet Sim" (TFD_X_IN)
    int tempMaxIters = 1000;         // "Temp Max Iterations"
    double tempMaxRelTol = 1.0e-4;   // "Temp Max Rel Tol"
    double tempMaxAbsTol = 1.0e-7;   // "Temp Max Abs Tol"
    int storage = KOFM_STORE_FP32;
    int device = 0;
};

class Reducer {
  public:
    Reducer(kofm_ctx* const* ctx, int field, int op) : ctx_(ctx), field_(field), op_(op) {}
    double reduceSingle() const;

  private:
    kofm_ctx* const* ctx_;
    int field_, op_;
};

class clVariablesLB;

class kOmega {
  public:
    explicit kOmega(clVariablesLB& lb);
    bool kOmegaSolverFlag = false;
    // kOmega.cpp:315-318
    Reducer sumKappa, sumOmega, minKappa, minOmega;
    // kOmega's time-stepping state, refreshed after every Solve()
    int stepsPerLB = 1;
    int timeSinceTimeStepChange = 0;
    double timeStep = 1.0;
    int lastOmegaIters = 0, lastKappaIters = 0;

    // kOmega::setInitialValues (kOmega.cpp:530-570): host arrays of k, omega
    // and nu_t (nu_t may be null); uploaded with the populations by
    // clVariablesLB::ini.
    void setInitialValues(const double* kappa, const double* omega, const double* nut);
    // kOmega::Solve (kOmega.cpp:31-73)
    void Solve();
    // kOmega::saveRestartFiles (kOmega.cpp:492): dir/lbkappa.bin, dir/lbomega.bin
    void saveRestartFiles(const std::string& dir) const;
    // the lbkappa / lbomega loads of kOmega::loadParams (kOmega.cpp:685-710)
    bool loadRestartFiles(const std::string& dir);

    // Sxy_array: the 3 strain-rate planes of the previous step (zero at a
    // start or restart, as the reference's zero-initialised buffer)
    std::vector<double> Kappa_array, Omega_array, Nut_array, Sxy_array;

  private:
    clVariablesLB& lb_;
};

class clVariablesLB {
  public:
    explicit clVariablesLB(const Params& p);
    ~clVariablesLB();
    clVariablesLB(const clVariablesLB&) = delete;
    clVariablesLB& operator=(const clVariablesLB&) = delete;

    Params p;
    kofm_ctx* ctx = nullptr;
    kOmega kOmegaClass;
    // clVariablesLB.cpp:343-345
    Reducer sumUx, sumUy, sumRo;
    int alter = 0;               // FA/FB alternation parity of the reference
    long long TimeN = 0;

    // Geometry of the channel (the arrays clVariablesLS and kOmega::iniWallD
    // produce): nType flags, wall distance and link fractions (4 planes
    // E,W,N,S; may be empty), interpolated bounce-back links.
    std::vector<int16_t> nType;
    std::vector<double> WallD, dXArr;
    std::vector<int32_t> ibbArr;
    std::vector<double> ibbDistArr;

    // Walls as heights per column (the polylines of clVariablesLS, through
    // (x, y_w[x])): when yBot / yTop are set, ini() builds the geometry above
    // on the device (kofm_set_walls) and copies it back; yBot0 / yTop0 are the
    // unfouled walls (empty: the same).  "Min dX Dist", "Wall D Search Rad".
    std::vector<double> yBot, yTop, yBot0, yTop0;
    double minDxDist = 0.001;
    int wallDSearchRad = 50;

    // Populations FA (9 planes) on the host
    std::vector<double> FA;

    // clVariablesLB::calcFeqVals (clVariablesLB.cpp:77-117)
    static void calcFeqVals(double* Feq_vals, double rho_val, double ux, double uy);
    // clVariablesLB::iniDists: weights (rest) on every node
    void iniDists();
    // clVariablesLB::iniDistsFromVel: equilibrium of given velocity planes
    void iniDistsFromVel(const double* ux, const double* uy);
    // clVariablesLB::ini: creates the device context and uploads geometry
    // and state (allocateBuffers + setKernelArgs of the reference)
    void ini();
    // clVariablesLB::Solve (clVariablesLB.h:375-441): collide + IBB, then
    // kOmegaClass.Solve() when the k-omega solver is on
    void Solve(int option = KOFM_OPTION_SAVE_MACRO_FIELDS);
    // clVariablesLB::calcUmean (clVariablesLB.cpp:122-125)
    double calcUmean() const;
    // clVariablesLB::getInitialFlow (clVariablesLB.cpp:170-232): nsteps of
    // Solve() with the progress print every `printEvery` steps
    void getInitialFlow(int nsteps, int printEvery = 1000);
    // clVariablesLB::saveRestartFiles (clVariablesLB.cpp:752-765):
    // dir/lbf.bin (+ k-omega files)
    void saveRestartFiles(const std::string& dir);
    // the lbf.bin load of clVariablesLB::loadParams (applied by ini())
    bool loadRestartFiles(const std::string& dir);
    // device -> host copies of the state (FA, k, omega, nu_t)
    void downloadState();
    // clVariablesLS::update + clVariablesLB::update (clVariablesLS.cpp:
    // 1020-1033, clVariablesLB.cpp:905-913): after the walls moved (yBot ...
    // changed), rebuilds flags, link fractions, interpolated links and wall
    // distance on the live context; nodes turned solid lose k, omega, nu_t
    void update();

    size_t fullSize() const { return (size_t)p.XsizeFull * (size_t)p.nY; }
};

// The thermal solver of the reference (clVariablesFD.h:20-452): the
// temperature field and its implicit finite-difference update over the
// context that clVariablesLB::ini created (Params::thermalSolverFlag on).
class clVariablesFD {
  public:
    explicit clVariablesFD(clVariablesLB& vlb);
    bool thermalSolverFlag = false;
    int stepsPerLB = 1, timeSinceTimeStepChange = 0;
    double timeStep = 1.0;
    int lastIters = 0;
    std::vector<double> tempArray;   // XsizeFull * nY, FP64
    std::vector<double> dXArr0;      // unfouled link fractions (may be empty)
    Reducer sumTemp;                 // clVariablesFD.cpp:266

    // clVariablesFD::ini (clVariablesFD.cpp:230-280): Tinitial everywhere
    // unless a temperature was loaded, then the upload
    void ini();
    // clVariablesFD::Solve (clVariablesFD.h:343-358)
    void Solve();
    // clVariablesFD::calcAverageT (clVariablesFD.cpp:139-142): the sum
    double calcAverageT() const { return sumTemp.reduceSingle(); }
    // dir/temp.bin (the "load/temp" file testRestartRun reads)
    void saveRestartFiles(const std::string& dir);
    bool loadRestartFiles(const std::string& dir);

  private:
    clVariablesLB& lb_;
};

// One time step of the reference's step loop without particles:
// Solve_no_TR (LBLS.cpp:185-205): collide + IBB, kOmega::Solve, and
// vfd.Solve() every tfdSteps steps when a thermal solver is attached.
class clProblem {
  public:
    explicit clProblem(clVariablesLB& vlb, clVariablesFD* vfd = nullptr) : vlb_(vlb), vfd_(vfd) {}
    void step();
    void Solve_no_TR() { step(); }

  private:
    clVariablesLB& vlb_;
    clVariablesFD* vfd_;
};

// Raw binary array files as Array::savebin writes them (Array.h:1178-1193).
bool saveBin(const std::string& path, const double* data, size_t n);
bool loadBin(const std::string& path, double* data, size_t n);

}  // namespace host
}  // namespace kofm
