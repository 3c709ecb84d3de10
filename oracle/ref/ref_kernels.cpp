// CPU build of the reference's own LB and k-omega kernels (checker only).
//
// oracle/Makefile preprocesses source/Kernels/{Heading,lbKernels,kOmegaKernels}.cl
// of the reference into oracle/_ref/gen/*.inc (vector literals such as
// "(double2)(a, b)" become "make_double2(a, b)"), and this file includes them
// inside `struct RefProgram`.  Each extern "C" entry point below runs one
// reference kernel over the same NDRange the reference host code enqueues:
//   collide kernels, Calc_Ro_J, the k-omega kernels: XsizeFull x nY work-items
//     (clVariablesLB.cpp:141-144, kOmega.cpp:119-125);
//   lbIBB: one work-item per IBB link (clVariablesLB.cpp:841-852).
// The kernels contain no barriers and no local memory, so a serial/OpenMP loop
// over (gx, gy) is an exact execution; the push-stream writes every output
// slot from exactly one work-item, so row-parallel OpenMP is race-free.
#include "cl_shim.hpp"
#include <cstdio>
#include <vector>

thread_local size_t g_ref_gid[3];

#define __kernel
#define __global
#define __local
#define __constant
#define constant
#define new new_
#undef RAND_MAX
#undef MAX
#undef MIN

// Program-build-time defines of the reference, as run-time members.
#define CHANNEL_LENGTH m_nx
#define CHANNEL_LENGTH_FULL m_nxf
#define CHANNEL_HEIGHT m_ny
#define DIST_SIZE m_dist
#define NTYPE_TYPE short
#define tau0 m_tau0
#define FTERM_VAL m_fterm
#define MU_NUMBER m_mu
#define MAX_TURB_VISC m_maxnut
#define LSC_NN m_lscnn
#define WALLD_SEARCH_RADIUS m_wallsr
// Define set used by the reference's default build (ConstDef.h:25 DEBUG_TURBARR
// -> DEBUG_ARRAYS via kOmega.cpp:662-664; USE_TURB_VEL_BC via
// clVariablesLB.cpp:868-871 with the default turbVelBCFlag = true).
#define DEBUG_ARRAYS
#define OPENCL_VERSION_1_2
#define USE_TURB_VEL_BC
#define WORKGROUPSIZE_IBB 256
// Particle-module defines referenced by helper functions in Heading.cl that
// the LB/k-omega path never calls.
#define TR_X_IND_START 0
#define FULLSIZEX_TR_PADDED 1
#define NUM_BL_BOT 0
#define BL_BOT_START 0
#define BL_TOP_START 0
#define BL_TOP_STOP 0
#define BL_BOT_STOP 0

#pragma GCC diagnostic push
#pragma GCC diagnostic ignored "-Wattributes"
#pragma GCC diagnostic ignored "-Wunknown-pragmas"
#pragma GCC diagnostic ignored "-Wunused-variable"
#pragma GCC diagnostic ignored "-Wunused-but-set-variable"
#pragma GCC diagnostic ignored "-Wsign-compare"

struct RefProgram {
    int m_nx, m_nxf, m_ny, m_dist;
    double m_tau0, m_fterm, m_mu, m_maxnut;
    int m_lscnn, m_wallsr;

    RefProgram(int nx, int nxf, int ny, double tau, double fterm, double mu,
               double maxnut, int lscnn, int wallsr)
        : m_nx(nx), m_nxf(nxf), m_ny(ny), m_dist(nxf * ny), m_tau0(tau),
          m_fterm(fterm), m_mu(mu), m_maxnut(maxnut), m_lscnn(lscnn),
          m_wallsr(wallsr) {}

#include "../_ref/gen/Heading.inc"
#include "../_ref/gen/lbKernels.inc"
#include "../_ref/gen/kOmegaKernels.inc"
#define SHEAR_CUTOFF_RADIUS m_cutoff
    double m_cutoff = 5.0;
#include "../_ref/gen/shear.inc"
#undef SHEAR_CUTOFF_RADIUS
// thermal program defines (clVariablesFD::setSourceDefines,
// clVariablesFD.cpp:684-698); the k-omega build adds USING_KOMEGA_SOLVER
#define LB_ALPHA_FLUID m_alpha_fluid
#define LB_ALPHA_FOUL m_alpha_foul
#define PR_TURB_NUMBER_INV m_prt_inv
#define TFD_X_IN_VAL m_tin
#define USING_KOMEGA_SOLVER
    double m_alpha_fluid = 0.0, m_alpha_foul = 0.0, m_prt_inv = 1.0, m_tin = 0.0;
#include "../_ref/gen/thermal.inc"
// level-set module: the polyline has LSC_UPDATE_M_NN + 1 points, the
// segment LSC_UPDATE_M_SKIP (bottom wall end -> top wall start) is not a
// wall (clVariablesLS.cpp:464-466)
#define LSC_UPDATE_M_NN m_lsc_nn1
#define LSC_UPDATE_M_SKIP m_lsc_skip
    int m_lsc_nn1 = 0, m_lsc_skip = -1;
#include "../_ref/gen/ls.inc"
#undef LSC_UPDATE_M_NN
#undef LSC_UPDATE_M_SKIP
#undef USING_KOMEGA_SOLVER
#undef LB_ALPHA_FLUID
#undef LB_ALPHA_FOUL
#undef PR_TURB_NUMBER_INV
#undef TFD_X_IN_VAL
};

#pragma GCC diagnostic pop
#undef new

struct RefCfg {
    int nx, nxf, ny;
    double tau0, fterm, mu, max_turb_visc;
};

static RefProgram make_prog(const RefCfg* c) {
    return RefProgram(c->nx, c->nxf, c->ny, c->tau0, c->fterm, c->mu,
                      c->max_turb_visc, 0, 50);
}

// 2-D NDRange XsizeFull x nY, rows in parallel.
template <class F>
static void ndrange2d(int gx_size, int gy_size, F&& body) {
#pragma omp parallel for schedule(static)
    for (int gy = 0; gy < gy_size; ++gy) {
        for (int gx = 0; gx < gx_size; ++gx) {
            g_ref_gid[0] = (size_t)gx;
            g_ref_gid[1] = (size_t)gy;
            g_ref_gid[2] = 0;
            body();
        }
    }
}

extern "C" {

// LB_collision_SRT_Fluid_w_kOmega (lbKernels.cl:345-633), USE_TURB_VEL_BC
// signature (the two extra arguments are unused by the kernel body).
int ref_collide_komega(const RefCfg* c, double* rho, double* ux, double* uy,
                       double* FA, double* FB, short* map, double* wallD,
                       double* nut, double* K, double* O, double* Sxy,
                       int options) {
    RefProgram p = make_prog(c);
    ndrange2d(c->nxf, c->ny, [&] {
        p.LB_collision_SRT_Fluid_w_kOmega(rho, ux, uy, FA, FB, map, wallD, nut,
                                          K, O, Sxy, nullptr, nullptr, options);
    });
    return 0;
}

// LB_collision_SRT_Fluid (lbKernels.cl:175-335).
int ref_collide_laminar(const RefCfg* c, double* rho, double* ux, double* uy,
                        double* FA, double* FB, short* map, int options) {
    RefProgram p = make_prog(c);
    ndrange2d(c->nxf, c->ny, [&] {
        p.LB_collision_SRT_Fluid(rho, ux, uy, FA, FB, map, options);
    });
    return 0;
}

// lbIBB (lbKernels.cl:640-668): one work-item per link, run in list order.
int ref_ibb(const RefCfg* c, int* ibbArr, double* distArr, double* FB, int n) {
    RefProgram p = make_prog(c);
    for (int i = 0; i < n; ++i) {
        g_ref_gid[0] = (size_t)i; g_ref_gid[1] = 0; g_ref_gid[2] = 0;
        p.lbIBB(ibbArr, distArr, FB, n);
    }
    return 0;
}

// Calc_Ro_J (lbKernels.cl:137-164).  The kernel adds one to get_global_id(1);
// rows 1..nY-1 are visited here (row nY-1 is solid and returns at once), which
// keeps every access inside the nX_full x nY arrays.
int ref_calc_ro_j(const RefCfg* c, double* rho, double* ux, double* uy,
                  double* F, short* map) {
    RefProgram p = make_prog(c);
    ndrange2d(c->nxf, c->ny - 1, [&] { p.Calc_Ro_J(rho, ux, uy, F, map); });
    return 0;
}

// Update_kOmega_Diffusivities (kOmegaKernels.cl:7-95).
int ref_komega_diffusivities(const RefCfg* c, short* map, double* K, double* O,
                             double* nut, double* wallD, double* Dk, double* Do,
                             double* F1, double* dkdxy, double* rho,
                             double* dX, double* dbg) {
    RefProgram p = make_prog(c);
    ndrange2d(c->nxf, c->ny, [&] {
        p.Update_kOmega_Diffusivities(map, K, O, nut, wallD, Dk, Do, F1, dkdxy,
                                      rho, dX, dbg);
    });
    return 0;
}

// Update_kOmega_Coeffs_Implicit (kOmegaKernels.cl:187-480).
int ref_komega_coeffs(const RefCfg* c, int* ind, double* K, double* O,
                      double* nut, double* Dk, double* Do, double* F1,
                      double* dkdo, double* Sxy, double* rho, double* ux,
                      double* uy, double* kA, double* oA, double* kb,
                      double* ob, double* dX, double* wallD, short* map,
                      double dt, double* dbg) {
    RefProgram p = make_prog(c);
    ndrange2d(c->nxf, c->ny, [&] {
        p.Update_kOmega_Coeffs_Implicit(ind, K, O, nut, Dk, Do, F1, dkdo, Sxy,
                                        rho, ux, uy, kA, oA, kb, ob, dX, wallD,
                                        nullptr, nullptr, map, dt, dbg);
    });
    return 0;
}

// TR_shear_1 (trKernelsShear.cl:175-222) over n shear nodes.
int ref_wall_shear_nodes(const RefCfg* c, double* rho, double* ux, double* uy, double* cfss,
                         double* FA, double* tau, int* nodes, double* nut, int n) {
    RefProgram p = make_prog(c);
    for (int i = 0; i < n; ++i) {
        g_ref_gid[0] = (size_t)i; g_ref_gid[1] = 0; g_ref_gid[2] = 0;
        double8 scratch[1];
        p.TR_shear_1(rho, ux, uy, reinterpret_cast<double8*>(cfss), FA, tau, nodes, nut, n, scratch);
    }
    return 0;
}

// TR_Find_Shear_Coeffs1 (trKernelsShear.cl:333-375) over n shear nodes.
int ref_shear_coeffs1(const RefCfg* c, int* nodes, short* map, double* cfss, int n, double cutoff) {
    RefProgram p = make_prog(c);
    p.m_cutoff = cutoff;
    for (int i = 0; i < n; ++i) {
        g_ref_gid[0] = (size_t)i; g_ref_gid[1] = 0; g_ref_gid[2] = 0;
        p.TR_Find_Shear_Coeffs1(nodes, map, cfss, n);
    }
    return 0;
}

// Update_T_Coeffs_Implicit (tfdKernels.cl:122-279) over XsizeFull x nY.
int ref_thermal_coeffs(const RefCfg* c, const double* th4, int* ind, short* map, double* dX0,
                       double* A, double* b, double* T, double* ux, double* uy, double* nut,
                       double dt) {
    RefProgram p = make_prog(c);
    p.m_alpha_fluid = th4[0]; p.m_alpha_foul = th4[1]; p.m_prt_inv = th4[2]; p.m_tin = th4[3];
    ndrange2d(c->nxf, c->ny, [&] {
        p.Update_T_Coeffs_Implicit(ind, map, dX0, A, b, T, nullptr, ux, uy, nut, dt);
    });
    return 0;
}

// updateIBBOnly (lsKernels.cl:428-492): one work-item per polyline segment
// i = 0 .. npts-2 (clVariablesLS.cpp:1085-1110), run in segment order.  C2
// holds the points (x, y) of the bottom wall left to right, then of the top
// wall right to left; writes up to cap links (population index, wall
// fraction) and returns the number the builder found in *count.
int ref_update_ibb_only(const RefCfg* c, const double* C2, int npts, short* map, int* ibb,
                        double* dist, int cap, int* count) {
    RefProgram p = make_prog(c);
    p.m_lsc_nn1 = npts - 1;
    p.m_lsc_skip = npts / 2 - 1;
    std::vector<double2> C((size_t)npts);
    for (int i = 0; i < npts; ++i) C[(size_t)i] = double2(C2[2 * i], C2[2 * i + 1]);
    int cnt = 0;
    for (int i = 0; i < npts - 1; ++i) {
        g_ref_gid[0] = (size_t)i; g_ref_gid[1] = 0; g_ref_gid[2] = 0;
        p.updateIBBOnly(C.data(), map, ibb, dist, &cnt, cap);
    }
    *count = cnt;
    return 0;
}

// updateNodeBoundaryInfo (lsKernels.cl:511-583) over nX x nY, in place:
// recomputes the per-direction wall bits and SOLID_BOUNDARY from the
// M_SOLID / M_FLUID bits, which it does not change (so the serial in-place
// run equals the reference's parallel one).
int ref_update_node_boundary_info(const RefCfg* c, short* map) {
    RefProgram p = make_prog(c);
    for (int gy = 0; gy < c->ny; ++gy)
        for (int gx = 0; gx < c->nx; ++gx) {
            g_ref_gid[0] = (size_t)gx; g_ref_gid[1] = (size_t)gy; g_ref_gid[2] = 0;
            p.updateNodeBoundaryInfo(map);
        }
    return 0;
}

// updateWallD (kOmegaKernels.cl:813-840) over nX x nY: the distance of each
// fluid node to the wall segments within WALLD_SEARCH_RADIUS of the column's
// segment (lsMap, clVariablesLS.cpp:895-918).  C2 as ref_update_ibb_only;
// lsmap [2][nxf] (bottom, top segment index of each column).
int ref_update_walld(const RefCfg* c, const double* C2, int npts, unsigned short* lsmap, short* map,
                     double* wallD, int radius) {
    RefProgram p(c->nx, c->nxf, c->ny, c->tau0, c->fterm, c->mu, c->max_turb_visc, npts, radius);
    std::vector<double2> C((size_t)npts);
    for (int i = 0; i < npts; ++i) C[(size_t)i] = double2(C2[2 * i], C2[2 * i + 1]);
    ndrange2d(c->nxf, c->ny, [&] { p.updateWallD(wallD, lsmap, C.data(), map); });
    return 0;
}

}  // extern "C"

// clVariablesLS::iniLSMap (clVariablesLS.cpp:893-918, host code) over the
// arrays it reads: the points C0, the segment table BL (point pairs) and the
// map lsMap(column, wall); writes outside the map go to a sink.
struct LsMapShim {
    typedef unsigned short cl_ushort;
    struct Params { int nX; } p;
    int nBL = 0, nxf = 0;
    const double* pts = nullptr;
    const int* bl = nullptr;
    unsigned short* map = nullptr;
    unsigned short sink = 0;
    struct Pt { double x, y; };
    Pt C0(int i) const { return Pt{pts[2 * i], pts[2 * i + 1]}; }
    int BL(int i, int k) const { return bl[2 * i + k]; }
    unsigned short& lsMap(int i, int j) { return (i >= 0 && i < nxf && j >= 0 && j < 2) ? map[j * nxf + i] : sink; }
#include "../_ref/gen/lsmap.inc"
};

// The host set-up of the E/W/N/S link fractions (inidXArrays /
// iniFillMap's dXArr part: 1 on fluid nodes, then bcFindNodes over every
// wall segment, clVariablesLS.cpp:650-667, 1195-1208) over the arrays it
// reads: points C (= C0), segments BL, nType, dXArr / dXArr0 [4][XsizeFull nY].
union cl_double2 {
    struct { double x, y; };
    double s[2];
};
union cl_int2 {
    struct { int x, y; };
    int s[2];
};
#undef MAX
#undef MIN
struct LsDxShim {
    enum { find_ibb, find_dx, find_dx0 };
    struct Params { int nX, nY; double eps; } p;
    struct Lb { cl_double2 Cxy_double[9]; int rev[9]; int Cx[9]; int Cy[9]; } vlb;
    struct Fl { double mindXDist; } vfl;
    LsDxShim& vls;  // read through the reference's global instance
    int nxf = 0;
    const cl_double2* C = nullptr;
    const cl_double2* C0 = nullptr;
    const int* bl = nullptr;
    const short* map = nullptr;
    double* dx = nullptr;
    double* dx0 = nullptr;
    LsDxShim() : vls(*this) {}
    int BL(int i, int k) const { return bl[2 * i + k]; }
    int nType(int i, int j) const { return (unsigned short)map[(size_t)j * nxf + i]; }
    double& dXArr(int i, int j, int k) { return dx[((size_t)k * p.nY + j) * nxf + i]; }
    double& dXArr0(int i, int j, int k) { return dx0[((size_t)k * p.nY + j) * nxf + i]; }
#include "../_ref/gen/lsdx.inc"
};
#undef Subtract2
#undef GETLEN
#undef DOT_PROD
#undef MOD
#undef MAX
#undef MIN

extern "C" {

// dx, dx0 [4][nxf*ny]: the fractions of the fouled (M_SOLID) and unfouled
// (M0_SOLID) walls the reference's host set-up computes for polyline pts and
// segments bl (nbl), with "Min dX Dist" mindx.
int ref_ini_dx(const double* pts, int npts, const int* bl, int nbl, const short* map, int nx, int nxf, int ny,
               double mindx, double* dx, double* dx0) {
    LsDxShim s;
    s.p.nX = nx; s.p.nY = ny; s.p.eps = 1.e-5;
    static const double cxy[9][2] = {{0., 0.}, {1., 0.}, {-1., 0.}, {0., 1.}, {0., -1.},
                                     {1., 1.}, {-1., -1.}, {1., -1.}, {-1., 1.}};
    static const int rev[9] = {0, 2, 1, 4, 3, 6, 5, 8, 7};
    for (int q = 0; q < 9; ++q) {
        s.vlb.Cxy_double[q].x = cxy[q][0]; s.vlb.Cxy_double[q].y = cxy[q][1];
        s.vlb.rev[q] = rev[q]; s.vlb.Cx[q] = (int)cxy[q][0]; s.vlb.Cy[q] = (int)cxy[q][1];
    }
    s.vfl.mindXDist = mindx;
    s.nxf = nxf;
    std::vector<cl_double2> C((size_t)npts);
    for (int i = 0; i < npts; ++i) { C[(size_t)i].x = pts[2 * i]; C[(size_t)i].y = pts[2 * i + 1]; }
    s.C = s.C0 = C.data();
    s.bl = bl; s.map = map; s.dx = dx; s.dx0 = dx0;
    const size_t plane = (size_t)nxf * ny;
    for (size_t k = 0; k < 4 * plane; ++k) { dx[k] = 0.0; dx0[k] = 0.0; }
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i)
            if (s.nType(i, j) & 0x2)                     // M_FLUID_NODE
                for (int k = 0; k < 4; ++k) { s.dXArr(i, j, k) = 1.0; s.dXArr0(i, j, k) = 1.0; }
    // the unfouled fractions follow M0_FLUID_NODE (0x8) nodes
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const bool f0 = (s.nType(i, j) & 0x8) != 0;
            for (int k = 0; k < 4; ++k) s.dXArr0(i, j, k) = f0 ? 1.0 : 0.0;
        }
    for (int i = 0; i < nbl; ++i) s.bcFindNodes(i, LsDxShim::find_dx0);
    for (int i = 0; i < nbl; ++i) s.bcFindNodes(i, LsDxShim::find_dx);
    return 0;
}

int ref_ini_lsmap(const double* pts, const int* bl, int nbl, int nx, int nxf, unsigned short* map) {
    LsMapShim s;
    s.p.nX = nx; s.nBL = nbl; s.nxf = nxf; s.pts = pts; s.bl = bl; s.map = map;
    s.iniLSMap();
    return 0;
}

int ref_abi_version(void) { return 1; }

}  // extern "C"
