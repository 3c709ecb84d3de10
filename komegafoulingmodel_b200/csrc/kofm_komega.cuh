// kofm_komega.cuh - fused k-omega system assembly for sm_100a.
//
// One kernel replaces the reference's Update_kOmega_Diffusivities and
// Update_kOmega_Coeffs_Implicit (Kernels/kOmegaKernels.cl:7-95, 187-480) and
// the GMRES updateRHS step (gmresKernels.cl:353-420, b -= A x0):
//   * a warp owns a strip of 30 columns and marches up a chunk of rows with
//     no shared memory and no block barrier: lane l holds column x0 - 1 + l,
//     so lanes 0 and 31 are the 1-node ring the strip's rows need;
//   * at row r the warp evaluates the blending function F1, the
//     cross-diffusion multipliers and the diffusivities D_k, D_w of row r
//     (k, omega neighbours in x by shuffles, in y from a register window);
//   * it then builds the backward-Euler rows for k and omega of row r - 1
//     (D neighbours in x by shuffles, in y from registers), normalised by the
//     diagonal (which is therefore 1 and not stored), with the wall-omega
//     Dirichlet row of kOmegaKernels.cl:389-403;
//   * the correction right-hand side b' = b - A x0 (x0 = current k / omega)
//     is formed in FP64 here, so the solver never re-reads x0 or b.
// D_k, D_w, F1 and the cross-diffusion terms never reach HBM (the reference
// writes and re-reads all of them).
#pragma once
#include "kofm_common.cuh"

namespace kofm {


// One implicit system (index 0: omega, 1: k) as the solver sees it.  The
// matrix stays FP64: an FP32-rounded operator would perturb every implicit
// update by ~1e-8 relative, and that bias accumulates over the time steps.
// The Krylov basis, residual and right-hand side are FP64 as well: an FP32
// basis loses orthogonality and stalls the first omega cycle near 1e-5
// relative residual.


// Multi-vector arrays (the 4 coefficients, the Krylov basis) are stored
// tile-interleaved: the NV values of the 32 nodes of one row segment (node
// index g = x + P y, P a multiple of 32) are contiguous, element (j, g) at
// ((g / 32) NV + j) 32 + g % 32.  A warp sweeping a strip of columns then
// reads one or two contiguous blocks per row instead of NV separate row
// pieces.
__host__ __device__ __forceinline__ long long ilv(int nv, int j, long long g) {
    return ((g >> 5) * nv + j) * 32 + (g & 31);
}

struct KoSystem {
    double* coef = nullptr;  // [4 x D] normalised off-diagonals E, W, N, S (interleaved)
    double* rhs = nullptr;    // [D] b' = b - A x0 (also the residual of restart 0)
    double* r = nullptr;      // [D] residual of restarts >= 1
    double* x = nullptr;     // [D] correction
    double* V = nullptr;      // [K x D] Krylov basis (orthogonalised, unscaled; interleaved),
                              // or the powers p_1 .. p_K of the one-sweep cycle
    double* x2 = nullptr;     // [D] correction and residual of alternate restarts
    double* r2 = nullptr;     //     (the one-sweep cycle's update reads one, writes the other)
};

struct AsmParams {
    const int16_t* ntype;
    const int32_t* dxidx;
    const DxRecord* dxrec;
    // node fields: FP32, or FP64 for the FP64 storage form (the kernel's FT)
    const void* wallD;
    const void* K;
    const void* O;
    const void* nut;
    const void* rho;
    const void* ux;
    const void* uy;
    const void* S;
    double* coef_o;
    double* rhs_o;
    double* coef_k;
    double* rhs_k;
    int nx, ny, P;
    int rows;  // rows per warp strip chunk
    long long D;
    double mu, dt;
};

struct Fd3 {
    double e, w, c;
};

// Non-uniform 3-point first-derivative weights from the link fractions, with
// the reference's clipping (>= 0.1) and fallback to the plain central
// difference when |centre weight| > 10 (kOmegaKernels.cl:37-55, 235-253).
__device__ __forceinline__ void fd_weights(double dpos, double dneg, Fd3& d1, Fd3& d2) {
    const double a = dpos < 0.1 ? 0.1 : dpos;
    const double b = dneg < 0.1 ? 0.1 : dneg;
    double s = a + b;
    s = s < 0.1 ? 0.1 : s;
    d1.e = b / (a * s);
    d1.w = -a / (b * s);
    d1.c = (a - b) / (a * b);
    if (fabs(d1.c) > 10.) { d1.e = 1.0 / s; d1.w = -1.0 / s; d1.c = 0.0; }
    d2.e = 2. / (a * s);
    d2.w = 2. / (b * s);
    d2.c = -2. / (a * b);
}

__device__ __forceinline__ double dmaxr(double a, double b) { return a < b ? b : a; }
__device__ __forceinline__ double dminr(double a, double b) { return b < a ? b : a; }

// Warp strips: KM_W interior columns per warp (lanes 1..30; lanes 0 and 31
// are the ring), KM_WARPS independent warps per block, KOFM_ASM_ROWS rows per
// warp (each chunk re-evaluates the closure of the ring rows above and below
// it: 2 of KOFM_ASM_ROWS + 2 rows).
constexpr int KM_W = 30;
#ifndef KOFM_ASM_WARPS
#define KOFM_ASM_WARPS 4
#endif
constexpr int KM_WARPS = KOFM_ASM_WARPS;
#ifndef KOFM_ASM_ROWS
#define KOFM_ASM_ROWS 16
#endif
#ifndef KOFM_ASM_MINBLOCKS
#define KOFM_ASM_MINBLOCKS 4  // resident blocks per SM the register budget is set for
#endif
#ifndef KOFM_ASM_CLOSURE_FP32
#define KOFM_ASM_CLOSURE_FP32 1
#endif

// Arithmetic type of the closure (F1, D_k, D_w, the cross-diffusion
// multipliers, grad D) for a field type.  FP32 fields: FP32 -- its inputs are
// FP32 fields and its rounding (~1e-7 relative) is the size of the FP32
// rounding of nu_t and k beside it; the rows, b' and the operator stay FP64.
// FP64 fields: FP64.
template <typename FT>
struct KoClosure {
    using type = double;
};
#if KOFM_ASM_CLOSURE_FP32
template <>
struct KoClosure<float> {
    using type = float;
};
#endif

__host__ __device__ __forceinline__ int km_wrap(int x, int nx) {
    x %= nx;
    return x < 0 ? x + nx : x;
}

// Blending function F1 (kOmegaKernels.cl:68-87), in the closure's type.
// The FP32 form's quotients are the fast ones (__fdividef, 2 ulp): F1 =
// tanh(a^4) carries four times the rounding of a either way.
__device__ __forceinline__ float ko_f1(float kv, float om, float yv, float rho, float cdx, float mu) {
    const float CDkw = fmaxf(rho * cdx, 1.0e-10f);
    float a = fmaxf(__fdividef(sqrtf(kv), (float)KO_BETA_STAR * om * yv), __fdividef(500.f * mu, yv * yv * om));
    a = fminf(a, __fdividef(4.f * kv * (float)KO_SIGMA_O2, CDkw * yv * yv));
    const float a2 = a * a;
    return tanhf(a2 * a2);
}
__device__ __forceinline__ double ko_f1(double kv, double om, double yv, double rho, double cdx,
                                        double mu) {
    const double CDkw = fmax(rho * cdx, 1.0e-10);
    double a = fmax(sqrt(kv) / (KO_BETA_STAR * om * yv), 500. * mu / (yv * yv * om));
    a = fmin(a, 4. * kv * KO_SIGMA_O2 / (CDkw * yv * yv));
    const double a2 = a * a;
    return tanh(a2 * a2);
}

__device__ __forceinline__ float km_div(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double km_div(double a, double b) { return a / b; }

// Weights of a node with a link-fraction record (NESW_BOUNDARY nodes whose
// dX differs from 1); rec < 0 means the unit weights d1 = (1/2, -1/2, 0),
// d2 = (1, 1, -2), which the code below applies as constants.
__device__ __forceinline__ int km_record(const AsmParams& p, int t, int g) {
    return (t & NESW_BOUNDARY) ? __ldg(p.dxidx + g) : -1;
}
__device__ __forceinline__ void km_weights(const AsmParams& p, int rec, Fd3& X, Fd3& X2, Fd3& Y, Fd3& Y2) {
    const DxRecord r = p.dxrec[rec];
    fd_weights(r.dx[0], r.dx[1], X, X2);
    fd_weights(r.dx[2], r.dx[3], Y, Y2);
}

// Closure of one fluid node (Update_kOmega_Diffusivities,
// kOmegaKernels.cl:24-94): neighbours c (centre), e, w, n, s.
template <typename CT, typename FT>
__device__ __forceinline__ void km_closure(const AsmParams& p, int rec, FT kc, FT ke, FT kw, FT kn, FT ks,
                                           FT oc, FT oe, FT ow, FT on, FT os, FT yv, FT rho, FT nt,
                                           CT& Dk, CT& Do, CT& F1, CT& mx, CT& my) {
    CT dOdx, dKdx, dOdy, dKdy;
    if (rec < 0) {
        // X.e E + X.w W + X.c C with (1/2, -1/2, 0): the same value as the
        // general form (scaling by 1/2 is exact)
        dOdx = CT(0.5) * (CT(oe) - CT(ow));
        dKdx = CT(0.5) * (CT(ke) - CT(kw));
        dOdy = CT(0.5) * (CT(on) - CT(os));
        dKdy = CT(0.5) * (CT(kn) - CT(ks));
    } else {
        Fd3 X, X2, Y, Y2;
        km_weights(p, rec, X, X2, Y, Y2);
        dOdx = CT(X.e) * CT(oe) + CT(X.w) * CT(ow) + CT(X.c) * CT(oc);
        dKdx = CT(X.e) * CT(ke) + CT(X.w) * CT(kw) + CT(X.c) * CT(kc);
        dOdy = CT(Y.e) * CT(on) + CT(Y.w) * CT(os) + CT(Y.c) * CT(oc);
        dKdy = CT(Y.e) * CT(kn) + CT(Y.w) * CT(ks) + CT(Y.c) * CT(kc);
    }
    const CT m = km_div(CT(2. * KO_SIGMA_O2), CT(oc));
    mx = m * dKdx;
    my = m * dKdy;
    F1 = ko_f1(CT(kc), CT(oc), CT(yv), CT(rho), mx * dOdx + my * dOdy, CT(p.mu));
    Dk = CT(p.mu) + (CT(KO_SIGMA_K1) * F1 + CT(KO_SIGMA_K2) * (CT(1) - F1)) * CT(nt);
    Do = CT(p.mu) + (CT(KO_SIGMA_O1) * F1 + CT(KO_SIGMA_O2) * (CT(1) - F1)) * CT(nt);
}

// Diagonal of a row, k or omega: advection velocity J, diffusivity d, time
// step dtr and sink Scr of the row.
template <bool UNIT>
__device__ __forceinline__ double km_diag(const Fd3& X, const Fd3& X2, const Fd3& Y, const Fd3& Y2, double Jx,
                                          double Jy, double d, double dtr, double Scr) {
    // unit weights: X.c = Y.c = 0, X2.c + Y2.c = -4
    if (UNIT) return 1. + dtr * (4. * d) - Scr;
    return 1. + dtr * (Jx * X.c + Jy * Y.c - d * (X2.c + Y2.c)) - Scr;
}

// One row normalised by the reciprocal ic of its diagonal: coefficients E, W,
// N, S at coef[cb + 32 j]; b - A x at rhs[g], with b = src ic and the sum in
// the CSR order S, W, C, E, N over the field x at the node and its
// neighbours.
template <bool UNIT, typename FT>
__device__ __forceinline__ void km_row(const Fd3& X, const Fd3& X2, const Fd3& Y, const Fd3& Y2, double Jx,
                                       double Jy, double d, double dtr, double ic, double src, FT xc, FT xe,
                                       FT xw, FT xn, FT xs, double* coef, int cb, double* rhs, int g) {
    const double f = dtr * ic;  // time step over the diagonal
    double e, w, n, s;
    if (UNIT) {
        // X2.e = X2.w = 1
        e = (0.5 * Jx - d) * f;
        w = (-0.5 * Jx - d) * f;
        n = (0.5 * Jy - d) * f;
        s = (-0.5 * Jy - d) * f;
    } else {
        e = (Jx * X.e - d * X2.e) * f;
        w = (Jx * X.w - d * X2.w) * f;
        n = (Jy * Y.e - d * Y2.e) * f;
        s = (Jy * Y.w - d * Y2.w) * f;
    }
    const double Ax = s * (double)xs + w * (double)xw + (double)xc + e * (double)xe + n * (double)xn;
    coef[cb] = e; coef[cb + 32] = w; coef[cb + 64] = n; coef[cb + 96] = s;
    rhs[g] = src * ic - Ax;
}

// Both rows of a node.  One FP64 reciprocal serves the three divisions of
// the node (the two diagonals and gamma / nu_t): r = 1 / (Kc Wc nu_t), then
// 1/Kc = Wc nu_t r, 1/Wc = Kc nu_t r, 1/nu_t = Kc Wc r (a few ulp from the
// quotients; a row's coefficients and right-hand side take the same factor).
template <bool UNIT, typename FT>
__device__ __forceinline__ void km_pair(const AsmParams& p, const Fd3& X, const Fd3& X2, const Fd3& Y,
                                        const Fd3& Y2, double Jxk, double Jyk, double Jxo, double Jyo,
                                        double dk, double dom, double dt, double dtw, double Sc, double Scw,
                                        double kv, double omw, double Pk, double gnum, double nt, int g, int cb,
                                        FT kc, FT ke, FT kw, FT kn, FT ks, FT oc, FT oe, FT ow, FT on, FT os) {
    const double Kc = km_diag<UNIT>(X, X2, Y, Y2, Jxk, Jyk, dk, dt, Sc);
    const double Wc = km_diag<UNIT>(X, X2, Y, Y2, Jxo, Jyo, dom, dtw, Scw);
    const double KW = Kc * Wc;
    const double r = 1. / (KW * nt);
    const double gam = gnum * (KW * r);
    km_row<UNIT>(X, X2, Y, Y2, Jxk, Jyk, dk, dt, (Wc * nt) * r, kv + dt * Pk, kc, ke, kw, kn, ks, p.coef_k, cb,
                 p.rhs_k, g);
    km_row<UNIT>(X, X2, Y, Y2, Jxo, Jyo, dom, dtw, (Kc * nt) * r, omw + dtw * (gam * Pk), oc, oe, ow, on, os,
                 p.coef_o, cb, p.rhs_o, g);
}

// Rows of one fluid node (Update_kOmega_Coeffs_Implicit,
// kOmegaKernels.cl:187-480), normalised by their diagonals, and
// b' = b - A x0.  D* are the diffusivities of the node and its neighbours;
// cb is the interleaved index of coefficient 0 of node g.
template <typename CT, typename FT>
__device__ __forceinline__ void km_rows(const AsmParams& p, double dt, int t, int rec, int g, int cb,
                                        CT dkc, CT dke, CT dkw, CT dkn, CT dks, CT doc, CT doe, CT dow,
                                        CT don, CT dos, CT F1, CT mx, CT my, FT kc, FT ke, FT kw, FT kn,
                                        FT ks, FT oc, FT oe, FT ow, FT on, FT os, FT fux, FT fuy,
                                        FT fsxx, FT fsxy, FT fsyy, FT fnt, FT frho, FT fyv) {
    const double dk = dkc, dom = doc;
    const double Ux = fux, Uy = fuy;
    const double Sxx = fsxx, Sxy = fsxy, Syy = fsyy;
    const double nt = fnt, rho = frho;
    const double om = dmaxr(0.0, (double)oc);
    const double kv = dmaxr(0.0, (double)kc);
    const double f1 = F1;
    double Pk = 2. * nt * (Sxx * Sxx + Syy * Syy + 2. * Sxy * Sxy) - 2. / 3. * kv * rho * (Sxx + Syy);
    Pk = dmaxr(dminr(Pk, 10. * KO_BETA_STAR * kv * om), 0.0);
    const double gnum = f1 * KO_GAMMA1 + (1. - f1) * KO_GAMMA2;  // gamma nu_t
    const double Sc = -KO_BETA_STAR * om;
    // the omega row of a node beside an E/W/N/S wall holds the wall value
    // (kOmegaKernels.cl:389-403): no time derivative, no source
    double dtw = dt, Scw = Sc, omw = om;
    if (t & NESW_BOUNDARY) {
        dtw = 0.;
        Scw = 0.;
        const double yp = fyv;
        const double ovis = (6. * p.mu / 0.075) / (yp * yp);
        const double olog = sqrt(kv) / (KO_C_MU_0_25 * KO_KAPPA * yp);
        omw = dminr(1000., sqrt(ovis * ovis + olog * olog));
    }
    if (rec < 0) {
        const Fd3 Z = {0., 0., 0.};  // unit weights: constants inside km_pair
        const double dk_dx = (double)(CT(0.5) * (dke - dkw));
        const double do_dx = (double)(CT(0.5) * (doe - dow));
        const double dk_dy = (double)(CT(0.5) * (dkn - dks));
        const double do_dy = (double)(CT(0.5) * (don - dos));
        km_pair<true>(p, Z, Z, Z, Z, Ux - dk_dx, Uy - dk_dy, Ux - do_dx - (double)mx, Uy - do_dy - (double)my,
                      dk, dom, dt, dtw, Sc, Scw, kv, omw, Pk, gnum, nt, g, cb, kc, ke, kw, kn, ks, oc, oe, ow,
                      on, os);
    } else {
        Fd3 X, X2, Y, Y2;
        km_weights(p, rec, X, X2, Y, Y2);
        const double dk_dx = X.e * (double)dke + X.w * (double)dkw + X.c * dk;
        const double do_dx = X.e * (double)doe + X.w * (double)dow + X.c * dom;
        const double dk_dy = Y.e * (double)dkn + Y.w * (double)dks + Y.c * dk;
        const double do_dy = Y.e * (double)don + Y.w * (double)dos + Y.c * dom;
        km_pair<false>(p, X, X2, Y, Y2, Ux - dk_dx, Uy - dk_dy, Ux - do_dx - (double)mx,
                       Uy - do_dy - (double)my, dk, dom, dt, dtw, Sc, Scw, kv, omw, Pk, gnum, nt, g, cb, kc,
                       ke, kw, kn, ks, oc, oe, ow, on, os);
    }
}

// Depth of each warp's row ring: the fields of a row are copied
// KM_RING - 1 rows before the row is used.
#ifndef KOFM_ASM_RING
#define KOFM_ASM_RING 4
#endif
constexpr int KM_R = KOFM_ASM_RING;
static_assert((KM_R & (KM_R - 1)) == 0 && KM_R >= 2, "ring depth: a power of two");
// Fields of one ring slot ([field][lane]): k, omega of row i + 1; k, omega of
// row i at the column beyond lanes 0 / 31; wall distance, rho, nu_t of row
// i; u_x, u_y, S_xx, S_xy, S_yy of row i - 1.
enum { KF_K, KF_O, KF_KX, KF_OX, KF_Y, KF_R, KF_N, KF_U, KF_V, KF_SA, KF_SB, KF_SC, KM_NF };

template <typename FT>
constexpr size_t km_smem_bytes() { return sizeof(FT) * KM_WARPS * KM_R * KM_NF * 32; }

template <typename FT>
__device__ __forceinline__ void km_cp(FT* dst, const FT* src) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
    if constexpr (sizeof(FT) == 4)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(src) : "memory");
}
__device__ __forceinline__ void km_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void km_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// The assembly: one warp per (strip of KM_W columns, chunk of p.rows rows).
// At row r the warp holds k, omega of rows r-2 .. r+1 (rows clamped to the
// lattice, as the halo of the tiles), the diffusivities of rows r-2 .. r and
// the closure outputs of row r-1.  The fields each step reads stream through
// a per-warp ring of KM_R slots in shared memory, copied with cp.async
// KM_R - 1 steps ahead; each lane reads back only the elements it copied, so
// the warp needs no barrier.
template <typename FT = float, bool DEVDT = false>
__global__ void __launch_bounds__(KM_WARPS * 32, KOFM_ASM_MINBLOCKS)
komega_assemble_kernel(const AsmParams p, const double* dt_dev) {
    using CT = typename KoClosure<FT>::type;
    constexpr unsigned FULL = 0xffffffffu;
    extern __shared__ __align__(16) unsigned char km_smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nx = p.nx, ny = p.ny;
    const int nstrips = (nx + KM_W - 1) / KM_W;
    const int nchunks = (ny + p.rows - 1) / p.rows;
    const int wid = blockIdx.x * KM_WARPS + warp;
    if (wid >= nstrips * nchunks) return;  // whole warps
    const int x0 = (wid % nstrips) * KM_W;
    const int y0 = (wid / nstrips) * p.rows;
    const int y1 = min(ny, y0 + p.rows);
    // 32-bit node offsets: the launch requires 4 D < 2^31
    const int P = p.P, D = (int)p.D;
    const int gxu = x0 - 1 + lane;
    const int cx = km_wrap(gxu, nx);
    // lanes 0 and 31 also read the column beyond them (their W / E neighbour)
    const int cxx = km_wrap(lane == 0 ? x0 - 2 : x0 + KM_W + 1, nx);
    const bool xl = lane == 0 || lane == 31;
    const bool icol = lane >= 1 && lane <= KM_W && gxu < nx;
    const int colb = ((cx >> 5) << 7) + (cx & 31);
    double dt = p.dt;
    if (DEVDT) dt = __ldg(dt_dev);
    const FT* pK = static_cast<const FT*>(p.K);
    const FT* pO = static_cast<const FT*>(p.O);
    const FT* pY = static_cast<const FT*>(p.wallD);
    const FT* pR = static_cast<const FT*>(p.rho);
    const FT* pN = static_cast<const FT*>(p.nut);
    const FT* pU = static_cast<const FT*>(p.ux);
    const FT* pV = static_cast<const FT*>(p.uy);
    const FT* pS = static_cast<const FT*>(p.S);
    auto crow = [ny](int y) -> int { return y < 0 ? 0 : (y >= ny ? ny - 1 : y); };
    FT* ring = reinterpret_cast<FT*>(km_smem) + warp * (KM_R * KM_NF * 32) + lane;
    // copies of the fields step i reads (i = y0 - 1 .. y1) into slot i mod KM_R
    auto stage = [&](int i) {
        FT* s = ring + ((i - y0 + 1) & (KM_R - 1)) * (KM_NF * 32);
        const int ga = crow(i + 1) * P;
        km_cp(s + KF_K * 32, pK + ga + cx);
        km_cp(s + KF_O * 32, pO + ga + cx);
        if (xl) {
            const int gx = crow(i) * P + cxx;
            km_cp(s + KF_KX * 32, pK + gx);
            km_cp(s + KF_OX * 32, pO + gx);
        }
        if (i >= 0 && i < ny) {
            const int g = i * P + cx;
            km_cp(s + KF_Y * 32, pY + g);
            km_cp(s + KF_R * 32, pR + g);
            km_cp(s + KF_N * 32, pN + g);
        }
        if (icol && i - 1 >= y0) {
            const int g = (i - 1) * P + cx;
            km_cp(s + KF_U * 32, pU + g);
            km_cp(s + KF_V * 32, pV + g);
            km_cp(s + KF_SA * 32, pS + g);
            km_cp(s + KF_SB * 32, pS + D + g);
            km_cp(s + KF_SC * 32, pS + 2 * D + g);
        }
    };
#pragma unroll
    for (int j = 0; j < KM_R - 1; ++j) {
        if (y0 - 1 + j <= y1) stage(y0 - 1 + j);
        km_commit();
    }

    // k, omega of rows r-2 .. r (start r = y0 - 1; row y0 - 3 is never used);
    // row r + 1 comes from the ring
    FT k0 = FT(0), o0 = FT(0);
    FT k1 = __ldg(pK + crow(y0 - 2) * P + cx), o1 = __ldg(pO + crow(y0 - 2) * P + cx);
    FT k2 = __ldg(pK + crow(y0 - 1) * P + cx), o2 = __ldg(pO + crow(y0 - 1) * P + cx);
    // flag of row r (loaded one step ahead)
    int t = y0 - 1 >= 0 ? (uint16_t)__ldg(p.ntype + (y0 - 1) * P + cx) : M_SOLID;
    // carried from row r - 1: flag, ring fields, closure
    int tm = M_SOLID;
    FT yvm = FT(0), rhm = FT(0), ntm = FT(0);
    CT f1m = CT(0), mxm = CT(0), mym = CT(0);
    // diffusivities of rows r-2 and r-1
    CT dk0 = CT(0), do0 = CT(0), dk1 = CT(0), do1 = CT(0);

    for (int r = y0 - 1; r <= y1; ++r) {
        // ---- this step's fields from the ring; the copies of step r + KM_R - 1
        km_wait<KM_R - 2>();
        const FT* s = ring + ((r - y0 + 1) & (KM_R - 1)) * (KM_NF * 32);
        const FT k3 = s[KF_K * 32], o3 = s[KF_O * 32];
        const FT kx = s[KF_KX * 32], ox = s[KF_OX * 32];
        const FT yv = s[KF_Y * 32], rh = s[KF_R * 32], nt = s[KF_N * 32];
        const FT u1 = s[KF_U * 32], v1 = s[KF_V * 32];
        const FT sa1 = s[KF_SA * 32], sb1 = s[KF_SB * 32], sc1 = s[KF_SC * 32];
        if (r + KM_R - 1 <= y1) stage(r + KM_R - 1);
        km_commit();
        int tn = M_SOLID;
        if (r + 1 < ny && r < y1) tn = (uint16_t)__ldg(p.ntype + (r + 1) * P + cx);
        // ---- closure of row r ----------------------------------------------
        FT ke = __shfl_down_sync(FULL, k2, 1), kw = __shfl_up_sync(FULL, k2, 1);
        FT oe = __shfl_down_sync(FULL, o2, 1), ow = __shfl_up_sync(FULL, o2, 1);
        if (lane == 31) { ke = kx; oe = ox; }
        if (lane == 0) { kw = kx; ow = ox; }
        CT dk2 = CT(0), do2 = CT(0), f1 = CT(0), mx = CT(0), my = CT(0);
        if (r >= 0 && r < ny && !(t & M_SOLID)) {
            const int rec = km_record(p, t, r * P + cx);
            km_closure<CT, FT>(p, rec, k2, ke, kw, k3, k1, o2, oe, ow, o3, o1, yv, rh, nt, dk2, do2, f1, mx, my);
        }
        // ---- rows of row q = r - 1 -----------------------------------------
        const CT dke = __shfl_down_sync(FULL, dk1, 1), dkw = __shfl_up_sync(FULL, dk1, 1);
        const CT doe = __shfl_down_sync(FULL, do1, 1), dow = __shfl_up_sync(FULL, do1, 1);
        const FT kem = __shfl_down_sync(FULL, k1, 1), kwm = __shfl_up_sync(FULL, k1, 1);
        const FT oem = __shfl_down_sync(FULL, o1, 1), owm = __shfl_up_sync(FULL, o1, 1);
        const int q = r - 1;
        if (icol && q >= y0) {
            const int g = q * P + cx;
            const int cb = 4 * q * P + colb;
            if (tm & M_SOLID) {
                p.coef_o[cb] = 0.0; p.coef_o[cb + 32] = 0.0; p.coef_o[cb + 64] = 0.0; p.coef_o[cb + 96] = 0.0;
                p.coef_k[cb] = 0.0; p.coef_k[cb + 32] = 0.0; p.coef_k[cb + 64] = 0.0; p.coef_k[cb + 96] = 0.0;
                p.rhs_o[g] = 0.0;
                p.rhs_k[g] = 0.0;
            } else {
                const int rec = km_record(p, tm, g);
                km_rows<CT, FT>(p, dt, tm, rec, g, cb, dk1, dke, dkw, dk2, dk0, do1, doe, dow, do2, do0,
                                f1m, mxm, mym, k1, kem, kwm, k2, k0, o1, oem, owm, o2, o0,
                                u1, v1, sa1, sb1, sc1, ntm, rhm, yvm);
            }
        }
        // ---- advance one row -------------------------------------------------
        k0 = k1; k1 = k2; k2 = k3;
        o0 = o1; o1 = o2; o2 = o3;
        dk0 = dk1; do0 = do1; dk1 = dk2; do1 = do2;
        f1m = f1; mxm = mx; mym = my;
        tm = t; yvm = yv; rhm = rh; ntm = nt;
        t = tn;
    }
    km_wait<0>();
}

}  // namespace kofm
