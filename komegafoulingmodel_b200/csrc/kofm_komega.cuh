// kofm_komega.cuh - fused k-omega system assembly for sm_100a.
//
// One kernel replaces the reference's Update_kOmega_Diffusivities and
// Update_kOmega_Coeffs_Implicit (Kernels/kOmegaKernels.cl:7-95, 187-480) and
// the GMRES updateRHS step (gmresKernels.cl:353-420, b -= A x0):
//   * a 32x8 tile of nodes stages k and omega with a 2-node halo in shared
//     memory;
//   * the blending function F1, the cross-diffusion multipliers and the
//     diffusivities D_k, D_w are evaluated on the tile plus a 1-node ring,
//     one node per thread (D_k, D_w are needed at the neighbours for grad D);
//   * each fluid node of the tile then builds its backward-Euler rows for k and
//     omega, normalised by the diagonal (which is therefore 1 and not
//     stored), with the wall-omega Dirichlet row of kOmegaKernels.cl:389-403;
//   * the correction right-hand side b' = b - A x0 (x0 = current k / omega)
//     is formed in FP64 here, so the solver never re-reads x0 or b.
// D_k, D_w, F1 and the cross-diffusion terms never reach HBM (the reference
// writes and re-reads all of them).
#pragma once
#include "kofm_common.cuh"

namespace kofm {

constexpr int KO_TX = 32, KO_TY = 8;

// One implicit system (index 0: omega, 1: k) as the solver sees it.  The
// matrix stays FP64: an FP32-rounded operator would perturb every implicit
// update by ~1e-8 relative, and that bias accumulates over the time steps.
// The Krylov basis, residual and right-hand side are FP64 as well: an FP32
// basis loses orthogonality and stalls the first omega cycle near 1e-5
// relative residual.
#ifndef KOFM_SOLVER_VEC
#define KOFM_SOLVER_VEC double
#endif
using vec_t = KOFM_SOLVER_VEC;  // storage type of the streamed solver vectors

struct KoSystem {
    double* coef = nullptr;  // [4][D] normalised off-diagonals E, W, N, S
    vec_t* rhs = nullptr;    // [D] b' = b - A x0 (also the residual of restart 0)
    vec_t* r = nullptr;      // [D] residual of restarts >= 1
    double* x = nullptr;     // [D] correction
    vec_t* V = nullptr;      // [K][D] Krylov basis (orthogonalised, unscaled)
};

struct AsmParams {
    const int16_t* ntype;
    const int32_t* dxidx;
    const DxRecord* dxrec;
    const float* wallD;
    const float* K;
    const float* O;
    const float* nut;
    const float* rho;
    const float* ux;
    const float* uy;
    const float* S;
    double* coef_o;
    vec_t* rhs_o;
    double* coef_k;
    vec_t* rhs_k;
    int nx, ny, P;
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

// Weights for unit link fractions (every node without an E/W/N/S wall link):
// d1 = (1/2, -1/2, 0), d2 = (1, 1, -2), exactly what fd_weights(1, 1) gives.
__device__ __forceinline__ void fd_unit(Fd3& d1, Fd3& d2) {
    d1.e = 0.5; d1.w = -0.5; d1.c = 0.0;
    d2.e = 1.0; d2.w = 1.0; d2.c = -2.0;
}

// Weights of one node: constants unless it has a dX record.
__device__ __forceinline__ void node_weights(const AsmParams& p, int t, long long g, Fd3& X,
                                             Fd3& X2, Fd3& Y, Fd3& Y2) {
    if (t & NESW_BOUNDARY) {
        const int r = p.dxidx[g];
        if (r >= 0) {
            const DxRecord rec = p.dxrec[r];
            fd_weights(rec.dx[0], rec.dx[1], X, X2);
            fd_weights(rec.dx[2], rec.dx[3], Y, Y2);
            return;
        }
    }
    fd_unit(X, X2);
    fd_unit(Y, Y2);
}

__device__ __forceinline__ double dmaxr(double a, double b) { return a < b ? b : a; }
__device__ __forceinline__ double dminr(double a, double b) { return b < a ? b : a; }

__device__ __forceinline__ int wrapx(int x, int nx) {
    return x < 0 ? x + nx : (x >= nx ? x - nx : x);
}

// One thread per node of the tile plus its 1-node ring (34 x 10 = 340 of the
// 352 threads), so the transcendental-heavy diffusivity phase takes one round;
// the threads of the 32 x 8 interior then build the rows.  Each thread loads
// its node's fields before the first barrier, so those loads overlap the
// staging of k and omega.
constexpr int KO_RX = KO_TX + 2, KO_RY = KO_TY + 2;
constexpr int KO_THREADS = 352;  // 11 warps >= KO_RX * KO_RY

__global__ void __launch_bounds__(KO_THREADS, 2)
komega_assemble_kernel(const AsmParams p) {
    constexpr int HX = KO_TX + 4, HY = KO_TY + 4;  // 2-ring halo
    __shared__ float sK[HY][HX];
    __shared__ float sO[HY][HX];
    __shared__ double sDk[KO_RY][KO_RX];
    __shared__ double sDo[KO_RY][KO_RX];

    const int tid = threadIdx.x;
    const int x0 = blockIdx.x * KO_TX, y0 = blockIdx.y * KO_TY;
    const int nx = p.nx, ny = p.ny, P = p.P;
    const long long D = p.D;

    // ---- this thread's ring node and its fields ---------------------------------
    const bool ring = tid < KO_RX * KO_RY;
    const int rx = ring ? tid % KO_RX : 0, ry = ring ? tid / KO_RX : 0;
    const int gxu = x0 - 1 + rx;  // unwrapped column
    const int gx = wrapx(gxu, nx);
    const int gy = y0 - 1 + ry;
    const bool inrow = ring && gy >= 0 && gy < ny;
    const bool interior = inrow && rx >= 1 && rx <= KO_TX && ry >= 1 && ry <= KO_TY && gxu < nx;
    const long long g = (long long)(inrow ? gy : 0) * P + gx;
    int t = M_SOLID;
    double yv = 1.0, rho = 0.0, nt = 0.0, Ux = 0.0, Uy = 0.0, Sxx = 0.0, Sxy = 0.0, Syy = 0.0;
    if (inrow) {
        t = (uint16_t)p.ntype[g];
        if (!(t & M_SOLID)) {
            yv = p.wallD[g];
            rho = p.rho[g];
            nt = p.nut[g];
            if (interior) {
                Ux = p.ux[g]; Uy = p.uy[g];
                Sxx = p.S[g]; Sxy = p.S[D + g]; Syy = p.S[2 * D + g];
            }
        }
    }

    // ---- stage k, omega (2-ring; x periodic over nx, rows clamped) -------
    for (int i = tid; i < HX * HY; i += KO_THREADS) {
        const int sy = i / HX, sx = i % HX;
        const int hx = wrapx(x0 - 2 + sx, nx);
        int hy = y0 - 2 + sy;
        hy = hy < 0 ? 0 : (hy >= ny ? ny - 1 : hy);
        const long long h = (long long)hy * P + hx;
        sK[sy][sx] = p.K[h];
        sO[sy][sx] = p.O[h];
    }
    __syncthreads();

    // ---- F1, cross-diffusion, diffusivities on the tile + 1 ring -------------
    // (Update_kOmega_Diffusivities, kOmegaKernels.cl:24-94)
    const int sy = ry + 1, sx = rx + 1;  // position in the 2-ring tile
    double Dk = 0.0, Do = 0.0, F1 = 0.0, mxv = 0.0, myv = 0.0;
    Fd3 X, Y, X2, Y2;
    if (inrow && !(t & M_SOLID)) {
        node_weights(p, t, g, X, X2, Y, Y2);
        const double om = sO[sy][sx], kv = sK[sy][sx];
        const double dOdx = X.e * sO[sy][sx + 1] + X.w * sO[sy][sx - 1] + X.c * om;
        const double dKdx = X.e * sK[sy][sx + 1] + X.w * sK[sy][sx - 1] + X.c * kv;
        const double dOdy = Y.e * sO[sy + 1][sx] + Y.w * sO[sy - 1][sx] + Y.c * om;
        const double dKdy = Y.e * sK[sy + 1][sx] + Y.w * sK[sy - 1][sx] + Y.c * kv;
        const double m = 2. * KO_SIGMA_O2 / om;
        mxv = m * dKdx;
        myv = m * dKdy;
        const double CDkw = dmaxr(rho * (mxv * dOdx + myv * dOdy), 1.0e-10);
        double a = dmaxr(sqrt(kv) / (KO_BETA_STAR * om * yv), 500. * p.mu / (yv * yv * om));
        a = dminr(a, 4. * kv * KO_SIGMA_O2 / (CDkw * yv * yv));
        const double a2 = a * a;
        F1 = tanh(a2 * a2);
        Dk = p.mu + (KO_SIGMA_K1 * F1 + KO_SIGMA_K2 * (1. - F1)) * nt;
        Do = p.mu + (KO_SIGMA_O1 * F1 + KO_SIGMA_O2 * (1. - F1)) * nt;
    }
    if (ring) {
        sDk[ry][rx] = Dk;
        sDo[ry][rx] = Do;
    }
    __syncthreads();

    // ---- rows of the tile's nodes (Update_kOmega_Coeffs_Implicit) ------------
    if (!interior) return;
    if (t & M_SOLID) {
        for (int c = 0; c < 4; ++c) { p.coef_o[c * D + g] = 0.0; p.coef_k[c * D + g] = 0.0; }
        p.rhs_o[g] = vec_t(0);
        p.rhs_k[g] = vec_t(0);
        return;
    }
    const double dk = Dk, dom = Do;
    const double dk_dx = X.e * sDk[ry][rx + 1] + X.w * sDk[ry][rx - 1] + X.c * dk;
    const double do_dx = X.e * sDo[ry][rx + 1] + X.w * sDo[ry][rx - 1] + X.c * dom;
    const double dk_dy = Y.e * sDk[ry + 1][rx] + Y.w * sDk[ry - 1][rx] + Y.c * dk;
    const double do_dy = Y.e * sDo[ry + 1][rx] + Y.w * sDo[ry - 1][rx] + Y.c * dom;
    const double Jxo = Ux - do_dx - mxv;
    const double Jyo = Uy - do_dy - myv;
    const double Jxk = Ux - dk_dx, Jyk = Uy - dk_dy;
    const double Kraw = sK[sy][sx], Oraw = sO[sy][sx];
    double om = dmaxr(0.0, Oraw);
    const double kv = dmaxr(0.0, Kraw);
    const double f1 = F1;
    double Pk = 2. * nt * (Sxx * Sxx + Syy * Syy + 2. * Sxy * Sxy) - 2. / 3. * kv * rho * (Sxx + Syy);
    Pk = dmaxr(dminr(Pk, 10. * KO_BETA_STAR * kv * om), 0.0);
    const double gam = (f1 * KO_GAMMA1 + (1. - f1) * KO_GAMMA2) / nt;
    double Sc = -KO_BETA_STAR * om;
    double dt = p.dt;

    double Kc = 1. + dt * (Jxk * X.c + Jyk * Y.c - dk * (X2.c + Y2.c)) - Sc;
    double Ke = dt * (Jxk * X.e - dk * X2.e);
    double Kw = dt * (Jxk * X.w - dk * X2.w);
    double Kn = dt * (Jyk * Y.e - dk * Y2.e);
    double Ks = dt * (Jyk * Y.w - dk * Y2.w);
    double Ksrc = kv + dt * Pk;
    const double iKc = 1. / Kc;
    Ke *= iKc; Kw *= iKc; Kn *= iKc; Ks *= iKc; Ksrc *= iKc;

    if (t & NESW_BOUNDARY) {
        dt = 0.;
        Sc = 0.;
        const double yp = yv;
        const double ovis = (6. * p.mu / 0.075) / (yp * yp);
        const double olog = sqrt(kv) / (KO_C_MU_0_25 * KO_KAPPA * yp);
        om = dminr(1000., sqrt(ovis * ovis + olog * olog));
    }
    double Wc = 1. + dt * (Jxo * X.c + Jyo * Y.c - dom * (X2.c + Y2.c)) - Sc;
    double We = dt * (Jxo * X.e - dom * X2.e);
    double Ww = dt * (Jxo * X.w - dom * X2.w);
    double Wn = dt * (Jyo * Y.e - dom * Y2.e);
    double Ws = dt * (Jyo * Y.w - dom * Y2.w);
    double Wsrc = om + dt * (gam * Pk);
    const double iWc = 1. / Wc;
    We *= iWc; Ww *= iWc; Wn *= iWc; Ws *= iWc; Wsrc *= iWc;

    // b' = b - A x0, summed in the CSR order of an interior row (S, W, C, E, N)
    const double kS = sK[sy - 1][sx], kW = sK[sy][sx - 1], kE = sK[sy][sx + 1], kN = sK[sy + 1][sx];
    const double oS = sO[sy - 1][sx], oW = sO[sy][sx - 1], oE = sO[sy][sx + 1], oN = sO[sy + 1][sx];
    const double Axk = Ks * kS + Kw * kW + Kraw + Ke * kE + Kn * kN;
    const double Axo = Ws * oS + Ww * oW + Oraw + We * oE + Wn * oN;
    p.coef_o[g] = We; p.coef_o[D + g] = Ww; p.coef_o[2 * D + g] = Wn; p.coef_o[3 * D + g] = Ws;
    p.coef_k[g] = Ke; p.coef_k[D + g] = Kw; p.coef_k[2 * D + g] = Kn; p.coef_k[3 * D + g] = Ks;
    p.rhs_o[g] = (vec_t)(Wsrc - Axo);
    p.rhs_k[g] = (vec_t)(Ksrc - Axk);
}

}  // namespace kofm
