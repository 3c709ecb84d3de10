// kofm_komega.cuh - fused k-omega system assembly for sm_100a.
//
// One kernel replaces the reference's Update_kOmega_Diffusivities and
// Update_kOmega_Coeffs_Implicit (Kernels/kOmegaKernels.cl:7-95, 187-480) and
// the GMRES updateRHS step (gmresKernels.cl:353-420, b -= A x0):
//   * a 32x8 tile of nodes stages k and omega with a 2-node halo, and rho,
//     nu_t, wall distance with a 1-node halo, in shared memory;
//   * the blending function F1, the cross-diffusion multipliers and the
//     diffusivities D_k, D_w are evaluated on the tile plus a 1-node ring
//     (they are needed at the neighbours for grad D);
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
// Krylov basis, residual and right-hand side only carry the per-step
// increment, so they are FP32 (all arithmetic is FP64); the accumulated
// correction x stays FP64.
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

__global__ void __launch_bounds__(KO_TX * KO_TY)
komega_assemble_kernel(const AsmParams p) {
    constexpr int HX = KO_TX + 4, HY = KO_TY + 4;  // 2-ring halo
    constexpr int RX = KO_TX + 2, RY = KO_TY + 2;  // 1-ring
    __shared__ float sK[HY][HX];
    __shared__ float sO[HY][HX];
    __shared__ double sDk[RY][RX];
    __shared__ double sDo[RY][RX];
    __shared__ double sF1[RY][RX];
    __shared__ double sMx[RY][RX];
    __shared__ double sMy[RY][RX];

    const int tx = threadIdx.x, ty = threadIdx.y;
    const int tid = ty * KO_TX + tx;
    const int x0 = blockIdx.x * KO_TX, y0 = blockIdx.y * KO_TY;
    const int nx = p.nx, ny = p.ny, P = p.P;

    // ---- stage k, omega (2-ring; x periodic over nx, rows clamped) -------
    for (int i = tid; i < HX * HY; i += KO_TX * KO_TY) {
        const int sy = i / HX, sx = i % HX;
        const int gx = wrapx(x0 - 2 + sx, nx);
        int gy = y0 - 2 + sy;
        gy = gy < 0 ? 0 : (gy >= ny ? ny - 1 : gy);
        const long long g = (long long)gy * P + gx;
        sK[sy][sx] = p.K[g];
        sO[sy][sx] = p.O[g];
    }
    __syncthreads();

    // ---- F1, cross-diffusion, diffusivities on the tile + 1 ring -------------
    // (Update_kOmega_Diffusivities, kOmegaKernels.cl:24-94)
    for (int i = tid; i < RX * RY; i += KO_TX * KO_TY) {
        const int ry = i / RX, rx = i % RX;
        const int gx = wrapx(x0 - 1 + rx, nx);
        const int gy = y0 - 1 + ry;
        double Dk = 0.0, Do = 0.0, F1 = 0.0, mxv = 0.0, myv = 0.0;
        if (gy >= 0 && gy < ny) {
            const long long g = (long long)gy * P + gx;
            const int t = (uint16_t)p.ntype[g];
            if (!(t & M_SOLID)) {
                Fd3 X, Y, X2, Y2;
                node_weights(p, t, g, X, X2, Y, Y2);
                const int sy = ry + 1, sx = rx + 1;  // position in the 2-ring tile
                const double om = sO[sy][sx], kv = sK[sy][sx];
                const double yv = p.wallD[g];
                const double dOdx = X.e * sO[sy][sx + 1] + X.w * sO[sy][sx - 1] + X.c * om;
                const double dKdx = X.e * sK[sy][sx + 1] + X.w * sK[sy][sx - 1] + X.c * kv;
                const double dOdy = Y.e * sO[sy + 1][sx] + Y.w * sO[sy - 1][sx] + Y.c * om;
                const double dKdy = Y.e * sK[sy + 1][sx] + Y.w * sK[sy - 1][sx] + Y.c * kv;
                const double m = 2. * KO_SIGMA_O2 / om;
                mxv = m * dKdx;
                myv = m * dKdy;
                const double CDkw = dmaxr((double)p.rho[g] * (mxv * dOdx + myv * dOdy), 1.0e-10);
                double a = dmaxr(sqrt(kv) / (KO_BETA_STAR * om * yv), 500. * p.mu / (yv * yv * om));
                a = dminr(a, 4. * kv * KO_SIGMA_O2 / (CDkw * yv * yv));
                const double a2 = a * a;
                F1 = tanh(a2 * a2);
                const double nt = p.nut[g];
                Dk = p.mu + (KO_SIGMA_K1 * F1 + KO_SIGMA_K2 * (1. - F1)) * nt;
                Do = p.mu + (KO_SIGMA_O1 * F1 + KO_SIGMA_O2 * (1. - F1)) * nt;
            }
        }
        sDk[ry][rx] = Dk;
        sDo[ry][rx] = Do;
        sF1[ry][rx] = F1;
        sMx[ry][rx] = mxv;
        sMy[ry][rx] = myv;
    }
    __syncthreads();

    // ---- rows of the tile's nodes (Update_kOmega_Coeffs_Implicit) ------------
    const int gx = x0 + tx, gy = y0 + ty;
    if (gx >= nx || gy >= ny) return;
    const long long g = (long long)gy * P + gx;
    const long long D = p.D;
    const int t = (uint16_t)p.ntype[g];
    if (t & M_SOLID) {
        for (int c = 0; c < 4; ++c) { p.coef_o[c * D + g] = 0.0; p.coef_k[c * D + g] = 0.0; }
        p.rhs_o[g] = vec_t(0);
        p.rhs_k[g] = vec_t(0);
        return;
    }
    Fd3 X, Y, X2, Y2;
    node_weights(p, t, g, X, X2, Y, Y2);
    const int ry = ty + 1, rx = tx + 1;
    const double dk = sDk[ry][rx], dom = sDo[ry][rx];
    const double dk_dx = X.e * sDk[ry][rx + 1] + X.w * sDk[ry][rx - 1] + X.c * dk;
    const double do_dx = X.e * sDo[ry][rx + 1] + X.w * sDo[ry][rx - 1] + X.c * dom;
    const double dk_dy = Y.e * sDk[ry + 1][rx] + Y.w * sDk[ry - 1][rx] + Y.c * dk;
    const double do_dy = Y.e * sDo[ry + 1][rx] + Y.w * sDo[ry - 1][rx] + Y.c * dom;
    const double Ux = p.ux[g], Uy = p.uy[g], Rho = p.rho[g];
    const double Jxo = Ux - do_dx - sMx[ry][rx];
    const double Jyo = Uy - do_dy - sMy[ry][rx];
    const double Jxk = Ux - dk_dx, Jyk = Uy - dk_dy;
    const int sy = ty + 2, sx = tx + 2;
    const double Kraw = sK[sy][sx], Oraw = sO[sy][sx];
    double om = dmaxr(0.0, Oraw);
    const double kv = dmaxr(0.0, Kraw);
    const double f1 = sF1[ry][rx], nt = p.nut[g];
    const double Sxx = p.S[g], Sxy = p.S[D + g], Syy = p.S[2 * D + g];
    double Pk = 2. * nt * (Sxx * Sxx + Syy * Syy + 2. * Sxy * Sxy) - 2. / 3. * kv * Rho * (Sxx + Syy);
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
        const double yp = p.wallD[g];
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
