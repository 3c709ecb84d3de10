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

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// One thread per node of the tile plus its 1-node ring (34 x 10 = 340 of the
// 352 threads), so the transcendental-heavy diffusivity phase takes one round;
// the threads of the 32 x 8 interior then build the rows.
//
// The kernel is persistent: a block walks the tiles tile += gridDim.x and,
// while it computes one tile, streams the next tile's k, omega halo and every
// thread's node fields into the other half of a double-buffered shared-memory
// stage with 4-byte cp.async (the node flag goes into a register), so the
// loads of a tile overlap the FP64 work of the previous one.
constexpr int KO_RX = KO_TX + 2, KO_RY = KO_TY + 2;
constexpr int KO_THREADS = 352;  // 11 warps >= KO_RX * KO_RY
constexpr int KO_HX = KO_TX + 4, KO_HY = KO_TY + 4;  // 2-ring halo
constexpr int KO_NF = 8;  // node fields: wallD, rho, nut, ux, uy, Sxx, Sxy, Syy

template <typename FT>
struct AsmStage {
    FT K[KO_HY][KO_HX];
    FT O[KO_HY][KO_HX];
    FT fld[KO_NF][KO_THREADS];
};

template <typename FT>
struct AsmSmem {
    AsmStage<FT> st[2];
    double Dk[KO_RY][KO_RX];
    double Do[KO_RY][KO_RX];
    double dt;  // the time step of this launch (p.dt, or read from p.dt_dev)
};

__device__ __forceinline__ void ko_cp4(float* smem, const float* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void ko_cp4(double* smem, const double* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}

// Geometry of this thread's ring node in tile (x0, y0).
struct KoNode {
    int rx, ry, gxu, gx, gy;
    bool inrow, interior;
    long long g;
};

__device__ __forceinline__ KoNode ko_node(const AsmParams& p, int tid, int x0, int y0) {
    KoNode n;
    const bool ring = tid < KO_RX * KO_RY;
    n.rx = ring ? tid % KO_RX : 0;
    n.ry = ring ? tid / KO_RX : 0;
    n.gxu = x0 - 1 + n.rx;
    n.gx = wrapx(n.gxu, p.nx);
    n.gy = y0 - 1 + n.ry;
    n.inrow = ring && n.gy >= 0 && n.gy < p.ny;
    n.interior = n.inrow && n.rx >= 1 && n.rx <= KO_TX && n.ry >= 1 && n.ry <= KO_TY && n.gxu < p.nx;
    n.g = (long long)(n.inrow ? n.gy : 0) * p.P + n.gx;
    return n;
}

// Issue the copies of tile (x0, y0) into stage S; returns the node flag.
template <typename FT>
__device__ __forceinline__ int ko_issue(const AsmParams& p, int tid, int x0, int y0, AsmStage<FT>& S) {
    const FT* pK = static_cast<const FT*>(p.K);
    const FT* pO = static_cast<const FT*>(p.O);
    for (int i = tid; i < KO_HX * KO_HY; i += KO_THREADS) {
        const int sy = i / KO_HX, sx = i % KO_HX;
        const int hx = wrapx(x0 - 2 + sx, p.nx);
        int hy = y0 - 2 + sy;
        hy = hy < 0 ? 0 : (hy >= p.ny ? p.ny - 1 : hy);
        const long long h = (long long)hy * p.P + hx;
        ko_cp4(&S.K[sy][sx], pK + h);
        ko_cp4(&S.O[sy][sx], pO + h);
    }
    const KoNode n = ko_node(p, tid, x0, y0);
    if (!n.inrow) return M_SOLID;
    const long long g = n.g, D = p.D;
    ko_cp4(&S.fld[0][tid], static_cast<const FT*>(p.wallD) + g);
    ko_cp4(&S.fld[1][tid], static_cast<const FT*>(p.rho) + g);
    ko_cp4(&S.fld[2][tid], static_cast<const FT*>(p.nut) + g);
    if (n.interior) {
        const FT* pS = static_cast<const FT*>(p.S);
        ko_cp4(&S.fld[3][tid], static_cast<const FT*>(p.ux) + g);
        ko_cp4(&S.fld[4][tid], static_cast<const FT*>(p.uy) + g);
        ko_cp4(&S.fld[5][tid], pS + g);
        ko_cp4(&S.fld[6][tid], pS + D + g);
        ko_cp4(&S.fld[7][tid], pS + 2 * D + g);
    }
    return (uint16_t)__ldg(p.ntype + g);
}

// Blending function F1 (kOmegaKernels.cl:68-87).  With FP32 fields in FP32:
// its inputs k, omega, rho, y are FP32 fields; F1 in [0, 1] enters D_k, D_w
// with an error ~1e-7, the size of the FP32 rounding of nu_t beside it.  With
// FP64 fields in FP64.
__device__ __forceinline__ double ko_f1(float, double kv, double om, double yv, double rho, double cdx,
                                        double mu) {
    const float CDkw = fmaxf((float)(rho * cdx), 1.0e-10f);
    const float kf = (float)kv, of = (float)om, yf = (float)yv;
    float a = fmaxf(sqrtf(kf) / ((float)KO_BETA_STAR * of * yf), 500.f * (float)mu / (yf * yf * of));
    a = fminf(a, 4.f * kf * (float)KO_SIGMA_O2 / (CDkw * yf * yf));
    const float a2 = a * a;
    return (double)tanhf(a2 * a2);
}
__device__ __forceinline__ double ko_f1(double, double kv, double om, double yv, double rho, double cdx,
                                        double mu) {
    const double CDkw = fmax(rho * cdx, 1.0e-10);
    double a = fmax(sqrt(kv) / (KO_BETA_STAR * om * yv), 500. * mu / (yv * yv * om));
    a = fmin(a, 4. * kv * KO_SIGMA_O2 / (CDkw * yv * yv));
    const double a2 = a * a;
    return tanh(a2 * a2);
}

// Phases 2 and 3 of one tile from stage S (all of S visible to the block).
template <typename FT, bool DEVDT>
__device__ __forceinline__ void ko_tile(const AsmParams& p, int tid, int x0, int y0, int t,
                                        const AsmStage<FT>& S, AsmSmem<FT>& M) {
    const KoNode n = ko_node(p, tid, x0, y0);
    const int rx = n.rx, ry = n.ry;
    const long long g = n.g;
    const bool ring = tid < KO_RX * KO_RY;

    // ---- F1, cross-diffusion, diffusivities on the tile + 1 ring -------------
    // (Update_kOmega_Diffusivities, kOmegaKernels.cl:24-94)
    const int sy = ry + 1, sx = rx + 1;  // position in the 2-ring tile
    double Dk = 0.0, Do = 0.0, F1 = 0.0, mxv = 0.0, myv = 0.0;
    double yv = 1.0, rho = 0.0, nt = 0.0;
    Fd3 X, Y, X2, Y2;
    const bool fluid = n.inrow && !(t & M_SOLID);
    if (fluid) {
        yv = S.fld[0][tid];
        rho = S.fld[1][tid];
        nt = S.fld[2][tid];
        node_weights(p, t, g, X, X2, Y, Y2);
        const double om = S.O[sy][sx], kv = S.K[sy][sx];
        const double dOdx = X.e * S.O[sy][sx + 1] + X.w * S.O[sy][sx - 1] + X.c * om;
        const double dKdx = X.e * S.K[sy][sx + 1] + X.w * S.K[sy][sx - 1] + X.c * kv;
        const double dOdy = Y.e * S.O[sy + 1][sx] + Y.w * S.O[sy - 1][sx] + Y.c * om;
        const double dKdy = Y.e * S.K[sy + 1][sx] + Y.w * S.K[sy - 1][sx] + Y.c * kv;
        const double m = 2. * KO_SIGMA_O2 / om;
        mxv = m * dKdx;
        myv = m * dKdy;
        F1 = ko_f1(FT(0), kv, om, yv, rho, mxv * dOdx + myv * dOdy, p.mu);
        Dk = p.mu + (KO_SIGMA_K1 * F1 + KO_SIGMA_K2 * (1. - F1)) * nt;
        Do = p.mu + (KO_SIGMA_O1 * F1 + KO_SIGMA_O2 * (1. - F1)) * nt;
    }
    if (ring) {
        M.Dk[ry][rx] = Dk;
        M.Do[ry][rx] = Do;
    }
    __syncthreads();

    // ---- rows of the tile's nodes (Update_kOmega_Coeffs_Implicit) ------------
    if (!n.interior) return;
    if (t & M_SOLID) {
        for (int c = 0; c < 4; ++c) { p.coef_o[ilv(4, c, g)] = 0.0; p.coef_k[ilv(4, c, g)] = 0.0; }
        p.rhs_o[g] = 0.0;
        p.rhs_k[g] = 0.0;
        return;
    }
    const double Ux = S.fld[3][tid], Uy = S.fld[4][tid];
    const double Sxx = S.fld[5][tid], Sxy = S.fld[6][tid], Syy = S.fld[7][tid];
    const double dk = Dk, dom = Do;
    const double dk_dx = X.e * M.Dk[ry][rx + 1] + X.w * M.Dk[ry][rx - 1] + X.c * dk;
    const double do_dx = X.e * M.Do[ry][rx + 1] + X.w * M.Do[ry][rx - 1] + X.c * dom;
    const double dk_dy = Y.e * M.Dk[ry + 1][rx] + Y.w * M.Dk[ry - 1][rx] + Y.c * dk;
    const double do_dy = Y.e * M.Do[ry + 1][rx] + Y.w * M.Do[ry - 1][rx] + Y.c * dom;
    const double Jxo = Ux - do_dx - mxv;
    const double Jyo = Uy - do_dy - myv;
    const double Jxk = Ux - dk_dx, Jyk = Uy - dk_dy;
    const double Kraw = S.K[sy][sx], Oraw = S.O[sy][sx];
    double om = dmaxr(0.0, Oraw);
    const double kv = dmaxr(0.0, Kraw);
    const double f1 = F1;
    double Pk = 2. * nt * (Sxx * Sxx + Syy * Syy + 2. * Sxy * Sxy) - 2. / 3. * kv * rho * (Sxx + Syy);
    Pk = dmaxr(dminr(Pk, 10. * KO_BETA_STAR * kv * om), 0.0);
    const double gam = (f1 * KO_GAMMA1 + (1. - f1) * KO_GAMMA2) / nt;
    double Sc = -KO_BETA_STAR * om;
    // the launch's time step: a kernel parameter (constant bank), or the value
    // the device-driven update keeps in device memory (staged in M.dt; loaded
    // here, where it is first used, so it holds no register through the tile)
    double dt = p.dt;
    if (DEVDT) {
        const unsigned a = (unsigned)__cvta_generic_to_shared(&M.dt);
        asm volatile("ld.shared.f64 %0, [%1];" : "=d"(dt) : "r"(a));
    }

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
    const double kS = S.K[sy - 1][sx], kW = S.K[sy][sx - 1], kE = S.K[sy][sx + 1], kN = S.K[sy + 1][sx];
    const double oS = S.O[sy - 1][sx], oW = S.O[sy][sx - 1], oE = S.O[sy][sx + 1], oN = S.O[sy + 1][sx];
    const double Axk = Ks * kS + Kw * kW + Kraw + Ke * kE + Kn * kN;
    const double Axo = Ws * oS + Ww * oW + Oraw + We * oE + Wn * oN;
    p.coef_o[ilv(4, 0, g)] = We; p.coef_o[ilv(4, 1, g)] = Ww; p.coef_o[ilv(4, 2, g)] = Wn; p.coef_o[ilv(4, 3, g)] = Ws;
    p.coef_k[ilv(4, 0, g)] = Ke; p.coef_k[ilv(4, 1, g)] = Kw; p.coef_k[ilv(4, 2, g)] = Kn; p.coef_k[ilv(4, 3, g)] = Ks;
    p.rhs_o[g] = (Wsrc - Axo);
    p.rhs_k[g] = (Ksrc - Axk);
}

#ifndef KOFM_ASM_MINBLOCKS
#define KOFM_ASM_MINBLOCKS 2  // resident blocks per SM (registers and the persistent grid)
#endif
template <typename FT = float, bool DEVDT = false>
__global__ void __launch_bounds__(KO_THREADS, KOFM_ASM_MINBLOCKS)
komega_assemble_kernel(const AsmParams p, const double* dt_dev) {
    extern __shared__ __align__(16) unsigned char ko_smem[];
    AsmSmem<FT>& M = *reinterpret_cast<AsmSmem<FT>*>(ko_smem);
    const int tid = threadIdx.x;
    const int tiles_x = (p.nx + KO_TX - 1) / KO_TX;
    const int ntiles = tiles_x * ((p.ny + KO_TY - 1) / KO_TY);
    int tile = blockIdx.x;
    if (tile >= ntiles) return;  // block-uniform
    // DEVDT: the time step is read from dt_dev (device-driven updates);
    // visible after the loop's first barrier
    if (DEVDT && tid == 0) M.dt = *dt_dev;
    int buf = 0;
    int t_cur = ko_issue(p, tid, (tile % tiles_x) * KO_TX, (tile / tiles_x) * KO_TY, M.st[0]);
    cp_async_commit();
    for (; tile < ntiles; tile += gridDim.x) {
        cp_async_wait_all();
        __syncthreads();  // stage `buf` complete for every thread; the previous tile is done
        const int next = tile + gridDim.x;
        int t_next = M_SOLID;
        if (next < ntiles)
            t_next = ko_issue(p, tid, (next % tiles_x) * KO_TX, (next / tiles_x) * KO_TY, M.st[buf ^ 1]);
        cp_async_commit();
        ko_tile<FT, DEVDT>(p, tid, (tile % tiles_x) * KO_TX, (tile / tiles_x) * KO_TY, t_cur, M.st[buf], M);
        t_cur = t_next;
        buf ^= 1;
    }
    cp_async_wait_all();
}

}  // namespace kofm
