// kofm_lb.cuh - D2Q9 pull-scheme collide-stream kernel (the reference's
// LB_collision_SRT_Fluid / LB_collision_SRT_Fluid_w_kOmega + lbIBB,
// Kernels/lbKernels.cl:175-335, 345-633, 640-668), re-designed for sm_100a.
//
// One thread owns 4 consecutive nodes of one row (x0..x0+3); a warp covers a
// 128-node row segment, a 32x4 block covers 4 rows.  Per population plane the
// warp issues one 16-byte (FP32) or 8-byte (FP16/BF16) load per thread of
// the upstream row; the +-1 x-shift of the pull is done with warp shuffles,
// lanes 0 / 31 fetch the single element across the segment edge (with the
// periodic wrap over nx).  Every plane row is read once and written once per
// step, so HBM traffic is the compulsory bytes.
//
// Pull vs the reference's push: the buffers hold post-collision populations
// G of the previous step; node x gathers G(x - c_q, q).  A link whose
// upstream node is solid (the node carries the bound flag of direction
// rev(q)) takes the node's own G(x, rev q): the reference's same-step
// half-way bounce-back (postCollisionBC, lbKernels.cl:166-171).  lbIBB's
// Bouzidi correction, which the reference applies to the post-stream buffer
// after the push, is applied here to the gathered values before collision:
//   2q <= 1: P(x, rev d) = 2q G(x, d) + (1 - 2q) P(x, d)
//   2q  > 1: P(x, rev d) = (G(x, d) + (2q - 1) G(x, rev d)) / (2q)
// where d is the link direction pointing into the wall.  All links of one node
// use the pre-correction values (the reference's list order only matters for
// a node with walls on two opposite sides).
//
// Collision in deviation form (d_q = f_q - w_q), exact-difference forcing
// with the product-form equilibrium (clVariablesLB.cpp:77-117):
//   rho = 1 + sum d,  u = j / rho,
//   feq_q - w_q = drho phx phy + dphx phy0 + phx0 dphy + dphx dphy,
//   d'_q = d_q - w (d_q - (feq_q - w_q)) + rho phy [phx(ux + F) - phx(ux)],
// with phi0(0) = 2/3, phi0(+-1) = 1/6, dphi(0, u) = -u^2,
// dphi(+-1, u) = (+-u + u^2)/2.  No term subtracts two O(1) numbers, so the
// FP32-stored deviations keep their relative precision.
#pragma once
#include "kofm_common.cuh"

// Resident 128-thread blocks per SM the register budget targets: 4 (at most
// 128 registers, a few spilled) measured 5% faster than the unconstrained
// 164-register build for the FP32 and 16-bit deviation forms; the f - feq form
// (about 200 registers) keeps its registers.
#ifndef KOFM_LB_MINBLOCKS
#define KOFM_LB_MINBLOCKS 4
#endif

namespace kofm {

struct LbParams {
    const void* gin;        // populations read (9 planes)
    void* gout;             // populations written (9 planes)
    const int16_t* ntype;
    const int32_t* rec;     // per-node IBB record index (-1: none)
    const IbbRecord* ibb;   // IBB records
    // node fields: FP32, or FP64 for the FP64 storage form (the kernel's FT)
    const void* wallD;
    void* K;
    void* O;
    void* S;                // 3 planes Sxx, Sxy, Syy
    void* nut;
    void* rho;
    void* ux;
    void* uy;
    double* partials;       // per block: sum rho, sum ux, sum uy (FP64)
    const float* ref_in;    // non-equilibrium form: reference rho, ux, uy of
    float* ref_out;         //   the populations read / written (3 planes)
    const float* rowref;    // row-reference form: rho, ux, uy of each row ([3][ny])
    int nx, ny, P;
    long long D;
    double tau, fterm, mu, maxnut;
    int options;
    int has_ibb;
};

template <typename AT>
__device__ __forceinline__ AT phi0(int c) { return c == 0 ? AT(2.0 / 3.0) : AT(1.0 / 6.0); }
template <typename AT>
__device__ __forceinline__ AT dphi(int c, AT u) {
    return c == 0 ? -u * u : AT(0.5) * (AT(c) * u + u * u);
}
// phi(c, u + g) - phi(c, u)
template <typename AT>
__device__ __forceinline__ AT dphiF(int c, AT u, AT g) {
    return c == 0 ? -g * (AT(2) * u + g) : AT(0.5) * g * (AT(c) + AT(2) * u + g);
}
template <typename AT>
__device__ __forceinline__ AT amax(AT a, AT b) { return a < b ? b : a; }
template <typename AT>
__device__ __forceinline__ AT amin(AT a, AT b) { return b < a ? b : a; }

template <typename ST>
__device__ __forceinline__ typename Store<ST>::vt ld1(const ST* base, long long idx) {
    return Store<ST>::to_f32(base[idx]);
}

// The 4 values of an FP32 plane row that the pull of a direction with x
// component cx brings to nodes x0..x0+3 (periodic in x; same shifts as the
// population gather).
__device__ __forceinline__ void pull_row_f32(const float* row, int cx, int lane, int x0, int nx,
                                             float v[4]) {
    const float4 c4 = __ldg(reinterpret_cast<const float4*>(row + x0));
    const float c[4] = {c4.x, c4.y, c4.z, c4.w};
    if (cx == 0) {
        v[0] = c[0]; v[1] = c[1]; v[2] = c[2]; v[3] = c[3];
    } else if (cx == 1) {
        float left = __shfl_up_sync(0xffffffffu, c[3], 1);
        if (lane == 0) left = __ldg(row + (x0 > 0 ? x0 - 1 : nx - 1));
        v[0] = left; v[1] = c[0]; v[2] = c[1]; v[3] = c[2];
    } else {
        float right = __shfl_down_sync(0xffffffffu, c[0], 1);
        if (lane == 31) right = __ldg(row + ((x0 + 4 < nx) ? x0 + 4 : 0));
        v[0] = c[1]; v[1] = c[2]; v[2] = c[3]; v[3] = right;
        const int jw = nx - 1 - x0;
        if (jw >= 0 && jw < 4) v[jw] = __ldg(row);
    }
}

// ---------------------------------------------------------------------------
// Quotients of the SST eddy viscosity: the fast FP32 quotient (__fdividef,
// 2 ulp) for the FP32 fields, whose rounding (~1e-7) already bounds nu_t;
// the IEEE quotient in FP64.
__device__ __forceinline__ float lb_div(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double lb_div(double a, double b) { return a / b; }

// ROW: populations stored as f - feq(reference moments of their row), FP16
// scaled as NEQ (KOFM_STORE_FP16_ROW); one reference (rho, u_x, u_y) per row,
// the same for all the nodes of a row within a collide (the host re-centres
// them between collides), so a warp decodes the values of one gathered row
// with one equilibrium per direction and encodes its own row's with another.
// NEQ: populations stored as f - feq(reference moments of the writing node),
// FP16 (KOFM_STORE_FP16_NEQ); see feq_dev_f32.  FT: type of the node fields
// (k, omega, strain rates, wall distance, nu_t, moments) -- FP32, or FP64 for
// the FP64 storage form, whose eddy viscosity is then evaluated in FP64 too.
//
// With NEQ and FP32 arithmetic (KOFM_STORE_FP16_NEQ32) the stored value is
// formed without the full population: relative to the node's own unforced
// moments (rho, u) it is (1 - w) neq + rho phi_y [phi_x(u + F) - phi_x(u)], both
// terms small and computed with relative precision, so the exact-difference
// force increment (~1e-7 of a population of ~0.1, a few FP32 ulps of it) is
// not rounded away; the equilibrium both sides subtract and add back is the
// same FP32 function feq_dev_f32 of the same FP32 moments.
//
// One block of 32 x 4 threads covers 128 columns x 4 rows: block (bx, by) of
// a lattice whose grid has gx = P / 128 block columns.  lb_step_kernel runs
// one lattice; lb_multi_kernel walks a table of such blocks over several
// lattices.
constexpr int LB_BLOCK_ROWS = 4;

template <typename ST, typename AT, bool KOMEGA, bool PHASE0, bool NEQ, typename FT, bool ROW = false>
__device__ __forceinline__ void lb_block(const LbParams& p, int bx, int by, int gx) {
    using VT = typename Store<ST>::vt;  // type a population is loaded into
    constexpr bool NEQ32 = NEQ && sizeof(AT) == 4;
    FT* const fK = static_cast<FT*>(p.K);
    FT* const fO = static_cast<FT*>(p.O);
    FT* const fS = static_cast<FT*>(p.S);
    const int lane = threadIdx.x;
    const int y = by * LB_BLOCK_ROWS + threadIdx.y;
    // Each warp owns one partial-sum slot; warps that leave early clear it.
    double* slot = nullptr;
    if (p.partials && (p.options & OPTION_SAVE_MACRO_FIELDS))
        slot = p.partials + (((long long)by * gx + bx) * 4 + threadIdx.y) * 3;
    if (y >= p.ny) {  // warp-uniform
        if (slot && lane == 0) { slot[0] = 0.0; slot[1] = 0.0; slot[2] = 0.0; }
        return;
    }
    const int x0 = (bx * 32 + lane) * 4;
    const ST* gin = static_cast<const ST*>(p.gin);
    ST* gout = static_cast<ST*>(p.gout);
    const long long rowoff = (long long)y * p.P;
    const long long D = p.D;

    int type[4];
    bool fl[4];
    {
        const short4 t4 = *reinterpret_cast<const short4*>(p.ntype + rowoff + x0);
        type[0] = (uint16_t)t4.x; type[1] = (uint16_t)t4.y;
        type[2] = (uint16_t)t4.z; type[3] = (uint16_t)t4.w;
#pragma unroll
        for (int j = 0; j < 4; ++j) fl[j] = (x0 + j < p.nx) && !(type[j] & M_SOLID);
    }
    const bool any_fluid = fl[0] | fl[1] | fl[2] | fl[3];
    if (!__any_sync(0xffffffffu, any_fluid)) {  // whole warp solid
        if (slot && lane == 0) { slot[0] = 0.0; slot[1] = 0.0; slot[2] = 0.0; }
        return;
    }

    AT d[9][4];
    float own_r[4] = {}, own_u[4] = {}, own_v[4] = {};  // NEQ: this node's reference moments
    // ROW: equilibrium deviation feq - w of the reference moments of row r
    auto row_feq = [&](int q, int r) -> float {
        return feq_dev_f32(q, p.rowref[r], p.rowref[p.ny + r], p.rowref[2 * p.ny + r]);
    };
    // own stored population of direction q, decoded
    auto own_pop = [&](int q, int j) -> AT {
        const VT raw = ld1(gin, q * D + rowoff + x0 + j);
        if (ROW) return AT(row_feq(q, y)) + AT(raw) * AT(NEQ_INV_SCALE);
        if (!NEQ) return AT(raw);
        return AT(feq_dev_f32(q, own_r[j], own_u[j], own_v[j])) + AT(raw) * AT(NEQ_INV_SCALE);
    };
    // ---- gather (pull) -----------------------------------------------------
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const int cx = cx_of(q), cy = cy_of(q);
        VT v[4];
        if (PHASE0) {
            Store<ST>::load4(gin + q * D + rowoff + x0, v);
        } else {
            int ys = y - cy;
            ys = ys < 0 ? 0 : (ys >= p.ny ? p.ny - 1 : ys);  // only solid rows clamp
            const ST* src = gin + q * D + (long long)ys * p.P;
            VT c[4];
            Store<ST>::load4(src + x0, c);
            if (cx == 0) {
                v[0] = c[0]; v[1] = c[1]; v[2] = c[2]; v[3] = c[3];
            } else if (cx == 1) {
                VT left = __shfl_up_sync(0xffffffffu, c[3], 1);
                if (lane == 0) {
                    const int xs = x0 > 0 ? x0 - 1 : p.nx - 1;
                    left = ld1(src, xs);
                }
                v[0] = left; v[1] = c[0]; v[2] = c[1]; v[3] = c[2];
            } else {
                VT right = __shfl_down_sync(0xffffffffu, c[0], 1);
                if (lane == 31) {
                    const int xs = (x0 + 4 < p.nx) ? x0 + 4 : 0;
                    right = ld1(src, xs);
                }
                v[0] = c[1]; v[1] = c[2]; v[2] = c[3]; v[3] = right;
                const int jw = p.nx - 1 - x0;  // node nx-1 wraps to x = 0
                if (jw >= 0 && jw < 4) v[jw] = ld1(src, 0);
            }
        }
        if (NEQ) {
            // reference moments of the 4 upstream nodes
            int ys = y - (PHASE0 ? 0 : cy);
            ys = ys < 0 ? 0 : (ys >= p.ny ? p.ny - 1 : ys);
            const int sx = PHASE0 ? 0 : cx;
            float rr[4], ru[4], rv[4];
            pull_row_f32(p.ref_in + (long long)ys * p.P, sx, lane, x0, p.nx, rr);
            pull_row_f32(p.ref_in + D + (long long)ys * p.P, sx, lane, x0, p.nx, ru);
            pull_row_f32(p.ref_in + 2 * D + (long long)ys * p.P, sx, lane, x0, p.nx, rv);
            if (q == 0) {
#pragma unroll
                for (int j = 0; j < 4; ++j) { own_r[j] = rr[j]; own_u[j] = ru[j]; own_v[j] = rv[j]; }
            }
#pragma unroll
            for (int j = 0; j < 4; ++j)
                d[q][j] = AT(feq_dev_f32(q, rr[j], ru[j], rv[j])) + AT(v[j]) * AT(NEQ_INV_SCALE);
        } else if (ROW) {
            // the reference of the row the 4 values were read from
            int ys = y - (PHASE0 ? 0 : cy);
            ys = ys < 0 ? 0 : (ys >= p.ny ? p.ny - 1 : ys);
            const AT fe = AT(row_feq(q, ys));
#pragma unroll
            for (int j = 0; j < 4; ++j) d[q][j] = fe + AT(v[j]) * AT(NEQ_INV_SCALE);
        } else {
#pragma unroll
            for (int j = 0; j < 4; ++j) d[q][j] = AT(v[j]);
        }
    }

    // ---- half-way bounce-back and interpolated bounce-back -----------------
    if (!PHASE0) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (!fl[j] || !(type[j] & BOUNDARY)) continue;
            const long long node = rowoff + x0 + j;
            AT pre[9];
#pragma unroll
            for (int q = 1; q < 9; ++q) {
                if (type[j] & bound_of(rev_of(q))) d[q][j] = own_pop(rev_of(q), j);
                pre[q] = d[q][j];
            }
            if (p.has_ibb) {
                const int r = p.rec[node];
                if (r >= 0) {
                    const IbbRecord rec = p.ibb[r];
#pragma unroll
                    for (int dd = 1; dd < 9; ++dd) {
                        const double qf = rec.q[dd - 1];
                        if (qf < 0.0) continue;
                        const int rd = rev_of(dd);
                        const AT q2 = AT(2.0 * qf);
                        if (q2 <= AT(1)) {
                            d[rd][j] = q2 * pre[rd] + (AT(1) - q2) * pre[dd];
                        } else {
                            const AT own = own_pop(rd, j);
                            d[rd][j] = (AT(1) / q2) * (pre[rd] + (q2 - AT(1)) * own);
                        }
                    }
                }
            }
        }
    }

    // ---- collision ----------------------------------------------------------
    const AT tau0 = AT(p.tau), fterm = AT(p.fterm), mu = AT(p.mu);
    FT o_rho[4], o_ux[4], o_uy[4], o_nut[4], o_s[3][4];
    float o_u0[4];  // NEQ32: the unforced u_x, the reference of the stored values
    FT kin[4], oin[4], win[4], sin3[3][4];
    if (KOMEGA) {
        fld_ld4(fK + rowoff + x0, kin);
        fld_ld4(fO + rowoff + x0, oin);
        fld_ldg4(static_cast<const FT*>(p.wallD) + rowoff + x0, win);
#pragma unroll
        for (int c = 0; c < 3; ++c) fld_ld4(fS + c * D + rowoff + x0, sin3[c]);
    }
    double bsum_rho = 0.0, bsum_ux = 0.0, bsum_uy = 0.0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if (!fl[j]) {
            o_rho[j] = FT(0); o_ux[j] = FT(0); o_uy[j] = FT(0); o_nut[j] = FT(0); o_u0[j] = 0.f;
            o_s[0][j] = FT(0); o_s[1][j] = FT(0); o_s[2][j] = FT(0);
#pragma unroll
            for (int q = 0; q < 9; ++q) d[q][j] = AT(0);
            continue;
        }
        AT drho = AT(0);
#pragma unroll
        for (int q = 0; q < 9; ++q) drho += d[q][j];
        const AT rho = AT(1) + drho;
        const AT jx = d[1][j] - d[2][j] + d[5][j] - d[6][j] + d[7][j] - d[8][j];
        const AT jy = d[3][j] - d[4][j] + d[5][j] - d[6][j] - d[7][j] + d[8][j];
        // ROW with FP32 arithmetic: u from FP64 sums of the deviations (an FP32
        // quotient of FP32 sums rounds u the same way at every node of a row
        // of equal values, step after step)
        double m64x = 0.0, m64y = 0.0;
        if (ROW && sizeof(AT) == 4) {
            double dr = 0.0;
#pragma unroll
            for (int q = 0; q < 9; ++q) dr += (double)d[q][j];
            const double ax = (double)d[1][j] - (double)d[2][j] + (double)d[5][j] - (double)d[6][j] +
                              (double)d[7][j] - (double)d[8][j];
            const double ay = (double)d[3][j] - (double)d[4][j] + (double)d[5][j] - (double)d[6][j] -
                              (double)d[7][j] + (double)d[8][j];
            m64x = ax / (1.0 + dr);
            m64y = ay / (1.0 + dr);
        }
        AT w = tau0;
        AT inv;  // 1 / rho
        if (KOMEGA) {
            // SST eddy viscosity (lbKernels.cl:400-451) in the fields' type:
            // FP32 for the FP32 fields (nu_t is stored in FP32; the relaxation
            // rate it sets changes the populations by ~1e-7 of their
            // non-equilibrium part, below the FP32 storage rounding), FP64 in
            // the FP64 form.
            FT om = oin[j], kv = kin[j];
            const FT yv = win[j];
            const long long node = rowoff + x0 + j;
            if (om < FT(0)) { om = fabs(om); fO[node] = om; }
            if (kv < FT(0)) { kv = FT(1e-16); fK[node] = FT(1e-16); }
            const FT mu_f = (FT)p.mu;
            const FT a = lb_div(FT(2) * sqrt(kv), (FT)KO_BETA_STAR * om * yv);
            const FT b = lb_div(FT(500) * mu_f, yv * yv * om);
            const FT arg = fmax(a, b);
            FT F2 = tanh(arg * arg);
            const FT sxx = sin3[0][j], sxy = sin3[1][j], syy = sin3[2][j];
            F2 *= sqrt(FT(2) * (sxx * sxx + FT(2) * sxy * sxy + syy * syy));
            const FT a1 = (FT)KO_A1;
            const FT nut = fmax(fmin((FT)p.maxnut, lb_div(a1 * kv, fmax(a1 * om, F2))), FT(1e-16));
            o_nut[j] = nut;
            // one reciprocal for 1 / rho and the relaxation rate
            // 1 / (3 (nu_t + mu) + 1/2): r = 1 / (rho den), 1/rho = den r, w = rho r
            const AT den = AT(3) * (AT(nut) + mu) + AT(0.5);
            const AT r = AT(1) / (rho * den);
            inv = den * r;
            w = rho * r;
        } else {
            inv = AT(1) / rho;
        }
        const AT ux = (ROW && sizeof(AT) == 4) ? AT(m64x) : inv * jx;
        const AT uy = (ROW && sizeof(AT) == 4) ? AT(m64y) : inv * jy;
        AT sxx_n = AT(0), sxy_n = AT(0), syy_n = AT(0);
        // NEQ32: the mass and momentum that the FP32 moments leave out -- rho
        // = 1 + drho rounded on the FP32 grid near 1 (up to 6e-8), u = j / rho
        // rounded -- kept apart and carried by the stored values unrelaxed, as
        // the collision conserves them
        AT cdr = AT(0), cdjx = AT(0), cdjy = AT(0);
        if (NEQ32) {
            // the rounding of the moment sums themselves (the same sums in the
            // same order, error-free transformation of each addition)
            auto lo = [](AT a, AT b, AT s) -> AT { const AT bp = s - a; return (a - (s - bp)) + (b - bp); };
            AT lr = AT(0), lx = AT(0), ly = AT(0);
            {
                AT sr = d[0][j];
#pragma unroll
                for (int q = 1; q < 9; ++q) { const AT t = sr + d[q][j]; lr += lo(sr, d[q][j], t); sr = t; }
                const int sx[6] = {1, 2, 5, 6, 7, 8}, gx[6] = {1, -1, 1, -1, 1, -1};
                const int sy[6] = {3, 4, 5, 6, 7, 8}, gy[6] = {1, -1, 1, -1, -1, 1};
                AT tx = d[1][j], ty = d[3][j];
#pragma unroll
                for (int i = 1; i < 6; ++i) {
                    const AT bx = gx[i] > 0 ? d[sx[i]][j] : -d[sx[i]][j];
                    const AT by = gy[i] > 0 ? d[sy[i]][j] : -d[sy[i]][j];
                    const AT nx_ = tx + bx, ny_ = ty + by;
                    lx += lo(tx, bx, nx_);
                    ly += lo(ty, by, ny_);
                    tx = nx_;
                    ty = ny_;
                }
            }
            cdr = (drho - (rho - AT(1))) + lr;
            cdjx = fma(-rho, ux, jx) + lx;
            cdjy = fma(-rho, uy, jy) + ly;
            // non-equilibrium parts against the FP32 equilibrium of the FP32
            // moments, with their mass and momentum (rounding) projected out
            // along w_q (1, 3 c_q): the non-conserved part the collision relaxes
            AT m0 = AT(0), mx = AT(0), my = AT(0);
#pragma unroll
            for (int q = 0; q < 9; ++q) {
                d[q][j] -= AT(feq_dev_f32(q, (float)rho, (float)ux, (float)uy));
                m0 += d[q][j];
                mx += AT(cx_of(q)) * d[q][j];
                my += AT(cy_of(q)) * d[q][j];
            }
#pragma unroll
            for (int q = 0; q < 9; ++q)
                d[q][j] -= AT(weight_of(q)) * (m0 + AT(3 * cx_of(q)) * mx + AT(3 * cy_of(q)) * my);
        }
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            const int cx = cx_of(q), cy = cy_of(q);
            const AT px0 = phi0<AT>(cx), py0 = phi0<AT>(cy);
            const AT dpx = dphi<AT>(cx, ux), dpy = dphi<AT>(cy, uy);
            const AT phy = py0 + dpy;
            const AT feqdev = NEQ32 ? AT(0)  // d already holds the non-equilibrium part
                                    : drho * (px0 + dpx) * phy + (dpx * py0 + px0 * dpy + dpx * dpy);
            const AT neq = d[q][j] - feqdev;
            if (KOMEGA) {
                if (cx != 0) sxx_n += neq;
                if (cy != 0) syy_n += neq;
                if (cx * cy == 1) sxy_n += neq;
                if (cx * cy == -1) sxy_n -= neq;
            }
            if (NEQ32)  // the post-collision value minus feq(rho, u) (stored as is)
                d[q][j] = (AT(1) - w) * neq + AT(weight_of(q)) * (cdr + AT(3 * cx) * cdjx + AT(3 * cy) * cdjy) +
                          rho * phy * dphiF<AT>(cx, ux, fterm);
            else
                d[q][j] = d[q][j] - w * neq + rho * phy * dphiF<AT>(cx, ux, fterm);
        }
        o_u0[j] = (float)ux;
        if (KOMEGA) {
            const AT s = AT(-1.5) * tau0 * inv;
            o_s[0][j] = (FT)(s * sxx_n);
            o_s[1][j] = (FT)(s * sxy_n);
            o_s[2][j] = (FT)(s * syy_n);
        }
        o_rho[j] = (FT)rho;
        o_ux[j] = (FT)(ux + fterm / AT(2));
        o_uy[j] = (FT)uy;
        bsum_rho += (double)rho;
        bsum_ux += (double)(ux + fterm / AT(2));
        bsum_uy += (double)uy;
    }

    // ---- stores -----------------------------------------------------------------
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        VT v[4];
        const AT fe_row = ROW ? AT(row_feq(q, y)) : AT(0);  // this row's reference
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (ROW)
                v[j] = fl[j] ? (VT)((d[q][j] - fe_row) * AT(NEQ_SCALE)) : VT(0);
            else if (NEQ32)
                v[j] = fl[j] ? (VT)(d[q][j] * AT(NEQ_SCALE)) : VT(0);
            else if (NEQ)
                v[j] = fl[j] ? (VT)((d[q][j] - AT(feq_dev_f32(q, o_rho[j], o_ux[j], o_uy[j]))) * AT(NEQ_SCALE))
                             : VT(0);
            else
                v[j] = (VT)d[q][j];
        }
        Store<ST>::store4(gout + q * D + rowoff + x0, v);
    }
    if (NEQ) {
        *reinterpret_cast<float4*>(p.ref_out + rowoff + x0) = make_float4(o_rho[0], o_rho[1], o_rho[2], o_rho[3]);
        if (NEQ32)
            *reinterpret_cast<float4*>(p.ref_out + D + rowoff + x0) = make_float4(o_u0[0], o_u0[1], o_u0[2], o_u0[3]);
        else
            *reinterpret_cast<float4*>(p.ref_out + D + rowoff + x0) = make_float4(o_ux[0], o_ux[1], o_ux[2], o_ux[3]);
        *reinterpret_cast<float4*>(p.ref_out + 2 * D + rowoff + x0) = make_float4(o_uy[0], o_uy[1], o_uy[2], o_uy[3]);
    }
    if (p.options & OPTION_SAVE_MACRO_FIELDS) {
        fld_st4(static_cast<FT*>(p.rho) + rowoff + x0, o_rho);
        fld_st4(static_cast<FT*>(p.ux) + rowoff + x0, o_ux);
        fld_st4(static_cast<FT*>(p.uy) + rowoff + x0, o_uy);
    }
    if (KOMEGA) {
        fld_st4(static_cast<FT*>(p.nut) + rowoff + x0, o_nut);
#pragma unroll
        for (int c = 0; c < 3; ++c) fld_st4(fS + c * D + rowoff + x0, o_s[c]);
    }

    // ---- per-block FP64 partial sums of rho, ux, uy ----------------------------
    if (slot) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            bsum_rho += __shfl_down_sync(0xffffffffu, bsum_rho, off);
            bsum_ux += __shfl_down_sync(0xffffffffu, bsum_ux, off);
            bsum_uy += __shfl_down_sync(0xffffffffu, bsum_uy, off);
        }
        if (lane == 0) { slot[0] = bsum_rho; slot[1] = bsum_ux; slot[2] = bsum_uy; }
    }
}

template <typename ST, typename AT, bool KOMEGA, bool PHASE0, bool NEQ = false, typename FT = float, bool ROW = false>
__global__ void __launch_bounds__(128, ((NEQ && sizeof(AT) == 8) || sizeof(FT) == 8) ? 1 : KOFM_LB_MINBLOCKS)
lb_step_kernel(const LbParams p) {
    lb_block<ST, AT, KOMEGA, PHASE0, NEQ, FT, ROW>(p, blockIdx.x, blockIdx.y, gridDim.x);
}

// A tile of the multi-lattice collide: `rows` block rows from `by` of block
// column `bx` of lattice `lat`.
struct LbTile {
    int lat, bx, by, rows;
};

// The collide of several lattices (same storage form and model) in one
// persistent launch: the blocks walk a tile table; each tile's lattice
// parameters are staged in shared memory.  Per node the same arithmetic and
// the same partial-sum slots as lb_step_kernel.
template <typename ST, typename AT, bool KOMEGA, bool NEQ = false, typename FT = float>
__global__ void __launch_bounds__(128, ((NEQ && sizeof(AT) == 8) || sizeof(FT) == 8) ? 1 : KOFM_LB_MINBLOCKS)
lb_multi_kernel(const LbParams* __restrict__ lats, const LbTile* __restrict__ tiles, int ntiles) {
    __shared__ LbParams sp;
    constexpr int NW = (int)(sizeof(LbParams) / sizeof(unsigned long long));
    static_assert(sizeof(LbParams) % sizeof(unsigned long long) == 0, "staged as 8-byte words");
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    int cur = -1;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const LbTile T = tiles[t];
        if (T.lat != cur) {  // block-uniform
            __syncthreads();  // every warp is done with the previous lattice's parameters
            if (tid < NW)
                reinterpret_cast<unsigned long long*>(&sp)[tid] =
                    reinterpret_cast<const unsigned long long*>(lats + T.lat)[tid];
            __syncthreads();
            cur = T.lat;
        }
        for (int r = 0; r < T.rows; ++r)
            lb_block<ST, AT, KOMEGA, false, NEQ, FT>(sp, T.bx, T.by + r, sp.P / 128);
    }
}

}  // namespace kofm
