// kofm_thermal.cuh - the thermal implicit finite-difference update
// (clVariablesFD::Solve, clVariablesFD.h:343-358) on the device (sm_100a).
//
//  * thermal_assemble_kernel: Update_T_Coeffs_Implicit (tfdKernels.cl:122-279)
//    fused with the sparsity pattern of the reference's non-periodic CSR_Inds
//    (SparseMatrix.cpp:57-209): one thread per node writes the four
//    off-diagonals (divided by the diagonal, which becomes 1) in the
//    interleaved layout ilv(4, q, g) and the right-hand side.
//  * bicgstab_kernel: BiCGStabSolver::solve (BiCGStabSolver.cpp:628-723) as
//    the reference enqueues it, in ONE cooperative launch.  The reference
//    never reduces omega (its omegaDotSqr kernels are built but not run), so
//    omega stays at the 1 its scalar buffer is filled with and the step-f9
//    reduction recomputes the same alpha; the convergence checks use L1 norms
//    (the "Norm" reduction, BiCGStabGenerator.cpp:259-262) against ||b||_1,
//    and the NaN / tenfold-growth test of reduceAndCheckConvergence
//    (BiCGStabSolver.cpp:509-545) ends the solve for the host's dt halving.
//    Instead of the reference's ~25 kernels and 4 host reads per iteration:
//      R: r = b - A x, r0 = r, ||b||_1, <r, r>         (once)
//      B: p = r + beta (p - omega v) on the fly at the node and its four
//         neighbours (iteration 0: p = r0), v = A p, <v, r0>   -> alpha
//      C: s = r - alpha v, ||s||_1                     -> first check
//      D: t = A s on the fly, x = (x + alpha p) + omega s, r = s - omega t,
//         ||r||_1, <r, r0>                             -> second check, beta
//    p and v are double-buffered (a pass reads the old values at the
//    neighbours while it writes the new ones); p of iteration 0 is r0 itself.
//    Threads take node pairs (16-byte loads and stores; the pair shares its
//    row neighbours).  Grid barriers, partial sums and the last-block serial
//    section are those of the k-omega solver.
#pragma once
#include "kofm_gmres.cuh"

namespace kofm {

// row kinds of the thermal system (CSR_Inds with M0_SOLID, M0_FLUID,
// SOLID_BOUNDARY0; clVariablesFD.h:40)
enum ThRow : int { TH_EMPTY = 0, TH_DIAG = 1, TH_FULL = 2 };

__device__ __forceinline__ int th_row(int t, int x, int nx) {
    if (x >= nx) return TH_EMPTY;
    if (t & M0_SOLID) return (t & SOLID_BOUNDARY0) ? TH_DIAG : TH_EMPTY;
    return TH_FULL;
}

struct ThermalAsm {
    const int16_t* ntype;
    const int32_t* dxidx;     // per-node link-fraction record (-1: all 1)
    const DxRecord* dxrec;
    const float* ux;
    const float* uy;
    const float* nut;         // nullptr without k-omega
    const double* T;
    double* Tprev;            // copy of T (first sub-step of an update), or nullptr
    double* coef;             // [4 x D] E, W, N, S (interleaved)
    double* b;                // [D]
    int nx, ny, P;
    double alpha_fluid, alpha_foul, prt_inv, t_in, dt;
};

// Update_T_Coeffs_Implicit for node (x, y); rows of unfouled-wall nodes and
// padding columns are left as they are.
__global__ void thermal_assemble_kernel(const ThermalAsm p) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= p.P || y >= p.ny) return;
    const long long g = (long long)y * p.P + x;
    if (p.Tprev) p.Tprev[g] = p.T[g];  // copyToPrevSolution (BiCGStabSolver.cpp:572-578)
    if (x >= p.nx) return;
    const int t = (uint16_t)p.ntype[g];
    if (t & M0_SOLID) return;
    // 3-point weights of the first and second derivatives; whole links (no
    // record) give the exact constants 1/2, -1/2, 0 and 1, 1, -2
    double dXe = 0.5, dXw = -0.5, dXc = 0.0, dYn = 0.5, dYs = -0.5, dYc = 0.0;
    double dX2e = 1.0, dX2w = 1.0, dX2c = -2.0, dY2n = 1.0, dY2s = 1.0, dY2c = -2.0;
    const int r = p.dxidx[g];
    if (r >= 0) {
        const DxRecord rec = p.dxrec[r];
        const double dxe = fmax(rec.dx[0], 0.1), dxw = fmax(rec.dx[1], 0.1), dxc = fmax(dxe + dxw, 0.1);
        const double dyn = fmax(rec.dx[2], 0.1), dys = fmax(rec.dx[3], 0.1), dyc = fmax(dyn + dys, 0.1);
        dXe = dxw / (dxe * dxc); dXw = -dxe / (dxw * dxc); dXc = (dxe - dxw) / (dxe * dxw);
        dYn = dys / (dyn * dyc); dYs = -dyn / (dys * dyc); dYc = (dyn - dys) / (dyn * dys);
        dX2e = 2. / (dxe * dxc); dX2w = 2. / (dxw * dxc); dX2c = -2. / (dxe * dxw);
        dY2n = 2. / (dyn * dyc); dY2s = 2. / (dys * dyc); dY2c = -2. / (dyn * dys);
        if (fabs(dXc) > 10.) { dXe = 1.0 / dxc; dXw = -1.0 / dxc; dXc = 0.0; }
        if (fabs(dYn) > 10.) { dYn = 1.0 / dyc; dYs = -1.0 / dyc; dYc = 0.0; }
    }
    double alpha = (t & M_SOLID) ? p.alpha_foul : p.alpha_fluid;
    const long long row = (long long)y * p.P;
    const long long gw = row + (x > 0 ? x - 1 : p.nx - 1), ge = row + (x < p.nx - 1 ? x + 1 : 0);
    double nu_c = 0.0, nu_e = 0.0, nu_w = 0.0, nu_n = 0.0, nu_s = 0.0;
    if (p.nut) {
        nu_c = p.nut[g]; nu_e = p.nut[ge]; nu_w = p.nut[gw];
        nu_n = p.nut[g + p.P]; nu_s = p.nut[g - p.P];
    }
    const double alphat = nu_c * p.prt_inv;
    const double Jx = (double)p.ux[g] - (p.prt_inv * (dXe * nu_e + dXw * nu_w + dXc * alphat));
    const double Jy = (double)p.uy[g] - (p.prt_inv * (dYn * nu_n + dYs * nu_s + dYc * alphat));
    alpha += alphat;
    double Tsrc = fmin(fmax(0.0, p.T[g]), p.t_in);
    double Cc = 1. + p.dt * (Jx * dXc + Jy * dYc - alpha * (dX2c + dY2c));
    const double Sc = p.dt * (Jy * dYs - alpha * dY2s);
    const double Wc = p.dt * (Jx * dXw - alpha * dX2w);
    if (x == 0) Tsrc -= p.t_in * Wc;           // inlet: fixed temperature
    const double Ec = p.dt * (Jx * dXe - alpha * dX2e);
    if (x == p.nx - 1) Cc += Ec;                // outlet: zero gradient
    Cc = 1. / Cc;
    p.coef[ilv(4, 0, g)] = x < p.nx - 1 ? Ec * Cc : 0.0;
    p.coef[ilv(4, 1, g)] = x > 0 ? Wc * Cc : 0.0;
    p.coef[ilv(4, 2, g)] = p.dt * (Jy * dYn - alpha * dY2n) * Cc;
    p.coef[ilv(4, 3, g)] = Sc * Cc;
    p.b[g] = Tsrc * Cc;
}

// ---- BiCGStab -------------------------------------------------------------------
struct ThermalCtl {
    int error;        // 1: barrier timeout
    int state;        // TH_RUNNING / TH_CONV / TH_RESET / TH_MAXIT / TH_TRIVIAL
    int iter;         // iterCount
    int checks;
    int first;        // next check sets the initial residual
    int exit_after_c; // stopped at the check after the s step (x += alpha p pending)
    int passes;
    int pad;
    double normb, rho, alpha, omega, beta, avg, residual, initial_residual;
};
enum ThState : int { TH_RUNNING = 0, TH_CONV = 1, TH_RESET = 2, TH_MAXIT = 3, TH_TRIVIAL = 4 };

struct ThermalArgs {
    const int16_t* ntype;
    const double* coef;
    double* x;                // T
    double* b;                // right-hand side, then the residual r (as the reference)
    double* r0;
    double* p[2];
    double* v[2];
    double* s;
    ThermalCtl* ctl;
    double* part;             // [GM_SLOTS][gridDim.x]
    GridBarrier* bar;
    int nx, ny, P;
    long long D;
    int max_iters;
    double rel_tol, abs_tol;
    int reset_flag;
    long long spin_limit;
};

enum ThSerial : int { TS_NONE = 0, TS_RES0, TS_ALPHA, TS_CHECK1, TS_CHECK2 };

// reduceAndCheckConvergence on the summed L1 norm of the current residual
__device__ void th_check(const ThermalArgs& a, ThermalCtl& C, double l1) {
    const double res = l1 / C.normb;
    C.checks += 1;
    C.residual = res;
    if (C.first) C.initial_residual = res;
    C.first = 0;
    if (a.reset_flag && (isnan(res) || (C.iter > 1 && res > 10. * C.avg))) { C.state = TH_RESET; return; }
    if (res <= a.rel_tol || res <= a.abs_tol * C.initial_residual) { C.state = TH_CONV; return; }
    C.avg = res;
}

__device__ void th_serial(const ThermalArgs& a, int kind, int nblocks) {
    __shared__ double tot[2];
    const int warp = threadIdx.x >> 5;
    const int used = (kind == TS_CHECK2 || kind == TS_RES0) ? 2 : 1;
    if (warp < used) {
        const double v = sum_slot_warp(a.part, nblocks, warp);
        if ((threadIdx.x & 31) == 0) tot[warp] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        ThermalCtl C;
        {
            const unsigned long long* src = reinterpret_cast<const unsigned long long*>(a.ctl);
            unsigned long long* dst = reinterpret_cast<unsigned long long*>(&C);
            for (int i = 0; i < (int)(sizeof(ThermalCtl) / 8); ++i) dst[i] = __ldcg(src + i);
        }
        switch (kind) {
            case TS_RES0:  // step 1 (||b||_1, the b == 0 exit) and step 4 (rho)
                C.normb = tot[0];
                if (C.normb <= 1.0e-16) C.state = TH_TRIVIAL;
                C.rho = tot[1];
                break;
            case TS_ALPHA: C.alpha = C.rho / tot[0]; break;
            case TS_CHECK1:
                th_check(a, C, tot[0]);
                if (C.state != TH_RUNNING) C.exit_after_c = 1;
                break;
            case TS_CHECK2:
                th_check(a, C, tot[0]);
                if (C.state == TH_RUNNING) {
                    C.iter += 1;
                    if (C.iter >= a.max_iters) {
                        C.state = TH_MAXIT;
                    } else {  // Sum_Rho_Calc_Beta (BiCGStabGenerator.cpp:128-142)
                        const double rho_new = tot[1];
                        C.beta = (rho_new / C.rho) * (C.alpha / C.omega);
                        C.rho = rho_new;
                    }
                }
                break;
            default: break;
        }
        C.passes += 1;
        const unsigned long long* src = reinterpret_cast<const unsigned long long*>(&C);
        unsigned long long* dst = reinterpret_cast<unsigned long long*>(a.ctl);
        for (int i = 0; i < (int)(sizeof(ThermalCtl) / 8); ++i) __stcg(dst + i, src[i]);
    }
}

// Bounded grid barrier; the last block to arrive runs the serial section.
__device__ bool th_sync(const ThermalArgs& a, int kind) {
    __shared__ int s_last;
    __shared__ unsigned int s_gen;
    const int nblocks = gridDim.x;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_gen = ld_acquire_u32(&a.bar->gen);
        const unsigned int ticket = atomicAdd(&a.bar->count, 1u);
        s_last = (ticket == (unsigned int)nblocks - 1u);
    }
    __syncthreads();
    if (s_last) {
        __threadfence();
        if (kind != TS_NONE) th_serial(a, kind, nblocks);
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) {
            atomicExch(&a.bar->count, 0u);
            __threadfence();
            atomicAdd(&a.bar->gen, 1u);
        }
    } else if (threadIdx.x == 0) {
        long long it = 0;
        while (ld_acquire_u32(&a.bar->gen) == s_gen) {
            if (++it > a.spin_limit || ldc(&a.ctl->error)) {
                atomicExch(&a.ctl->error, 1);
                break;
            }
            __nanosleep(100);
        }
    }
    __syncthreads();
    return ldc(&a.ctl->error) == 0;
}

__device__ __forceinline__ double2 ld2(const double* p) { return __ldcg(reinterpret_cast<const double2*>(p)); }
__device__ __forceinline__ void st2(double* p, double u, double v) {
    __stcg(reinterpret_cast<double2*>(p), make_double2(u, v));
}

// A times a vector on the node pair (g, g+1), g even: val2(n) gives the
// vector on nodes n, n+1 (n even), val1(n) on one node.  Rows in CSR order
// (S, W, C, E, N); wall-boundary rows are the identity, inner-wall and
// padding rows are empty.
template <typename F2, typename F1>
__device__ __forceinline__ double2 th_apply2(const ThermalArgs& a, long long g, int x, int k0, int k1,
                                             F2&& val2, F1&& val1) {
    if (k0 == TH_EMPTY && k1 == TH_EMPTY) return make_double2(0.0, 0.0);
    const double2 c = val2(g);
    double r0 = k0 == TH_DIAG ? c.x : 0.0, r1 = k1 == TH_DIAG ? c.y : 0.0;
    if (k0 == TH_FULL || k1 == TH_FULL) {
        const double2 sv = val2(g - a.P), nv = val2(g + a.P);
        if (k0 == TH_FULL) {
            double acc = __ldg(a.coef + ilv(4, 3, g)) * sv.x;
            if (x > 0) acc += __ldg(a.coef + ilv(4, 1, g)) * val1(g - 1);
            acc += c.x;
            if (x < a.nx - 1) acc += __ldg(a.coef + ilv(4, 0, g)) * c.y;
            acc += __ldg(a.coef + ilv(4, 2, g)) * nv.x;
            r0 = acc;
        }
        if (k1 == TH_FULL) {
            const long long g1 = g + 1;
            double acc = __ldg(a.coef + ilv(4, 3, g1)) * sv.y;
            acc += __ldg(a.coef + ilv(4, 1, g1)) * c.x;  // x + 1 > 0
            acc += c.y;
            if (x + 1 < a.nx - 1) acc += __ldg(a.coef + ilv(4, 0, g1)) * val1(g + 2);
            acc += __ldg(a.coef + ilv(4, 2, g1)) * nv.y;
            r1 = acc;
        }
    }
    return make_double2(r0, r1);
}

__global__ void __launch_bounds__(GM_THREADS, 4) bicgstab_kernel(const ThermalArgs a) {
    const long long npairs = a.D / 2;
    const long long stride = (long long)gridDim.x * GM_THREADS;
    const long long t0 = (long long)blockIdx.x * GM_THREADS + threadIdx.x;
    auto kinds = [&](long long g, int x, int& k0, int& k1) {
        const unsigned int t2 = *reinterpret_cast<const unsigned int*>(a.ntype + g);
        k0 = th_row((int)(t2 & 0xffff), x, a.nx);
        k1 = th_row((int)(t2 >> 16), x + 1, a.nx);
    };

    // ---- R: steps 1-4: ||b||_1; r = b - A x; r0 = r; rho = <r, r> -------------------
    {
        double acc[2] = {0.0, 0.0};
        auto x2 = [&](long long n) { return ld2(a.x + n); };
        auto x1 = [&](long long n) { return __ldcg(a.x + n); };
        for (long long pr = t0; pr < npairs; pr += stride) {
            const long long g = 2 * pr;
            const int x = (int)(g % a.P);
            int k0, k1;
            kinds(g, x, k0, k1);
            const double2 ax = th_apply2(a, g, x, k0, k1, x2, x1);
            const double2 b = ld2(a.b + g);
            const double r0 = b.x - ax.x, r1 = b.y - ax.y;
            st2(a.b + g, r0, r1);
            st2(a.r0 + g, r0, r1);
            acc[0] += fabs(b.x) + fabs(b.y);
            acc[1] += r0 * r0 + r1 * r1;
        }
        block_reduce_slots<2>(acc, 2, a.part, 0);
    }
    if (!th_sync(a, TS_RES0)) return;
    if (ldc(&a.ctl->state) == TH_TRIVIAL) {
        // b == 0: x = b (BiCGStabSolver.cpp:654-658); b holds r = b - A x now,
        // so b is rebuilt as r + A x into s first, then copied to x and b
        auto x2 = [&](long long n) { return ld2(a.x + n); };
        auto x1 = [&](long long n) { return __ldcg(a.x + n); };
        for (long long pr = t0; pr < npairs; pr += stride) {
            const long long g = 2 * pr;
            const int x = (int)(g % a.P);
            int k0, k1;
            kinds(g, x, k0, k1);
            const double2 ax = th_apply2(a, g, x, k0, k1, x2, x1);
            const double2 r = ld2(a.b + g);
            st2(a.s + g, r.x + ax.x, r.y + ax.y);
        }
        if (!th_sync(a, TS_NONE)) return;
        for (long long pr = t0; pr < npairs; pr += stride) {
            const long long g = 2 * pr;
            const double2 v = ld2(a.s + g);
            st2(a.x + g, v.x, v.y);
            st2(a.b + g, v.x, v.y);
        }
        return;
    }

    const double* pcur = a.r0;  // p of the last iteration (iteration 0: r0 = r)
    int vc = 0;                 // v of the last iteration
    for (int it = 0; it < a.max_iters; ++it) {
        // ---- B: p = r + beta (p - omega v), v = A p, <v, r0> -------------------------
        double* pnew = (pcur == a.p[0]) ? a.p[1] : a.p[0];
        {
            const double beta = ldc(&a.ctl->beta), omega = ldc(&a.ctl->omega);
            const double* vold = a.v[vc];
            double* vnew = a.v[vc ^ 1];
            auto p2 = [&](long long n) -> double2 {
                const double2 po = ld2(pcur + n);
                if (it == 0) return po;
                const double2 r = ld2(a.b + n), vo = ld2(vold + n);
                return make_double2(r.x + beta * (po.x - omega * vo.x), r.y + beta * (po.y - omega * vo.y));
            };
            auto p1 = [&](long long n) -> double {
                const double po = __ldcg(pcur + n);
                if (it == 0) return po;
                return __ldcg(a.b + n) + beta * (po - omega * __ldcg(vold + n));
            };
            double acc[1] = {0.0};
            for (long long pr = t0; pr < npairs; pr += stride) {
                const long long g = 2 * pr;
                const int x = (int)(g % a.P);
                int k0, k1;
                kinds(g, x, k0, k1);
                const double2 v = th_apply2(a, g, x, k0, k1, p2, p1);
                if (it > 0) {
                    const double2 pv = p2(g);
                    st2(pnew + g, pv.x, pv.y);
                }
                st2(vnew + g, v.x, v.y);
                const double2 rr = ld2(a.r0 + g);
                acc[0] += v.x * rr.x + v.y * rr.y;
            }
            block_reduce_slots<1>(acc, 1, a.part, 0);
        }
        if (it > 0) pcur = pnew;
        vc ^= 1;
        if (!th_sync(a, TS_ALPHA)) return;
        // ---- C: s = r - alpha v, ||s||_1 ---------------------------------------------
        const double alpha = ldc(&a.ctl->alpha);
        {
            const double* v = a.v[vc];
            double acc[1] = {0.0};
            for (long long pr = t0; pr < npairs; pr += stride) {
                const long long g = 2 * pr;
                const double2 r = ld2(a.b + g), vv = ld2(v + g);
                const double s0 = r.x - alpha * vv.x, s1 = r.y - alpha * vv.y;
                st2(a.s + g, s0, s1);
                acc[0] += fabs(s0) + fabs(s1);
            }
            block_reduce_slots<1>(acc, 1, a.part, 0);
        }
        if (!th_sync(a, TS_CHECK1)) return;
        if (ldc(&a.ctl->state) != TH_RUNNING) {
            // shCalc's x += alpha p and r = s stand (BiCGStabSolver.cpp:694-701)
            for (long long pr = t0; pr < npairs; pr += stride) {
                const long long g = 2 * pr;
                const double2 xv = ld2(a.x + g), pv = ld2(pcur + g), sv = ld2(a.s + g);
                st2(a.x + g, xv.x + alpha * pv.x, xv.y + alpha * pv.y);
                st2(a.b + g, sv.x, sv.y);
            }
            return;
        }
        // ---- D: t = A s, x = (x + alpha p) + omega s, r = s - omega t ------------------
        {
            const double omega = ldc(&a.ctl->omega);
            auto s2 = [&](long long n) { return ld2(a.s + n); };
            auto s1 = [&](long long n) { return __ldcg(a.s + n); };
            double acc[2] = {0.0, 0.0};
            for (long long pr = t0; pr < npairs; pr += stride) {
                const long long g = 2 * pr;
                const int x = (int)(g % a.P);
                int k0, k1;
                kinds(g, x, k0, k1);
                const double2 t = th_apply2(a, g, x, k0, k1, s2, s1);
                const double2 sv = ld2(a.s + g), xv = ld2(a.x + g), pv = ld2(pcur + g);
                const double xh0 = xv.x + alpha * pv.x, xh1 = xv.y + alpha * pv.y;
                st2(a.x + g, xh0 + omega * sv.x, xh1 + omega * sv.y);
                const double r0 = sv.x - omega * t.x, r1 = sv.y - omega * t.y;
                st2(a.b + g, r0, r1);
                const double2 rr = ld2(a.r0 + g);
                acc[0] += fabs(r0) + fabs(r1);
                acc[1] += r0 * rr.x + r1 * rr.y;
            }
            block_reduce_slots<2>(acc, 2, a.part, 0);
        }
        if (!th_sync(a, TS_CHECK2)) return;
        if (ldc(&a.ctl->state) != TH_RUNNING) return;
    }
}

}  // namespace kofm
