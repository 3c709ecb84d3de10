// kofm_gmres.cuh - device-resident restarted "simpler GMRES" for the two
// k-omega systems (sm_100a).
//
// Algorithm: the reference's GMRESSolver::solve (GMRESSolver.cpp:227-355)
// with the kernels it enqueues (gmresKernels.cl:33-279, GMRESGenerator.cpp
// NormalizeResidual / addInitialGuess): Walker & Zhou's simpler GMRES on the
// correction system A d = b - A x0 with classical Gram-Schmidt, the truncation
// tests on diag(R) and on xi, the residual estimator rho *= sin(acos(xi/rho)),
// the back-substitution with the reference's R indexing, and x = x0 + d.
//
// B200 design: ONE cooperative launch per k-omega update solves both systems
// (omega and k, independent in the reference: kOmega.cpp:68-70) with no host
// round-trip.  The reference needs >= 4 blocking host synchronisations and
// ~40 kernel launches per restart.  Here every sweep is a grid-stride pass
// over node pairs (16-byte FP64 loads); the matrix is applied matrix-free as a
// 5-point stencil with the stored normalised off-diagonals (diagonal = 1);
// Krylov vectors are stored un-normalised and scaled lazily, which removes
// the reference's separate normalisation sweep; dot products are reduced per
// block and combined by the last block to arrive at the grid barrier, which
// also runs the scalar logic (the reference's host code) before releasing
// the grid.  The barrier spin is bounded: on expiry the kernel records
// a timeout in the control block and every block returns.
#pragma once
#include "kofm_common.cuh"
#include "kofm_komega.cuh"

#ifndef KOFM_MAX_KRYLOV
#define KOFM_MAX_KRYLOV 12
#endif

namespace kofm {

constexpr int GM_THREADS = 256;
constexpr int GM_SLOTS = 32;  // partial-sum slots per block (2 systems x 16)

struct GmresSys {
    int active;     // still iterating this restart
    int nan;        // NaN residual seen (resetTimeFunc path)
    int conv;       // converged
    int restarts;   // restart cycles entered
    int iters;      // iterCount
    int kk;         // number of update coefficients used
    double rho0, norm_rhs, rinv, rho, prev_err;
    double s[KOFM_MAX_KRYLOV];   // 1 / ||u_j||
    double h[KOFM_MAX_KRYLOV];   // Gram-Schmidt coefficients of the current k
    double xi[KOFM_MAX_KRYLOV];
    double c[KOFM_MAX_KRYLOV];   // update coefficients
    double R[KOFM_MAX_KRYLOV * KOFM_MAX_KRYLOV];
    double sums[16];
};

struct GmresControl {
    GmresSys sys[2];
    int error;        // 0 ok, 1 barrier timeout
    int passes;       // grid sweeps performed
    int any_active;
    int pad;
};

struct GridBarrier {
    unsigned int count;
    unsigned int gen;
};

struct GmresArgs {
    KoSystem sys[2];
    float* field[2];          // omega, k (FP32 fields, updated in place)
    const int16_t* ntype;
    GmresControl* ctl;
    double* part;             // [gridDim.x][GM_SLOTS]
    GridBarrier* bar;
    int nx, ny, P;
    long long D;
    int K;                    // Krylov dimension
    int max_restarts;
    double rel_tol, abs_tol;
    long long spin_limit;     // barrier spin bound (iterations of ~100 ns)
};

// ---- memory helpers: vectors written inside the launch are read through L2 --
__device__ __forceinline__ double2 ldv2(const double* p) { return __ldcg(reinterpret_cast<const double2*>(p)); }
__device__ __forceinline__ double ldv(const double* p) { return __ldcg(p); }
__device__ __forceinline__ void stv2(double* p, double a, double b) {
    __stcg(reinterpret_cast<double2*>(p), make_double2(a, b));
}

// The control block is written by whichever block runs a serial section and
// read by all blocks, so every access bypasses L1 (ld.cg / st.cg).
template <typename T>
__device__ __forceinline__ T ldc(const T* p) { return __ldcg(p); }

__device__ void sys_load(GmresSys& dst, const GmresSys* src) {
    static_assert(sizeof(GmresSys) % 8 == 0, "GmresSys must be 8-byte granular");
    const unsigned long long* s = reinterpret_cast<const unsigned long long*>(src);
    unsigned long long* d = reinterpret_cast<unsigned long long*>(&dst);
    for (int i = 0; i < (int)(sizeof(GmresSys) / 8); ++i) d[i] = __ldcg(s + i);
}
__device__ void sys_store(GmresSys* dst, const GmresSys& src) {
    const unsigned long long* s = reinterpret_cast<const unsigned long long*>(&src);
    unsigned long long* d = reinterpret_cast<unsigned long long*>(dst);
    for (int i = 0; i < (int)(sizeof(GmresSys) / 8); ++i) __stcg(d + i, s[i]);
}

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// ---- block reduction of NS slots into part[blockIdx.x][base + s] ------------
template <int NS>
__device__ __forceinline__ void block_reduce_slots(double (&acc)[NS], int nused, double* part, int base) {
    __shared__ double red[GM_THREADS / 32][GM_SLOTS];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        if (s < nused) {
            double v = acc[s];
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
            if (lane == 0) red[warp][s] = v;
        }
    }
    __syncthreads();
    if (threadIdx.x < nused) {
        double v = 0.0;
#pragma unroll
        for (int w = 0; w < GM_THREADS / 32; ++w) v += red[w][threadIdx.x];
        part[(long long)blockIdx.x * GM_SLOTS + base + threadIdx.x] = v;
    }
    __syncthreads();
}

// Sum slot `slot` of all blocks in block order (deterministic); one warp.
__device__ __forceinline__ double sum_slot_warp(const double* part, int nblocks, int slot) {
    const int lane = threadIdx.x & 31;
    double v = 0.0;
    // each lane sums a contiguous run of blocks, then a fixed tree combines
    const int per = (nblocks + 31) / 32;
    const int b0 = lane * per, b1 = min(nblocks, b0 + per);
    for (int b = b0; b < b1; ++b) v += __ldcg(part + (long long)b * GM_SLOTS + slot);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    return __shfl_sync(0xffffffffu, v, 0);
}

// Phases of the serial section run by the last block at a barrier.
enum SerialKind : int {
    SER_NONE = 0,
    SER_RESIDUAL,   // after r = b' - A x : rho0, convergence
    SER_PROD0,      // after u0 = A r : R(0,0), xi0
    SER_PRODK,      // after z = A u_{k-1} : Gram-Schmidt coefficients h_j
    SER_GS2,        // after u_k = z - sum h_j u_j : R(:,k), xi_k; end of cycle at k = K-1
};

// End of one restart cycle for one system (GMRESSolver.cpp:300-350).
__device__ void cycle_logic(GmresSys& S, int K, double rel_tol) {
    int k = K;
    for (int i = 0; i < k; ++i)
        if (fabs(S.R[i + i * k]) < rel_tol * S.R[0]) { k = i; break; }
    const int full = k;
    for (int i = 0; i < k; ++i) {
        S.iters += 1;
        if (S.xi[i] >= S.rho || S.xi[i] <= -S.rho) { k = i; break; }
        S.rho *= sin(acos(S.xi[i] / S.rho));
    }
    for (int i2 = k - 1; i2 > -1; --i2) {
        for (int j = i2 + 1; j < k; ++j) S.xi[i2] -= S.R[i2 + j * full] * S.xi[j];
        S.xi[i2] /= S.R[i2 + i2 * full];
    }
    for (int i = 0; i < k; ++i) S.xi[i] *= S.rho0;
    for (int i = 0; i < K; ++i) S.c[i] = S.xi[i];
    S.kk = k;
    S.prev_err = fabs(S.rho * S.rho0 / S.norm_rhs);
}

// Serial section: executed by all threads of the last-arriving block.
__device__ void serial_section(const GmresArgs& a, int kind, int kcur, int restart, int nblocks) {
    GmresControl* ctl = a.ctl;
    __shared__ double tot[GM_SLOTS];
    // 1) deterministic totals of the used slots
    const int warp = threadIdx.x >> 5, nwarps = GM_THREADS / 32;
    for (int slot = warp; slot < GM_SLOTS; slot += nwarps) {
        const double v = sum_slot_warp(a.part, nblocks, slot);
        if ((threadIdx.x & 31) == 0) tot[slot] = v;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    int any = 0;
    for (int s = 0; s < 2; ++s) {
        GmresSys S;
        sys_load(S, &ctl->sys[s]);
        if (!S.active) continue;
        const double* t = tot + 16 * s;
        switch (kind) {
            case SER_RESIDUAL: {
                S.rho0 = sqrt(t[0]);
                if (restart == 0) S.norm_rhs = S.rho0;
                S.rinv = 1.0 / S.rho0;
                S.rho = 1.0;
                const double resid = S.rho0 / S.norm_rhs;
                if (isnan(resid)) { S.nan = 1; S.active = 0; }
                else if (resid <= a.rel_tol || S.rho0 <= a.abs_tol) { S.conv = 1; S.active = 0; }
                else { S.restarts += 1; }
                break;
            }
            case SER_PROD0: {
                const double n0 = sqrt(t[0]);
                S.s[0] = 1.0 / n0;
                for (int i = 0; i < a.K * a.K; ++i) S.R[i] = 0.0;
                S.R[0] = S.rinv * n0;                  // ||A r|| with r = r_raw / rho0
                S.xi[0] = S.rinv * t[1] * S.s[0];      // <r, v_0>
                if (a.K == 1) cycle_logic(S, a.K, a.rel_tol);
                break;
            }
            case SER_PRODK: {
                for (int j = 0; j < kcur; ++j) S.h[j] = S.s[kcur - 1] * S.s[j] * t[j];
                break;
            }
            case SER_GS2: {
                const double nk = sqrt(t[0]);
                S.s[kcur] = 1.0 / nk;
                for (int j = 0; j < kcur; ++j) S.R[j + kcur * a.K] = S.h[j];
                S.R[kcur + kcur * a.K] = nk;
                S.xi[kcur] = S.rinv * t[1] * S.s[kcur];
                if (kcur == a.K - 1) cycle_logic(S, a.K, a.rel_tol);
                break;
            }
            default: break;
        }
        any |= S.active;
        sys_store(&ctl->sys[s], S);
    }
    __stcg(&ctl->any_active, any);
    __stcg(&ctl->passes, ldc(&ctl->passes) + 1);
}

// Bounded grid barrier with a serial section run by the last block to arrive.
// Returns false if the wait expired (the control block's error is set).
__device__ bool grid_sync(const GmresArgs& a, int kind, int kcur, int restart) {
    __shared__ int s_last;
    __shared__ unsigned int s_gen;
    const int nblocks = gridDim.x;
    __threadfence();  // this thread's vector and partial-sum stores, device-wide
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_gen = ld_acquire_u32(&a.bar->gen);
        const unsigned int ticket = atomicAdd(&a.bar->count, 1u);
        s_last = (ticket == (unsigned int)nblocks - 1u);
    }
    __syncthreads();
    bool ok = true;
    if (s_last) {
        __threadfence();
        if (kind != SER_NONE) serial_section(a, kind, kcur, restart, nblocks);
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
    if (ldc(&a.ctl->error)) ok = false;
    return ok;
}

// ---- 5-point stencil application on a node pair -----------------------------
// y = v + cE v_e + cW v_w + cN v_n + cS v_s, in the CSR order of an interior
// row (S, W, C, E, N).  scale multiplies v (lazy normalisation).
struct PairCtx {
    long long g;     // node index of the left node of the pair
    int x, y;
    bool f0, f1;     // fluid flags
};

__device__ __forceinline__ void stencil_pair(const GmresArgs& a, const double* coef,
                                             const double* v, const PairCtx& pc, double scale,
                                             double& y0, double& y1, double& c0, double& c1) {
    const long long D = a.D, g = pc.g;
    const double2 cc = ldv2(v + g);
    const double2 nn = ldv2(v + g + a.P);
    const double2 ss = ldv2(v + g - a.P);
    const long long row = (long long)pc.y * a.P;
    const int x = pc.x, nx = a.nx;
    // periodic neighbours over nx: west of x, east of x, east of x+1
    const double vw0 = ldv(v + row + (x > 0 ? x - 1 : nx - 1));
    const double ve0 = x + 1 < nx ? cc.y : ldv(v + row);
    const double ve1 = x + 2 < nx ? ldv(v + row + x + 2) : ldv(v + row + (x + 2 - nx));
    const double2 cE = __ldg(reinterpret_cast<const double2*>(coef + g));
    const double2 cW = __ldg(reinterpret_cast<const double2*>(coef + D + g));
    const double2 cN = __ldg(reinterpret_cast<const double2*>(coef + 2 * D + g));
    const double2 cS = __ldg(reinterpret_cast<const double2*>(coef + 3 * D + g));
    const double r0 = cS.x * ss.x + cW.x * vw0 + cc.x + cE.x * ve0 + cN.x * nn.x;
    const double r1 = cS.y * ss.y + cW.y * cc.x + cc.y + cE.y * ve1 + cN.y * nn.y;
    y0 = pc.f0 ? scale * r0 : 0.0;
    y1 = pc.f1 ? scale * r1 : 0.0;
    c0 = cc.x;
    c1 = cc.y;
}

__device__ __forceinline__ bool pair_ctx(const GmresArgs& a, long long pair, PairCtx& pc) {
    pc.g = pair * 2;
    pc.y = (int)(pc.g / a.P);
    pc.x = (int)(pc.g - (long long)pc.y * a.P);
    if (pc.x >= a.nx) return false;
    const unsigned int t2 = *reinterpret_cast<const unsigned int*>(a.ntype + pc.g);
    const int t0 = t2 & 0xffff, t1 = t2 >> 16;
    pc.f0 = !(t0 & M_SOLID);
    pc.f1 = (pc.x + 1 < a.nx) && !(t1 & M_SOLID);
    return pc.f0 || pc.f1;
}

// ---- the solver kernel ----------------------------------------------------------
__global__ void __launch_bounds__(GM_THREADS)
gmres_kernel(const GmresArgs a) {
    GmresControl* ctl = a.ctl;
    const long long npairs = a.D / 2;
    const long long stride = (long long)gridDim.x * GM_THREADS;
    const long long t0 = (long long)blockIdx.x * GM_THREADS + threadIdx.x;
    const int K = a.K;
    __shared__ double sh_c[2][KOFM_MAX_KRYLOV];
    __shared__ int sh_act[2];

    for (int restart = 0; restart < a.max_restarts; ++restart) {
        // ---- P0: residual r = b' - A x (restart 0: x = 0, r = b') ------------
        for (int s = 0; s < 2; ++s) {
            if (threadIdx.x == 0) sh_act[s] = ldc(&ctl->sys[s].active);
        }
        __syncthreads();
        for (int s = 0; s < 2; ++s) {
            double acc[1] = {0.0};
            if (sh_act[s]) {
                const KoSystem& S = a.sys[s];
                for (long long pr = t0; pr < npairs; pr += stride) {
                    PairCtx pc;
                    if (!pair_ctx(a, pr, pc)) continue;
                    double r0, r1;
                    if (restart == 0) {
                        const double2 b = ldv2(S.rhs + pc.g);
                        r0 = pc.f0 ? b.x : 0.0;
                        r1 = pc.f1 ? b.y : 0.0;
                    } else {
                        double y0, y1, c0, c1;
                        stencil_pair(a, S.coef, S.x, pc, 1.0, y0, y1, c0, c1);
                        const double2 b = ldv2(S.rhs + pc.g);
                        r0 = pc.f0 ? b.x - y0 : 0.0;
                        r1 = pc.f1 ? b.y - y1 : 0.0;
                    }
                    stv2(S.r + pc.g, r0, r1);
                    acc[0] += r0 * r0 + r1 * r1;
                }
            }
            block_reduce_slots<1>(acc, sh_act[s] ? 1 : 0, a.part, 16 * s);
        }
        if (!grid_sync(a, SER_RESIDUAL, 0, restart)) return;
        if (!ldc(&ctl->any_active)) break;

        // ---- k = 0: u0 = A r ----------------------------------------------------
        for (int s = 0; s < 2; ++s) {
            if (threadIdx.x == 0) sh_act[s] = ldc(&ctl->sys[s].active);
        }
        __syncthreads();
        for (int s = 0; s < 2; ++s) {
            double acc[2] = {0.0, 0.0};
            if (sh_act[s]) {
                const KoSystem& S = a.sys[s];
                for (long long pr = t0; pr < npairs; pr += stride) {
                    PairCtx pc;
                    if (!pair_ctx(a, pr, pc)) continue;
                    double y0, y1, c0, c1;
                    stencil_pair(a, S.coef, S.r, pc, 1.0, y0, y1, c0, c1);
                    stv2(S.V + pc.g, y0, y1);
                    acc[0] += y0 * y0 + y1 * y1;
                    acc[1] += c0 * y0 + c1 * y1;
                }
            }
            block_reduce_slots<2>(acc, sh_act[s] ? 2 : 0, a.part, 16 * s);
        }
        if (!grid_sync(a, SER_PROD0, 0, restart)) return;

        for (int k = 1; k < K; ++k) {
            // ---- z = A u_{k-1} (stored in V[k]); <z, u_j>, j < k ---------------
            for (int s = 0; s < 2; ++s) {
                if (threadIdx.x == 0) sh_act[s] = ldc(&ctl->sys[s].active);
            }
            __syncthreads();
            for (int s = 0; s < 2; ++s) {
                double acc[KOFM_MAX_KRYLOV];
#pragma unroll
                for (int j = 0; j < KOFM_MAX_KRYLOV; ++j) acc[j] = 0.0;
                if (sh_act[s]) {
                    const KoSystem& S = a.sys[s];
                    const double* up = S.V + (long long)(k - 1) * a.D;
                    double* zp = S.V + (long long)k * a.D;
                    for (long long pr = t0; pr < npairs; pr += stride) {
                        PairCtx pc;
                        if (!pair_ctx(a, pr, pc)) continue;
                        double y0, y1, c0, c1;
                        stencil_pair(a, S.coef, up, pc, 1.0, y0, y1, c0, c1);
                        stv2(zp + pc.g, y0, y1);
#pragma unroll
                        for (int j = 0; j < KOFM_MAX_KRYLOV; ++j) {
                            if (j < k - 1) {
                                const double2 u = ldv2(S.V + (long long)j * a.D + pc.g);
                                acc[j] += y0 * u.x + y1 * u.y;
                            } else if (j == k - 1) {
                                acc[j] += y0 * c0 + y1 * c1;
                            }
                        }
                    }
                }
                block_reduce_slots<KOFM_MAX_KRYLOV>(acc, sh_act[s] ? k : 0, a.part, 16 * s);
            }
            if (!grid_sync(a, SER_PRODK, k, restart)) return;

            // ---- u_k = s_{k-1} z - sum_j h_j s_j u_j ; ||u_k||^2, <r, u_k> ------
            for (int s = 0; s < 2; ++s) {
                if (threadIdx.x < k) sh_c[s][threadIdx.x] =
                    ldc(&ctl->sys[s].h[threadIdx.x]) * ldc(&ctl->sys[s].s[threadIdx.x]);
                if (threadIdx.x == 0) sh_act[s] = ldc(&ctl->sys[s].active);
            }
            __syncthreads();
            for (int s = 0; s < 2; ++s) {
                double acc[2] = {0.0, 0.0};
                if (sh_act[s]) {
                    const KoSystem& S = a.sys[s];
                    const double sk1 = ldc(&ctl->sys[s].s[k - 1]);
                    double* zp = S.V + (long long)k * a.D;
                    for (long long pr = t0; pr < npairs; pr += stride) {
                        PairCtx pc;
                        if (!pair_ctx(a, pr, pc)) continue;
                        const double2 z = ldv2(zp + pc.g);
                        double v0 = sk1 * z.x, v1 = sk1 * z.y;
#pragma unroll
                        for (int j = 0; j < KOFM_MAX_KRYLOV; ++j) {
                            if (j < k) {
                                const double2 u = ldv2(S.V + (long long)j * a.D + pc.g);
                                v0 -= sh_c[s][j] * u.x;
                                v1 -= sh_c[s][j] * u.y;
                            }
                        }
                        if (!pc.f0) v0 = 0.0;
                        if (!pc.f1) v1 = 0.0;
                        stv2(zp + pc.g, v0, v1);
                        const double2 r = ldv2(S.r + pc.g);
                        acc[0] += v0 * v0 + v1 * v1;
                        acc[1] += r.x * v0 + r.y * v1;
                    }
                }
                block_reduce_slots<2>(acc, sh_act[s] ? 2 : 0, a.part, 16 * s);
            }
            if (!grid_sync(a, SER_GS2, k, restart)) return;
        }
        // ---- x += c0 rinv r + sum_{j>=1} c_j s_{j-1} u_{j-1} --------------------------
        for (int s = 0; s < 2; ++s) {
            if (threadIdx.x == 0) {
                sh_act[s] = ldc(&ctl->sys[s].active);
            }
            if (threadIdx.x < K) {
                const GmresSys* S = &ctl->sys[s];
                const int j = threadIdx.x;
                const int kk = ldc(&S->kk);
                sh_c[s][j] = j == 0 ? ldc(&S->c[0]) * ldc(&S->rinv)
                                    : (j < kk ? ldc(&S->c[j]) * ldc(&S->s[j - 1]) : 0.0);
            }
        }
        __syncthreads();
        for (int s = 0; s < 2; ++s) {
            if (!sh_act[s]) continue;
            const KoSystem& S = a.sys[s];
            for (long long pr = t0; pr < npairs; pr += stride) {
                PairCtx pc;
                if (!pair_ctx(a, pr, pc)) continue;
                double2 xv = make_double2(0.0, 0.0);
                if (restart > 0) xv = ldv2(S.x + pc.g);
                const double2 r = ldv2(S.r + pc.g);
                double v0 = xv.x + sh_c[s][0] * r.x, v1 = xv.y + sh_c[s][0] * r.y;
                for (int j = 1; j < K; ++j) {
                    const double cj = sh_c[s][j];
                    if (cj == 0.0) continue;
                    const double2 u = ldv2(S.V + (long long)(j - 1) * a.D + pc.g);
                    v0 += cj * u.x;
                    v1 += cj * u.y;
                }
                stv2(S.x + pc.g, v0, v1);
            }
        }
        if (!grid_sync(a, SER_NONE, 0, restart)) return;
    }

    // ---- x_new = x0 + d on fluid nodes; solid-boundary rows -> 0 -----------------
    for (int s = 0; s < 2; ++s) {
        const KoSystem& S = a.sys[s];
        float* f = a.field[s];
        const bool has_x = ldc(&ctl->sys[s].restarts) > 0;
        for (long long pr = t0; pr < npairs; pr += stride) {
            const long long g = pr * 2;
            const int y = (int)(g / a.P), x = (int)(g - (long long)y * a.P);
            if (x >= a.nx) continue;
            const unsigned int t2 = *reinterpret_cast<const unsigned int*>(a.ntype + g);
            const int tt[2] = {(int)(t2 & 0xffff), (int)(t2 >> 16)};
            const double2 xv = has_x ? ldv2(S.x + g) : make_double2(0.0, 0.0);
            const double dv[2] = {xv.x, xv.y};
            for (int j = 0; j < 2; ++j) {
                if (x + j >= a.nx) continue;
                if (!(tt[j] & M_SOLID)) f[g + j] = (float)((double)f[g + j] + dv[j]);
                else if (tt[j] & SOLID_BOUNDARY) f[g + j] = 0.f;
            }
        }
    }
}

}  // namespace kofm
