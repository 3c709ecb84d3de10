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
// B200 design
//  * ONE cooperative launch per k-omega update solves both systems (omega and
//    k are independent in the reference, kOmega.cpp:68-70) with no host
//    round-trip; the reference needs >= 4 blocking host synchronisations and
//    ~40 kernel launches per restart.
//  * One fused sweep per Krylov vector.  For vector k a block stages, for a
//    64x8 tile, u_{k-1} on a 2-node ring and the stencil coefficients on a
//    1-node ring in shared memory, recomputes z_k = A u_{k-1} on the 1-ring,
//    orthogonalises u_k = s_{k-1} z_k - sum_j h_j s_j u_j there (classical
//    Gram-Schmidt, the reference's order), writes u_k, and applies the
//    stencil once more to get w = A u_k for the NEXT vector's Gram-Schmidt
//    dot products -- so each vector costs one sweep and one grid barrier
//    instead of the reference's product / two Gram-Schmidt stages / normalise.
//    Krylov vectors are kept un-normalised; the scales 1/||u_j|| are applied
//    lazily in FP64.
//  * Streamed vectors (basis, residual, coefficients, right-hand side) are
//    FP32 in HBM; every product and dot product is FP64.
//  * Dot products are reduced per block and combined, in a fixed order, by
//    the last block to reach the grid barrier, which also runs the scalar
//    logic (the reference's host code) before releasing the grid.  The
//    barrier spin is bounded: on expiry the control block records a timeout
//    and every block returns.
#pragma once
#include "kofm_common.cuh"
#include "kofm_komega.cuh"

#ifndef KOFM_MAX_KRYLOV
#define KOFM_MAX_KRYLOV 12
#endif

namespace kofm {

constexpr int GM_THREADS = 256;
constexpr int GM_SLOTS = 32;                    // partial-sum slots per block
constexpr int GM_SYS_SLOTS = 16;                // per system
constexpr int TW = 64, TH = 8;                  // tile
constexpr int R1W = TW + 2, R1H = TH + 2;       // tile + 1-node ring
constexpr int R2W = TW + 4, R2H = TH + 4;       // tile + 2-node ring

struct GmresSys {
    int active;     // still iterating this restart
    int nan;        // NaN residual seen (resetTimeFunc path)
    int conv;       // converged
    int restarts;   // restart-loop iterations entered (restart_count + 1 at exit)
    int cycles;     // Krylov cycles run (restarts that did not converge)
    int iters;      // iterCount
    int kk;         // number of update coefficients used
    int pad;
    double rho0, norm_rhs, rinv, rho, prev_err;
    double s[KOFM_MAX_KRYLOV];   // 1 / ||u_j||
    double h[KOFM_MAX_KRYLOV];   // Gram-Schmidt coefficients for the next vector
    double xi[KOFM_MAX_KRYLOV];
    double c[KOFM_MAX_KRYLOV];   // update coefficients
    double R[KOFM_MAX_KRYLOV * KOFM_MAX_KRYLOV];
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
    long long spin_limit;     // barrier spin bound (polls of >= 100 ns)
    int tiles_x, tiles_y;
};

// ---- coherent access to data written inside the launch (bypass L1) --------
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
    __shared__ double red[GM_THREADS / 32][GM_SYS_SLOTS];
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
    const int per = (nblocks + 31) / 32;
    const int b0 = lane * per, b1 = min(nblocks, b0 + per);
    for (int b = b0; b < b1; ++b) v += __ldcg(part + (long long)b * GM_SLOTS + slot);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    return __shfl_sync(0xffffffffu, v, 0);
}

enum SerialKind : int {
    SER_NONE = 0,
    SER_RESIDUAL,   // after the residual pass: rho0, convergence test
    SER_KRYLOV,     // after the pass that made u_k (kcur = k)
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
    __shared__ GmresSys sS;  // working copy of one system's scalars (thread 0)
    const int warp = threadIdx.x >> 5, nwarps = GM_THREADS / 32;
    for (int slot = warp; slot < GM_SLOTS; slot += nwarps) {
        const double v = sum_slot_warp(a.part, nblocks, slot);
        if ((threadIdx.x & 31) == 0) tot[slot] = v;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    int any = 0;
    for (int s = 0; s < 2; ++s) {
        GmresSys& S = sS;
        sys_load(S, &ctl->sys[s]);
        if (!S.active) continue;
        const double* t = tot + GM_SYS_SLOTS * s;
        if (kind == SER_RESIDUAL) {
            S.rho0 = sqrt(t[0]);
            if (restart == 0) S.norm_rhs = S.rho0;
            S.rinv = 1.0 / S.rho0;
            S.rho = 1.0;
            S.restarts += 1;
            const double resid = S.rho0 / S.norm_rhs;
            if (isnan(resid)) { S.nan = 1; S.active = 0; }
            else if (resid <= a.rel_tol || S.rho0 <= a.abs_tol) { S.conv = 1; S.active = 0; }
            else { S.cycles += 1; }
        } else if (kind == SER_KRYLOV) {
            // t[0] = ||u_k||^2, t[1] = <r_raw, u_k>, t[2 + j] = <A u_k, u_j> (j <= k)
            const int k = kcur, K = a.K;
            const double nk = sqrt(t[0]);
            S.s[k] = 1.0 / nk;
            if (k == 0) {
                for (int i = 0; i < K * K; ++i) S.R[i] = 0.0;
                S.R[0] = S.rinv * nk;  // ||A r|| with r = r_raw / rho0
            } else {
                for (int j = 0; j < k; ++j) S.R[j + k * K] = S.h[j];
                S.R[k + k * K] = nk;
            }
            S.xi[k] = S.rinv * t[1] * S.s[k];  // <r, v_k>
            if (k < K - 1) {
                // h_j = <A v_k, v_j> with v = s u
                for (int j = 0; j <= k; ++j) S.h[j] = S.s[k] * S.s[j] * t[2 + j];
            } else {
                cycle_logic(S, K, a.rel_tol);
            }
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
    return ldc(&a.ctl->error) == 0;
}

__device__ __forceinline__ int wrap_mod(int x, int n) {
    int r = x % n;
    return r < 0 ? r + n : r;
}

__device__ __forceinline__ bool is_fluid(const int16_t* nt, long long g) {
    return !((uint16_t)nt[g] & M_SOLID);
}

// ---- shared tile of one Krylov pass -------------------------------------------
struct KTile {
    double U1[R2H][R2W];        // stencil input u_{k-1} (or r) on the 2-ring
    double C[4][R1H][R1W];      // coefficients E, W, N, S on the 1-ring
    double UK[R1H][R1W];        // u_k on the 1-ring
    unsigned char F[R2H][R2W];  // fluid flags on the 2-ring
    double g[KOFM_MAX_KRYLOV];  // h_j s_j
    double sk1;                 // s_{k-1}
};

// 5-point stencil in the CSR order of an interior row (S, W, C, E, N) on a
// value grid V centred at (cy, cx), coefficients of the 1-ring at (ry, rx).
template <typename VG>
__device__ __forceinline__ double tile_stencil(const VG& V, int cy, int cx, const KTile& T,
                                               int ry, int rx) {
    return (double)T.C[3][ry][rx] * V[cy - 1][cx] + (double)T.C[1][ry][rx] * V[cy][cx - 1] +
           V[cy][cx] + (double)T.C[0][ry][rx] * V[cy][cx + 1] +
           (double)T.C[2][ry][rx] * V[cy + 1][cx];
}

// One fused Krylov pass for vector k of system S over one tile.  The tile is
// a window onto the periodic lattice: column positions map to x mod nx, so
// positions at or beyond nx alias columns 0, 1, ... (computed, never stored).
//   k == 0: u_0 = A r                  (r = residual, un-normalised)
//   k >= 1: u_k = s_{k-1} A u_{k-1} - sum_j g_j u_j
// then, if k < K-1, w = A u_k on the tile.  Accumulates ||u_k||^2, <r, u_k>
// and <w, u_j> (j <= k) into acc.
__device__ __forceinline__ void krylov_tile(const GmresArgs& a, const KoSystem& S,
                                            const float* rsrc, int k, int tile, KTile& T,
                                            double (&acc)[2 + KOFM_MAX_KRYLOV]) {
    const int tx = tile % a.tiles_x, ty = tile / a.tiles_x;
    const int x0 = tx * TW, y0 = ty * TH;
    const int nx = a.nx, ny = a.ny, P = a.P;
    const long long D = a.D;
    const float* src = (k == 0) ? rsrc : S.V + (long long)(k - 1) * D;
    // 1) u_{k-1} (or r) and fluid flags on the 2-ring
    for (int p = threadIdx.x; p < R2H * R2W; p += GM_THREADS) {
        const int ry = p / R2W, rx = p % R2W;
        const int gy = y0 - 2 + ry;
        const int gx = wrap_mod(x0 - 2 + rx, nx);
        double v = 0.0;
        unsigned char f = 0;
        if (gy >= 0 && gy < ny) {
            const long long g = (long long)gy * P + gx;
            f = is_fluid(a.ntype, g);
            if (f) v = (double)__ldcg(src + g);
        }
        T.U1[ry][rx] = v;
        T.F[ry][rx] = f;
    }
    __syncthreads();
    // 2) coefficients on the 1-ring
    for (int p = threadIdx.x; p < R1H * R1W; p += GM_THREADS) {
        const int ry = p / R1W, rx = p % R1W;
        const int gy = y0 - 1 + ry;
        const int gx = wrap_mod(x0 - 1 + rx, nx);
        double c0 = 0.0, c1 = 0.0, c2 = 0.0, c3 = 0.0;
        if (T.F[ry + 1][rx + 1]) {
            const long long g = (long long)gy * P + gx;
            c0 = __ldg(S.coef + g);
            c1 = __ldg(S.coef + D + g);
            c2 = __ldg(S.coef + 2 * D + g);
            c3 = __ldg(S.coef + 3 * D + g);
        }
        T.C[0][ry][rx] = c0; T.C[1][ry][rx] = c1; T.C[2][ry][rx] = c2; T.C[3][ry][rx] = c3;
    }
    __syncthreads();
    // 3) z = A u_{k-1} on the 1-ring, scaled; Gram-Schmidt with u_{k-1} last
    for (int p = threadIdx.x; p < R1H * R1W; p += GM_THREADS) {
        const int ry = p / R1W, rx = p % R1W;
        double u = 0.0;
        if (T.F[ry + 1][rx + 1]) {
            const double z = tile_stencil(T.U1, ry + 1, rx + 1, T, ry, rx);
            if (k == 0) {
                u = z;
            } else {
                u = T.sk1 * z;
                const int gy = y0 - 1 + ry;
                const int gx = wrap_mod(x0 - 1 + rx, nx);
                const long long g = (long long)gy * P + gx;
                for (int j = 0; j < k - 1; ++j)
                    u -= T.g[j] * (double)__ldcg(S.V + (long long)j * D + g);
                u -= T.g[k - 1] * T.U1[ry + 1][rx + 1];
            }
            u = (double)(float)u;  // the stored (FP32) value defines u_k
        }
        T.UK[ry][rx] = u;
    }
    __syncthreads();
    // 4) interior: store u_k, dot products, w = A u_k
    const bool need_w = k < a.K - 1;
    for (int p = threadIdx.x; p < TW * TH; p += GM_THREADS) {
        const int iy = p / TW, ix = p % TW;
        const int gy = y0 + iy, gxr = x0 + ix;
        if (gy >= ny || gxr >= nx) continue;  // padding / alias columns
        const long long g = (long long)gy * P + gxr;
        const double u = T.UK[iy + 1][ix + 1];
        __stcg(S.V + (long long)k * D + g, (float)u);
        if (!T.F[iy + 2][ix + 2]) continue;
        const double r = (double)__ldcg(rsrc + g);
        acc[0] += u * u;
        acc[1] += r * u;
        if (need_w) {
            const double w = tile_stencil(T.UK, iy + 1, ix + 1, T, iy + 1, ix + 1);
            const double um1 = T.U1[iy + 2][ix + 2];
#pragma unroll
            for (int j = 0; j < KOFM_MAX_KRYLOV; ++j) {
                if (j < k - 1) acc[2 + j] += w * (double)__ldcg(S.V + (long long)j * D + g);
                else if (j == k - 1) acc[2 + j] += w * um1;
                else if (j == k) acc[2 + j] += w * u;
            }
        }
    }
    __syncthreads();
}

// ---- the solver kernel ---------------------------------------------------------
__global__ void __launch_bounds__(GM_THREADS)
gmres_kernel(const GmresArgs a) {
    GmresControl* ctl = a.ctl;
    __shared__ KTile T;
    __shared__ double sh_c[2][KOFM_MAX_KRYLOV];
    __shared__ int sh_act[2];
    const long long npairs = a.D / 2;
    const long long stride = (long long)gridDim.x * GM_THREADS;
    const long long t0 = (long long)blockIdx.x * GM_THREADS + threadIdx.x;
    const int ntiles = a.tiles_x * a.tiles_y;
    const int K = a.K;

    for (int restart = 0; restart < a.max_restarts; ++restart) {
        // ---- residual: restart 0 uses b' itself; later r = b' - A x ---------
        if (threadIdx.x < 2) sh_act[threadIdx.x] = ldc(&ctl->sys[threadIdx.x].active);
        __syncthreads();
        for (int s = 0; s < 2; ++s) {
            double acc[1] = {0.0};
            if (sh_act[s]) {
                const KoSystem& S = a.sys[s];
                for (long long pr = t0; pr < npairs; pr += stride) {
                    const long long g = pr * 2;
                    const int y = (int)(g / a.P), x = (int)(g - (long long)y * a.P);
                    if (x >= a.nx) continue;
                    const unsigned int t2 = *reinterpret_cast<const unsigned int*>(a.ntype + g);
                    const bool f0 = !((t2 & 0xffff) & M_SOLID);
                    const bool f1 = (x + 1 < a.nx) && !((t2 >> 16) & M_SOLID);
                    if (!f0 && !f1) {
                        if (restart > 0) __stcg(reinterpret_cast<float2*>(S.r + g), make_float2(0.f, 0.f));
                        continue;
                    }
                    if (restart == 0) {
                        const float2 b = __ldcg(reinterpret_cast<const float2*>(S.rhs + g));
                        const double b0 = f0 ? (double)b.x : 0.0, b1 = f1 ? (double)b.y : 0.0;
                        acc[0] += b0 * b0 + b1 * b1;
                    } else {
                        double rr[2];
                        for (int j = 0; j < 2; ++j) {
                            const int xj = x + j;
                            const bool fj = j == 0 ? f0 : f1;
                            rr[j] = 0.0;
                            if (!fj) continue;
                            const long long gj = g + j;
                            const long long row = (long long)y * a.P;
                            const int xw = xj > 0 ? xj - 1 : a.nx - 1;
                            const int xe = xj + 1 < a.nx ? xj + 1 : 0;
                            const double Ax =
                                (double)__ldg(S.coef + 3 * a.D + gj) * __ldcg(S.x + gj - a.P) +
                                (double)__ldg(S.coef + a.D + gj) * __ldcg(S.x + row + xw) +
                                __ldcg(S.x + gj) +
                                (double)__ldg(S.coef + gj) * __ldcg(S.x + row + xe) +
                                (double)__ldg(S.coef + 2 * a.D + gj) * __ldcg(S.x + gj + a.P);
                            rr[j] = (double)(float)((double)__ldcg(S.rhs + gj) - Ax);
                        }
                        __stcg(reinterpret_cast<float2*>(S.r + g), make_float2((float)rr[0], (float)rr[1]));
                        acc[0] += rr[0] * rr[0] + rr[1] * rr[1];
                    }
                }
            }
            block_reduce_slots<1>(acc, sh_act[s] ? 1 : 0, a.part, GM_SYS_SLOTS * s);
        }
        if (!grid_sync(a, SER_RESIDUAL, 0, restart)) return;
        if (!ldc(&ctl->any_active)) break;

        // ---- K fused Krylov passes ---------------------------------------------
        for (int k = 0; k < K; ++k) {
            if (threadIdx.x < 2) sh_act[threadIdx.x] = ldc(&ctl->sys[threadIdx.x].active);
            __syncthreads();
            for (int s = 0; s < 2; ++s) {
                double acc[2 + KOFM_MAX_KRYLOV];
#pragma unroll
                for (int j = 0; j < 2 + KOFM_MAX_KRYLOV; ++j) acc[j] = 0.0;
                const int nslots = k < K - 1 ? 3 + k : 2;
                if (sh_act[s]) {
                    const KoSystem& S = a.sys[s];
                    const GmresSys* C = &ctl->sys[s];
                    if (threadIdx.x < k) T.g[threadIdx.x] = ldc(&C->h[threadIdx.x]) * ldc(&C->s[threadIdx.x]);
                    if (threadIdx.x == 0 && k > 0) T.sk1 = ldc(&C->s[k - 1]);
                    __syncthreads();
                    const float* rsrc = restart == 0 ? S.rhs : S.r;
                    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
                        krylov_tile(a, S, rsrc, k, tile, T, acc);
                }
                block_reduce_slots<2 + KOFM_MAX_KRYLOV>(acc, sh_act[s] ? nslots : 0, a.part,
                                                        GM_SYS_SLOTS * s);
            }
            if (!grid_sync(a, SER_KRYLOV, k, restart)) return;
        }

        // ---- x += c0 rinv r + sum_{j>=1} c_j s_{j-1} u_{j-1} ----------------------
        for (int s = 0; s < 2; ++s) {
            if (threadIdx.x == 0) sh_act[s] = ldc(&ctl->sys[s].active);
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
            const float* rsrc = restart == 0 ? S.rhs : S.r;
            for (long long pr = t0; pr < npairs; pr += stride) {
                const long long g = pr * 2;
                double2 xv = make_double2(0.0, 0.0);
                if (restart > 0) xv = __ldcg(reinterpret_cast<const double2*>(S.x + g));
                const float2 r = __ldcg(reinterpret_cast<const float2*>(rsrc + g));
                double v0 = xv.x + sh_c[s][0] * (double)r.x, v1 = xv.y + sh_c[s][0] * (double)r.y;
                for (int j = 1; j < K; ++j) {
                    const double cj = sh_c[s][j];
                    if (cj == 0.0) continue;
                    const float2 u = __ldcg(reinterpret_cast<const float2*>(S.V + (long long)(j - 1) * a.D + g));
                    v0 += cj * (double)u.x;
                    v1 += cj * (double)u.y;
                }
                __stcg(reinterpret_cast<double2*>(S.x + g), make_double2(v0, v1));
            }
        }
        if (!grid_sync(a, SER_NONE, 0, restart)) return;
    }

    // ---- x_new = x0 + d on fluid nodes; solid-boundary rows -> 0 -----------------
    for (int s = 0; s < 2; ++s) {
        const KoSystem& S = a.sys[s];
        float* f = a.field[s];
        const bool has_x = ldc(&ctl->sys[s].cycles) > 0;
        for (long long pr = t0; pr < npairs; pr += stride) {
            const long long g = pr * 2;
            const int y = (int)(g / a.P), x = (int)(g - (long long)y * a.P);
            if (x >= a.nx) continue;
            const unsigned int t2 = *reinterpret_cast<const unsigned int*>(a.ntype + g);
            const int tt[2] = {(int)(t2 & 0xffff), (int)(t2 >> 16)};
            const double2 xv = has_x ? __ldcg(reinterpret_cast<const double2*>(S.x + g)) : make_double2(0.0, 0.0);
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
