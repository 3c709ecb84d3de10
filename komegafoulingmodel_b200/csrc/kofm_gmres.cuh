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
//  * One fused sweep per Krylov vector.  A warp marches down a strip of 32
//    columns; per row it computes z_k = A u_{k-1}, orthogonalises
//    u_k = s_{k-1} z_k - sum_j h_j s_j u_j (classical Gram-Schmidt, the
//    reference's order), writes u_k, and accumulates the dot products
//    <A u_k, u_j> of the NEXT vector's Gram-Schmidt step row by row -- so
//    each vector costs one sweep and one grid barrier instead of the
//    reference's product / two Gram-Schmidt stages / normalise.
//    Krylov vectors are kept un-normalised; the scales 1/||u_j|| are applied
//    lazily.  Vectors and matrix are FP64 (an FP32 basis stalls the first
//    cycle near 1e-5 relative residual on the omega wall rows).
//  * Dot products are reduced per block and combined, in a fixed order, by
//    the last block to reach the grid barrier, which also runs the scalar
//    logic (the reference's host code) before releasing the grid.  The
//    barrier spin is bounded: on expiry the control block records a timeout
//    and every block returns.
#pragma once
#include "kofm_common.cuh"
#include "kofm_komega.cuh"

#ifndef KOFM_MAX_KRYLOV
#define KOFM_MAX_KRYLOV 10
#endif

namespace kofm {

constexpr int GM_THREADS = 256;
#ifndef KOFM_GM_MINBLOCKS
#define KOFM_GM_MINBLOCKS 2  // resident blocks per SM the register budget targets
#endif
constexpr int GM_SLOTS = 32;                    // partial-sum slots per block
constexpr int GM_SYS_SLOTS = 16;                // per system

struct GmresSys {
    int active;     // still iterating this restart
    int nan;        // NaN residual seen (resetTimeFunc path)
    int conv;       // converged
    int restarts;   // restart-loop iterations entered (restart_count + 1 at exit)
    int cycles;     // Krylov cycles run (restarts that did not converge)
    int iters;      // iterCount
    int kk;         // number of update coefficients used
    int done;       // current cycle finished (no more Krylov vectors needed)
    int vecs;       // Krylov vectors built (all cycles)
    int vec_index_sum;  // sum over built vectors of their index k in the cycle
    int update_terms;   // sum over cycles of the update's coefficient count kk
    int inject;         // test hook: report a NaN residual at the first check
    int lev;            // one-sweep cycle: powers computed so far in this cycle
    int ext;            // one-sweep cycle: 1 = more powers needed before the cut
    int powers;         // one-sweep cycle: powers computed (all rounds and cycles)
    int lnext;          // one-sweep cycle: first-round powers chosen for the next cycle (0: none yet)
    // one-sweep cycle run as separate phase launches: the restart whose
    // vectors are in use (buffer parity), the levels of the pending powers
    // round (lfrom + 1 .. lto), a finished cycle waiting for its update and
    // residual sweeps, and the field write-back done
    int rst, lfrom, lto, ready, written;
    double rho0, norm_rhs, rinv, rho, prev_err;
    double abytes;      // one-sweep cycle: algorithmic bytes per node of the sweeps so far
    double s[KOFM_MAX_KRYLOV];   // 1 / ||u_j||
    double h[KOFM_MAX_KRYLOV];   // Gram-Schmidt coefficients for the next vector
    double xi[KOFM_MAX_KRYLOV];
    double c[KOFM_MAX_KRYLOV];   // update coefficients
    double R[KOFM_MAX_KRYLOV * KOFM_MAX_KRYLOV];
};

constexpr int GM_TRACE = 32;
struct GmresControl {
    GmresSys sys[2];
    int error;        // 0 ok, 1 barrier timeout
    int passes;       // grid sweeps performed
    int any_active;
    int ntrace;       // grid barriers recorded in trace
    int any_ext;      // one-sweep cycle: a system asks for more powers
    int rounds;       // phase-launch solve: rounds run
    int launches;     // phase-launch solve: kernel launches of the solve
    int pad;
    unsigned long long t_start;           // %globaltimer at the first block's start (ns)
    unsigned long long trace[GM_TRACE];   // %globaltimer at each grid barrier's release
};

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Records the release time of a grid barrier (called by the last block).
__device__ __forceinline__ void trace_barrier(GmresControl* ctl) {
    const int n = __ldcg(&ctl->ntrace);
    if (n < GM_TRACE) __stcg(&ctl->trace[n], globaltimer_ns());
    __stcg(&ctl->ntrace, n + 1);
}

struct GridBarrier {
    unsigned int count;
    unsigned int gen;
};

struct GmresArgs {
    KoSystem sys[2];
    void* field[2];           // omega, k (updated in place): FP32, or FP64 when f64
    int f64;
    const int16_t* ntype;
    GmresControl* ctl;
    double* part;             // [GM_SLOTS][gridDim.x] (slot-major)
    GridBarrier* bar;
    int nx, ny, P;
    long long D;
    int K;                    // Krylov dimension
    int max_restarts;
    double rel_tol, abs_tol;
    long long spin_limit;     // barrier spin bound (polls of >= 100 ns)
    int full_cycle;           // 1: build all K vectors before the truncation tests
    int strips;               // strips of WS_OWN (30) own columns
};

// ---- coherent access to data written inside the launch (bypass L1) --------
template <typename T>
__device__ __forceinline__ T ldc(const T* p) { return __ldcg(p); }

// pair loads / stores of solver vectors (coherent: written inside the launch)
__device__ __forceinline__ double2 ldvec2(const double* p) {
    return __ldcg(reinterpret_cast<const double2*>(p));
}
__device__ __forceinline__ void stvec2(double* p, double a, double b) {
    __stcg(reinterpret_cast<double2*>(p), make_double2(a, b));
}

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// ---- block reduction of NS slots into part[base + s][blockIdx.x] ------------
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
        part[(long long)(base + threadIdx.x) * gridDim.x + blockIdx.x] = v;
    }
    __syncthreads();
}

// Sum slot `slot` of all blocks in a fixed order (deterministic); one warp,
// lane l adding blocks l, l + 32, ... (coalesced: slot-major partials).
__device__ __forceinline__ double sum_slot_warp(const double* part, int nblocks, int slot) {
    const int lane = threadIdx.x & 31;
    const double* ps = part + (long long)slot * nblocks;
    // four independent partial sums per lane (loads in flight together),
    // combined in a fixed order
    double v0 = 0.0, v1 = 0.0, v2 = 0.0, v3 = 0.0;
    int b = lane;
    for (; b + 96 < nblocks; b += 128) {
        v0 += __ldcg(ps + b);
        v1 += __ldcg(ps + b + 32);
        v2 += __ldcg(ps + b + 64);
        v3 += __ldcg(ps + b + 96);
    }
    for (; b < nblocks; b += 32) v0 += __ldcg(ps + b);
    double v = (v0 + v1) + (v2 + v3);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    return __shfl_sync(0xffffffffu, v, 0);
}

enum SerialKind : int {
    SER_NONE = 0,
    SER_RESIDUAL,   // after the residual pass: rho0, convergence test
    SER_KRYLOV,     // after the pass that made u_k (kcur = k)
};

// Back-substitution and update coefficients for a cycle cut at k with R
// indexed by stride `full` (GMRESSolver.cpp:330-343).
__device__ void cycle_finish(GmresSys& S, int K, int k, int full) {
    for (int i2 = k - 1; i2 > -1; --i2) {
        for (int j = i2 + 1; j < k; ++j) S.xi[i2] -= S.R[i2 + j * full] * S.xi[j];
        S.xi[i2] /= S.R[i2 + i2 * full];
    }
    for (int i = 0; i < k; ++i) S.xi[i] *= S.rho0;
    for (int i = 0; i < K; ++i) S.c[i] = S.xi[i];
    S.kk = k;
    S.update_terms += k;
    S.prev_err = fabs(S.rho * S.rho0 / S.norm_rhs);
    S.done = 1;
}

// The reference's tests applied as vector k becomes available: the diag(R)
// cut at k (then full = k), else one xi-test iteration (iterCount += 1;
// |xi_k| >= rho cuts at k with full = K), else the estimator update.
__device__ void cycle_step(GmresSys& S, int K, int k, double rel_tol) {
    if (fabs(S.R[k + k * K]) < rel_tol * S.R[0]) { cycle_finish(S, K, k, k); return; }
    S.iters += 1;
    if (S.xi[k] >= S.rho || S.xi[k] <= -S.rho) { cycle_finish(S, K, k, K); return; }
    S.rho *= sin(acos(S.xi[k] / S.rho));
    if (k == K - 1) cycle_finish(S, K, K, K);
}

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
    S.update_terms += k;
    S.prev_err = fabs(S.rho * S.rho0 / S.norm_rhs);
    S.done = 1;
}

// Serial section: executed by all threads of the last-arriving block.  The
// block sums the partials and stages each system's scalars in shared memory;
// thread 0 runs the scalar logic.
__device__ void serial_section(const GmresArgs& a, int kind, int kcur, int restart, int nblocks) {
    GmresControl* ctl = a.ctl;
    __shared__ double tot[GM_SLOTS];
    __shared__ GmresSys sS;
    __shared__ int s_any;
    const int warp = threadIdx.x >> 5, nwarps = GM_THREADS / 32;
    // only the slots this pass filled: 1 per system after a residual sweep,
    // 3 + k (2 for the last vector of a cycle) after Krylov sweep k
    const int used = kind == SER_RESIDUAL ? 1 : (kcur < a.K - 1 ? 3 + kcur : 2);
    for (int i = warp; i < 2 * used; i += nwarps) {
        const int slot = (i < used ? 0 : GM_SYS_SLOTS) + (i < used ? i : i - used);
        const double v = sum_slot_warp(a.part, nblocks, slot);
        if ((threadIdx.x & 31) == 0) tot[slot] = v;
    }
    if (threadIdx.x == 0) s_any = 0;
    constexpr int NW = (int)(sizeof(GmresSys) / 8);
    for (int s = 0; s < 2; ++s) {
        __syncthreads();
        {
            const unsigned long long* src = reinterpret_cast<const unsigned long long*>(&ctl->sys[s]);
            unsigned long long* dst = reinterpret_cast<unsigned long long*>(&sS);
            for (int i = threadIdx.x; i < NW; i += GM_THREADS) dst[i] = __ldcg(src + i);
        }
        __syncthreads();
        if (threadIdx.x == 0 && sS.active && !(kind == SER_KRYLOV && sS.done)) {
            GmresSys& S = sS;
            const double* t = tot + GM_SYS_SLOTS * s;
            if (kind == SER_RESIDUAL) {
                S.rho0 = sqrt(t[0]);
                if (restart == 0) S.norm_rhs = S.rho0;
                S.rinv = 1.0 / S.rho0;
                S.rho = 1.0;
                S.restarts += 1;
                const double resid = S.rho0 / S.norm_rhs;
                if (isnan(resid) || (restart == 0 && S.inject)) { S.nan = 1; S.active = 0; }
                else if (resid <= a.rel_tol || S.rho0 <= a.abs_tol) { S.conv = 1; S.active = 0; }
                else { S.cycles += 1; S.done = 0; }
            } else if (kind == SER_KRYLOV) {
                // t[0] = ||u_k||^2, t[1] = <r_raw, u_k>, t[2 + j] = <A u_k, u_j> (j <= k)
                const int k = kcur, K = a.K;
                const double nk = sqrt(t[0]);
                S.vecs += 1;
                S.vec_index_sum += k;
                S.s[k] = 1.0 / nk;
                if (k == 0) {
                    for (int i = 0; i < K * K; ++i) S.R[i] = 0.0;
                    S.R[0] = S.rinv * nk;  // ||A r|| with r = r_raw / rho0
                } else {
                    for (int j = 0; j < k; ++j) S.R[j + k * K] = S.h[j];
                    S.R[k + k * K] = nk;
                }
                S.xi[k] = S.rinv * t[1] * S.s[k];  // <r, v_k>
                if (a.full_cycle) {
                    if (k == K - 1) cycle_logic(S, K, a.rel_tol);
                } else {
                    cycle_step(S, K, k, a.rel_tol);
                }
                if (!S.done && k < K - 1) {
                    // h_j = <A v_k, v_j> with v = s u
                    for (int j = 0; j <= k; ++j) S.h[j] = S.s[k] * S.s[j] * t[2 + j];
                }
            }
            s_any |= kind == SER_KRYLOV ? (S.active && !S.done) : S.active;
        }
        __syncthreads();
        {
            const unsigned long long* src = reinterpret_cast<const unsigned long long*>(&sS);
            unsigned long long* dst = reinterpret_cast<unsigned long long*>(&ctl->sys[s]);
            for (int i = threadIdx.x; i < NW; i += GM_THREADS) __stcg(dst + i, src[i]);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __stcg(&ctl->any_active, s_any);
        __stcg(&ctl->passes, ldc(&ctl->passes) + 1);
    }
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
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) {
            trace_barrier(a.ctl);
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

// ---- warp-strip Krylov pass ---------------------------------------------------
// A work unit is a strip of WS_OWN = 30 columns times a range of rows, owned by
// ONE warp, which marches down the rows.  Lane l holds column x0 - 1 + l: lanes
// 1..30 are the strip's own columns, lanes 0 and 31 the neighbouring strips'
// edge columns (x0 - 1 and x0 + 30), computed like any other column so that
// every lane runs the same instructions:
//   row y:  u_k(y) = s_{k-1} A u_{k-1} - sum_j g_j u_j; own lanes store u_k(y)
//           and add ||u_k||^2 and <r, u_k>;
//           <A u_k, u_j> split by rows: row y adds u_j(y) (u_k + W u_k(x-1) +
//           E u_k(x+1) + S u_k(y-1)) and the N term of row y-1,
//           u_k(y) N(y-1) u_j(y-1), carried in registers as q_j.
// x neighbours come from warp shuffles; lanes 0 and 31 also read u_{k-1} one
// column further out (x0 - 2, x0 + 31).  Every lane streams its column's
// inputs of the rows ahead into its own slots of a shared-memory ring
// (cp.async, 8 bytes each, addresses advanced by a fixed row stride) while row
// y computes, so the pass needs no block-level synchronisation.  Vectors and
// coefficients are zero on non-fluid nodes and rows outside the lattice read
// as zero.  Columns are taken modulo nx (periodic x; lanes past the last
// column of the last strip alias real columns and are neither stored nor
// counted).
constexpr int WS_OWN = 30;                  // own columns of a strip
constexpr int WS_KV = KOFM_MAX_KRYLOV - 2;  // u_j for j < k-1 <= K-2
static_assert(KOFM_MAX_KRYLOV == 10, "krylov_strip is instantiated for k = 0..9");
constexpr int GM_WARPS = GM_THREADS / 32;

// One ring slot of a warp: everything row y needs, laid out per k (the
// number of basis vectors read depends on the vector being built):
//   cf[4][32]     E, W, N, S of row y
//   vj[k-1][32]   u_j(y), j < k-1
//   r[32]         r(y) (k >= 1)
//   up[32]        u_{k-1}(y+1)
//   gout[2]       u_{k-1}(y) at x0 - 2 (lane 0) and x0 + 31 (lane 31)
// The warp's ring region holds as many slots of that size as fit (up to 6),
// so small k prefetch deeper.
constexpr int WS_RING_DOUBLES = 3 * ((4 + WS_KV + 2) * 32 + 2);

template <int k>
struct SlotView {
    static constexpr int NV = k > 1 ? k - 1 : 0;
    static constexpr int NR = k > 0 ? 1 : 0;
    static constexpr int O_VJ = 4 * 32;
    static constexpr int O_R = O_VJ + NV * 32;
    static constexpr int O_UP = O_R + NR * 32;
    static constexpr int O_GOUT = O_UP + 32;
    static constexpr int DOUBLES = O_GOUT + 2;
    static constexpr int FIT = WS_RING_DOUBLES / DOUBLES;
    static constexpr int SLOTS = FIT > 6 ? 6 : FIT;
    static_assert(SLOTS >= 3, "ring too small");
};

struct SolverSmem {
    double ring[GM_WARPS][WS_RING_DOUBLES];
    double g[KOFM_MAX_KRYLOV];  // h_j s_j
    double sk1;                 // s_{k-1}
};

__device__ __forceinline__ int wrap_mod(int x, int n) {
    int r = x % n;
    return r < 0 ? r + n : r;
}

__device__ __forceinline__ void cp8(unsigned saddr, const double* gmem) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(saddr), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }
__device__ __forceinline__ void st_zero(unsigned saddr) {
    asm volatile("st.shared.f64 [%0], %1;\n" ::"r"(saddr), "d"(0.0) : "memory");
}

// Per-lane addressing of one strip: element offsets of the lane's column in
// the plain, coefficient (4 interleaved) and basis (K interleaved) arrays, and
// the row strides (P is a multiple of 32, so a row moves every interleaved
// array by a fixed stride).
struct StripAddr {
    long long oP, oC, oV, oSrc, oOut;  // oOut: u_{k-1} one column further out
    long long sC, sV, sSrc;            // row strides (plain: P)
};

// The lane's inputs of row y into the slot at shared address sb:
// u_{k-1}(y+1), u_{k-1}(y) one column out (lanes 0 / 31), and for rows inside
// the lattice the coefficients, u_j (j < k-1) and r.
template <int k>
__device__ __forceinline__ void ws_issue(const GmresArgs& a, const KoSystem& S, const double* src,
                                         const double* rsrc, const StripAddr& A, int y, int lane,
                                         bool ghost, unsigned sb) {
    using SV = SlotView<k>;
    const unsigned sl = sb + 8u * lane;
    if (y + 1 >= 0 && y + 1 < a.ny) cp8(sl + 8u * SV::O_UP, src + (long long)(y + 1) * A.sSrc + A.oSrc);
    else st_zero(sl + 8u * SV::O_UP);
    const unsigned so = sb + 8u * (SV::O_GOUT + (lane == 0 ? 0 : 1));
    if (y < 0 || y >= a.ny) {
        if (ghost) st_zero(so);
#pragma unroll
        for (int q = 0; q < 4; ++q) st_zero(sl + 8u * (q * 32));
#pragma unroll
        for (int j = 0; j < k - 1; ++j) st_zero(sl + 8u * (SV::O_VJ + j * 32));
        if (k > 0) st_zero(sl + 8u * SV::O_R);
        return;
    }
    if (ghost) cp8(so, src + (long long)y * A.sSrc + A.oOut);
    const double* pc = S.coef + (long long)y * A.sC + A.oC;
#pragma unroll
    for (int q = 0; q < 4; ++q) cp8(sl + 8u * (q * 32), pc + q * 32);
    const double* pv = S.V + (long long)y * A.sV + A.oV;
#pragma unroll
    for (int j = 0; j < k - 1; ++j) cp8(sl + 8u * (SV::O_VJ + j * 32), pv + j * 32);
    if (k > 0) cp8(sl + 8u * SV::O_R, rsrc + (long long)y * a.P + A.oP);
}

// One warp: rows [ya, yb) of the strip whose own columns start at x0.
// k (the vector being built) is a template parameter, so every loop over the
// older basis vectors has its exact length.
template <int k>
__device__ void krylov_strip(const GmresArgs& a, const KoSystem& S, const double* rsrc,
                             int x0, int ya, int yb, SolverSmem& T, double* ring,
                             double (&acc)[2 + KOFM_MAX_KRYLOV]) {
    using SV = SlotView<k>;
    constexpr int NS = SV::SLOTS;  // rows of loads in flight: NS - 1
    const int lane = threadIdx.x & 31;
    const int K = a.K;
    // u_{k-1}: r (plain layout) for k = 0, else basis vector k-1 (interleaved)
    const double* src = (k == 0) ? rsrc : S.V;
    const bool need_w = k < K - 1;
    const int xl = wrap_mod(x0 - 1 + lane, a.nx);
    const bool own = lane >= 1 && lane <= WS_OWN && x0 - 1 + lane < a.nx;
    const bool ghost = lane == 0 || lane == 31;
    const int xo = wrap_mod(lane == 0 ? x0 - 2 : x0 + WS_OWN + 1, a.nx);
    StripAddr A;
    A.oP = xl;
    A.oC = (long long)(xl >> 5) * 128 + (xl & 31);
    A.oV = (long long)(xl >> 5) * (K * 32) + (xl & 31);
    A.sC = 4LL * a.P;
    A.sV = (long long)K * a.P;
    if (k == 0) {
        A.oSrc = A.oP; A.oOut = xo; A.sSrc = a.P;
    } else {
        A.oSrc = A.oV + (k - 1) * 32;
        A.oOut = (long long)(xo >> 5) * (K * 32) + (xo & 31) + (k - 1) * 32;
        A.sSrc = A.sV;
    }
    auto ld = [&](int y) -> double {
        if (y < 0 || y >= a.ny) return 0.0;
        return __ldcg(src + (long long)y * A.sSrc + A.oSrc);
    };
    // rolling u_{k-1} window (rows y-1, y) of the lane's column
    double um = ld(ya - 2), u0 = ld(ya - 1);
    const unsigned ring_s = (unsigned)__cvta_generic_to_shared(ring);
    constexpr unsigned SLOT_BYTES = 8u * SV::DOUBLES;
    int sw = 0;  // slot of the next row to issue
#pragma unroll
    for (int i = 0; i < NS - 1; ++i) {
        if (ya - 1 + i <= yb) ws_issue<k>(a, S, src, rsrc, A, ya - 1 + i, lane, ghost, ring_s + sw * SLOT_BYTES);
        cp_commit();
        sw = sw + 1 == NS ? 0 : sw + 1;
    }
    int sr = 0;  // slot of row y

    const double* g = T.g;  // Gram-Schmidt weights of this vector (shared)
    const double sk1 = T.sk1;
    double q[WS_KV];
#pragma unroll
    for (int j = 0; j < WS_KV; ++j) q[j] = 0.0;
    double nprev = 0.0, ukprev = 0.0;
    for (int y = ya - 1; y <= yb; ++y) {
        if (y + NS - 1 <= yb) ws_issue<k>(a, S, src, rsrc, A, y + NS - 1, lane, ghost, ring_s + sw * SLOT_BYTES);
        cp_commit();
        sw = sw + 1 == NS ? 0 : sw + 1;
        cp_wait<NS - 1>();
        const double* W = ring + sr * SV::DOUBLES;
        sr = sr + 1 == NS ? 0 : sr + 1;
        const double up = W[SV::O_UP + lane];
        const double cE = W[lane], cW = W[32 + lane], cN = W[64 + lane], cS = W[96 + lane];
        double v[WS_KV];
#pragma unroll
        for (int j = 0; j < WS_KV; ++j) v[j] = j < k - 1 ? W[SV::O_VJ + j * 32 + lane] : 0.0;
        double left = __shfl_up_sync(0xffffffffu, u0, 1);
        double right = __shfl_down_sync(0xffffffffu, u0, 1);
        if (lane == 0) left = W[SV::O_GOUT];
        if (lane == 31) right = W[SV::O_GOUT + 1];
        // CSR order of an interior row: S, W, C, E, N
        const double z = cS * um + cW * left + u0 + cE * right + cN * up;
        double uk;
        if (k == 0) {
            uk = z;
        } else {
            uk = sk1 * z;
#pragma unroll
            for (int j = 0; j < WS_KV; ++j)
                if (j < k - 1) uk -= g[j] * v[j];
            uk -= g[k > 0 ? k - 1 : 0] * u0;
        }
        const bool rowin = y >= ya && y < yb;
        if (rowin && own) {
            const double rr = k == 0 ? u0 : W[SV::O_R + lane];
            __stcg(S.V + (long long)y * A.sV + A.oV + k * 32, uk);
            acc[0] += uk * uk;
            acc[1] += rr * uk;
        }
        if (need_w) {
            const double ukl = __shfl_up_sync(0xffffffffu, uk, 1);
            const double ukr = __shfl_down_sync(0xffffffffu, uk, 1);
            if (own && (rowin || y == yb)) {
                // row y's own part (zero on the halo row yb) plus row y-1's N term
                const double aw = rowin ? uk + cW * ukl + cE * ukr + cS * ukprev : 0.0;
                const double am = rowin ? u0 : 0.0, ak = rowin ? uk : 0.0;
#pragma unroll
                for (int j = 0; j < KOFM_MAX_KRYLOV; ++j) {
                    double t = 0.0;
                    if (j < WS_KV && j < k - 1)
                        t = (rowin ? v[j < WS_KV ? j : 0] : 0.0) * aw + uk * q[j < WS_KV ? j : 0];
                    else if (j == k - 1)
                        t = am * aw + uk * (nprev * um);
                    else if (j == k)
                        t = ak * aw + uk * (nprev * ukprev);
                    acc[2 + j] += t;
                }
            }
            // carry the N terms of row y (zero for rows outside the unit)
            const double nrow = rowin ? cN : 0.0;
#pragma unroll
            for (int j = 0; j < WS_KV; ++j) q[j] = nrow * v[j];
            nprev = nrow;
        }
        ukprev = uk;
        um = u0;
        u0 = up;
    }
    cp_wait<0>();
}

// ---- the solver kernel ---------------------------------------------------------
__global__ void __launch_bounds__(GM_THREADS, KOFM_GM_MINBLOCKS)
gmres_kernel(const GmresArgs a) {
    GmresControl* ctl = a.ctl;
    if (blockIdx.x == 0 && threadIdx.x == 0) __stcg(&ctl->t_start, globaltimer_ns());
    extern __shared__ __align__(16) unsigned char gm_smem[];
    SolverSmem& T = *reinterpret_cast<SolverSmem*>(gm_smem);  // dynamic: larger than 48 KiB
    double* ring = T.ring[threadIdx.x >> 5];
    const int wib = threadIdx.x >> 5;  // warp in block
    __shared__ double sh_c[2][KOFM_MAX_KRYLOV];
    __shared__ int sh_act[2];
    const long long npairs = a.D / 2;
    const long long stride = (long long)gridDim.x * GM_THREADS;
    const long long t0 = (long long)blockIdx.x * GM_THREADS + threadIdx.x;
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
                        if (restart > 0) stvec2(S.r + g, 0.0, 0.0);
                        continue;
                    }
                    if (restart == 0) {
                        const double2 b = ldvec2(S.rhs + g);
                        const double b0 = f0 ? b.x : 0.0, b1 = f1 ? b.y : 0.0;
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
                                (double)__ldg(S.coef + ilv(4, 3, gj)) * __ldcg(S.x + gj - a.P) +
                                (double)__ldg(S.coef + ilv(4, 1, gj)) * __ldcg(S.x + row + xw) +
                                __ldcg(S.x + gj) +
                                (double)__ldg(S.coef + ilv(4, 0, gj)) * __ldcg(S.x + row + xe) +
                                (double)__ldg(S.coef + ilv(4, 2, gj)) * __ldcg(S.x + gj + a.P);
                            rr[j] = __ldcg(S.rhs + gj) - Ax;
                        }
                        stvec2(S.r + g, rr[0], rr[1]);
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
            if (threadIdx.x < 2)
                sh_act[threadIdx.x] = ldc(&ctl->sys[threadIdx.x].active) && !ldc(&ctl->sys[threadIdx.x].done);
            __syncthreads();
            if (!sh_act[0] && !sh_act[1]) break;  // block-uniform, same in every block
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
                    const double* rsrc = restart == 0 ? S.rhs : S.r;
                    {
                        // The block takes a share of the flattened (group, row)
                        // sequence, a group being GM_WARPS adjacent strips; its
                        // warps march the same rows of neighbouring strips side
                        // by side, so their ghost-column reads hit L1 / L2.
                        const int groups = (a.strips + GM_WARPS - 1) / GM_WARPS;
                        const long long total = (long long)groups * a.ny;
                        long long f = total * blockIdx.x / gridDim.x;
                        const long long f1 = total * (blockIdx.x + 1) / gridDim.x;
                        while (f < f1) {
                            const int grp = (int)(f / a.ny), ya = (int)(f - (long long)grp * a.ny);
                            const int yb = (int)min((long long)a.ny, (long long)ya + (f1 - f));
                            const int strip = grp * GM_WARPS + wib;
                            if (strip < a.strips) {
                                switch (k) {
#define KOFM_KSTRIP(n) \
    case n: krylov_strip<n>(a, S, rsrc, strip * WS_OWN, ya, yb, T, ring, acc); break;
                                    KOFM_KSTRIP(0) KOFM_KSTRIP(1) KOFM_KSTRIP(2) KOFM_KSTRIP(3)
                                    KOFM_KSTRIP(4) KOFM_KSTRIP(5) KOFM_KSTRIP(6) KOFM_KSTRIP(7)
                                    KOFM_KSTRIP(8) KOFM_KSTRIP(9)
#undef KOFM_KSTRIP
                                    default: break;
                                }
                            }
                            f += yb - ya;
                        }
                    }
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
            const double* rsrc = restart == 0 ? S.rhs : S.r;
            for (long long pr = t0; pr < npairs; pr += stride) {
                const long long g = pr * 2;
                double2 xv = make_double2(0.0, 0.0);
                if (restart > 0) xv = __ldcg(reinterpret_cast<const double2*>(S.x + g));
                const double2 r = ldvec2(rsrc + g);
                double v0 = xv.x + sh_c[s][0] * r.x, v1 = xv.y + sh_c[s][0] * r.y;
                for (int j = 1; j < K; ++j) {
                    const double cj = sh_c[s][j];
                    if (cj == 0.0) continue;
                    const double2 u = ldvec2(S.V + ilv(K, j - 1, g));  // g even: g, g+1 adjacent
                    v0 += cj * u.x;
                    v1 += cj * u.y;
                }
                __stcg(reinterpret_cast<double2*>(S.x + g), make_double2(v0, v1));
            }
        }
        if (!grid_sync(a, SER_NONE, 0, restart)) return;
    }

    // ---- x_new = x0 + d on fluid nodes; solid-boundary rows -> 0 -----------------
    // A solve that met a NaN residual leaves its field as it was before the
    // solve (the reference adds the correction of the cycles before the NaN,
    // GMRESSolver.cpp:350-353, and its copyFromPrevSolution restores nothing).
    for (int s = 0; s < 2; ++s) {
        const KoSystem& S = a.sys[s];
        float* f = static_cast<float*>(a.field[s]);
        double* f8 = static_cast<double*>(a.field[s]);
        const bool has_x = ldc(&ctl->sys[s].cycles) > 0 && !ldc(&ctl->sys[s].nan);
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
                if (a.f64) {
                    if (!(tt[j] & M_SOLID)) f8[g + j] = f8[g + j] + dv[j];
                    else if (tt[j] & SOLID_BOUNDARY) f8[g + j] = 0.0;
                } else {
                    if (!(tt[j] & M_SOLID)) f[g + j] = (float)((double)f[g + j] + dv[j]);
                    else if (tt[j] & SOLID_BOUNDARY) f[g + j] = 0.f;
                }
            }
        }
    }
}

}  // namespace kofm
