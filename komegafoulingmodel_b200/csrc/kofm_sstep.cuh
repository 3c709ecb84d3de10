// kofm_sstep.cuh - the k-omega solve with all Krylov directions of a cycle
// built in one sweep (sm_100a).
//
// Algorithm: the reference's restarted "simpler GMRES" (GMRESSolver::solve,
// GMRESSolver.cpp:227-355; Walker & Zhou 1994) on the correction system
// A d = b' with the same restart loop, convergence test, truncation tests
// (diag(R) against relTol R(0,0), then |xi_k| >= rho), residual estimator
// rho *= sin(acos(xi/rho)), back-substitution with the reference's R
// indexing, and x = x0 + d.  What changes is how the Krylov basis is formed.
//
// The rows are normalised by their diagonal, so A = I + N with N the four
// off-diagonals.  The Krylov space of A on r equals that of N, spanned by the
// powers p_0 = r, p_{j+1} = N p_j.  One grid sweep (the "powers" phase)
// computes p_1 .. p_L of a cycle at once: every thread owns one column of a
// 256-column strip and marches down the rows, level j working one row behind
// level j-1 (a skewed wavefront), so each coefficient row is read from HBM
// once for all L levels; the row's coefficients and level-0 value are staged
// ahead in a per-thread shared-memory ring by cp.async; x neighbours come from
// warp shuffles, across warps from a shared-memory edge buffer written the
// step before (one block barrier per row).  A pointwise sweep then forms the
// Gram matrix G = P^T P of [p_0 .. p_L], and the serial section runs the
// simpler GMRES steps in the (L+1)-dimensional coefficient space with the
// inner product a^T G b: with A p_j = p_j + p_{j+1}, every vector of the
// method (r/||r||, A z, the orthonormal v_k, the update) is a combination of
// the p_j, and R, xi, rho and the tests are the reference's quantities.  Two
// pointwise sweeps apply d += sum c_j p_j and form the next residual
// b' - A d with its norm, so the next restart's test needs no extra sweep.
//
// L follows the cycle lengths seen so far (two more powers than the last
// cycle used, kept per system across solves); a cycle whose tests have not
// fired by then gets the remaining powers up to the Krylov dimension in a
// second powers + Gram round and is re-run from its first vector.
//
// Per cycle: 4 sweeps (powers, Gram, update, residual) instead of one per
// Krylov vector plus residual and update sweeps, and the orthogonalisation
// reads no basis vector.  In exact arithmetic the iterates are those of the
// reference's classical Gram-Schmidt; in FP64 the truncation tests see
// rounding of the size the reference's own classical Gram-Schmidt has (both
// lose orthogonality like eps cond^2), so the cut of a converged cycle moves
// by a vector or two while restart counts and the solution agree to far below
// the tolerance.
#pragma once
#include "kofm_gmres.cuh"

namespace kofm {

constexpr int SS_THREADS = 256;
constexpr int SS_WARPS = SS_THREADS / 32;
constexpr int SS_MAXL = KOFM_MAX_KRYLOV;                  // levels of one sweep
constexpr int SS_NG = (SS_MAXL + 1) * (SS_MAXL + 2) / 2;  // Gram entries per system
constexpr int SS_SLOTS = 2 * SS_NG;                       // partial sums per block
constexpr int SS_PF = 6;                                  // rows staged ahead by the powers sweep
constexpr int SS_RING = 8;                                // ring rows (power of two > SS_PF + 1)
static_assert(SS_RING > SS_PF + 1 && (SS_RING & (SS_RING - 1)) == 0, "ring");
constexpr int SS_RF = 5;                                  // ring fields: level 0, cE, cW, cN, cS
constexpr int SS_MINL = 4;                                // fewest powers of a first round

struct SsArgs {
    KoSystem sys[2];          // x / x2 and r / r2 alternate between restarts
    void* field[2];           // omega, k (updated in place at the end): FP32, or FP64 when f64
    int f64;
    const int16_t* ntype;
    GmresControl* ctl;
    double* part;             // [SS_SLOTS][gridDim.x] (slot-major)
    GridBarrier* bar;
    int* lhint;               // [2] powers of a first round, kept across solves (0: K)
    int nx, ny, P;
    long long D;
    int K;                    // Krylov dimension
    int max_restarts;
    double rel_tol, abs_tol;
    long long spin_limit;
    int pstrips;              // powers strips of SS_THREADS - 2K own columns
    int prows;                // row ranges per powers strip
};

// Gram entry (i, j), i <= j, of one system: slot j (j + 1) / 2 + i.
__host__ __device__ constexpr int ss_gslot(int i, int j) { return j * (j + 1) / 2 + i; }

struct SsSmem {
    double edge[2][SS_WARPS][2][SS_MAXL];  // [step parity][warp][left/right lane][level]
    double red[SS_WARPS][SS_NG];           // block reduction of the Gram partials
    double c[2][SS_MAXL + 1];              // update coefficients on p_0 .. p_K
    int act[2];
    int kk[2];
    int lfrom[2], lto[2];                  // powers of this round: levels lfrom+1 .. lto
};

// Dynamic shared memory of the powers phase: per thread (column) a ring of
// SS_RING rows of SS_RF doubles, [row][field][thread] (conflict-free).
constexpr size_t SS_DSMEM = sizeof(double) * SS_RING * SS_RF * SS_THREADS;

__device__ __forceinline__ int ss_first_levels(const SsArgs& a, int s) {
    int l = __ldcg(a.lhint + s);
    if (l <= 0 || l > a.K) l = a.K;
    return l < SS_MINL ? (a.K < SS_MINL ? a.K : SS_MINL) : l;
}

// ---- coefficient-space simpler GMRES (serial step, one warp per system) --------
// G: (L+1) x (L+1) Gram of p_0 .. p_L (full, symmetric, row-major in shared
// memory).  Builds the cycle's vectors in order and applies the reference's
// tests after each (the same cycle_step as the one-vector-per-sweep solver).
// Lane i holds coefficient i (on p_i) of every vector; the products with G
// and the inner products a^T G b are formed across the warp, the scalar
// tests on lane 0 (S lives in shared memory).  Returns the vectors built;
// S.done = 0 when L < K vectors passed every test (more powers needed).  On a
// finished cycle, cP gets the update y_0 r/rho0 + sum_{j>=1} y_j v_{j-1} on
// p_0 .. p_L.
__device__ __forceinline__ double ss_warp_sum(double x) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
    return __shfl_sync(0xffffffffu, x, 0);
}

__device__ int ss_cycle_warp(GmresSys& S, const double* G, int L, int K, double rel_tol, double* cP, int cap) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int n = L + 1;
    const double rinv = S.rinv;
    const double z0 = lane == 0 ? rinv : 0.0;  // r / ||r|| = p_0 / rho0
    const int iters0 = S.iters;
    for (int i = lane; i < K * K; i += 32) S.R[i] = 0.0;
    __syncwarp();
    if (lane == 0) {
        S.rho = 1.0;
        S.done = 0;
    }
    __syncwarp();
    double V[SS_MAXL], GV[SS_MAXL];
    int built = 0;
#pragma unroll
    for (int k = 0; k < SS_MAXL; ++k) {
        if (k >= L || k >= K || k >= cap) break;
        // w = A z, z = r / rho0 (k = 0) or v_{k-1}; A p_j = p_j + p_{j+1}
        const double z = k == 0 ? z0 : V[k - 1];
        const double zm = __shfl_up_sync(FULL, z, 1);
        double w = lane < n ? (lane == 0 ? z : z + zm) : 0.0;
        double Gw = 0.0;
        for (int j = 0; j < n; ++j) {
            const double wj = __shfl_sync(FULL, w, j);
            if (lane < n) Gw += G[lane * n + j] * wj;
        }
        // classical Gram-Schmidt: R(j, k) = <w, v_j> with the unmodified w
        double h[SS_MAXL];
#pragma unroll
        for (int j = 0; j < k; ++j) h[j] = ss_warp_sum(w * GV[j]);
#pragma unroll
        for (int j = 0; j < k; ++j) {
            w -= h[j] * V[j];
            Gw -= h[j] * GV[j];
        }
        const double nk2 = ss_warp_sum(w * Gw);
        const double nk = nk2 > 0.0 ? sqrt(nk2) : 0.0;  // a vanishing direction cuts (diag test)
        const double inv = nk > 0.0 ? 1.0 / nk : 0.0;
        V[k] = w * inv;
        GV[k] = Gw * inv;
        const double xi = rinv * __shfl_sync(FULL, GV[k], 0);  // z0^T G v_k
        if (lane == 0) {
#pragma unroll
            for (int j = 0; j < k; ++j) S.R[j + k * K] = h[j];
            S.R[k + k * K] = nk;
            S.xi[k] = xi;
            cycle_step(S, K, k, rel_tol);
        }
        __syncwarp();
        built = k + 1;
        if (S.done) break;
    }
    if (!S.done && built >= cap && cap < L && cap < K) {
        // the powers past level cap are numerically dependent on the earlier
        // ones: the cycle ends with the vectors built (back-substitution as
        // for a xi cut), and the next restart goes on from its residual
        if (lane == 0) cycle_finish(S, K, built, K);
        __syncwarp();
    }
    if (!S.done) {
        __syncwarp();
        if (lane == 0) S.iters = iters0;  // the cycle is re-run with more powers
        __syncwarp();
        return built;
    }
    // coefficient 0 is applied even when the cycle is cut at k = 0, as the
    // reference's update does (its xi(0) then unscaled)
    const int kk = S.kk;
    double cp = S.c[0] * z0;
#pragma unroll
    for (int j = 1; j < SS_MAXL; ++j)
        if (j < kk) cp += S.c[j] * V[j - 1];
    if (lane < n) cP[lane] = cp;
    __syncwarp();
    return built;
}

// Shared scratch of one warp's serial step.
struct SsCycleSmem {
    double G[(SS_MAXL + 1) * (SS_MAXL + 1)];
    double cP[SS_MAXL + 1];
    int cap;  // vectors the cycle may build (numerical rank of the power basis)
};

// Smallest pivot of the unit-diagonal Gram Cholesky accepted for a level.
constexpr double SS_PIVOT_MIN = 1.0e-9;

// One system's serial step after a Gram round, run by one warp: t holds
// G(i, j) of p_0 .. p_L (slots ss_gslot), the round computed powers
// lfrom + 1 .. L; `first` marks restart 0's first round, which also takes the
// restart-0 convergence test from G(0, 0) = ||b'||^2 (GMRESSolver::solve's
// checkConvergence).  A cycle whose tests have not fired asks for the
// remaining powers (ext); a finished one leaves its update coefficients on
// p_0 .. p_L in S.h.
__device__ __noinline__ void ss_gram_step(const SsArgs& a, GmresSys& S, int s, const double* t, int L,
                                          int lfrom, bool first, SsCycleSmem& cs) {
    const int lane = threadIdx.x & 31;
    const double rho0 = sqrt(t[0]);
    if (lane == 0) {
        // this round's powers (level 0 and coefficients in, levels lfrom+1 .. L
        // out) and Gram (levels 0 .. L in), per node
        S.abytes += 8.0 + 32.0 + 8.0 * (L - lfrom) + 8.0 * (L + 1);
        S.powers += L - lfrom;
        if (first) {
            S.rho0 = rho0;
            S.norm_rhs = rho0;
            S.restarts += 1;
            const double resid = S.rho0 / S.norm_rhs;
            if (isnan(resid) || S.inject) { S.nan = 1; S.active = 0; }
            else if (resid <= a.rel_tol || S.rho0 <= a.abs_tol) { S.conv = 1; S.active = 0; }
            else S.cycles += 1;
        }
        if (!S.active) S.lfrom = S.lto = 0;
        else {
            S.rho0 = rho0;
            S.rinv = 1.0 / rho0;
        }
    }
    __syncwarp();
    if (!S.active) return;
    const int n = L + 1;
    for (int e = lane; e < n * n; e += 32) {
        const int i = e / n, j = e - i * n;
        cs.G[e] = t[i <= j ? ss_gslot(i, j) : ss_gslot(j, i)];
    }
    __syncwarp();
    // Numerical rank of the power basis: Cholesky of the Gram matrix scaled
    // to a unit diagonal, whose j-th pivot is sin^2 of the angle between p_j
    // and span(p_0 .. p_{j-1}).  Levels from the first pivot below
    // SS_PIVOT_MIN on carry too few correct digits for the coefficient-space
    // orthogonalisation (the monomial basis turns towards the dominant
    // eigenvector as the operator's convective part grows), so the cycle
    // uses at most that many levels.
    // Right-looking, lane i holding row i of the scaled Gram (its trailing
    // Schur complement after each step); every lane learns the pivots by
    // broadcast, so the first one below SS_PIVOT_MIN ends the loop in step.
    {
        double row[SS_MAXL + 1];
        const double gii = lane < n ? cs.G[lane * n + lane] : 0.0;
#pragma unroll
        for (int k = 0; k <= SS_MAXL; ++k) {
            double v = 0.0;
            if (lane < n && k < n) {
                const double gkk = cs.G[k * n + k];
                v = (gii > 0.0 && gkk > 0.0) ? cs.G[lane * n + k] / sqrt(gii * gkk) : 0.0;
            }
            row[k] = v;
        }
        int m = n;
#pragma unroll
        for (int j = 0; j <= SS_MAXL; ++j) {
            if (j >= n) break;
            const double v = __shfl_sync(0xffffffffu, row[j], j);
            if (!(v > SS_PIVOT_MIN)) { m = j; break; }  // levels 0 .. j-1 usable
            const double d = sqrt(v);
            const double lij = lane > j ? row[j] / d : 0.0;
#pragma unroll
            for (int k = j + 1; k <= SS_MAXL; ++k) {
                const double lkj = __shfl_sync(0xffffffffu, lij, k);
                if (lane > j) row[k] -= lij * lkj;
            }
        }
        if (lane == 0) cs.cap = m - 1 < 1 ? 1 : m - 1;  // vector k uses levels up to k + 1
    }
    __syncwarp();
    const int built = ss_cycle_warp(S, cs.G, L, a.K, a.rel_tol, cs.cP, cs.cap);
    if (lane == 0) {
        S.lev = L;
        if (!S.done) {
            S.ext = 1;  // more powers, then the cycle again
            S.lfrom = L;
            S.lto = a.K;
        } else {
            S.ext = 0;
            S.vecs += built;
            S.vec_index_sum += built * (built - 1) / 2;
            // the update sweep reads c on p_0 .. p_{kk-1}
            for (int i = 0; i < a.K; ++i) S.h[i] = i < n ? cs.cP[i] : 0.0;
            int nl = built + 2;
            nl = nl > a.K ? a.K : nl;
            __stcg(a.lhint + s, nl);
            S.lnext = nl;
            S.ready = 1;
            S.lfrom = S.lto = 0;
        }
    }
    __syncwarp();
}

// One system's serial step after the residual sweep of restart `restart`:
// rr = ||b' - A d||^2, the residual of the next restart (GMRESSolver.cpp:248-256).
__device__ __noinline__ void ss_resid_step(const SsArgs& a, GmresSys& S, int s, double rr, int restart) {
    // the update (p_0 .. p_{kk-1} and the previous correction in, the
    // correction out) and the residual (correction, four coefficients and b'
    // in, r out), per node
    S.abytes += 8.0 * (S.kk > 1 ? S.kk : 1) + (restart > 0 ? 8.0 : 0.0) + 8.0 + 56.0;
    const int next = restart + 1;
    if (next < a.max_restarts) {
        S.rho0 = sqrt(rr);
        S.restarts += 1;
        const double resid = S.rho0 / S.norm_rhs;
        if (isnan(resid)) { S.nan = 1; S.active = 0; }
        else if (resid <= a.rel_tol || S.rho0 <= a.abs_tol) { S.conv = 1; S.active = 0; }
        else S.cycles += 1;
    } else {
        S.active = 0;  // iteration cap: the loop ends without a test
    }
    S.rst = next;
    S.ready = 0;
    S.lfrom = 0;
    S.lto = S.active ? ss_first_levels(a, s) : 0;
}

enum SsSerial : int { SS_SER_NONE = 0, SS_SER_GRAM, SS_SER_RESID };

// Serial section (last block to reach a barrier).  SS_SER_GRAM: the Gram of
// this round's powers is complete (restart 0, round 0 also takes its
// convergence test from G(0,0) = ||b'||^2); SS_SER_RESID: the residual sweep
// left ||r||^2 of the next restart in slot 0.
__device__ void ss_serial(const SsArgs& a, int kind, int restart, int round, int nblocks) {
    GmresControl* ctl = a.ctl;
    __shared__ double tot[SS_SLOTS];
    __shared__ GmresSys sS[2];
    __shared__ int s_any, s_ext;
    __shared__ int s_L[2];
    const int warp = threadIdx.x >> 5;
    constexpr int NW = (int)(sizeof(GmresSys) / 8);
    for (int s = 0; s < 2; ++s) {
        const unsigned long long* src = reinterpret_cast<const unsigned long long*>(&ctl->sys[s]);
        unsigned long long* dst = reinterpret_cast<unsigned long long*>(&sS[s]);
        for (int i = threadIdx.x; i < NW; i += SS_THREADS) dst[i] = __ldcg(src + i);
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        // the levels of this round, as every block chose them
        const int s = threadIdx.x;
        const GmresSys& S = sS[s];
        int L = 0;
        if (S.active && kind == SS_SER_GRAM) {
            if (round == 0) L = ss_first_levels(a, s);
            else L = S.ext ? a.K : 0;
        }
        s_L[s] = L;
    }
    if (threadIdx.x == 0) { s_any = 0; s_ext = 0; }
    __syncthreads();
    int used[2];
    for (int s = 0; s < 2; ++s)
        used[s] = kind == SS_SER_GRAM ? (s_L[s] + 1) * (s_L[s] + 2) / 2 : 1;
    for (int i = warp; i < used[0] + used[1]; i += SS_WARPS) {
        const int s = i < used[0] ? 0 : 1;
        const int slot = s * SS_NG + (i - s * used[0]);
        const double v = sum_slot_warp(a.part, nblocks, slot);
        if ((threadIdx.x & 31) == 0) tot[slot] = v;
    }
    __syncthreads();
    // one warp per system (warps 0 and 1)
    __shared__ SsCycleSmem cs[2];
    if (warp < 2) {
        const int s = warp;
        GmresSys& S = sS[s];
        const double* t = tot + SS_NG * s;
        const bool act = S.active;
        if (act && kind == SS_SER_GRAM && s_L[s] > 0)
            ss_gram_step(a, S, s, t, s_L[s], round == 0 ? 0 : S.lev, restart == 0 && round == 0, cs[s]);
        if ((threadIdx.x & 31) == 0) {
            if (act && kind == SS_SER_RESID) ss_resid_step(a, S, s, t[0], restart);
            atomicOr(&s_any, S.active);
            atomicOr(&s_ext, S.active && S.ext);
        }
    }
    __syncthreads();
    for (int s = 0; s < 2; ++s) {
        const unsigned long long* src = reinterpret_cast<const unsigned long long*>(&sS[s]);
        unsigned long long* dst = reinterpret_cast<unsigned long long*>(&ctl->sys[s]);
        for (int i = threadIdx.x; i < NW; i += SS_THREADS) __stcg(dst + i, src[i]);
    }
    if (threadIdx.x == 0) {
        __stcg(&ctl->any_active, s_any);
        __stcg(&ctl->any_ext, s_ext);
        __stcg(&ctl->passes, ldc(&ctl->passes) + 1);
    }
}

// Bounded grid barrier with the serial section run by the last block to
// arrive (the same protocol as the one-vector-per-sweep solver's).
__device__ bool ss_sync(const SsArgs& a, int kind, int restart, int round) {
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
        if (kind != SS_SER_NONE) ss_serial(a, kind, restart, round, nblocks);
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

__device__ __forceinline__ void ss_cp8(unsigned saddr, const double* gmem) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(saddr), "l"(gmem) : "memory");
}

// ---- powers phase ----------------------------------------------------------------
// One block: levels lfrom+1 .. lfrom+L of the rows [ya, yb) of the strip
// whose own columns start at x0, from level lfrom (p0 plain, or basis slot
// lfrom - 1).  Thread t holds column x0 - L + t (periodic); level j is valid
// on threads j .. 255 - j.  Step tau takes level 0 at row tau and computes
// level j at row tau - j from level j-1 at rows tau-j-1, tau-j (x
// neighbours, by warp shuffles and across warps from the edge buffer the
// step before wrote) and tau-j+1.  The thread's level-0 value and four
// coefficients of row tau + SS_PF are copied into its ring slot (cp.async)
// while row tau computes; level 1 takes the coefficients of its row from the
// ring and later levels reuse them from registers.  Rows outside the lattice
// are zero.  Level j is stored in basis slot lfrom + j - 1 (interleaved
// layout).
//
// The step loop is unrolled U = 3 ceil(L / 3) times so that both register
// windows are circular buffers with compile-time slots: level j's last three
// rows (row y in slot (step - j) mod 3 of H[j]) and the coefficients of the
// last U rows (row y in slot (y - t0) mod U).  The step count is rounded up
// to a multiple of U (the extra steps march past the last row: zero input,
// nothing stored).
template <int L>
__device__ void ss_powers(const SsArgs& a, const KoSystem& S, const double* p0, bool p0_basis,
                          int lfrom, int x0, int own_w, int ya, int yb, SsSmem& sm, double* ring) {
    constexpr int U = (L + 2) / 3 * 3;
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int xs = x0 - L + t;
    const int xc = ((xs % a.nx) + a.nx) % a.nx;
    const bool own = t >= L && t < L + own_w && xs < a.nx;
    const long long cbase = (long long)(xc >> 5) * 128 + (xc & 31);
    const long long cstride = 4LL * a.P;
    const long long vbase = (long long)(xc >> 5) * (a.K * 32) + (xc & 31);
    const long long vstride = (long long)a.K * a.P;
    // level-0 source: plain layout (stride P) or a basis slot (interleaved)
    const double* src0 = p0_basis ? S.V + vbase + (long long)(lfrom - 1) * 32 : p0 + xc;
    const long long s0 = p0_basis ? vstride : (long long)a.P;
    double* myring = ring + t;  // [slot][field][thread]
    const unsigned ring_s = (unsigned)__cvta_generic_to_shared(myring);
    auto issue = [&](int row) {
        const int r = row & (SS_RING - 1);
        if (row >= 0 && row < a.ny) {
            ss_cp8(ring_s + 8u * (unsigned)(r * SS_RF * SS_THREADS), src0 + (long long)row * s0);
            const double* c = S.coef + (long long)row * cstride + cbase;
#pragma unroll
            for (int q = 0; q < 4; ++q)
                ss_cp8(ring_s + 8u * (unsigned)((r * SS_RF + 1 + q) * SS_THREADS), c + 32 * q);
        } else {
#pragma unroll
            for (int f = 0; f < SS_RF; ++f) myring[(r * SS_RF + f) * SS_THREADS] = 0.0;
        }
    };
    double H[L][3];
    double cE[U], cW[U], cN[U], cS[U];
#pragma unroll
    for (int j = 0; j < L; ++j) H[j][0] = H[j][1] = H[j][2] = 0.0;
#pragma unroll
    for (int j = 0; j < U; ++j) { cE[j] = 0.0; cW[j] = 0.0; cN[j] = 0.0; cS[j] = 0.0; }
    const int t0 = ya - L, t1 = yb + L;
    const int nsteps = (t1 - t0 + U - 1) / U * U;
#pragma unroll 1
    for (int i = 0; i < SS_PF; ++i) {
        issue(t0 + i);
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    }
    // store address of level 1 at row tau - 1; level j is (j - 1) rows and slots further
    double* vrow = S.V + (long long)(t0 - 1) * vstride + vbase + (long long)lfrom * 32;
#pragma unroll 1
    for (int b = 0; b < nsteps; b += U) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int tau = t0 + b + u;
            issue(tau + SS_PF);
            asm volatile("cp.async.commit_group;\n" ::: "memory");
            asm volatile("cp.async.wait_group %0;\n" ::"n"(SS_PF) : "memory");  // rows <= tau landed
            {
                // coefficients of row tau - 1 (level 1's row)
                const int c1 = (u + U - 1) % U;
                const double* q = myring + ((tau - 1) & (SS_RING - 1)) * SS_RF * SS_THREADS;
                cE[c1] = q[1 * SS_THREADS];
                cW[c1] = q[2 * SS_THREADS];
                cN[c1] = q[3 * SS_THREADS];
                cS[c1] = q[4 * SS_THREADS];
            }
            H[0][u % 3] = myring[(tau & (SS_RING - 1)) * SS_RF * SS_THREADS];
            __syncthreads();  // the edge values of step tau - 1 are visible
            const int par = tau & 1;
            const int yl = tau - L;  // the last level's row
            const bool st_row = own && tau - 1 >= ya && yl < yb;
            // x neighbours of every level at its row of the step before
            // (level j at row tau - 1 - j)
            double lft[L], rgt[L];
#pragma unroll
            for (int j = 0; j < L; ++j) {
                const double mine = H[j][((u - 1 - j) % 3 + 3) % 3];
                lft[j] = __shfl_up_sync(0xffffffffu, mine, 1);
                rgt[j] = __shfl_down_sync(0xffffffffu, mine, 1);
            }
            if (lane == 0) {
#pragma unroll
                for (int j = 0; j < L; ++j) lft[j] = w > 0 ? sm.edge[par ^ 1][w - 1][1][j] : 0.0;
            }
            if (lane == 31) {
#pragma unroll
                for (int j = 0; j < L; ++j) rgt[j] = w < SS_WARPS - 1 ? sm.edge[par ^ 1][w + 1][0][j] : 0.0;
            }
#pragma unroll
            for (int j = 1; j <= L; ++j) {
                const int y = tau - j;
                // level j-1 at rows y + 1 (newest) and y - 1
                const int sN = ((u - (j - 1)) % 3 + 3) % 3;
                const int sS = ((u - j - 1) % 3 + 3) % 3;
                const int cs = ((u - j) % U + U) % U;
                // N p in the CSR order of an interior row without its centre: S, W, E, N
                const double v = cS[cs] * H[j - 1][sS] + cW[cs] * lft[j - 1] + cE[cs] * rgt[j - 1] +
                                 cN[cs] * H[j - 1][sN];
                if (j < L) H[j][((u - j) % 3 + 3) % 3] = v;
                if (st_row && y >= ya && y < yb) __stcg(vrow - (long long)(j - 1) * vstride + (j - 1) * 32, v);
            }
            // level j's newest row (tau - j) for the neighbours' next step
            if (lane == 0) {
#pragma unroll
                for (int j = 0; j < L; ++j) sm.edge[par][w][0][j] = H[j][((u - j) % 3 + 3) % 3];
            }
            if (lane == 31) {
#pragma unroll
                for (int j = 0; j < L; ++j) sm.edge[par][w][1][j] = H[j][((u - j) % 3 + 3) % 3];
            }
            vrow += vstride;
        }
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();  // the edge buffer and the ring are reused by the next unit
}

// ---- Gram phase -------------------------------------------------------------------
// Nodes [g0, g1) of one system, U per thread and iteration (the U (L+1)
// loads in flight together): the (L+1)(L+2)/2 products of p_0 .. p_L summed
// per thread.
template <int L, int U = 2>
__device__ __forceinline__ void ss_gram(const SsArgs& a, const KoSystem& S, const double* p0, long long g0,
                                        long long g1, double* acc) {
    constexpr int NGL = (L + 1) * (L + 2) / 2;
    double s[NGL];
#pragma unroll
    for (int i = 0; i < NGL; ++i) s[i] = 0.0;
    long long g = g0 + threadIdx.x;
    for (; g + (U - 1) * SS_THREADS < g1; g += U * SS_THREADS) {
        double p[U][L + 1];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const long long gu = g + u * SS_THREADS;
            p[u][0] = __ldcg(p0 + gu);
            const long long vb = (gu >> 5) * (a.K * 32) + (gu & 31);
#pragma unroll
            for (int j = 1; j <= L; ++j) p[u][j] = __ldcg(S.V + vb + (j - 1) * 32);
        }
#pragma unroll
        for (int j = 0; j <= L; ++j)
#pragma unroll
            for (int i = 0; i <= j; ++i) {
                double t = p[0][i] * p[0][j];
#pragma unroll
                for (int u = 1; u < U; ++u) t += p[u][i] * p[u][j];
                s[ss_gslot(i, j)] += t;
            }
    }
    if (U > 1 && g < g1) {
        double p[L + 1];
        p[0] = __ldcg(p0 + g);
        const long long vb = (g >> 5) * (a.K * 32) + (g & 31);
#pragma unroll
        for (int j = 1; j <= L; ++j) p[j] = __ldcg(S.V + vb + (j - 1) * 32);
#pragma unroll
        for (int j = 0; j <= L; ++j)
#pragma unroll
            for (int i = 0; i <= j; ++i) s[ss_gslot(i, j)] += p[i] * p[j];
    }
#pragma unroll
    for (int i = 0; i < NGL; ++i) acc[i] = s[i];
}

// The same sums with each thread's node values streamed through a ring of
// SP_GRAM_RING nodes in dynamic shared memory ([slot][level][thread],
// cp.async SP_GRAM_RING - 1 nodes ahead): the (L+1)(L+2)/2 sums hold most of
// a thread's registers, so the loads in flight come from the ring, not from
// more warps.  Each thread reads back only what it copied: no barrier.
constexpr int SP_GRAM_RING = 4;
__host__ __device__ constexpr size_t sp_gram_dsmem(int L) {
    return sizeof(double) * SP_GRAM_RING * (L + 1) * SS_THREADS;
}
__device__ __forceinline__ void ss_cp8(double* dst, const double* src) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(src) : "memory");
}
template <int L>
__device__ __forceinline__ void ss_gram_ring(const SsArgs& a, const KoSystem& S, const double* p0, long long g0,
                                             long long g1, double* ring, double* acc) {
    constexpr int NGL = (L + 1) * (L + 2) / 2;
    constexpr int R = SP_GRAM_RING;
    double s[NGL];
#pragma unroll
    for (int i = 0; i < NGL; ++i) s[i] = 0.0;
    double* mine = ring + threadIdx.x;
    auto issue = [&](long long g, int slot) {
        if (g < g1) {
            double* d = mine + slot * (L + 1) * SS_THREADS;
            ss_cp8(d, p0 + g);
            const long long vb = (g >> 5) * (a.K * 32) + (g & 31);
#pragma unroll
            for (int j = 1; j <= L; ++j) ss_cp8(d + j * SS_THREADS, S.V + vb + (j - 1) * 32);
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };
    long long g = g0 + threadIdx.x;
#pragma unroll
    for (int k = 0; k < R - 1; ++k) issue(g + k * SS_THREADS, k);
    for (int slot = 0; g < g1; g += SS_THREADS, slot = (slot + 1) & (R - 1)) {
        // the copies of node g + (R - 1) threads-strides ahead go into the slot
        // read in the previous iteration
        issue(g + (R - 1) * SS_THREADS, (slot + R - 1) & (R - 1));
        asm volatile("cp.async.wait_group %0;\n" ::"n"(R - 1) : "memory");
        const double* d = mine + slot * (L + 1) * SS_THREADS;
        double p[L + 1];
#pragma unroll
        for (int j = 0; j <= L; ++j) p[j] = d[j * SS_THREADS];
#pragma unroll
        for (int j = 0; j <= L; ++j)
#pragma unroll
            for (int i = 0; i <= j; ++i) s[ss_gslot(i, j)] += p[i] * p[j];
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < NGL; ++i) acc[i] = s[i];
}

__device__ void ss_block_reduce(const double* v, int n, double* part, int base, SsSmem& sm) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int s = 0; s < n; ++s) {
        double x = v[s];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
        if (lane == 0) sm.red[warp][s] = x;
    }
    __syncthreads();
    for (int s = threadIdx.x; s < n; s += SS_THREADS) {
        double x = 0.0;
#pragma unroll
        for (int w = 0; w < SS_WARPS; ++w) x += sm.red[w][s];
        part[(long long)(base + s) * gridDim.x + blockIdx.x] = x;
    }
    __syncthreads();
}

// ---- the solver kernel ------------------------------------------------------------------
__global__ void __launch_bounds__(SS_THREADS, 1)
sstep_kernel(const SsArgs a) {
    GmresControl* ctl = a.ctl;
    __shared__ SsSmem sm;
    extern __shared__ __align__(16) double ss_ring[];
    double* ring = ss_ring;
    if (blockIdx.x == 0 && threadIdx.x == 0) __stcg(&ctl->t_start, globaltimer_ns());
    const long long stride = (long long)gridDim.x * SS_THREADS;
    const long long t0 = (long long)blockIdx.x * SS_THREADS + threadIdx.x;
    for (int restart = 0; restart < a.max_restarts; ++restart) {
        for (int round = 0;; ++round) {
            // ---- levels of this round ----------------------------------------------------
            if (threadIdx.x < 2) {
                const int s = threadIdx.x;
                const int act = ldc(&ctl->sys[s].active);
                int lf = 0, lt = 0;
                if (act) {
                    if (round == 0) lt = ss_first_levels(a, s);
                    else if (ldc(&ctl->sys[s].ext)) { lf = ldc(&ctl->sys[s].lev); lt = a.K; }
                }
                sm.act[s] = act;
                sm.lfrom[s] = lf;
                sm.lto[s] = lt;
            }
            __syncthreads();
            // ---- powers ---------------------------------------------------------------
            {
                const int units = a.pstrips * a.prows;
                for (int u = blockIdx.x; u < 2 * units; u += gridDim.x) {
                    const int s = u / units, r = u % units;
                    const int lf = sm.lfrom[s], L = sm.lto[s] - lf;
                    if (L <= 0) continue;  // block-uniform
                    const int strip = r % a.pstrips, rr = r / a.pstrips;
                    const int ya = (int)((long long)rr * a.ny / a.prows);
                    const int yb = (int)((long long)(rr + 1) * a.ny / a.prows);
                    const KoSystem& S = a.sys[s];
                    const double* p0 = restart == 0 ? S.rhs : ((restart & 1) ? S.r2 : S.r);
                    // strips are laid out for K levels of halo: own columns x0 .. x0 + 255 - 2K
                    const int ow = SS_THREADS - 2 * a.K;
                    const int x0 = strip * ow;
                    switch (L) {
#define KOFM_SSP(n) \
    case n: ss_powers<n>(a, S, p0, lf > 0, lf, x0, ow, ya, yb, sm, ring); break;
                        KOFM_SSP(1) KOFM_SSP(2) KOFM_SSP(3) KOFM_SSP(4) KOFM_SSP(5)
                        KOFM_SSP(6) KOFM_SSP(7) KOFM_SSP(8) KOFM_SSP(9) KOFM_SSP(10)
#undef KOFM_SSP
                        default: break;
                    }
                }
            }
            if (!ss_sync(a, SS_SER_NONE, restart, round)) return;
            // ---- Gram of p_0 .. p_lto ----------------------------------------------------
            for (int s = 0; s < 2; ++s) {
                double acc[SS_NG];
                const int L = sm.lto[s];
                const int ng = (L + 1) * (L + 2) / 2;
                if (L > 0) {
                    const KoSystem& S = a.sys[s];
                    const double* p0 = restart == 0 ? S.rhs : ((restart & 1) ? S.r2 : S.r);
                    // a fixed contiguous node range per block (deterministic sums)
                    const long long n32 = a.D / 32;
                    const long long g0 = n32 * blockIdx.x / gridDim.x * 32;
                    const long long g1 = n32 * (blockIdx.x + 1) / gridDim.x * 32;
                    switch (L) {
#define KOFM_SSG(n) \
    case n: ss_gram<n>(a, S, p0, g0, g1, acc); break;
                        KOFM_SSG(1) KOFM_SSG(2) KOFM_SSG(3) KOFM_SSG(4) KOFM_SSG(5)
                        KOFM_SSG(6) KOFM_SSG(7) KOFM_SSG(8) KOFM_SSG(9) KOFM_SSG(10)
#undef KOFM_SSG
                        default: break;
                    }
                }
                ss_block_reduce(acc, L > 0 ? ng : 0, a.part, SS_NG * s, sm);
            }
            if (!ss_sync(a, SS_SER_GRAM, restart, round)) return;
            if (!ldc(&ctl->any_ext)) break;
        }
        if (!ldc(&ctl->any_active)) break;
        // ---- d = d_prev + sum c_j p_j (pointwise) -------------------------------------
        if (threadIdx.x < 2) {
            const int s = threadIdx.x;
            sm.act[s] = ldc(&ctl->sys[s].active);
            sm.kk[s] = ldc(&ctl->sys[s].kk);
        }
        if (threadIdx.x < 2 * (SS_MAXL + 1)) {
            const int s = threadIdx.x / (SS_MAXL + 1), i = threadIdx.x % (SS_MAXL + 1);
            sm.c[s][i] = i < a.K ? ldc(&ctl->sys[s].h[i]) : 0.0;
        }
        __syncthreads();
        // restart n reads the residual and correction of parity n and writes
        // those of parity n + 1 (restart 0: b' and d = 0)
        for (int s = 0; s < 2; ++s) {
            if (!sm.act[s]) continue;
            const KoSystem& S = a.sys[s];
            const double* p0 = restart == 0 ? S.rhs : ((restart & 1) ? S.r2 : S.r);
            const double* xin = restart == 0 ? nullptr : ((restart & 1) ? S.x2 : S.x);
            double* xout = (restart & 1) ? S.x : S.x2;
            double cr[SS_MAXL];
#pragma unroll
            for (int j = 0; j < SS_MAXL; ++j) cr[j] = sm.c[s][j];
            const int kk = sm.kk[s];
            const long long npairs = a.D / 2;
            // two node pairs per thread and iteration: their loads in flight together
            for (long long pr = t0; pr < npairs; pr += 2 * stride) {
                const long long pb = pr + stride < npairs ? pr + stride : pr;
                const long long g[2] = {pr * 2, pb * 2};  // g, g + 1 share a 32-node group
                double2 d[2], r[2];
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    d[u] = xin ? __ldcg(reinterpret_cast<const double2*>(xin + g[u])) : make_double2(0.0, 0.0);
                    r[u] = __ldcg(reinterpret_cast<const double2*>(p0 + g[u]));
                }
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    d[u].x += cr[0] * r[u].x;
                    d[u].y += cr[0] * r[u].y;
                }
#pragma unroll
                for (int j = 1; j < SS_MAXL; ++j) {
                    if (j >= kk) break;
                    double2 p[2];
#pragma unroll
                    for (int u = 0; u < 2; ++u)
                        p[u] = __ldcg(reinterpret_cast<const double2*>(
                            S.V + (g[u] >> 5) * (a.K * 32) + (g[u] & 31) + (j - 1) * 32));
#pragma unroll
                    for (int u = 0; u < 2; ++u) {
                        d[u].x += cr[j] * p[u].x;
                        d[u].y += cr[j] * p[u].y;
                    }
                }
#pragma unroll
                for (int u = 0; u < 2; ++u) __stcg(reinterpret_cast<double2*>(xout + g[u]), d[u]);
            }
        }
        if (!ss_sync(a, SS_SER_NONE, restart, 0)) return;
        // ---- r = b' - A d, ||r||^2 -------------------------------------------------------
        for (int s = 0; s < 2; ++s) {
            double acc = 0.0;
            if (sm.act[s]) {
                const KoSystem& S = a.sys[s];
                const double* xd = (restart & 1) ? S.x : S.x2;
                double* rout = (restart & 1) ? S.r : S.r2;
                const long long npairs = a.D / 2;
                for (long long pr = t0; pr < npairs; pr += stride) {
                    const long long g = pr * 2;
                    const int y = (int)(g / a.P), x = (int)(g - (long long)y * a.P);
                    double rr[2] = {0.0, 0.0};
                    const long long row = (long long)y * a.P;
#pragma unroll
                    for (int j = 0; j < 2; ++j) {
                        const int xj = x + j;
                        if (xj >= a.nx) continue;
                        const long long gj = g + j;
                        const int xw = xj > 0 ? xj - 1 : a.nx - 1;
                        const int xe = xj + 1 < a.nx ? xj + 1 : 0;
                        const double* cf = S.coef + ilv(4, 0, gj);
                        // rows 0 and ny-1 are solid: their off-diagonals are 0
                        const double dS = y > 0 ? __ldcg(xd + gj - a.P) : 0.0;
                        const double dN = y + 1 < a.ny ? __ldcg(xd + gj + a.P) : 0.0;
                        // CSR order of an interior row: S, W, C, E, N
                        const double Ad = __ldg(cf + 96) * dS + __ldg(cf + 32) * __ldcg(xd + row + xw) +
                                          __ldcg(xd + gj) + __ldg(cf) * __ldcg(xd + row + xe) +
                                          __ldg(cf + 64) * dN;
                        rr[j] = __ldg(S.rhs + gj) - Ad;
                    }
                    __stcg(reinterpret_cast<double2*>(rout + g), make_double2(rr[0], rr[1]));
                    acc += rr[0] * rr[0] + rr[1] * rr[1];
                }
            }
            ss_block_reduce(&acc, sm.act[s] ? 1 : 0, a.part, SS_NG * s, sm);
        }
        if (!ss_sync(a, SS_SER_RESID, restart, 0)) return;
        if (!ldc(&ctl->any_active)) break;
    }

    // ---- x_new = x0 + d on fluid nodes; solid-boundary rows -> 0 -----------------
    // A solve that met a NaN residual leaves its field as it was.
    const long long npairs = a.D / 2;
    for (int s = 0; s < 2; ++s) {
        const KoSystem& S = a.sys[s];
        float* f = static_cast<float*>(a.field[s]);
        double* f8 = static_cast<double*>(a.field[s]);
        // the correction of the last of `cycles` updates is in parity `cycles`
        const int cyc = ldc(&ctl->sys[s].cycles);
        const bool has_x = cyc > 0 && !ldc(&ctl->sys[s].nan);
        const double* xf = (cyc & 1) ? S.x2 : S.x;
        for (long long pr = t0; pr < npairs; pr += stride) {
            const long long g = pr * 2;
            const int y = (int)(g / a.P), x = (int)(g - (long long)y * a.P);
            if (x >= a.nx) continue;
            const unsigned int t2 = *reinterpret_cast<const unsigned int*>(a.ntype + g);
            const int tt[2] = {(int)(t2 & 0xffff), (int)(t2 >> 16)};
            const double2 xv = has_x ? __ldcg(reinterpret_cast<const double2*>(xf + g)) : make_double2(0.0, 0.0);
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

// ---- the same solver as separate phase launches -----------------------------------------
// sstep_kernel's sweeps and serial steps, each sweep its own launch with its
// own grid and register budget (the pointwise sweeps run at full occupancy,
// the powers and Gram sweeps are compiled per level count).  The host
// enqueues one round at a time: per system its powers and Gram sweeps, then
// the update, residual and write-back sweeps of both systems; each sweep
// reads what it has to do from the control block (a system whose cycle asks
// for more powers skips the update; a finished one is written back once), and
// the host reads the control block after the round to enqueue the next (an
// extension round, or the next restart) while a system is still iterating.
// The serial steps run in the last block to finish a sweep (ticket counter,
// no grid barrier and no spin-wait).

// Launch shapes of the phase sweeps (host side, per level count).
struct SsLaunch {
    int pow_grid[SS_MAXL + 1];   // powers sweep of L levels: blocks
    int pow_prows[SS_MAXL + 1];  // and row ranges per strip
    int gram_grid[SS_MAXL + 1];  // Gram sweep of p_0 .. p_L: blocks
    int pt_grid;                 // update / residual / write-back sweeps: blocks
};

// blocks per SM the powers sweep of L levels is compiled for (its per-thread
// state is 9 L doubles)
__host__ __device__ constexpr int sp_pow_minb(int L) { return L <= 5 ? 2 : 1; }

// True in every thread of the block that finishes a sweep last; that block
// then sees every other block's partial sums.  Resets the ticket counter for
// the next sweep on the stream.
__device__ __forceinline__ bool sp_last_block(GridBarrier* bar) {
    __shared__ int s_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned int ticket = atomicAdd(&bar->count, 1u);
        s_last = ticket == gridDim.x - 1u;
        if (s_last) atomicExch(&bar->count, 0u);
    }
    __syncthreads();
    if (s_last) __threadfence();
    return s_last;
}

__device__ __forceinline__ void sp_sys_load(const GmresControl* ctl, int s, GmresSys& dst) {
    constexpr int NW = (int)(sizeof(GmresSys) / 8);
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(&ctl->sys[s]);
    unsigned long long* d = reinterpret_cast<unsigned long long*>(&dst);
    for (int i = threadIdx.x; i < NW; i += blockDim.x) d[i] = __ldcg(src + i);
}

__device__ __forceinline__ void sp_sys_store(GmresControl* ctl, int s, const GmresSys& src) {
    constexpr int NW = (int)(sizeof(GmresSys) / 8);
    const unsigned long long* sp = reinterpret_cast<const unsigned long long*>(&src);
    unsigned long long* d = reinterpret_cast<unsigned long long*>(&ctl->sys[s]);
    for (int i = threadIdx.x; i < NW; i += blockDim.x) __stcg(d + i, sp[i]);
}

// Block reduction of N per-thread sums into part[base + i][blockIdx.x].
template <int N>
__device__ __forceinline__ void sp_block_reduce(const double (&v)[N], double* part, int base, SsSmem& sm) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int s = 0; s < N; ++s) {
        double x = v[s];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
        if (lane == 0) sm.red[warp][s] = x;
    }
    __syncthreads();
    for (int s = threadIdx.x; s < N; s += SS_THREADS) {
        double x = 0.0;
#pragma unroll
        for (int w = 0; w < SS_WARPS; ++w) x += sm.red[w][s];
        part[(long long)(base + s) * gridDim.x + blockIdx.x] = x;
    }
    __syncthreads();
}

// Sub-stepping state of one context (device memory; the host pushes a reset
// when a state is loaded and reads it back when it synchronises).
struct KoStepState {
    double dt;             // kOmega::timeStep (first member: the assembly reads it by address)
    int steps_per_lb;      // kOmega::stepsPerLB
    int time_since_change; // kOmega::timeSinceTimeStepChange
    int cur;               // sub-step of the running update
    int status;            // KOFM_OK, or the error that stopped updates (sticky until a reset)
    int fail_solves;       // kofm_debug_fail_solves: solves still to report a NaN
    int fail_mask;
    int substeps;          // solves of the last update
    int launches;          // kernel launches of the last update
    long long updates;     // updates run since the last reset
    long long launches_total;  // kernel launches of all updates since the last reset
};

// Control block of a solve: both systems iterating, restart 0, first round
// of L0 / L1 powers (chosen by the host from the cycle lengths seen so far);
// a pending failure injection (kofm_debug_fail_solves) is taken from st.
__global__ void sp_init_kernel(GmresControl* ctl, GridBarrier* bar, KoStepState* st, int L0, int L1) {
    constexpr int NW = (int)(sizeof(GmresControl) / sizeof(unsigned int));
    unsigned int* w = reinterpret_cast<unsigned int*>(ctl);
    for (int i = threadIdx.x; i < NW; i += blockDim.x) w[i] = 0u;
    __syncthreads();
    if (threadIdx.x == 0) {
        int inject = 0;
        if (st->fail_solves > 0) {
            inject = st->fail_mask;
            st->fail_solves--;
        }
        for (int s = 0; s < 2; ++s) {
            ctl->sys[s].active = 1;
            ctl->sys[s].inject = (inject >> s) & 1;
            ctl->sys[s].lto = s == 0 ? L0 : L1;
        }
        ctl->any_active = 1;
        ctl->t_start = globaltimer_ns();
        bar->count = 0u;
        bar->gen = 0u;
    }
}

// The pending round of system s as the host launched it; false (and the
// error word set to 2) if the control block disagrees.
__device__ __forceinline__ bool sp_round(const SsArgs& a, int s, int lev, bool powers, int& lf, int& lt,
                                         int& rst) {
    const GmresSys* S = &a.ctl->sys[s];
    const int act = ldc(&S->active);
    lf = ldc(&S->lfrom);
    lt = ldc(&S->lto);
    rst = ldc(&S->rst);
    if (!act || lt <= lf) return false;
    if ((powers ? lt - lf : lt) != lev) {
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicExch(&a.ctl->error, 2);
        return false;
    }
    return true;
}

// Powers lfrom + 1 .. lto (= lfrom + L) of system s; units (strip, row
// range) of its lattice over the grid.
template <int L>
__global__ void __launch_bounds__(SS_THREADS, sp_pow_minb(L))
sp_powers_kernel(const SsArgs a, int s) {
    __shared__ SsSmem sm;
    extern __shared__ __align__(16) double ss_ring[];
    int lf, lt, rst;
    if (!sp_round(a, s, L, true, lf, lt, rst)) return;
    const KoSystem& S = a.sys[s];
    const double* p0 = rst == 0 ? S.rhs : ((rst & 1) ? S.r2 : S.r);
    const int ow = SS_THREADS - 2 * a.K;
    const int units = a.pstrips * a.prows;
    for (int u = blockIdx.x; u < units; u += gridDim.x) {
        const int strip = u % a.pstrips, rr = u / a.pstrips;
        const int ya = (int)((long long)rr * a.ny / a.prows);
        const int yb = (int)((long long)(rr + 1) * a.ny / a.prows);
        ss_powers<L>(a, S, p0, lf > 0, lf, strip * ow, ow, ya, yb, sm, ss_ring);
    }
}

// Gram of p_0 .. p_L of system s; the last block runs the system's serial
// step (the simpler-GMRES cycle in the power basis, one warp).  Each block
// takes a fixed contiguous range of nodes (deterministic sums); a thread
// takes one node per iteration, its L + 1 values copied SP_GRAM_RING - 1
// iterations ahead (dynamic shared memory: sp_gram_dsmem(L)).
template <int L>
__global__ void __launch_bounds__(SS_THREADS)
sp_gram_kernel(const SsArgs a, int s) {
    constexpr int NGL = (L + 1) * (L + 2) / 2;
    __shared__ SsSmem sm;
    int lf, lt, rst;
    if (!sp_round(a, s, L, false, lf, lt, rst)) return;
    const KoSystem& S = a.sys[s];
    const double* p0 = rst == 0 ? S.rhs : ((rst & 1) ? S.r2 : S.r);
    const int tid = threadIdx.x;
    {
        const long long n32 = a.D / 32;
        const long long g0 = n32 * blockIdx.x / gridDim.x * 32;
        const long long g1 = n32 * (blockIdx.x + 1) / gridDim.x * 32;
        extern __shared__ __align__(16) double sp_gram_ring_smem[];
        double acc[SS_NG];
        ss_gram_ring<L>(a, S, p0, g0, g1, sp_gram_ring_smem, acc);
        double v[NGL];
#pragma unroll
        for (int i = 0; i < NGL; ++i) v[i] = acc[i];
        sp_block_reduce<NGL>(v, a.part, 0, sm);
    }
    if (!sp_last_block(a.bar)) return;
    __shared__ double tot[SS_NG];
    __shared__ GmresSys sS;
    sp_sys_load(a.ctl, s, sS);
    const int warp = tid >> 5;
    for (int i = warp; i < NGL; i += SS_WARPS) {
        const double v = sum_slot_warp(a.part, gridDim.x, i);
        if ((tid & 31) == 0) tot[i] = v;
    }
    __syncthreads();
    __shared__ SsCycleSmem cs;
    if (warp == 0) ss_gram_step(a, sS, s, tot, L, lf, rst == 0 && lf == 0, cs);
    if (tid == 0) {
        trace_barrier(a.ctl);
        __stcg(&a.ctl->passes, ldc(&a.ctl->passes) + 1);
    }
    __syncthreads();
    sp_sys_store(a.ctl, s, sS);
}

// d = d_prev + sum_j c_j p_j of every system with a finished cycle
// (pointwise; restart n reads the correction of parity n and writes parity
// n + 1, restart 0 starts from d = 0).
__global__ void __launch_bounds__(SS_THREADS)
sp_update_kernel(const SsArgs a) {
    __shared__ double c[2][SS_MAXL];
    __shared__ int act[2], kk[2], rs[2];
    if (threadIdx.x < 2) {
        const int s = threadIdx.x;
        const GmresSys* S = &a.ctl->sys[s];
        act[s] = ldc(&S->active) && ldc(&S->ready);
        kk[s] = ldc(&S->kk);
        rs[s] = ldc(&S->rst);
    }
    if (threadIdx.x < 2 * SS_MAXL) {
        const int s = threadIdx.x / SS_MAXL, i = threadIdx.x % SS_MAXL;
        c[s][i] = i < a.K ? ldc(&a.ctl->sys[s].h[i]) : 0.0;
    }
    __syncthreads();
    const long long stride = (long long)gridDim.x * SS_THREADS;
    const long long npairs = a.D / 2;
    for (int s = 0; s < 2; ++s) {
        if (!act[s]) continue;
        const KoSystem& S = a.sys[s];
        const int restart = rs[s];
        const double* p0 = restart == 0 ? S.rhs : ((restart & 1) ? S.r2 : S.r);
        const double* xin = restart == 0 ? nullptr : ((restart & 1) ? S.x2 : S.x);
        double* xout = (restart & 1) ? S.x : S.x2;
        double cr[SS_MAXL];
#pragma unroll
        for (int j = 0; j < SS_MAXL; ++j) cr[j] = c[s][j];
        const int n = kk[s];
        for (long long pr = (long long)blockIdx.x * SS_THREADS + threadIdx.x; pr < npairs; pr += stride) {
            const long long g = pr * 2;  // g, g + 1 share a 32-node group
            double2 d = xin ? __ldcg(reinterpret_cast<const double2*>(xin + g)) : make_double2(0.0, 0.0);
            const double2 r = __ldcg(reinterpret_cast<const double2*>(p0 + g));
            double2 p[SS_MAXL - 1];
            const double* vb = S.V + (g >> 5) * (a.K * 32) + (g & 31);
            // coefficients past kk are exact zeros: their directions are not read
#pragma unroll
            for (int j = 1; j < SS_MAXL; ++j)
                p[j - 1] = j < n ? __ldcg(reinterpret_cast<const double2*>(vb + (j - 1) * 32)) : make_double2(0.0, 0.0);
            d.x += cr[0] * r.x;
            d.y += cr[0] * r.y;
#pragma unroll
            for (int j = 1; j < SS_MAXL; ++j) {
                d.x += cr[j] * p[j - 1].x;
                d.y += cr[j] * p[j - 1].y;
            }
            __stcg(reinterpret_cast<double2*>(xout + g), d);
        }
    }
}

// r = b' - A d and ||r||^2 of every system with a finished cycle; the last
// block runs their serial steps (the next restart's convergence test).
__global__ void __launch_bounds__(SS_THREADS)
sp_resid_kernel(const SsArgs a) {
    __shared__ SsSmem sm;
    __shared__ int act[2], rs[2];
    if (threadIdx.x < 2) {
        const int s = threadIdx.x;
        act[s] = ldc(&a.ctl->sys[s].active) && ldc(&a.ctl->sys[s].ready);
        rs[s] = ldc(&a.ctl->sys[s].rst);
    }
    __syncthreads();
    if (!act[0] && !act[1]) return;
    // units of (row, chunk of 2 x 256 columns): one 32-bit division per unit
    const int cpr = (a.P / 2 + SS_THREADS - 1) / SS_THREADS;
    const int units = a.ny * cpr;
    for (int s = 0; s < 2; ++s) {
        double acc[1] = {0.0};
        if (act[s]) {
            const KoSystem& S = a.sys[s];
            const int restart = rs[s];
            const double* xd = (restart & 1) ? S.x : S.x2;
            double* rout = (restart & 1) ? S.r : S.r2;
            for (int u = blockIdx.x; u < units; u += gridDim.x) {
                const int y = u / cpr;
                const int x = ((u - y * cpr) * SS_THREADS + threadIdx.x) * 2;
                if (x >= a.P) continue;
                const long long g = (long long)y * a.P + x;
                double rr[2] = {0.0, 0.0};
                const long long row = (long long)y * a.P;
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    const int xj = x + j;
                    if (xj >= a.nx) continue;
                    const long long gj = g + j;
                    const int xw = xj > 0 ? xj - 1 : a.nx - 1;
                    const int xe = xj + 1 < a.nx ? xj + 1 : 0;
                    const double* cf = S.coef + ilv(4, 0, gj);
                    // rows 0 and ny-1 are solid: their off-diagonals are 0
                    const double dS = y > 0 ? __ldcg(xd + gj - a.P) : 0.0;
                    const double dN = y + 1 < a.ny ? __ldcg(xd + gj + a.P) : 0.0;
                    // CSR order of an interior row: S, W, C, E, N
                    const double Ad = __ldg(cf + 96) * dS + __ldg(cf + 32) * __ldcg(xd + row + xw) +
                                      __ldcg(xd + gj) + __ldg(cf) * __ldcg(xd + row + xe) +
                                      __ldg(cf + 64) * dN;
                    rr[j] = __ldg(S.rhs + gj) - Ad;
                }
                __stcg(reinterpret_cast<double2*>(rout + g), make_double2(rr[0], rr[1]));
                acc[0] += rr[0] * rr[0] + rr[1] * rr[1];
            }
        }
        sp_block_reduce<1>(acc, a.part, SS_NG * s, sm);
    }
    if (!sp_last_block(a.bar)) return;
    __shared__ double tot[2];
    __shared__ GmresSys sS[2];
    sp_sys_load(a.ctl, 0, sS[0]);
    sp_sys_load(a.ctl, 1, sS[1]);
    const int warp = threadIdx.x >> 5;
    if (warp < 2) {
        const double v = sum_slot_warp(a.part, gridDim.x, SS_NG * warp);
        if ((threadIdx.x & 31) == 0) tot[warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < 2 && act[threadIdx.x])
        ss_resid_step(a, sS[threadIdx.x], threadIdx.x, tot[threadIdx.x], rs[threadIdx.x]);
    if (threadIdx.x == 0) {
        trace_barrier(a.ctl);
        __stcg(&a.ctl->passes, ldc(&a.ctl->passes) + 1);
    }
    __syncthreads();
    sp_sys_store(a.ctl, 0, sS[0]);
    sp_sys_store(a.ctl, 1, sS[1]);
    if (threadIdx.x == 0) __stcg(&a.ctl->any_active, (int)(sS[0].active || sS[1].active));
}

// x_new = x0 + d on fluid nodes and 0 on solid-boundary rows, once per
// system, as soon as it has stopped iterating; a solve that met a NaN
// residual leaves its field as it was.
__global__ void __launch_bounds__(SS_THREADS)
sp_write_kernel(const SsArgs a) {
    __shared__ int wr[2], hx[2], cy[2];
    if (threadIdx.x < 2) {
        const int s = threadIdx.x;
        const GmresSys* S = &a.ctl->sys[s];
        wr[s] = !ldc(&S->active) && !ldc(&S->written);
        cy[s] = ldc(&S->cycles);
        hx[s] = cy[s] > 0 && !ldc(&S->nan);
    }
    __syncthreads();
    if (!wr[0] && !wr[1]) return;
    const int cpr = (a.P / 2 + SS_THREADS - 1) / SS_THREADS;
    const int units = a.ny * cpr;
    for (int s = 0; s < 2; ++s) {
        if (!wr[s]) continue;
        const KoSystem& S = a.sys[s];
        float* f = static_cast<float*>(a.field[s]);
        double* f8 = static_cast<double*>(a.field[s]);
        // the correction of the last of `cycles` updates is in parity `cycles`
        const double* xf = (cy[s] & 1) ? S.x2 : S.x;
        for (int u = blockIdx.x; u < units; u += gridDim.x) {
            const int y = u / cpr;
            const int x = ((u - y * cpr) * SS_THREADS + threadIdx.x) * 2;
            if (x >= a.nx) continue;
            const long long g = (long long)y * a.P + x;
            const unsigned int t2 = *reinterpret_cast<const unsigned int*>(a.ntype + g);
            const int tt[2] = {(int)(t2 & 0xffff), (int)(t2 >> 16)};
            const double2 xv = hx[s] ? __ldcg(reinterpret_cast<const double2*>(xf + g)) : make_double2(0.0, 0.0);
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
    if (sp_last_block(a.bar) && threadIdx.x < 2 && wr[threadIdx.x])
        __stcg(&a.ctl->sys[threadIdx.x].written, 1);
}

// ---- the update as a device-driven graph -------------------------------------------------
// kOmega::Solve (kOmega.cpp:31-73: the doubling test, then sub-steps of
// assembly + both solves, halving dt on a NaN residual) with every decision
// taken on the device: these kernels set the conditions of the graph's WHILE
// and SWITCH nodes (cudaGraphSetConditional), so a time step needs no host
// round trip.  The loops are bounded by counters the kernels keep: a solve by
// its round cap, an update by the halving cap (steps_per_lb <= 2^20) and a
// total of KU_MAX_SUBSTEPS solves.

constexpr int KU_MAX_SUBSTEPS = (1 << 21) + 64;  // above any sequence the halving cap allows

__global__ void ku_reset_kernel(KoStepState* st, double dt, int steps_per_lb) {
    if (threadIdx.x) return;
    st->dt = dt;
    st->steps_per_lb = steps_per_lb;
    st->time_since_change = 0;
    st->cur = 0;
    st->status = 0;
    st->substeps = 0;
    st->launches = 0;
    st->updates = 0;
    st->launches_total = 0;
}

__global__ void ku_fail_kernel(KoStepState* st, int n, int mask) {
    if (threadIdx.x) return;
    st->fail_solves = n;
    st->fail_mask = mask;
}

// Start of an update: the doubling test (doubleTimeStep, kOmega.cpp:401-414)
// and the sub-step loop's condition.
// The assembly node of the update graph takes its time step as a kernel
// parameter (constant bank) that these kernels rewrite whenever dt changes
// (asm_node non-null); else the assembly reads dt from st.
__device__ __forceinline__ void ku_set_dt(cudaGraphDeviceNode_t asm_node, size_t dt_offset, double dt) {
    if (asm_node) cudaGraphKernelNodeSetParam(asm_node, dt_offset, &dt, sizeof(double));
}

__global__ void ku_begin_kernel(KoStepState* st, cudaGraphConditionalHandle sub, cudaGraphDeviceNode_t asm_node,
                                unsigned long long dt_offset) {
    if (threadIdx.x) return;
    if (st->status) {
        cudaGraphSetConditional(sub, 0);
        return;
    }
    st->time_since_change++;
    if (st->time_since_change >= 20) {
        st->time_since_change = 0;
        if (st->steps_per_lb != 1) {
            st->steps_per_lb /= 2;
            st->dt *= 2.0;
        }
    }
    ku_set_dt(asm_node, dt_offset, st->dt);
    st->cur = 0;
    st->substeps = 0;
    st->launches = 1;  // this kernel
    st->launches_total++;
    st->updates++;
    cudaGraphSetConditional(sub, st->cur < st->steps_per_lb ? 1u : 0u);
}

// Control block of one solve (as sp_init_kernel), the first round's levels
// from the cycle lengths kept per system, a pending failure injection, and
// the round loop's condition.
__global__ void ku_init_kernel(GmresControl* ctl, GridBarrier* bar, KoStepState* st, const int* lhint, int K,
                               cudaGraphConditionalHandle round) {
    constexpr int NW = (int)(sizeof(GmresControl) / sizeof(unsigned int));
    unsigned int* w = reinterpret_cast<unsigned int*>(ctl);
    for (int i = threadIdx.x; i < NW; i += blockDim.x) w[i] = 0u;
    __syncthreads();
    if (threadIdx.x == 0) {
        int inject = 0;
        if (st->fail_solves > 0) {
            inject = st->fail_mask;
            st->fail_solves--;
        }
        for (int s = 0; s < 2; ++s) {
            int l = lhint[s];
            l = l <= 0 || l > K ? K : l;
            l = l < SS_MINL ? (K < SS_MINL ? K : SS_MINL) : l;
            ctl->sys[s].active = 1;
            ctl->sys[s].inject = (inject >> s) & 1;
            ctl->sys[s].lto = l;
        }
        ctl->any_active = 1;
        ctl->t_start = globaltimer_ns();
        bar->count = 0u;
        bar->gen = 0u;
        cudaGraphSetConditional(round, 1u);
    }
}

// The kernels of this round: SWITCH values L - 1 for the powers sweep of L
// levels and the Gram sweep of p_0 .. p_L of each system (SS_MAXL: none).
__global__ void ku_select_kernel(GmresControl* ctl, cudaGraphConditionalHandle p0, cudaGraphConditionalHandle p1,
                                 cudaGraphConditionalHandle g0, cudaGraphConditionalHandle g1) {
    if (threadIdx.x) return;
    int n = 5;  // select, update, residual, write-back, end
    unsigned pv[2], gv[2];
    for (int s = 0; s < 2; ++s) {
        const GmresSys& S = ctl->sys[s];
        const bool run = S.active && S.lto > S.lfrom;
        pv[s] = run ? (unsigned)(S.lto - S.lfrom - 1) : (unsigned)SS_MAXL;
        gv[s] = run ? (unsigned)(S.lto - 1) : (unsigned)SS_MAXL;
        n += run ? 2 : 0;
    }
    ctl->launches += n;
    cudaGraphSetConditional(p0, pv[0]);
    cudaGraphSetConditional(p1, pv[1]);
    cudaGraphSetConditional(g0, gv[0]);
    cudaGraphSetConditional(g1, gv[1]);
}

// End of a round: the round loop goes on while a system iterates, up to
// max_rounds (a solve past that cap, or a failed sweep, stops the update).
__global__ void ku_round_end_kernel(GmresControl* ctl, KoStepState* st, int max_rounds,
                                    cudaGraphConditionalHandle round) {
    if (threadIdx.x) return;
    const int r = ++ctl->rounds;
    const bool any = ctl->sys[0].active || ctl->sys[1].active;
    unsigned go = any ? 1u : 0u;
    if (ctl->error) {
        st->status = ctl->error == 2 ? KOFM_ERR_STATE : KOFM_ERR_TIMEOUT;
        go = 0u;
    } else if (any && r >= max_rounds) {
        st->status = KOFM_ERR_STATE;
        go = 0u;
    }
    cudaGraphSetConditional(round, go);
}

// End of a sub-step: halveTimeStep on a NaN residual (omega first, then k;
// kOmega.cpp:68-70, 387-399), the halving cap, and the sub-step loop's
// condition.
__global__ void ku_substep_kernel(const GmresControl* ctl, KoStepState* st, cudaGraphConditionalHandle sub,
                                  cudaGraphDeviceNode_t asm_node, unsigned long long dt_offset) {
    if (threadIdx.x) return;
    const int n = ctl->launches + 3;  // the rounds' kernels + assembly, control-block init, this kernel
    st->launches += n;
    st->launches_total += n;
    st->substeps++;
    if (st->status) {
        cudaGraphSetConditional(sub, 0u);
        return;
    }
    for (int s = 0; s < 2; ++s) {
        if (ctl->sys[s].nan) {
            st->steps_per_lb *= 2;
            st->dt /= 2.0;
            st->cur = 0;
            st->time_since_change = 0;
        }
    }
    if (st->steps_per_lb > (1 << 20) || st->substeps >= KU_MAX_SUBSTEPS) {
        st->status = KOFM_ERR_NAN;  // runaway halving
        cudaGraphSetConditional(sub, 0u);
        return;
    }
    st->cur++;
    ku_set_dt(asm_node, dt_offset, st->dt);
    cudaGraphSetConditional(sub, st->cur < st->steps_per_lb ? 1u : 0u);
}

}  // namespace kofm
