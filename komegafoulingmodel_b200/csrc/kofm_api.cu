// kofm_api.cu - context, memory management and the C ABI (include/kofm.h).
//
// Everything the hot path needs lives in device memory owned by the context;
// host arrays in the reference's padded FP64 layout cross the boundary only in
// kofm_set_* / kofm_get_*.  All work is enqueued on the context's stream.
#include "kofm.h"
#include "kofm_common.cuh"
#include "kofm_lb.cuh"
#include "kofm_komega.cuh"
#include "kofm_gmres.cuh"
#include "kofm_sstep.cuh"
#include "kofm_thermal.cuh"

#include <cuda_runtime.h>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <utility>
#include <vector>

using namespace kofm;

struct kofm_ctx;
namespace kofm {
int th_solver_alloc(kofm_ctx* c);
int ko_solver_alloc(KoSystem* sys, GmresControl** ctl, double** part, unsigned int** bar,
                    int* nblocks, int P, int ny, int K, int dev, int max_blocks);
int ss_solver_alloc(double** part, int** lhint, int* nblocks, int* pstrips, int* prows, int nx,
                    int ny, int K, int dev, int max_blocks);
int sp_solver_alloc(kofm_ctx* c);
void ko_system_free(KoSystem* s);
static int ug_pull(kofm_ctx* c);
static void ug_reset(kofm_ctx* c);
}  // namespace kofm

namespace {

constexpr int RED_BLOCKS = 256;  // fixed => deterministic reduction order

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

}  // namespace

// device work memory of kofm_adjoint, kept between calls
struct AdjWork {
    float* cps = nullptr;  size_t cps_b = 0;   // checkpoints
    float* seg = nullptr;  size_t seg_b = 0;   // recomputed states of a segment
    float* lam = nullptr;  size_t lam_b = 0;   // adjoint of the gathered populations
    float* nu = nullptr;   size_t nu_b = 0;    // adjoint of the post-collision state
    double* jpart = nullptr; size_t jpart_b = 0;
    double* dq = nullptr;  size_t dq_b = 0;
    double* sgrad = nullptr; size_t sgrad_b = 0;  // shear-term gradients of a segment
    int8_t* cls = nullptr; size_t cls_b = 0;      // node classes of the transposed gather
    long long cap = -1;    // bytes for stored states (< 0: half the free memory)
};

struct kofm_ctx {
    kofm_desc desc{};
    int P = 0;            // device row pitch (nodes)
    long long D = 0;      // plane stride (nodes)
    int dev = 0;
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    size_t store_bytes = 4;

    // lattice state
    void* g[2] = {nullptr, nullptr};  // population buffers (9 planes each)
    float* ref[2] = {nullptr, nullptr};  // KOFM_STORE_FP16_NEQ: reference rho, ux, uy of g[b]
    float* rowref = nullptr;             // KOFM_STORE_FP16_ROW: rho, ux, uy of each row ([3][ny])
    float* rowref_next = nullptr;        //   the next references (re-centring)
    long long row_steps = 0;             //   collides since the last re-centring
    int cur = 0;                      // buffer holding the current state
    int phase = 0;                    // 0: FA form, 1: post-collision (pull)
    int16_t* ntype = nullptr;
    int32_t* rec = nullptr;           // per-node IBB record index
    IbbRecord* ibb = nullptr;
    int n_ibb_rec = 0;
    std::vector<std::pair<long long, int>> ibb_links;  // input order: (device node, direction)
    int32_t* dxrec_idx = nullptr;     // per-node dX record index
    DxRecord* dxrec = nullptr;
    // node fields: FP32, or FP64 in the FP64 storage form (f64; fbytes = 8)
    bool f64 = false;
    size_t fbytes = 4;
    void* wallD = nullptr;
    void* K = nullptr;
    void* O = nullptr;
    void* S = nullptr;                // 3 planes
    void* nut = nullptr;
    void* rho = nullptr;
    void* ux = nullptr;
    void* uy = nullptr;
    double* lb_partials = nullptr;
    long long n_lb_partials = 0;
    double* red_partials = nullptr;   // RED_BLOCKS
    double* red_out = nullptr;        // 1
    double* h_red = nullptr;          // pinned, 64 doubles
    double* staging = nullptr;        // FP64 host-layout staging
    size_t staging_elems = 0;
    bool have_geometry = false;
    bool have_state = false;

    // k-omega solver
    KoSystem sys[2];                  // 0: omega, 1: k
    GmresControl* ctl = nullptr;      // device control block
    GmresControl* h_ctl = nullptr;    // pinned mirror
    double* gpart = nullptr;          // solver partial sums
    unsigned int* bar = nullptr;      // grid barrier words
    int solver_blocks = 0;
    // one-sweep-per-cycle solver (kofm_sstep.cuh): partial sums, grid and
    // the strips of its powers and update sweeps
    double* spart = nullptr;
    int* ss_lhint = nullptr;          // powers of a cycle's first round, per system
    int ss_blocks = 0, ss_pstrips = 0, ss_prows = 0;
    SsLaunch sp{};                    // the same solver as separate phase launches
    int ss_hint[2] = {0, 0};          // host copy of ss_lhint (first-round powers)
    // the k-omega update as a device-driven CUDA graph (kofm_stepgraph.inc)
    KoStepState* kst = nullptr;       // sub-stepping state (device)
    KoStepState* h_kst = nullptr;     // pinned copy
    cudaGraph_t ug = nullptr;
    cudaGraphExec_t ugx = nullptr;
    bool ug_pending = false;          // updates launched since the state was last read back
    bool ug_devupd = false;           // the graph's assembly node takes dt as a device-updated parameter
    long long launches_host = 0;      // k-omega kernel launches the host loop made since set_state
    int steps_per_lb = 1;
    int time_since_change = 0;
    double dt = 1.0;
    int fail_solves = 0;              // kofm_debug_fail_solves
    int fail_mask = 0;
    kofm_stats stats{};

    // wall shear (kofm_set_shear / kofm_wall_shear)
    int32_t* shear_nodes = nullptr;   // [n] node index of the padded host layout
    double* shear_cfss = nullptr;     // [n][16]
    double* shear_tau = nullptr;      // [n]
    int32_t* shear_bl_nodes = nullptr;// [n_bl][4]
    double* shear_bl_w = nullptr;     // [n_bl][4]
    double* shear_bl_tau = nullptr;   // [n_bl]
    int shear_n = 0, shear_nbl = 0;
    int32_t* shear_idx = nullptr;     // per device node: shear-node index or -1
    AdjWork adj;
    int n_dxrec = -1, n_dxrec0 = -1;  // FD records (-1: not built)
    // room in the record tables, and the device builder's work buffers (kept
    // so that a builder call on a live context allocates nothing)
    size_t ibb_cap = 0, dxrec_cap = 0, dxrec0_cap = 0;
    int32_t* ibb_node = nullptr;  // host-layout node of each IBB record [ibb_cap]
    double* geo_walls = nullptr;  size_t geo_walls_n = 0;
    int* geo_rows = nullptr;      size_t geo_rows_n = 0;

    // thermal implicit FD (kofm_thermal_*)
    double* T = nullptr;              // [D] temperature (tempArray), FP64
    double* Tprev = nullptr;          // [D] tempPrev (restored on a dt halving)
    double* tb = nullptr;             // [D] right-hand side, then the residual
    double* tr0 = nullptr;            // [D] r0hat
    double* tp[2] = {nullptr, nullptr};
    double* tv[2] = {nullptr, nullptr};
    double* ts = nullptr;
    double* tcoef = nullptr;          // [4 x D] interleaved E, W, N, S
    int32_t* dxrec0_idx = nullptr;    // per-node dXArr0 record (-1: all 1)
    DxRecord* dxrec0 = nullptr;
    bool have_dx0 = false;            // kofm_set_thermal_geometry was called
    bool have_temp = false;
    ThermalCtl* tctl = nullptr;
    ThermalCtl* h_tctl = nullptr;     // pinned mirror
    double* tpart = nullptr;
    unsigned int* tbar = nullptr;
    int th_blocks = 0;
    int th_steps_per_lb = 1;
    int th_time_since_change = 0;
    double th_dt = 1.0;
    long long time_n = 0;             // p.TimeN of the step loop
};

namespace {

#define KOFM_CUDA_TRY(call, code)                                                 \
    do {                                                                          \
        cudaError_t _e = (call);                                                  \
        if (_e != cudaSuccess) {                                                  \
            fprintf(stderr, "kofm: %s failed: %s\n", #call, cudaGetErrorString(_e)); \
            return (code);                                                        \
        }                                                                         \
    } while (0)

int dalloc(void** p, size_t bytes) {
    if (cudaMalloc(p, bytes) != cudaSuccess) return KOFM_ERR_BUFFER_ALLOCATION;
    if (cudaMemset(*p, 0, bytes) != cudaSuccess) return KOFM_ERR_BUFFER_ALLOCATION;
    return KOFM_OK;
}

template <typename T>
int dalloc_t(T** p, size_t n) {
    return dalloc(reinterpret_cast<void**>(p), n * sizeof(T));
}

int ensure_staging(kofm_ctx* c, size_t elems) {
    if (c->staging_elems >= elems) return KOFM_OK;
    if (c->staging) cudaFree(c->staging);
    c->staging = nullptr;
    c->staging_elems = 0;
    int st = dalloc_t(&c->staging, elems);
    if (st) return st;
    c->staging_elems = elems;
    return KOFM_OK;
}

// ---- conversion kernels ----------------------------------------------------
// host-layout FP64 populations (FA) -> device deviations; solid/padding -> 0
template <typename ST>
__global__ void k_fa_in(const double* __restrict__ f, ST* __restrict__ g,
                        const int16_t* __restrict__ nt, int nx, int nxf, int ny,
                        int P, long long D) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= P) return;
    const long long node = (long long)y * P + x;
    const bool fluid = x < nx && !((uint16_t)nt[node] & M_SOLID);
    const long long Dh = (long long)nxf * ny;
    for (int q = 0; q < 9; ++q) {
        double v = 0.0;
        if (fluid) v = f[q * Dh + (long long)y * nxf + x] - weight_of(q);
        g[q * D + node] = Store<ST>::from_f64(v);
    }
}

// host-layout FP64 FA -> non-equilibrium form: reference = the node's own
// moments rounded to FP32, e = f - feq(reference), scaled, in FP16
__global__ void k_fa_in_neq(const double* __restrict__ f, __half* __restrict__ g,
                            float* __restrict__ ref, const int16_t* __restrict__ nt, int nx,
                            int nxf, int ny, int P, long long D) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= P) return;
    const long long node = (long long)y * P + x;
    const bool fluid = x < nx && !((uint16_t)nt[node] & M_SOLID);
    const long long Dh = (long long)nxf * ny;
    double fv[9];
    double rho = 0.0, jx = 0.0, jy = 0.0;
    for (int q = 0; q < 9; ++q) {
        fv[q] = fluid ? f[q * Dh + (long long)y * nxf + x] : 0.0;
        rho += fv[q];
        jx += cx_of(q) * fv[q];
        jy += cy_of(q) * fv[q];
    }
    const float r = fluid ? (float)rho : 0.f;
    const float u = fluid ? (float)(jx / rho) : 0.f, v = fluid ? (float)(jy / rho) : 0.f;
    ref[node] = r;
    ref[D + node] = u;
    ref[2 * D + node] = v;
    for (int q = 0; q < 9; ++q) {
        const float e = fluid ? (float)((fv[q] - weight_of(q)) - (double)feq_dev_f32(q, r, u, v)) : 0.f;
        g[q * D + node] = __float2half_rn(e * NEQ_SCALE);
    }
}

// Reference of the stored populations of a non-equilibrium form: per node
// (KOFM_STORE_FP16_NEQ*: rho, ux, uy planes of D) or per row
// (KOFM_STORE_FP16_ROW: [3][ny]); neither for the f - w forms.
struct PopRef {
    const float* node;
    const float* row;
};

// Row references of KOFM_STORE_FP16_ROW from the host-layout FP64 FA: the
// mean density of the row's fluid nodes and its mean velocity (momentum over
// mass); 1, 0, 0 for a row without fluid.  One block per row.
__global__ void k_row_ref(const double* __restrict__ f, float* __restrict__ rowref,
                          const int16_t* __restrict__ nt, int nx, int nxf, int ny, int P) {
    const int y = blockIdx.x;
    const long long Dh = (long long)nxf * ny;
    double s[4] = {0.0, 0.0, 0.0, 0.0};  // rho, jx, jy, nodes
    for (int x = threadIdx.x; x < nx; x += blockDim.x) {
        if ((uint16_t)nt[(long long)y * P + x] & M_SOLID) continue;
        for (int q = 0; q < 9; ++q) {
            const double fq = f[q * Dh + (long long)y * nxf + x];
            s[0] += fq;
            s[1] += cx_of(q) * fq;
            s[2] += cy_of(q) * fq;
        }
        s[3] += 1.0;
    }
    __shared__ double red[4][8];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int k = 0; k < 4; ++k) {
        double v = s[k];
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if (lane == 0) red[k][w] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t[4] = {0.0, 0.0, 0.0, 0.0};
        for (int k = 0; k < 4; ++k)
            for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t[k] += red[k][i];
        const bool any = t[3] > 0.0 && t[0] > 0.0;
        rowref[y] = any ? (float)(t[0] / t[3]) : 1.f;
        rowref[ny + y] = any ? (float)(t[1] / t[0]) : 0.f;
        rowref[2 * ny + y] = any ? (float)(t[2] / t[0]) : 0.f;
    }
}

// host-layout FP64 FA -> row-reference form: e = f - feq(reference of the
// node's row), scaled, in FP16
__global__ void k_fa_in_row(const double* __restrict__ f, __half* __restrict__ g,
                            const float* __restrict__ rowref, const int16_t* __restrict__ nt, int nx,
                            int nxf, int ny, int P, long long D) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= P) return;
    const long long node = (long long)y * P + x;
    const bool fluid = x < nx && !((uint16_t)nt[node] & M_SOLID);
    const long long Dh = (long long)nxf * ny;
    const float r = rowref[y], u = rowref[ny + y], v = rowref[2 * ny + y];
    for (int q = 0; q < 9; ++q) {
        const double fq = fluid ? f[q * Dh + (long long)y * nxf + x] : 0.0;
        const float e = fluid ? (float)((fq - weight_of(q)) - (double)feq_dev_f32(q, r, u, v)) : 0.f;
        g[q * D + node] = __float2half_rn(e * NEQ_SCALE);
    }
}

// Collide arithmetic of KOFM_STORE_FP16_ROW.
#ifndef KOFM_ROW_AT
#define KOFM_ROW_AT float
#endif
// Collides between re-centrings of the row references (KOFM_STORE_FP16_ROW).
#ifndef KOFM_ROW_RECENTRE
#define KOFM_ROW_RECENTRE 32
#endif

// Row references from the moments the last collide wrote: the row's mean
// density and its mean velocity (momentum over mass) over its fluid nodes.
__global__ void k_row_ref_fields(const float* __restrict__ rho, const float* __restrict__ ux,
                                 const float* __restrict__ uy, float* __restrict__ rowref,
                                 const int16_t* __restrict__ nt, int nx, int ny, int P) {
    const int y = blockIdx.x;
    double s[4] = {0.0, 0.0, 0.0, 0.0};  // rho, jx, jy, nodes
    for (int x = threadIdx.x; x < nx; x += blockDim.x) {
        const long long n = (long long)y * P + x;
        if ((uint16_t)nt[n] & M_SOLID) continue;
        const double r = rho[n];
        s[0] += r;
        s[1] += r * ux[n];
        s[2] += r * uy[n];
        s[3] += 1.0;
    }
    __shared__ double red[4][8];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int k = 0; k < 4; ++k) {
        double v = s[k];
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if (lane == 0) red[k][w] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t[4] = {0.0, 0.0, 0.0, 0.0};
        for (int k = 0; k < 4; ++k)
            for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t[k] += red[k][i];
        const bool any = t[3] > 0.0 && t[0] > 0.0;
        rowref[y] = any ? (float)(t[0] / t[3]) : 1.f;
        rowref[ny + y] = any ? (float)(t[1] / t[0]) : 0.f;
        rowref[2 * ny + y] = any ? (float)(t[2] / t[0]) : 0.f;
    }
}

// Re-encodes the stored populations of every fluid node against the new
// references of its row: e' = e + feq(old) - feq(new) (scaled, FP16).
__global__ void k_row_recentre(__half* __restrict__ g, const float* __restrict__ oldref,
                               const float* __restrict__ newref, const int16_t* __restrict__ nt, int nx,
                               int ny, int P, long long D) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= nx) return;
    const long long node = (long long)y * P + x;
    if ((uint16_t)nt[node] & M_SOLID) return;
    const float r0 = oldref[y], u0 = oldref[ny + y], v0 = oldref[2 * ny + y];
    const float r1 = newref[y], u1 = newref[ny + y], v1 = newref[2 * ny + y];
    for (int q = 0; q < 9; ++q) {
        const float e = __half2float(g[q * D + node]) +
                        (feq_dev_f32(q, r0, u0, v0) - feq_dev_f32(q, r1, u1, v1)) * NEQ_SCALE;
        g[q * D + node] = __float2half_rn(e);
    }
}

// device state -> host-layout FP64 FA.  phase 0: own deviations; phase 1:
// gather + bounce-back + interpolated bounce-back (the next step's pull).
// Deviations f - w of the populations FA of fluid node (x, y) -- the
// reference's post-stream, bounced and interpolated state -- from the device
// state: phase 0 holds them at the node; phase 1 gathers the previous step's
// post-collision values and applies bounce-back and interpolated bounce-back
// (the next step's pull).  ref != nullptr: non-equilibrium form (decode with
// the stored reference of the node each value was read from).
template <typename ST>
__device__ void fa_node(const ST* __restrict__ g, int type, const int32_t* __restrict__ rec,
                        const IbbRecord* __restrict__ ibb, int has_ibb, int nx, int ny, int P,
                        long long D, int phase, PopRef ref, int x, int y, double d[9]) {
    auto dec = [&](int q, long long n) -> double {
        const double raw = Store<ST>::to_f64(g[q * D + n]);
        if (ref.node) {
            const float* rf = ref.node;
            return (double)(feq_dev_f32(q, rf[n], rf[D + n], rf[2 * D + n]) + (float)raw * NEQ_INV_SCALE);
        }
        if (ref.row) {
            const int r = (int)(n / P);
            const float* rr = ref.row;
            return (double)(feq_dev_f32(q, rr[r], rr[ny + r], rr[2 * ny + r]) + (float)raw * NEQ_INV_SCALE);
        }
        return raw;
    };
    const long long node = (long long)y * P + x;
    for (int q = 0; q < 9; ++q) {
        if (phase == 0) {
            d[q] = dec(q, node);
        } else {
            int xs = x - cx_of(q);
            xs = xs < 0 ? xs + nx : (xs >= nx ? xs - nx : xs);
            int ys = y - cy_of(q);
            ys = ys < 0 ? 0 : (ys >= ny ? ny - 1 : ys);
            d[q] = dec(q, (long long)ys * P + xs);
        }
    }
    if (phase == 1 && (type & BOUNDARY)) {
        double pre[9];
        pre[0] = d[0];
        for (int q = 1; q < 9; ++q) {
            if (type & bound_of(rev_of(q))) d[q] = dec(rev_of(q), node);
            pre[q] = d[q];
        }
        if (has_ibb && rec[node] >= 0) {
            const IbbRecord r = ibb[rec[node]];
            for (int dd = 1; dd < 9; ++dd) {
                const double qf = r.q[dd - 1];
                if (qf < 0.0) continue;
                const int rd = rev_of(dd);
                const double q2 = 2.0 * qf;
                if (q2 <= 1.0) d[rd] = q2 * pre[rd] + (1.0 - q2) * pre[dd];
                else d[rd] = (1.0 / q2) * (pre[rd] + (q2 - 1.0) * dec(rd, node));
            }
        }
    }
}

// device state -> host-layout FP64 FA (see fa_node)
template <typename ST>
__global__ void k_fa_out(const ST* __restrict__ g, const int16_t* __restrict__ nt,
                         const int32_t* __restrict__ rec, const IbbRecord* __restrict__ ibb,
                         int has_ibb, double* __restrict__ f, int nx, int nxf, int ny,
                         int P, long long D, int phase, PopRef ref) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= nxf) return;
    const long long Dh = (long long)nxf * ny;
    const long long hnode = (long long)y * nxf + x;
    const int type = x < nx ? (uint16_t)nt[(long long)y * P + x] : M_SOLID;
    if (type & M_SOLID) {
        for (int q = 0; q < 9; ++q) f[q * Dh + hnode] = 0.0;
        return;
    }
    double d[9];
    fa_node<ST>(g, type, rec, ibb, has_ibb, nx, ny, P, D, phase, ref, x, y, d);
    for (int q = 0; q < 9; ++q) f[q * Dh + hnode] = d[q] + weight_of(q);
}

// Wall shear at the shear nodes (TR_shear_1, Kernels/trKernelsShear.cl:131-222):
// f_neq = FA - feq(rho, u) of the node's populations 1..8 (rho, u the moments
// the last step wrote), tau = |(f_neq . cx_row, f_neq . cy_row)| (nu + nu_t)
// / (3 (nu + nu_t) + 1/2) / rho, with the sign of its x component.
template <typename ST, typename FT = float>
__global__ void k_shear_nodes(const ST* __restrict__ g, const int16_t* __restrict__ nt,
                              const int32_t* __restrict__ rec, const IbbRecord* __restrict__ ibb,
                              int has_ibb, int nx, int ny, int P, long long D, int phase,
                              PopRef ref, const FT* __restrict__ rho,
                              const FT* __restrict__ ux, const FT* __restrict__ uy,
                              const FT* __restrict__ nut, double mu, const int32_t* __restrict__ nodes,
                              const double* __restrict__ cfss, int n, int nxf, double* __restrict__ tau) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int hn = nodes[i];
    const int y = hn / nxf, x = hn - y * nxf;
    const long long node = (long long)y * P + x;
    const int type = (uint16_t)nt[node];
    double d[9];
    fa_node<ST>(g, type, rec, ibb, has_ibb, nx, ny, P, D, phase, ref, x, y, d);
    const double r = rho[node], u = ux[node], v = uy[node];
    double tx = 0.0, ty = 0.0;
    for (int q = 1; q < 9; ++q) {
        const int cx = cx_of(q), cy = cy_of(q);
        const double phx = cx == 0 ? 2.0 / 3.0 - u * u : 0.5 * (1.0 / 3.0 + cx * u + u * u);
        const double phy = cy == 0 ? 2.0 / 3.0 - v * v : 0.5 * (1.0 / 3.0 + cy * v + v * v);
        const double fneq = (d[q] + weight_of(q)) - r * phx * phy;
        tx += fneq * cfss[16 * (long long)i + (q - 1)];
        ty += fneq * cfss[16 * (long long)i + 8 + (q - 1)];
    }
    double visc = (nut ? (double)nut[node] : 0.0) + mu;
    visc *= 1.0 / (3.0 * visc + 0.5);
    const double t = sqrt(tx * tx * visc * visc + ty * ty * visc * visc) / r;
    tau[i] = tx < 0.0 ? -t : t;
}

// Shear of every boundary link: weighted mean of its four nearest shear
// nodes (TR_shear_2, trKernelsShear.cl:300-316); index -1 contributes nothing.
__global__ void k_shear_links(const double* __restrict__ tau_nodes, const int32_t* __restrict__ sind,
                              const double* __restrict__ w, int nbl, double* __restrict__ out) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nbl) return;
    double acc = 0.0;
    for (int a = 0; a < 4; ++a) {
        const int j = sind[4 * b + a];
        if (j >= 0) acc += w[4 * b + a] * tau_nodes[j];
    }
    out[b] = acc;
}

// FP64 host-layout scalar field <-> device field (FP32, or FP64 in the FP64 form)
template <typename FT>
__global__ void k_field_in(const double* __restrict__ h, FT* __restrict__ dv, int nxf,
                           int ny, int P) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= P) return;
    dv[(long long)y * P + x] = x < nxf ? (FT)h[(long long)y * nxf + x] : FT(0);
}
template <typename FT>
__global__ void k_field_out(const FT* __restrict__ dv, double* __restrict__ h, int nxf,
                            int ny, int P) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= nxf) return;
    h[(long long)y * nxf + x] = (double)dv[(long long)y * P + x];
}

// ---- deterministic reductions -------------------------------------------------
// Block b sums the fixed contiguous range [b*n/B, (b+1)*n/B) of the padded
// field (rows of P nodes; columns >= nxf excluded), then one block combines the
// B partials in order.
template <int OP>
__device__ __forceinline__ double red_op(double a, double b) {
    return OP == KOFM_OP_SUM ? a + b : (OP == KOFM_OP_MIN ? fmin(a, b) : fmax(a, b));
}
template <int OP>
__device__ __forceinline__ double red_init() {
    return OP == KOFM_OP_SUM ? 0.0 : (OP == KOFM_OP_MIN ? 1.0e308 : -1.0e308);
}

template <int OP, typename T = float>
__global__ void k_reduce_field(const T* __restrict__ v, long long nnodes, int P, int nxf,
                               double* __restrict__ part) {
    __shared__ double sh[32];
    const long long s = (long long)((double)blockIdx.x * nnodes / gridDim.x);
    const long long e = (long long)((double)(blockIdx.x + 1) * nnodes / gridDim.x);
    double acc = red_init<OP>();
    for (long long i = s + threadIdx.x; i < e; i += blockDim.x) {
        if ((int)(i % P) < nxf) acc = red_op<OP>(acc, (double)v[i]);
    }
    for (int off = 16; off > 0; off >>= 1) acc = red_op<OP>(acc, __shfl_down_sync(0xffffffffu, acc, off));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        acc = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : red_init<OP>();
        for (int off = 16; off > 0; off >>= 1) acc = red_op<OP>(acc, __shfl_down_sync(0xffffffffu, acc, off));
        if (threadIdx.x == 0) part[blockIdx.x] = acc;
    }
}

template <int OP>
__global__ void k_reduce_final(const double* __restrict__ part, int n, double* __restrict__ out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double acc = red_init<OP>();
        for (int i = 0; i < n; ++i) acc = red_op<OP>(acc, part[i]);
        out[0] = acc;
    }
}

// wall-shear integrand: rho (mu + nu_t) 2 |Sxy| on fluid nodes with an N or S
// wall link, summed per block.
template <typename FT>
__global__ void k_wall_shear(const int16_t* __restrict__ nt, const FT* __restrict__ rho,
                             const FT* __restrict__ nut, const FT* __restrict__ S,
                             long long nnodes, long long D, int P, int nx, double mu,
                             double* __restrict__ part) {
    __shared__ double sh[32];
    const long long s = (long long)((double)blockIdx.x * nnodes / gridDim.x);
    const long long e = (long long)((double)(blockIdx.x + 1) * nnodes / gridDim.x);
    double acc = 0.0;
    for (long long i = s + threadIdx.x; i < e; i += blockDim.x) {
        const int t = (uint16_t)nt[i];
        if ((int)(i % P) < nx && !(t & M_SOLID) && (t & (N_BOUND | S_BOUND)))
            acc += (double)rho[i] * (mu + (double)nut[i]) * 2.0 * fabs((double)S[D + i]);
    }
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        acc = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
        for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
        if (threadIdx.x == 0) part[blockIdx.x] = acc;
    }
}

// ---- LB step dispatch ------------------------------------------------------------
template <typename ST, typename AT, bool NEQ = false, typename FT = float, bool ROW = false>
cudaError_t launch_lb(kofm_ctx* c, const LbParams& p, bool komega, bool phase0) {
    dim3 block(32, 4);
    dim3 grid(c->P / 128, (c->desc.ny + 3) / 4);
    if (komega) {
        if (phase0) lb_step_kernel<ST, AT, true, true, NEQ, FT, ROW><<<grid, block, 0, c->stream>>>(p);
        else lb_step_kernel<ST, AT, true, false, NEQ, FT, ROW><<<grid, block, 0, c->stream>>>(p);
    } else {
        if (phase0) lb_step_kernel<ST, AT, false, true, NEQ, FT, ROW><<<grid, block, 0, c->stream>>>(p);
        else lb_step_kernel<ST, AT, false, false, NEQ, FT, ROW><<<grid, block, 0, c->stream>>>(p);
    }
    return cudaGetLastError();
}

int validate_desc(const kofm_desc* d) {
    if (!d) return KOFM_ERR_INVALID_ARG;
    if (d->nx < 4 || d->ny < 3 || d->nx_full < d->nx) return KOFM_ERR_LOADING_PARAMS;
    if ((long long)d->nx_full * d->ny > (1LL << 31) - 1) return KOFM_ERR_LOADING_PARAMS;
    if (d->storage < KOFM_STORE_FP32 || d->storage > KOFM_STORE_FP16_ROW) return KOFM_ERR_LOADING_PARAMS;
    // the FP64 form is the precision study's reference form: no thermal update
    if (d->storage == KOFM_STORE_FP64 && d->use_thermal) return KOFM_ERR_LOADING_PARAMS;
    if (!(d->tau > 0.0 && d->tau < 2.0)) return KOFM_ERR_LOADING_PARAMS;
    if (d->krylov_dim < 1 || d->krylov_dim > KOFM_MAX_KRYLOV) return KOFM_ERR_LOADING_PARAMS;
    if (d->komega_max_iters < 1) return KOFM_ERR_LOADING_PARAMS;
    if (d->solver_max_blocks < 0) return KOFM_ERR_LOADING_PARAMS;
    if (d->komega_classic < 0 || d->komega_classic > 3) return KOFM_ERR_LOADING_PARAMS;
    if (d->use_thermal) {
        if (d->thermal_every < 1 || d->thermal_max_iters < 1) return KOFM_ERR_LOADING_PARAMS;
        if (!(d->pr_number > 0.0) || !(d->pr_turb_number > 0.0) || !(d->thermal_dt > 0.0))
            return KOFM_ERR_LOADING_PARAMS;
    }
    return KOFM_OK;
}

}  // namespace

// =============================================================================
extern "C" {

int kofm_abi_version(void) { return KOFM_ABI_VERSION; }

const char* kofm_error_string(int s) {
    switch (s) {
        case KOFM_OK: return "ok";
        case KOFM_ERR_BUFFER_ALLOCATION: return "device buffer allocation failed";
        case KOFM_ERR_MEMORY_COPY: return "host/device copy failed";
        case KOFM_ERR_CALLING_KERNEL: return "kernel launch or execution failed";
        case KOFM_ERR_LOADING_PARAMS: return "invalid run parameters";
        case KOFM_ERR_INITIALIZING_KOMEGA: return "k-omega initialisation failed";
        case KOFM_ERR_INITIALIZING_VLS: return "invalid geometry";
        case KOFM_ERR_INITIALIZING_VLB: return "LB initialisation failed";
        case KOFM_ERR_INVALID_ARG: return "invalid argument";
        case KOFM_ERR_NO_DEVICE: return "no usable CUDA device";
        case KOFM_ERR_NOT_CONVERGED: return "k-omega solve reached its iteration cap";
        case KOFM_ERR_NAN: return "NaN residual in the k-omega solve (dt halved)";
        case KOFM_ERR_TIMEOUT: return "bounded device wait expired";
        case KOFM_ERR_STATE: return "geometry or state not set";
        case KOFM_ERR_TOO_LARGE: return "input larger than the fixed scratch allows";
        default: return "unknown status";
    }
}

int kofm_desc_default(kofm_desc* d) {
    if (!d) return KOFM_ERR_INVALID_ARG;
    memset(d, 0, sizeof(*d));
    d->nx = 256; d->nx_full = 256; d->ny = 64;
    d->use_komega = 0;
    d->tau = 1.25;                // rate; LB_TAU_NUMBER is 1.99
    d->fterm = 0.0;
    d->mu = (1.0 / 1.25 - 0.5) / 3.0;
    d->max_turb_visc = 10.0;      // MAX_TURB_VISC
    d->storage = KOFM_STORE_FP32;
    d->device = 0;
    d->komega_max_iters = 1000;   // KOMEGA_MAX_ITERS
    d->krylov_dim = 10;           // GMRES_KRYLOV_DIM_SIZE
    d->komega_rel_tol = 1.0e-4;   // KOMEGA_MAX_REL_TOL
    d->komega_abs_tol = 1.0e-7;   // KOMEGA_MAX_ABS_TOL
    d->komega_dt = 1.0;           // p.dTlb
    d->komega_full_cycle = 0;     // end each cycle at its first truncation
    d->use_thermal = 0;
    d->thermal_every = 1;         // LB_STEPS_PER_FD
    d->pr_number = 0.708;         // PR_NUMBER
    d->pr_turb_number = 0.9;      // PR_TURB_NUMBER
    d->alpha_foul = 0.0;          // no fouling layer
    d->t_in = 2.0;                // TFD_X_IN
    d->thermal_max_iters = 1000;  // THERMAL_MAX_ITERS
    d->thermal_rel_tol = 1.0e-4;  // THERMAL_MAX_REL_TOL
    d->thermal_abs_tol = 1.0e-7;  // THERMAL_MAX_ABS_TOL
    d->thermal_dt = 1.0;          // dTtfd = tfdSteps
    return KOFM_OK;
}

int kofm_destroy(kofm_ctx* c) {
    if (!c) return KOFM_ERR_INVALID_ARG;
    cudaSetDevice(c->dev);
    if (c->stream) cudaStreamSynchronize(c->stream);
    void* bufs[] = {c->g[0], c->g[1], c->ref[0], c->ref[1], c->rowref, c->rowref_next, c->ntype, c->rec, c->ibb, c->dxrec_idx, c->dxrec,
                    c->wallD, c->K, c->O, c->S, c->nut, c->rho, c->ux, c->uy,
                    c->lb_partials, c->red_partials, c->red_out, c->staging, c->ctl,
                    c->gpart, c->spart, c->ss_lhint, c->bar, c->shear_nodes, c->shear_cfss, c->shear_tau,
                    c->shear_bl_nodes, c->shear_bl_w, c->shear_bl_tau, c->T, c->Tprev, c->tb,
                    c->tr0, c->tp[0], c->tp[1], c->tv[0], c->tv[1], c->ts, c->tcoef,
                    c->dxrec0_idx, c->dxrec0, c->tctl, c->tpart, c->tbar, c->shear_idx,
                    c->adj.cps, c->adj.seg, c->adj.lam, c->adj.nu, c->adj.jpart, c->adj.dq, c->adj.sgrad, c->adj.cls,
                    c->ibb_node, c->geo_walls, c->geo_rows, c->kst};
    if (c->ugx) cudaGraphExecDestroy(c->ugx);
    if (c->ug) cudaGraphDestroy(c->ug);
    for (void* b : bufs)
        if (b) cudaFree(b);
    for (int s = 0; s < 2; ++s) ko_system_free(&c->sys[s]);
    if (c->h_red) cudaFreeHost(c->h_red);
    if (c->h_ctl) cudaFreeHost(c->h_ctl);
    if (c->h_kst) cudaFreeHost(c->h_kst);
    if (c->h_tctl) cudaFreeHost(c->h_tctl);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return KOFM_OK;
}

int kofm_create(const kofm_desc* d, kofm_ctx** out) {
    if (!out) return KOFM_ERR_INVALID_ARG;
    *out = nullptr;
    int st = validate_desc(d);
    if (st) return st;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= d->device || d->device < 0)
        return KOFM_ERR_NO_DEVICE;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, d->device) != cudaSuccess) return KOFM_ERR_NO_DEVICE;
    if (prop.major < 10) return KOFM_ERR_NO_DEVICE;  // built for sm_100a only
    kofm_ctx* c = new (std::nothrow) kofm_ctx();
    if (!c) return KOFM_ERR_BUFFER_ALLOCATION;
    c->desc = *d;
    c->dev = d->device;
    c->num_sms = prop.multiProcessorCount;
    c->P = ((d->nx_full + 127) / 128) * 128;
    c->D = (long long)c->P * d->ny;
    c->store_bytes = d->storage == KOFM_STORE_FP64 ? 8 : (d->storage == KOFM_STORE_FP32 ? 4 : 2);
    c->f64 = d->storage == KOFM_STORE_FP64;
    c->fbytes = c->f64 ? 8 : 4;
    c->dt = d->komega_dt;
    c->steps_per_lb = (int)(1.0 / d->komega_dt);
    if (c->steps_per_lb < 1) c->steps_per_lb = 1;
    if (cudaSetDevice(c->dev) != cudaSuccess) { delete c; return KOFM_ERR_NO_DEVICE; }
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return KOFM_ERR_NO_DEVICE;
    }
    const long long D = c->D;
#define ALLOC(ptr, n)                                       \
    do {                                                    \
        int _s = dalloc_t(&(ptr), (size_t)(n));             \
        if (_s) { kofm_destroy(c); return _s; }             \
    } while (0)
    for (int b = 0; b < 2; ++b) {
        int _s = dalloc(&c->g[b], (size_t)(9 * D) * c->store_bytes);
        if (_s) { kofm_destroy(c); return _s; }
    }
    if (d->storage == KOFM_STORE_FP16_NEQ || d->storage == KOFM_STORE_FP16_NEQ32) {
        ALLOC(c->ref[0], 3 * D);
        ALLOC(c->ref[1], 3 * D);
    }
    if (d->storage == KOFM_STORE_FP16_ROW) {
        ALLOC(c->rowref, 3 * d->ny);
        ALLOC(c->rowref_next, 3 * d->ny);
    }
#define ALLOC_FIELD(ptr, n)                                         \
    do {                                                            \
        int _s = dalloc(&(ptr), (size_t)(n) * c->fbytes);           \
        if (_s) { kofm_destroy(c); return _s; }                     \
    } while (0)
    ALLOC(c->ntype, D);
    ALLOC(c->rec, D);
    ALLOC(c->dxrec_idx, D);
    ALLOC_FIELD(c->rho, D);
    ALLOC_FIELD(c->ux, D);
    ALLOC_FIELD(c->uy, D);
    c->n_lb_partials = (long long)(c->P / 128) * ((d->ny + 3) / 4) * 4 * 3;
    ALLOC(c->lb_partials, c->n_lb_partials);
    ALLOC(c->red_partials, RED_BLOCKS);
    ALLOC(c->red_out, 8);
    if (d->use_komega) {
        ALLOC_FIELD(c->wallD, D);
        ALLOC_FIELD(c->K, D);
        ALLOC_FIELD(c->O, D);
        ALLOC_FIELD(c->S, 3 * D);
        ALLOC_FIELD(c->nut, D);
        int s2 = ko_solver_alloc(c->sys, &c->ctl, &c->gpart, &c->bar, &c->solver_blocks,
                                 c->P, d->ny, d->krylov_dim, c->dev, d->solver_max_blocks);
        if (s2) { kofm_destroy(c); return s2; }
        s2 = ss_solver_alloc(&c->spart, &c->ss_lhint, &c->ss_blocks, &c->ss_pstrips, &c->ss_prows,
                             d->nx, d->ny, d->krylov_dim, c->dev, d->solver_max_blocks);
        if (!s2) s2 = sp_solver_alloc(c);
        if (s2) { kofm_destroy(c); return s2; }
        if (cudaMallocHost(&c->h_ctl, sizeof(GmresControl)) != cudaSuccess ||
            cudaMallocHost(&c->h_kst, sizeof(KoStepState)) != cudaSuccess) {
            kofm_destroy(c);
            return KOFM_ERR_BUFFER_ALLOCATION;
        }
        memset(c->h_kst, 0, sizeof(KoStepState));
        ALLOC(c->kst, 1);
    }
    if (d->use_thermal) {
        ALLOC(c->T, D);
        ALLOC(c->Tprev, D);
        ALLOC(c->tb, D);
        ALLOC(c->tr0, D);
        for (int b = 0; b < 2; ++b) { ALLOC(c->tp[b], D); ALLOC(c->tv[b], D); }
        ALLOC(c->ts, D);
        ALLOC(c->tcoef, 4 * D);
        ALLOC(c->dxrec0_idx, D);
        int s3 = th_solver_alloc(c);
        if (s3) { kofm_destroy(c); return s3; }
        c->th_dt = d->thermal_dt;
        c->th_steps_per_lb = (int)(1.0 / d->thermal_dt);
        if (c->th_steps_per_lb < 1) c->th_steps_per_lb = 1;
        cudaMemset(c->dxrec0_idx, 0xff, D * sizeof(int32_t));
    }
#undef ALLOC
#undef ALLOC_FIELD
    if (cudaMallocHost(&c->h_red, 64 * sizeof(double)) != cudaSuccess) {
        kofm_destroy(c);
        return KOFM_ERR_BUFFER_ALLOCATION;
    }
    // rec / dxrec_idx default to -1 (no record)
    cudaMemset(c->rec, 0xff, D * sizeof(int32_t));
    cudaMemset(c->dxrec_idx, 0xff, D * sizeof(int32_t));
    c->stats.steps_per_lb = c->steps_per_lb;
    c->stats.dt = c->dt;
    *out = c;
    return KOFM_OK;
}

void* kofm_stream(kofm_ctx* c) { return c ? (void*)c->stream : nullptr; }

int kofm_set_geometry(kofm_ctx* c, const int16_t* ntype, const double* wallD,
                      const double* dX4, const int32_t* ibb_idx, const double* ibb_q,
                      int32_t n_ibb) {
    if (!c || !ntype) return KOFM_ERR_INVALID_ARG;
    const kofm_desc& d = c->desc;
    if (d.use_komega && (!wallD || !dX4)) return KOFM_ERR_INVALID_ARG;
    if (d.use_thermal && !dX4) return KOFM_ERR_INVALID_ARG;
    if (n_ibb < 0 || (n_ibb > 0 && (!ibb_idx || !ibb_q))) return KOFM_ERR_INVALID_ARG;
    cudaSetDevice(c->dev);
    const int nx = d.nx, nxf = d.nx_full, ny = d.ny, P = c->P;
    const long long Dh = (long long)nxf * ny;
    // rows 0 and ny-1 may hold no fluid node (clVariablesLS.cpp:935-937)
    for (int x = 0; x < nx; ++x) {
        if (!((uint16_t)ntype[x] & M_SOLID) || !((uint16_t)ntype[(long long)(ny - 1) * nxf + x] & M_SOLID))
            return KOFM_ERR_INITIALIZING_VLS;
    }
    std::vector<int16_t> nt((size_t)c->D, (int16_t)M_SOLID);
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) nt[(size_t)y * P + x] = ntype[(long long)y * nxf + x];
    // interpolated bounce-back records, one per node that owns a link
    std::vector<int32_t> rec((size_t)c->D, -1);
    std::vector<IbbRecord> recs;
    std::vector<std::pair<long long, int>> links;
    for (int i = 0; i < n_ibb; ++i) {
        const long long loc = ibb_idx[i];
        const int dir = (int)(loc / Dh);
        const long long hnode = loc - (long long)dir * Dh;
        if (dir < 1 || dir > 8 || hnode < 0 || hnode >= Dh) return KOFM_ERR_INITIALIZING_VLS;
        const int x = (int)(hnode % nxf), y = (int)(hnode / nxf);
        if (x >= nx) return KOFM_ERR_INITIALIZING_VLS;
        const size_t node = (size_t)y * P + x;
        if (rec[node] < 0) {
            IbbRecord r;
            for (int k = 0; k < 8; ++k) r.q[k] = -1.0;
            rec[node] = (int32_t)recs.size();
            recs.push_back(r);
        }
        recs[rec[node]].q[dir - 1] = ibb_q[i];
        links.emplace_back((long long)node, dir);
    }
    // FD link-fraction records for nodes whose dX differs from 1
    std::vector<int32_t> dxi((size_t)c->D, -1);
    std::vector<DxRecord> dxr;
    std::vector<double> wd;   // FP64 wall distance, stored in the fields' type
    if (d.use_komega || d.use_thermal) {
        if (d.use_komega) wd.assign((size_t)c->D, 0.0);
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                const long long h = (long long)y * nxf + x;
                const size_t node = (size_t)y * P + x;
                if (d.use_komega) wd[node] = wallD[h];
                // records for the LB-fluid nodes (k-omega rows) and, with the
                // thermal update, for the fouling-layer nodes of its rows
                const int tt = (uint16_t)ntype[h];
                if ((tt & M_SOLID) && !(d.use_thermal && !(tt & M0_SOLID))) continue;
                DxRecord r;
                bool unit = true;
                for (int k = 0; k < 4; ++k) {
                    r.dx[k] = dX4[k * Dh + h];
                    if (r.dx[k] != 1.0) unit = false;
                }
                if (!unit) {
                    dxi[node] = (int32_t)dxr.size();
                    dxr.push_back(r);
                }
            }
    }
    // from here on the context's tables change: a failure leaves it without
    // a geometry (and state), so that it cannot step on half-written tables
    auto fail = [&](int code) {
        c->have_geometry = false;
        c->have_state = false;
        c->n_ibb_rec = 0;
        c->ibb_links.clear();
        return code;
    };
    if (c->ibb) { cudaFree(c->ibb); c->ibb = nullptr; }
    if (c->dxrec) { cudaFree(c->dxrec); c->dxrec = nullptr; }
    c->n_ibb_rec = (int)recs.size();
    c->ibb_cap = recs.size();
    c->dxrec_cap = dxr.size();
    if (c->ibb_node) { cudaFree(c->ibb_node); c->ibb_node = nullptr; }
    c->n_dxrec = (d.use_komega || d.use_thermal) ? (int)dxr.size() : -1;
    c->ibb_links.swap(links);
    if (!recs.empty()) {
        if (dalloc_t(&c->ibb, recs.size())) return fail(KOFM_ERR_BUFFER_ALLOCATION);
        if (cudaMemcpy(c->ibb, recs.data(), recs.size() * sizeof(IbbRecord), cudaMemcpyHostToDevice) != cudaSuccess) return fail(KOFM_ERR_MEMORY_COPY);
    }
    if (!dxr.empty()) {
        if (dalloc_t(&c->dxrec, dxr.size())) return fail(KOFM_ERR_BUFFER_ALLOCATION);
        if (cudaMemcpy(c->dxrec, dxr.data(), dxr.size() * sizeof(DxRecord), cudaMemcpyHostToDevice) != cudaSuccess) return fail(KOFM_ERR_MEMORY_COPY);
    }
    if (cudaMemcpy(c->ntype, nt.data(), nt.size() * sizeof(int16_t), cudaMemcpyHostToDevice) != cudaSuccess) return fail(KOFM_ERR_MEMORY_COPY);
    if (cudaMemcpy(c->rec, rec.data(), rec.size() * sizeof(int32_t), cudaMemcpyHostToDevice) != cudaSuccess) return fail(KOFM_ERR_MEMORY_COPY);
    if (cudaMemcpy(c->dxrec_idx, dxi.data(), dxi.size() * sizeof(int32_t), cudaMemcpyHostToDevice) != cudaSuccess) return fail(KOFM_ERR_MEMORY_COPY);
    if (d.use_komega) {
        cudaError_t e;
        if (c->f64) {
            e = cudaMemcpy(c->wallD, wd.data(), wd.size() * sizeof(double), cudaMemcpyHostToDevice);
        } else {
            std::vector<float> wf(wd.size());
            for (size_t i = 0; i < wd.size(); ++i) wf[i] = (float)wd[i];
            e = cudaMemcpy(c->wallD, wf.data(), wf.size() * sizeof(float), cudaMemcpyHostToDevice);
        }
        if (e != cudaSuccess) return fail(KOFM_ERR_MEMORY_COPY);
    }
    c->have_geometry = true;
    return KOFM_OK;
}

// Plane `plane` of a device field (of the context's field type).
static inline void* field_plane(kofm_ctx* c, void* f, int plane) {
    return static_cast<char*>(f) + (size_t)plane * c->D * c->fbytes;
}

static int upload_field(kofm_ctx* c, const double* h, void* dv) {
    const kofm_desc& d = c->desc;
    const size_t n = (size_t)d.nx_full * d.ny;
    KOFM_CUDA_TRY(cudaMemcpyAsync(c->staging, h, n * sizeof(double), cudaMemcpyHostToDevice, c->stream), KOFM_ERR_MEMORY_COPY);
    dim3 grid((c->P + 255) / 256, d.ny);
    if (c->f64) k_field_in<double><<<grid, 256, 0, c->stream>>>(c->staging, (double*)dv, d.nx_full, d.ny, c->P);
    else k_field_in<float><<<grid, 256, 0, c->stream>>>(c->staging, (float*)dv, d.nx_full, d.ny, c->P);
    KOFM_CUDA_TRY(cudaGetLastError(), KOFM_ERR_CALLING_KERNEL);
    return KOFM_OK;
}

static int download_field(kofm_ctx* c, const void* dv, double* h) {
    const kofm_desc& d = c->desc;
    const size_t n = (size_t)d.nx_full * d.ny;
    dim3 grid((d.nx_full + 255) / 256, d.ny);
    if (c->f64) k_field_out<double><<<grid, 256, 0, c->stream>>>((const double*)dv, c->staging, d.nx_full, d.ny, c->P);
    else k_field_out<float><<<grid, 256, 0, c->stream>>>((const float*)dv, c->staging, d.nx_full, d.ny, c->P);
    KOFM_CUDA_TRY(cudaGetLastError(), KOFM_ERR_CALLING_KERNEL);
    KOFM_CUDA_TRY(cudaMemcpyAsync(h, c->staging, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream), KOFM_ERR_MEMORY_COPY);
    KOFM_CUDA_TRY(cudaStreamSynchronize(c->stream), KOFM_ERR_MEMORY_COPY);
    return KOFM_OK;
}

int kofm_set_state(kofm_ctx* c, const double* f, const double* k, const double* omega,
                   const double* nut, const double* sxy) {
    if (!c || !f) return KOFM_ERR_INVALID_ARG;
    if (!c->have_geometry) return KOFM_ERR_STATE;
    const kofm_desc& d = c->desc;
    if (d.use_komega && (!k || !omega || !sxy)) return KOFM_ERR_INVALID_ARG;
    cudaSetDevice(c->dev);
    const size_t Dh = (size_t)d.nx_full * d.ny;
    int st = ensure_staging(c, 9 * Dh);
    if (st) return st;
    KOFM_CUDA_TRY(cudaMemcpyAsync(c->staging, f, 9 * Dh * sizeof(double), cudaMemcpyHostToDevice, c->stream), KOFM_ERR_MEMORY_COPY);
    dim3 grid((c->P + 127) / 128, d.ny);
    c->cur = 0;
    switch (d.storage) {
        case KOFM_STORE_FP32:
            k_fa_in<float><<<grid, 128, 0, c->stream>>>(c->staging, (float*)c->g[0], c->ntype, d.nx, d.nx_full, d.ny, c->P, c->D);
            break;
        case KOFM_STORE_FP16_DEV:
            k_fa_in<__half><<<grid, 128, 0, c->stream>>>(c->staging, (__half*)c->g[0], c->ntype, d.nx, d.nx_full, d.ny, c->P, c->D);
            break;
        case KOFM_STORE_FP16_NEQ:
        case KOFM_STORE_FP16_NEQ32:
            k_fa_in_neq<<<grid, 128, 0, c->stream>>>(c->staging, (__half*)c->g[0], c->ref[0], c->ntype, d.nx, d.nx_full, d.ny, c->P, c->D);
            break;
        case KOFM_STORE_FP16_ROW:
            k_row_ref<<<d.ny, 256, 0, c->stream>>>(c->staging, c->rowref, c->ntype, d.nx, d.nx_full, d.ny, c->P);
            c->row_steps = 0;
            k_fa_in_row<<<grid, 128, 0, c->stream>>>(c->staging, (__half*)c->g[0], c->rowref, c->ntype, d.nx, d.nx_full, d.ny, c->P, c->D);
            break;
        case KOFM_STORE_FP64:
            k_fa_in<double><<<grid, 128, 0, c->stream>>>(c->staging, (double*)c->g[0], c->ntype, d.nx, d.nx_full, d.ny, c->P, c->D);
            break;
        default:
            k_fa_in<__nv_bfloat16><<<grid, 128, 0, c->stream>>>(c->staging, (__nv_bfloat16*)c->g[0], c->ntype, d.nx, d.nx_full, d.ny, c->P, c->D);
    }
    KOFM_CUDA_TRY(cudaGetLastError(), KOFM_ERR_CALLING_KERNEL);
    if (d.use_komega) {
        if ((st = upload_field(c, k, c->K))) return st;
        if ((st = upload_field(c, omega, c->O))) return st;
        if (nut) {
            if ((st = upload_field(c, nut, c->nut))) return st;
        }
        for (int s = 0; s < 3; ++s)
            if ((st = upload_field(c, sxy + s * Dh, field_plane(c, c->S, s)))) return st;
    }
    KOFM_CUDA_TRY(cudaStreamSynchronize(c->stream), KOFM_ERR_MEMORY_COPY);
    c->phase = 0;
    c->have_state = true;
    c->stats.phase = 0;
    // a loaded state starts the k-omega sub-stepping again (kOmega::ini)
    c->dt = d.komega_dt;
    c->steps_per_lb = (int)(1.0 / d.komega_dt);
    if (c->steps_per_lb < 1) c->steps_per_lb = 1;
    c->time_since_change = 0;
    if (d.use_komega) {
        ug_pull(c);  // updates still in flight finish first
        ug_reset(c);
        c->launches_host = 0;
        c->stats.solver_launches_total = 0;
    }
    return KOFM_OK;
}

int kofm_get_state(kofm_ctx* c, double* f, double* k, double* omega, double* nut, double* sxy) {
    if (!c) return KOFM_ERR_INVALID_ARG;
    if (!c->have_state) return KOFM_ERR_STATE;
    const kofm_desc& d = c->desc;
    cudaSetDevice(c->dev);
    const size_t Dh = (size_t)d.nx_full * d.ny;
    int st = ensure_staging(c, 9 * Dh);
    if (st) return st;
    if (f) {
        dim3 grid((d.nx_full + 127) / 128, d.ny);
        const int has_ibb = c->n_ibb_rec > 0;
        switch (d.storage) {
            case KOFM_STORE_FP32:
                k_fa_out<float><<<grid, 128, 0, c->stream>>>((const float*)c->g[c->cur], c->ntype, c->rec, c->ibb, has_ibb, c->staging, d.nx, d.nx_full, d.ny, c->P, c->D, c->phase, PopRef{nullptr, nullptr});
                break;
            case KOFM_STORE_FP16_DEV:
                k_fa_out<__half><<<grid, 128, 0, c->stream>>>((const __half*)c->g[c->cur], c->ntype, c->rec, c->ibb, has_ibb, c->staging, d.nx, d.nx_full, d.ny, c->P, c->D, c->phase, PopRef{nullptr, nullptr});
                break;
            case KOFM_STORE_FP16_NEQ:
            case KOFM_STORE_FP16_NEQ32:
                k_fa_out<__half><<<grid, 128, 0, c->stream>>>((const __half*)c->g[c->cur], c->ntype, c->rec, c->ibb, has_ibb, c->staging, d.nx, d.nx_full, d.ny, c->P, c->D, c->phase, PopRef{c->ref[c->cur], nullptr});
                break;
            case KOFM_STORE_FP16_ROW:
                k_fa_out<__half><<<grid, 128, 0, c->stream>>>((const __half*)c->g[c->cur], c->ntype, c->rec, c->ibb, has_ibb, c->staging, d.nx, d.nx_full, d.ny, c->P, c->D, c->phase, PopRef{nullptr, c->rowref});
                break;
            case KOFM_STORE_FP64:
                k_fa_out<double><<<grid, 128, 0, c->stream>>>((const double*)c->g[c->cur], c->ntype, c->rec, c->ibb, has_ibb, c->staging, d.nx, d.nx_full, d.ny, c->P, c->D, c->phase, PopRef{nullptr, nullptr});
                break;
            default:
                k_fa_out<__nv_bfloat16><<<grid, 128, 0, c->stream>>>((const __nv_bfloat16*)c->g[c->cur], c->ntype, c->rec, c->ibb, has_ibb, c->staging, d.nx, d.nx_full, d.ny, c->P, c->D, c->phase, PopRef{nullptr, nullptr});
        }
        KOFM_CUDA_TRY(cudaGetLastError(), KOFM_ERR_CALLING_KERNEL);
        KOFM_CUDA_TRY(cudaMemcpyAsync(f, c->staging, 9 * Dh * sizeof(double), cudaMemcpyDeviceToHost, c->stream), KOFM_ERR_MEMORY_COPY);
        KOFM_CUDA_TRY(cudaStreamSynchronize(c->stream), KOFM_ERR_MEMORY_COPY);
    }
    if (d.use_komega) {
        if (k && (st = download_field(c, c->K, k))) return st;
        if (omega && (st = download_field(c, c->O, omega))) return st;
        if (nut && (st = download_field(c, c->nut, nut))) return st;
        if (sxy)
            for (int s = 0; s < 3; ++s)
                if ((st = download_field(c, field_plane(c, c->S, s), sxy + s * Dh))) return st;
    }
    return KOFM_OK;
}

int kofm_set_shear(kofm_ctx* c, const int32_t* nodes, int32_t n_nodes, const double* cfss,
                   const int32_t* bl_nodes, const double* bl_weights, int32_t n_bl) {
    if (!c || n_nodes < 1 || !nodes || !cfss || n_bl < 0 || (n_bl > 0 && (!bl_nodes || !bl_weights)))
        return KOFM_ERR_INVALID_ARG;
    if (!c->have_geometry) return KOFM_ERR_STATE;
    const kofm_desc& d = c->desc;
    const long long nh = (long long)d.nx_full * d.ny;
    for (int i = 0; i < n_nodes; ++i) {
        if (nodes[i] < 0 || nodes[i] >= nh || nodes[i] % d.nx_full >= d.nx) return KOFM_ERR_INVALID_ARG;
    }
    for (long long i = 0; i < 4LL * n_bl; ++i)
        if (bl_nodes[i] < -1 || bl_nodes[i] >= n_nodes) return KOFM_ERR_INVALID_ARG;
    cudaSetDevice(c->dev);
    void* old[] = {c->shear_nodes, c->shear_cfss, c->shear_tau, c->shear_bl_nodes, c->shear_bl_w, c->shear_bl_tau,
                   c->shear_idx};
    for (void* b : old)
        if (b) cudaFree(b);
    c->shear_nodes = nullptr; c->shear_cfss = nullptr; c->shear_tau = nullptr; c->shear_idx = nullptr;
    c->shear_bl_nodes = nullptr; c->shear_bl_w = nullptr; c->shear_bl_tau = nullptr;
    c->shear_n = c->shear_nbl = 0;
    int st;
    if ((st = dalloc_t(&c->shear_nodes, (size_t)n_nodes))) return st;
    if ((st = dalloc_t(&c->shear_cfss, (size_t)16 * n_nodes))) return st;
    if ((st = dalloc_t(&c->shear_tau, (size_t)n_nodes))) return st;
    if (n_bl > 0) {
        if ((st = dalloc_t(&c->shear_bl_nodes, (size_t)4 * n_bl))) return st;
        if ((st = dalloc_t(&c->shear_bl_w, (size_t)4 * n_bl))) return st;
        if ((st = dalloc_t(&c->shear_bl_tau, (size_t)n_bl))) return st;
    }
    KOFM_CUDA_TRY(cudaMemcpy(c->shear_nodes, nodes, sizeof(int32_t) * n_nodes, cudaMemcpyHostToDevice), KOFM_ERR_MEMORY_COPY);
    KOFM_CUDA_TRY(cudaMemcpy(c->shear_cfss, cfss, sizeof(double) * 16 * n_nodes, cudaMemcpyHostToDevice), KOFM_ERR_MEMORY_COPY);
    if (n_bl > 0) {
        KOFM_CUDA_TRY(cudaMemcpy(c->shear_bl_nodes, bl_nodes, sizeof(int32_t) * 4 * n_bl, cudaMemcpyHostToDevice), KOFM_ERR_MEMORY_COPY);
        KOFM_CUDA_TRY(cudaMemcpy(c->shear_bl_w, bl_weights, sizeof(double) * 4 * n_bl, cudaMemcpyHostToDevice), KOFM_ERR_MEMORY_COPY);
    }
    {
        std::vector<int32_t> idx((size_t)c->D, -1);
        for (int i = 0; i < n_nodes; ++i) {
            const int yy = nodes[i] / d.nx_full, xx = nodes[i] - yy * d.nx_full;
            idx[(size_t)yy * c->P + xx] = i;
        }
        if ((st = dalloc_t(&c->shear_idx, (size_t)c->D))) return st;
        KOFM_CUDA_TRY(cudaMemcpy(c->shear_idx, idx.data(), idx.size() * sizeof(int32_t), cudaMemcpyHostToDevice),
                      KOFM_ERR_MEMORY_COPY);
    }
    c->shear_n = n_nodes;
    c->shear_nbl = n_bl;
    return KOFM_OK;
}

int kofm_wall_shear(kofm_ctx* c, double* node_tau, double* bl_tau) {
    if (!c) return KOFM_ERR_INVALID_ARG;
    if (!c->have_state || c->shear_n < 1) return KOFM_ERR_STATE;
    const kofm_desc& d = c->desc;
    cudaSetDevice(c->dev);
    const int n = c->shear_n;
    const int has_ibb = c->n_ibb_rec > 0;
    const PopRef ref = (d.storage == KOFM_STORE_FP16_NEQ || d.storage == KOFM_STORE_FP16_NEQ32)
                           ? PopRef{c->ref[c->cur], nullptr}
                           : PopRef{nullptr, d.storage == KOFM_STORE_FP16_ROW ? c->rowref : nullptr};
    const int nb = (n + 127) / 128;
    const float* frho = (const float*)c->rho;
    const float* fux = (const float*)c->ux;
    const float* fuy = (const float*)c->uy;
    const float* fnut = (const float*)c->nut;
    switch (d.storage) {
        case KOFM_STORE_FP32:
            k_shear_nodes<float><<<nb, 128, 0, c->stream>>>((const float*)c->g[c->cur], c->ntype, c->rec, c->ibb, has_ibb, d.nx, d.ny, c->P, c->D, c->phase, PopRef{nullptr, nullptr}, frho, fux, fuy, fnut, d.mu, c->shear_nodes, c->shear_cfss, n, d.nx_full, c->shear_tau);
            break;
        case KOFM_STORE_BF16_DEV:
            k_shear_nodes<__nv_bfloat16><<<nb, 128, 0, c->stream>>>((const __nv_bfloat16*)c->g[c->cur], c->ntype, c->rec, c->ibb, has_ibb, d.nx, d.ny, c->P, c->D, c->phase, PopRef{nullptr, nullptr}, frho, fux, fuy, fnut, d.mu, c->shear_nodes, c->shear_cfss, n, d.nx_full, c->shear_tau);
            break;
        case KOFM_STORE_FP64:
            k_shear_nodes<double, double><<<nb, 128, 0, c->stream>>>((const double*)c->g[c->cur], c->ntype, c->rec, c->ibb, has_ibb, d.nx, d.ny, c->P, c->D, c->phase, PopRef{nullptr, nullptr}, (const double*)c->rho, (const double*)c->ux, (const double*)c->uy, (const double*)c->nut, d.mu, c->shear_nodes, c->shear_cfss, n, d.nx_full, c->shear_tau);
            break;
        default:  // FP16 forms
            k_shear_nodes<__half><<<nb, 128, 0, c->stream>>>((const __half*)c->g[c->cur], c->ntype, c->rec, c->ibb, has_ibb, d.nx, d.ny, c->P, c->D, c->phase, ref, frho, fux, fuy, fnut, d.mu, c->shear_nodes, c->shear_cfss, n, d.nx_full, c->shear_tau);
    }
    KOFM_CUDA_TRY(cudaGetLastError(), KOFM_ERR_CALLING_KERNEL);
    if (c->shear_nbl > 0) {
        k_shear_links<<<(c->shear_nbl + 127) / 128, 128, 0, c->stream>>>(c->shear_tau, c->shear_bl_nodes, c->shear_bl_w, c->shear_nbl, c->shear_bl_tau);
        KOFM_CUDA_TRY(cudaGetLastError(), KOFM_ERR_CALLING_KERNEL);
    }
    if (node_tau)
        KOFM_CUDA_TRY(cudaMemcpyAsync(node_tau, c->shear_tau, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream), KOFM_ERR_MEMORY_COPY);
    if (bl_tau && c->shear_nbl > 0)
        KOFM_CUDA_TRY(cudaMemcpyAsync(bl_tau, c->shear_bl_tau, sizeof(double) * c->shear_nbl, cudaMemcpyDeviceToHost, c->stream), KOFM_ERR_MEMORY_COPY);
    KOFM_CUDA_TRY(cudaStreamSynchronize(c->stream), KOFM_ERR_CALLING_KERNEL);
    return KOFM_OK;
}

int kofm_get_macro(kofm_ctx* c, double* rho, double* ux, double* uy) {
    if (!c) return KOFM_ERR_INVALID_ARG;
    cudaSetDevice(c->dev);
    const kofm_desc& d = c->desc;
    int st = ensure_staging(c, (size_t)d.nx_full * d.ny);
    if (st) return st;
    if (rho && (st = download_field(c, c->rho, rho))) return st;
    if (ux && (st = download_field(c, c->ux, ux))) return st;
    if (uy && (st = download_field(c, c->uy, uy))) return st;
    return KOFM_OK;
}

}  // extern "C"

namespace {

// Parameters of the collide from buffer parity cur (read g[cur], write g[cur ^ 1]).
LbParams lb_params(const kofm_ctx* c, int32_t options, int cur) {
    const kofm_desc& d = c->desc;
    LbParams p;
    p.gin = c->g[cur];
    p.gout = c->g[cur ^ 1];
    p.ntype = c->ntype;
    p.rec = c->rec;
    p.ibb = c->ibb;
    p.wallD = c->wallD;
    p.K = c->K; p.O = c->O; p.S = c->S; p.nut = c->nut;
    p.rho = c->rho; p.ux = c->ux; p.uy = c->uy;
    p.partials = c->lb_partials;
    p.ref_in = c->ref[cur];
    p.ref_out = c->ref[cur ^ 1];
    p.rowref = c->rowref;
    p.nx = d.nx; p.ny = d.ny; p.P = c->P; p.D = c->D;
    p.tau = d.tau; p.fterm = d.fterm; p.mu = d.mu; p.maxnut = d.max_turb_visc;
    p.options = options;
    p.has_ibb = c->n_ibb_rec > 0;
    return p;
}

// Host-side record of a collide enqueued for c.
void lb_done(kofm_ctx* c) {
    c->cur ^= 1;
    c->phase = 1;
    c->stats.phase = 1;
    c->stats.steps += 1;
}

}  // namespace

extern "C" {

int kofm_lb_step(kofm_ctx* c, int32_t options) {
    if (!c) return KOFM_ERR_INVALID_ARG;
    if (!c->have_state) return KOFM_ERR_STATE;
    const kofm_desc& d = c->desc;
    const LbParams p = lb_params(c, options, c->cur);
    const bool ko = d.use_komega != 0, ph0 = c->phase == 0;
    cudaError_t e;
    switch (d.storage) {
        case KOFM_STORE_FP32: e = launch_lb<float, double>(c, p, ko, ph0); break;
        case KOFM_STORE_FP16_DEV: e = launch_lb<__half, float>(c, p, ko, ph0); break;
        case KOFM_STORE_FP16_NEQ: e = launch_lb<__half, double, true>(c, p, ko, ph0); break;
        case KOFM_STORE_FP64: e = launch_lb<double, double, false, double>(c, p, ko, ph0); break;
        case KOFM_STORE_FP16_NEQ32: e = launch_lb<__half, float, true>(c, p, ko, ph0); break;
        case KOFM_STORE_FP16_ROW: e = launch_lb<__half, KOFM_ROW_AT, false, float, true>(c, p, ko, ph0); break;
        default: e = launch_lb<__nv_bfloat16, float>(c, p, ko, ph0); break;
    }
    if (e != cudaSuccess) {
        fprintf(stderr, "kofm: lb step launch failed: %s\n", cudaGetErrorString(e));
        return KOFM_ERR_CALLING_KERNEL;
    }
    lb_done(c);
    if (d.storage == KOFM_STORE_FP16_ROW && (options & KOFM_OPTION_SAVE_MACRO_FIELDS) &&
        ++c->row_steps >= KOFM_ROW_RECENTRE) {
        // the row references follow the flow: the row means of the moments
        // this collide wrote, the stored values re-encoded against them
        k_row_ref_fields<<<d.ny, 256, 0, c->stream>>>((const float*)c->rho, (const float*)c->ux,
                                                      (const float*)c->uy, c->rowref_next, c->ntype,
                                                      d.nx, d.ny, c->P);
        dim3 grid((c->P + 127) / 128, d.ny);
        k_row_recentre<<<grid, 128, 0, c->stream>>>((__half*)c->g[c->cur], c->rowref, c->rowref_next,
                                                    c->ntype, d.nx, d.ny, c->P, c->D);
        KOFM_CUDA_TRY(cudaGetLastError(), KOFM_ERR_CALLING_KERNEL);
        std::swap(c->rowref, c->rowref_next);
        c->row_steps = 0;
    }
    return KOFM_OK;
}

int kofm_reduce(kofm_ctx* c, int32_t field, int32_t op, double* out) {
    if (!c || !out) return KOFM_ERR_INVALID_ARG;
    const kofm_desc& d = c->desc;
    const void* v = nullptr;
    switch (field) {
        case KOFM_FIELD_RHO: v = c->rho; break;
        case KOFM_FIELD_UX: v = c->ux; break;
        case KOFM_FIELD_UY: v = c->uy; break;
        case KOFM_FIELD_K: v = c->K; break;
        case KOFM_FIELD_OMEGA: v = c->O; break;
        case KOFM_FIELD_NUT: v = c->nut; break;
        case KOFM_FIELD_WALL_SHEAR: break;
        case KOFM_FIELD_TEMP: break;
        default: return KOFM_ERR_INVALID_ARG;
    }
    if (field == KOFM_FIELD_TEMP && !c->T) return KOFM_ERR_STATE;
    if (field != KOFM_FIELD_WALL_SHEAR && field != KOFM_FIELD_TEMP && !v) return KOFM_ERR_STATE;
    if (op < KOFM_OP_SUM || op > KOFM_OP_MAX) return KOFM_ERR_INVALID_ARG;
    cudaSetDevice(c->dev);
    const long long n = c->D;
    if (field == KOFM_FIELD_WALL_SHEAR) {
        if (!d.use_komega || op != KOFM_OP_SUM) return KOFM_ERR_INVALID_ARG;
        if (c->f64)
            k_wall_shear<double><<<RED_BLOCKS, 256, 0, c->stream>>>(c->ntype, (const double*)c->rho, (const double*)c->nut, (const double*)c->S, n, c->D, c->P, d.nx, d.mu, c->red_partials);
        else
            k_wall_shear<float><<<RED_BLOCKS, 256, 0, c->stream>>>(c->ntype, (const float*)c->rho, (const float*)c->nut, (const float*)c->S, n, c->D, c->P, d.nx, d.mu, c->red_partials);
        k_reduce_final<KOFM_OP_SUM><<<1, 32, 0, c->stream>>>(c->red_partials, RED_BLOCKS, c->red_out);
    } else if (field == KOFM_FIELD_TEMP) {
        if (op == KOFM_OP_SUM) k_reduce_field<KOFM_OP_SUM, double><<<RED_BLOCKS, 256, 0, c->stream>>>(c->T, n, c->P, d.nx_full, c->red_partials);
        else if (op == KOFM_OP_MIN) k_reduce_field<KOFM_OP_MIN, double><<<RED_BLOCKS, 256, 0, c->stream>>>(c->T, n, c->P, d.nx_full, c->red_partials);
        else k_reduce_field<KOFM_OP_MAX, double><<<RED_BLOCKS, 256, 0, c->stream>>>(c->T, n, c->P, d.nx_full, c->red_partials);
        if (op == KOFM_OP_SUM) k_reduce_final<KOFM_OP_SUM><<<1, 32, 0, c->stream>>>(c->red_partials, RED_BLOCKS, c->red_out);
        else if (op == KOFM_OP_MIN) k_reduce_final<KOFM_OP_MIN><<<1, 32, 0, c->stream>>>(c->red_partials, RED_BLOCKS, c->red_out);
        else k_reduce_final<KOFM_OP_MAX><<<1, 32, 0, c->stream>>>(c->red_partials, RED_BLOCKS, c->red_out);
    } else if (c->f64) {
        const double* fv = (const double*)v;
        if (op == KOFM_OP_SUM) k_reduce_field<KOFM_OP_SUM, double><<<RED_BLOCKS, 256, 0, c->stream>>>(fv, n, c->P, d.nx_full, c->red_partials);
        else if (op == KOFM_OP_MIN) k_reduce_field<KOFM_OP_MIN, double><<<RED_BLOCKS, 256, 0, c->stream>>>(fv, n, c->P, d.nx_full, c->red_partials);
        else k_reduce_field<KOFM_OP_MAX, double><<<RED_BLOCKS, 256, 0, c->stream>>>(fv, n, c->P, d.nx_full, c->red_partials);
        if (op == KOFM_OP_SUM) k_reduce_final<KOFM_OP_SUM><<<1, 32, 0, c->stream>>>(c->red_partials, RED_BLOCKS, c->red_out);
        else if (op == KOFM_OP_MIN) k_reduce_final<KOFM_OP_MIN><<<1, 32, 0, c->stream>>>(c->red_partials, RED_BLOCKS, c->red_out);
        else k_reduce_final<KOFM_OP_MAX><<<1, 32, 0, c->stream>>>(c->red_partials, RED_BLOCKS, c->red_out);
    } else if (op == KOFM_OP_SUM) {
        k_reduce_field<KOFM_OP_SUM><<<RED_BLOCKS, 256, 0, c->stream>>>((const float*)v, n, c->P, d.nx_full, c->red_partials);
        k_reduce_final<KOFM_OP_SUM><<<1, 32, 0, c->stream>>>(c->red_partials, RED_BLOCKS, c->red_out);
    } else if (op == KOFM_OP_MIN) {
        k_reduce_field<KOFM_OP_MIN><<<RED_BLOCKS, 256, 0, c->stream>>>((const float*)v, n, c->P, d.nx_full, c->red_partials);
        k_reduce_final<KOFM_OP_MIN><<<1, 32, 0, c->stream>>>(c->red_partials, RED_BLOCKS, c->red_out);
    } else {
        k_reduce_field<KOFM_OP_MAX><<<RED_BLOCKS, 256, 0, c->stream>>>((const float*)v, n, c->P, d.nx_full, c->red_partials);
        k_reduce_final<KOFM_OP_MAX><<<1, 32, 0, c->stream>>>(c->red_partials, RED_BLOCKS, c->red_out);
    }
    KOFM_CUDA_TRY(cudaGetLastError(), KOFM_ERR_CALLING_KERNEL);
    KOFM_CUDA_TRY(cudaMemcpyAsync(c->h_red, c->red_out, sizeof(double), cudaMemcpyDeviceToHost, c->stream), KOFM_ERR_MEMORY_COPY);
    KOFM_CUDA_TRY(cudaStreamSynchronize(c->stream), KOFM_ERR_CALLING_KERNEL);
    *out = c->h_red[0];
    return KOFM_OK;
}

int kofm_sync(kofm_ctx* c) {
    if (!c) return KOFM_ERR_INVALID_ARG;
    cudaSetDevice(c->dev);
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
        fprintf(stderr, "kofm: stream error: %s\n", cudaGetErrorString(e));
        return KOFM_ERR_CALLING_KERNEL;
    }
    // the status the device-driven k-omega updates stopped with, if any
    if (c->desc.use_komega) return ug_pull(c);
    return KOFM_OK;
}

int kofm_get_stats(kofm_ctx* c, kofm_stats* out) {
    if (!c || !out) return KOFM_ERR_INVALID_ARG;
    if (c->desc.use_komega) {
        cudaSetDevice(c->dev);
        ug_pull(c);
    }
    c->stats.steps_per_lb = c->steps_per_lb;
    c->stats.time_since_change = c->time_since_change;
    c->stats.dt = c->dt;
    c->stats.thermal_steps_per_lb = c->th_steps_per_lb;
    c->stats.thermal_time_since_change = c->th_time_since_change;
    c->stats.thermal_dt = c->th_dt;
    *out = c->stats;
    return KOFM_OK;
}

}  // extern "C"

// k-omega entry points live in kofm_komega_api.inc (same translation unit).
#include "kofm_komega_api.inc"
// batched lattices (CUDA graph over several contexts)
#include "kofm_batch.inc"
// thermal implicit FD
#include "kofm_thermal_api.inc"
// discrete adjoint of the laminar step
#include "kofm_adjoint.inc"
#include "kofm_geometry.inc"
