// kofm_common.cuh - shared definitions of the sm_100a kernels.
//
// Device layout (private to the library):
//   pitch P = nx_full rounded up to a multiple of 128 nodes; plane stride
//   D = P * ny; node (x, y) at x + P*y; population q of node at q*D + node.
//   Populations are stored as deviations d_q = f_q - w_q (w_q = D2Q9 weight),
//   in FP32 (collide arithmetic FP64) or FP16/BF16 (collide arithmetic FP32).
//   The buffers hold either the reference's FA form (pre-collision, right
//   after kofm_set_state: "phase 0") or post-collision values that the next
//   step gathers from the neighbours ("phase 1", pull scheme).
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <stdint.h>

namespace kofm {

// nType bits (reference Kernels/Heading.cl:223-251).
constexpr int M_SOLID = 0x0001;
constexpr int M_FLUID = 0x0002;
constexpr int M0_SOLID = 0x0004;         // wall of the unfouled geometry
constexpr int M0_FLUID = 0x0008;
constexpr int SOLID_BOUNDARY = 0x0010;
constexpr int SOLID_BOUNDARY0 = 0x0020;  // boundary of the unfouled wall
constexpr int E_BOUND = 0x0100, W_BOUND = 0x0200, N_BOUND = 0x0400, S_BOUND = 0x0800;
constexpr int NE_BOUND = 0x1000, SW_BOUND = 0x2000, SE_BOUND = 0x4000, NW_BOUND = 0x8000;
constexpr int NESW_BOUNDARY = 0x0F00;
constexpr int BOUNDARY = 0xFF00;
constexpr int OPTION_SAVE_MACRO_FIELDS = 0x2;

// D2Q9 direction order C,E,W,N,S,NE,SW,SE,NW (Heading.cl:197-205).
__host__ __device__ constexpr int cx_of(int q) {
    return q == 1 || q == 5 || q == 7 ? 1 : (q == 2 || q == 6 || q == 8 ? -1 : 0);
}
__host__ __device__ constexpr int cy_of(int q) {
    return q == 3 || q == 5 || q == 8 ? 1 : (q == 4 || q == 6 || q == 7 ? -1 : 0);
}
__host__ __device__ constexpr int rev_of(int q) {
    return q == 0 ? 0 : (q % 2 == 1 ? q + 1 : q - 1);
}
__host__ __device__ constexpr int bound_of(int q) {
    return q == 0 ? 0 : (0x0100 << (q - 1));
}
// w_q = phi0(cx) * phi0(cy), phi0(0) = 2/3, phi0(+-1) = 1/6.
__host__ __device__ constexpr double weight_of(int q) {
    return (cx_of(q) == 0 ? 2.0 / 3.0 : 1.0 / 6.0) * (cy_of(q) == 0 ? 2.0 / 3.0 : 1.0 / 6.0);
}

// SST constants (Heading.cl:396-410).
constexpr double KO_BETA_STAR = 9.0 / 100.0;
constexpr double KO_SIGMA_K1 = 0.85, KO_SIGMA_K2 = 1.0;
constexpr double KO_SIGMA_O1 = 0.5, KO_SIGMA_O2 = 0.856;
constexpr double KO_A1 = 0.31, KO_KAPPA = 0.41, KO_C_MU_0_25 = 0.5477225575;
constexpr double KO_GAMMA1 = 5.0 / 9.0, KO_GAMMA2 = 0.44;

// ---- storage conversions ------------------------------------------------
template <typename ST> struct Store;
// vt: the type a population is loaded into and stored from (FP32 for the
// 32- and 16-bit forms, FP64 for the FP64 form)
template <> struct Store<double> {
    using vt = double;
    __device__ static double to_f32(double v) { return v; }
    __device__ static double to_f64(double v) { return v; }
    __device__ static double from_f64(double v) { return v; }
    __device__ static void load4(const double* p, double o[4]) {
        const double2 a = __ldg(reinterpret_cast<const double2*>(p));
        const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
        o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
    }
    __device__ static void store4(double* p, const double v[4]) {
        reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
        reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
    }
};
template <> struct Store<float> {
    using vt = float;
    using vec4 = float4;
    __device__ static float to_f32(float v) { return v; }
    __device__ static float from_f32(float v) { return v; }
    __device__ static double to_f64(float v) { return (double)v; }
    __device__ static float from_f64(double v) { return (float)v; }
    __device__ static void load4(const float* p, float o[4]) {
        float4 v = __ldg(reinterpret_cast<const float4*>(p));
        o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
    }
    __device__ static void store4(float* p, const float v[4]) {
        *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
    }
};
template <> struct Store<__half> {
    using vt = float;
    __device__ static float to_f32(__half v) { return __half2float(v); }
    __device__ static double to_f64(__half v) { return (double)__half2float(v); }
    __device__ static __half from_f32(float v) { return __float2half_rn(v); }
    __device__ static __half from_f64(double v) { return __double2half(v); }
    __device__ static void load4(const __half* p, float o[4]) {
        uint2 raw = __ldg(reinterpret_cast<const uint2*>(p));
        __half2 a = *reinterpret_cast<__half2*>(&raw.x);
        __half2 b = *reinterpret_cast<__half2*>(&raw.y);
        float2 fa = __half22float2(a), fb = __half22float2(b);
        o[0] = fa.x; o[1] = fa.y; o[2] = fb.x; o[3] = fb.y;
    }
    __device__ static void store4(__half* p, const float v[4]) {
        __half2 a = __floats2half2_rn(v[0], v[1]);
        __half2 b = __floats2half2_rn(v[2], v[3]);
        uint2 raw;
        raw.x = *reinterpret_cast<uint32_t*>(&a);
        raw.y = *reinterpret_cast<uint32_t*>(&b);
        *reinterpret_cast<uint2*>(p) = raw;
    }
};
template <> struct Store<__nv_bfloat16> {
    using vt = float;
    __device__ static float to_f32(__nv_bfloat16 v) { return __bfloat162float(v); }
    __device__ static double to_f64(__nv_bfloat16 v) { return (double)__bfloat162float(v); }
    __device__ static __nv_bfloat16 from_f32(float v) { return __float2bfloat16_rn(v); }
    __device__ static __nv_bfloat16 from_f64(double v) { return __double2bfloat16(v); }
    __device__ static void load4(const __nv_bfloat16* p, float o[4]) {
        uint2 raw = __ldg(reinterpret_cast<const uint2*>(p));
        __nv_bfloat162 a = *reinterpret_cast<__nv_bfloat162*>(&raw.x);
        __nv_bfloat162 b = *reinterpret_cast<__nv_bfloat162*>(&raw.y);
        float2 fa = __bfloat1622float2(a), fb = __bfloat1622float2(b);
        o[0] = fa.x; o[1] = fa.y; o[2] = fb.x; o[3] = fb.y;
    }
    __device__ static void store4(__nv_bfloat16* p, const float v[4]) {
        __nv_bfloat162 a = __floats2bfloat162_rn(v[0], v[1]);
        __nv_bfloat162 b = __floats2bfloat162_rn(v[2], v[3]);
        uint2 raw;
        raw.x = *reinterpret_cast<uint32_t*>(&a);
        raw.y = *reinterpret_cast<uint32_t*>(&b);
        *reinterpret_cast<uint2*>(p) = raw;
    }
};

// ---- 4 consecutive field values (16-byte aligned FP32, 32-byte FP64) ---------
__device__ __forceinline__ void fld_ld4(const float* p, float o[4]) {
    const float4 v = *reinterpret_cast<const float4*>(p);
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
}
__device__ __forceinline__ void fld_ld4(const double* p, double o[4]) {
    const double2 a = reinterpret_cast<const double2*>(p)[0];
    const double2 b = reinterpret_cast<const double2*>(p)[1];
    o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
}
__device__ __forceinline__ void fld_ldg4(const float* p, float o[4]) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(p));
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
}
__device__ __forceinline__ void fld_ldg4(const double* p, double o[4]) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
}
__device__ __forceinline__ void fld_st4(float* p, const float v[4]) {
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void fld_st4(double* p, const double v[4]) {
    reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
    reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
}

// ---- non-equilibrium storage form (KOFM_STORE_FP16_NEQ) ----------------------
// A stored population is e_q = f_q - feq_q(rho_r, u_r): its distance from the
// product-form equilibrium of a reference moment triple (rho_r, u_r) that the
// writing node stores in FP32 beside it (its rho, reported u_x, u_y).  e is
// O(f_neq), far smaller than the f - w deviation, so FP16 keeps ~3 more
// decimal digits of the population.  e is scaled by 2^12 before rounding so
// that the small values stay in FP16's normal range.  Encoder and decoder use
// the same FP32 function of the same FP32 reference values.
constexpr float NEQ_SCALE = 4096.0f;
constexpr float NEQ_INV_SCALE = 1.0f / 4096.0f;

// feq_q(rho, u) - w_q in FP32 (deviation form of the product equilibrium)
__device__ __forceinline__ float feq_dev_f32(int q, float rho, float ux, float uy) {
    const int cx = cx_of(q), cy = cy_of(q);
    const float drho = rho - 1.0f;
    const float px0 = cx == 0 ? 2.0f / 3.0f : 1.0f / 6.0f;
    const float py0 = cy == 0 ? 2.0f / 3.0f : 1.0f / 6.0f;
    const float dpx = cx == 0 ? -ux * ux : 0.5f * ((float)cx * ux + ux * ux);
    const float dpy = cy == 0 ? -uy * uy : 0.5f * ((float)cy * uy + uy * uy);
    return __fadd_rn(__fmul_rn(__fmul_rn(drho, __fadd_rn(px0, dpx)), __fadd_rn(py0, dpy)),
                     __fadd_rn(__fadd_rn(__fmul_rn(dpx, py0), __fmul_rn(px0, dpy)), __fmul_rn(dpx, dpy)));
}

// Interpolated bounce-back record of one wall-adjacent node: wall fraction q
// of each link direction 1..8 (q < 0: no interpolated correction on that
// link).  Built on the host from the reference's ibbArr / ibbDistArr list.
struct IbbRecord {
    double q[8];
};

// Per-node FD link fractions for nodes with an E/W/N/S wall link (dXArr of
// the reference, planes E,W,N,S); every other fluid node has all four = 1.
struct DxRecord {
    double dx[4];
};

}  // namespace kofm
