// OpenCL-C -> C++ shim used ONLY to compile the reference's own kernel
// sources (source/Kernels/Heading.cl, lbKernels.cl, kOmegaKernels.cl, the
// wall-shear functions of trKernelsShear.cl, the implicit thermal assembly of
// tfdKernels.cl and the interpolated-link list builder of lsKernels.cl) for the
// CPU, so the oracle can be checked against the reference code itself.
//
// This file is test infrastructure (the checker), never part of the product.
// The kernel sources are not copied into this repository: oracle/Makefile
// preprocesses them from the reference tree into oracle/_ref/ (git-ignored)
// and ref_kernels.cpp #includes them inside `struct RefProgram`, so that the
// program-build-time `#define`s of the reference (CHANNEL_LENGTH, DIST_SIZE,
// tau0, FTERM_VAL, MU_NUMBER, ...) become per-instance members, set at run
// time instead of by the OpenCL compiler.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

typedef unsigned int uint;
typedef unsigned long ulong;
typedef unsigned short ushort;
typedef unsigned char uchar;

struct int2 { int x, y; };
struct uint2 { uint x, y; };
struct double2 {
    double x, y;
    double2() = default;
    double2(double s) : x(s), y(s) {}          // OpenCL scalar -> vector
    double2(double a, double b) : x(a), y(b) {}
};
struct double4 { double x, y, z, w; };
// double8 with the .s0 .. .s7 and .lo / .hi views used by the shear kernels
struct double8 {
    union {
        struct { double s0, s1, s2, s3, s4, s5, s6, s7; };
        struct { double4 lo, hi; };
    };
};
struct float4 { float x, y, z, w; };

static inline int2 make_int2(int a, int b) { return int2{a, b}; }
static inline uint2 make_uint2(uint a, uint b) { return uint2{a, b}; }
static inline double2 make_double2(double a, double b) { return double2{a, b}; }
static inline double4 make_double4(double a, double b, double c, double d) { return double4{a, b, c, d}; }
static inline double8 make_double8(double a, double b, double c, double d, double e, double f,
                                   double g, double h) {
    double8 r;
    r.s0 = a; r.s1 = b; r.s2 = c; r.s3 = d; r.s4 = e; r.s5 = f; r.s6 = g; r.s7 = h;
    return r;
}
static inline double8 operator*(double8 a, double s) {
    return make_double8(a.s0 * s, a.s1 * s, a.s2 * s, a.s3 * s, a.s4 * s, a.s5 * s, a.s6 * s, a.s7 * s);
}
static inline double dot(double4 a, double4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
static inline float4 make_float4(float a, float b, float c, float d) { return float4{a, b, c, d}; }

static inline double2 operator+(double2 a, double2 b) { return {a.x + b.x, a.y + b.y}; }
static inline double2 operator-(double2 a, double2 b) { return {a.x - b.x, a.y - b.y}; }
static inline double2 operator*(double s, double2 a) { return {s * a.x, s * a.y}; }
static inline double2 operator*(double2 a, double s) { return {s * a.x, s * a.y}; }
static inline double2 operator/(double2 a, double s) { return {a.x / s, a.y / s}; }
static inline double2& operator/=(double2& a, double s) { a.x /= s; a.y /= s; return a; }
static inline double2& operator*=(double2& a, double s) { a.x *= s; a.y *= s; return a; }
static inline double dot(double2 a, double2 b) { return a.x * b.x + a.y * b.y; }
static inline double length(double2 a) { return std::sqrt(a.x * a.x + a.y * a.y); }
static inline double2 normalize(double2 a) { const double l = length(a); return {a.x / l, a.y / l}; }
static inline double2 ceil(double2 a) { return {std::ceil(a.x), std::ceil(a.y)}; }
static inline int2 convert_int2(double2 a) { return {(int)a.x, (int)a.y}; }
static inline double2 convert_double2(int2 a) { return {(double)a.x, (double)a.y}; }
static inline double convert_double(uint a) { return (double)a; }

// OpenCL max/min for scalars: "returns y if x < y, otherwise x" (and the
// mirrored rule for min).
static inline double max(double a, double b) { return a < b ? b : a; }
static inline double min(double a, double b) { return b < a ? b : a; }
static inline int max(int a, int b) { return a < b ? b : a; }
static inline int min(int a, int b) { return b < a ? b : a; }
static inline double pown(double x, int n) { return std::pow(x, (double)n); }
using std::sqrt; using std::tanh; using std::fabs; using std::exp; using std::log;
using std::isfinite;

static inline uint mad_hi(uint a, uint b, uint c) {
    return (uint)(((unsigned long long)a * (unsigned long long)b) >> 32) + c;
}
// the list builder's slot counter; its work-items run one after another
static inline int atomic_add(int* p, int v) { const int old = *p; *p += v; return old; }
static inline ulong atom_cmpxchg(volatile ulong* p, ulong cmp, ulong val) {
    return __sync_val_compare_and_swap(p, cmp, val);
}

// Work-item indices: set by the NDRange loop in ref_kernels.cpp. One OpenMP
// thread runs one work-item at a time, so thread_local storage suffices (the
// LB/k-omega kernels use no barriers or local memory).
extern thread_local size_t g_ref_gid[3];
static inline size_t get_global_id(int d) { return g_ref_gid[d]; }
// one work-item per work-group slot: local arrays are indexed by slot 0
static inline size_t get_local_id(int) { return 0; }
