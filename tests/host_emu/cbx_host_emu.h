// Host emulation of the CUDA constructs used by the integrator headers.
//
// Test infrastructure: lets the generated integrator translation unit be
// compiled by g++ and executed one thread at a time on the CPU, so the
// device logic can be checked against the oracle without a GPU.  Warp
// intrinsics act on a single lane (each emulated thread runs alone).
#pragma once
#define CBX_HOST_EMULATION 1
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>

#define __device__
#define __host__
#define __global__
#define __forceinline__ inline
#define __constant__ static
#define __shared__ static
#define __launch_bounds__(...)

using std::ceil;
using std::fabs;
using std::floor;
using std::fmax;
using std::fmin;
using std::isfinite;
using std::isnan;
using std::pow;
using std::sqrt;
inline float sqrtf(float v) { return std::sqrt(v); }
inline float powf(float a, float b) { return std::pow(a, b); }

struct float4 {
    float x, y, z, w;
};
inline float4 make_float4(float x, float y, float z, float w) { return float4{x, y, z, w}; }
struct uint4 {
    unsigned x, y, z, w;
};
inline uint4 make_uint4(unsigned x, unsigned y, unsigned z, unsigned w) { return uint4{x, y, z, w}; }
struct double2 {
    double x, y;
};
inline double2 make_double2(double x, double y) { return double2{x, y}; }

struct cbx_dim3 {
    unsigned x, y, z;
};
extern cbx_dim3 threadIdx, blockIdx, blockDim, gridDim;

template <class T> inline T __ldg(const T* p) { return *p; }
inline void __syncthreads() {}
inline unsigned long long atomicAdd(unsigned long long* a, unsigned long long v) {
    unsigned long long old = *a;
    *a += v;
    return old;
}
inline unsigned __activemask() { return 1u << (threadIdx.x & 31u); }
inline int __ffs(unsigned v) { return v ? __builtin_ctz(v) + 1 : 0; }
inline int __popc(unsigned v) { return __builtin_popcount(v); }
// round-to-nearest adds that the device compiler never fuses into an FMA;
// the host build contracts nothing, so they are plain adds here
inline float __fadd_rn(float a, float b) { return a + b; }
inline double __dadd_rn(double a, double b) { return a + b; }
template <class T> inline T __shfl_sync(unsigned, T v, int) { return v; }
inline bool __any_sync(unsigned, bool v) { return v; }
