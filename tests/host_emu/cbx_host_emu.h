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
template <class T> inline T __shfl_sync(unsigned, T v, int) { return v; }
inline bool __any_sync(unsigned, bool v) { return v; }
