// Common definitions for the batch ODE integrator device code.
//
// Compiled at run time by NVRTC for sm_100a together with a generated
// system struct and a generated configuration struct (see
// cubie_b200/kernelgen.py).  Everything here is header-only device code.
#pragma once

// Functions whose body is large and called from many places (the class-
// grouped right-hand side and J v of the warp layout) are kept as one copy:
// inlined at every call site of every unrolled stage they multiplied the
// kernel's code size until instruction fetch, not arithmetic, bounded it.
#ifdef CBX_HOST_EMULATION
#define CBX_NOINLINE __attribute__((noinline))
#else
#define CBX_NOINLINE __noinline__
#endif

namespace cbx {

// Per-run status bits; values match the reference's CUBIE_RESULT_CODES
// (src/cubie/result_codes.py:50-58).
enum Status : int {
    SUCCESS = 0,
    MAX_NEWTON_ITERATIONS_EXCEEDED = 2,
    MAX_LINEAR_ITERATIONS_EXCEEDED = 4,
    STEP_TOO_SMALL = 8,
    DT_EFF_EFFECTIVELY_ZERO = 16,
    MAX_LOOP_ITERS_EXCEEDED = 32,
    STAGNATION = 64,
    BICGSTAB_BREAKDOWN = 128,
    NEWTON_DIVERGENCE = 256,
};

// Algorithm families and linear solvers selected by the configuration.
enum Algo : int { ALGO_ERK = 0, ALGO_DIRK = 1, ALGO_FIRK = 2, ALGO_ROSENBROCK = 3 };
enum Lin : int { LIN_MR = 0, LIN_SD = 1, LIN_BICGSTAB = 2, LIN_GMRES = 3, LIN_DIRECT = 4 };
enum Ctrl : int { CTRL_FIXED = 0, CTRL_I = 1, CTRL_PI = 2, CTRL_PID = 3, CTRL_GUSTAFSSON = 4 };

// Python's max/min semantics for two arguments (the reference uses the
// Python builtins, which keep the first argument unless the second is
// strictly larger/smaller; this decides NaN propagation).
template <class T> __device__ __forceinline__ T pymax(T a, T b) { return (b > a) ? b : a; }
template <class T> __device__ __forceinline__ T pymin(T a, T b) { return (b < a) ? b : a; }
template <class T> __device__ __forceinline__ T clampv(T v, T lo, T hi) { return pymax(lo, pymin(v, hi)); }

template <class T> __device__ __forceinline__ T absv(T v) { return v < T(0) ? -v : v; }

// A round-to-nearest add the compiler never fuses with the multiply that
// produced an operand.  Used where a value crosses from the step function
// into the loop's state update: whether an FMA forms there otherwise depends
// on the surrounding control flow, and the adjoint's replay must reproduce
// the forward bit for bit from different surroundings.
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }

// Type selection (A when B holds, else Bt) without the standard library,
// which NVRTC does not provide.
template <bool B, class A, class Bt> struct Pick { using type = A; };
template <class A, class Bt> struct Pick<false, A, Bt> { using type = Bt; };

__device__ __forceinline__ bool is_finite(float v) { return isfinite(v); }
__device__ __forceinline__ bool is_finite(double v) { return isfinite(v); }
__device__ __forceinline__ bool is_nan(float v) { return isnan(v); }
__device__ __forceinline__ bool is_nan(double v) { return isnan(v); }

__device__ __forceinline__ float sqrt_t(float v) { return sqrtf(v); }
__device__ __forceinline__ double sqrt_t(double v) { return sqrt(v); }
__device__ __forceinline__ float pow_t(float a, float b) { return powf(a, b); }
__device__ __forceinline__ double pow_t(double a, double b) { return pow(a, b); }
__device__ __forceinline__ float log2_t(float a) { return log2f(a); }
__device__ __forceinline__ double log2_t(double a) { return log2(a); }
__device__ __forceinline__ float exp2_t(float a) { return exp2f(a); }
__device__ __forceinline__ double exp2_t(double a) { return exp2(a); }

template <class T> struct Limits;
template <> struct Limits<float> {
    static __device__ __forceinline__ float huge() { return 3.4028234663852886e38f; }
    static __device__ __forceinline__ float eps() { return 1.1920928955078125e-07f; }
};
template <> struct Limits<double> {
    static __device__ __forceinline__ double huge() { return 1.7976931348623157e308; }
    static __device__ __forceinline__ double eps() { return 2.220446049250313e-16; }
};

// Compensated (Kahan) accumulation of a sum of terms in type T.
template <class T> struct Kahan {
    T sum, comp;
    __device__ __forceinline__ Kahan() : sum(T(0)), comp(T(0)) {}
    __device__ __forceinline__ void add(T term) {
        T y = term - comp;
        T s = sum + y;
        comp = (s - sum) - y;
        sum = s;
    }
};

}  // namespace cbx
