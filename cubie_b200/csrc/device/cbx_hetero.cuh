// One persistent launch over runs of several configurations ("families":
// different systems, algorithms, precisions, tolerances, outputs).  No
// counterpart in the reference, which compiles and launches one kernel per
// system.
//
// Global run r belongs to family k when first_run[k] <= r < first_run[k+1]
// and is run r - first_run[k] of that family's own cbx_solve_args (its own
// inputs, outputs and status words).  Every family has its own run counter
// (work_counter[k]).  A warp drains one family at a time with that family's
// persistent loop (lanes claim the family's next run the moment their run
// ends), then moves on to the next family that still has runs; warps start
// at different families (rotated by warp index) so all families progress
// together and the launch ends when the last family's runs are done.
// Within a family, claims follow its run_order when one is given (most
// estimated work first, as in the single-family persistent launch).  Each
// family's loop is its own function instantiation with its own loop state,
// value-initialised where it is declared: left uninitialised, its values
// entered each family's loop undefined, and the compiler kept them live
// across the loop over families, so the registers added up over the
// families (124 for the three of the mixed batch, against 47 to 56 for
// each alone).  Initialised, a lane needs about the most any one family
// needs (64).
#pragma once
#include "cbx_loop.cuh"

namespace cbx {

template <class Cfg>
__device__ __forceinline__ void drain_family(const cbx_solve_args& a, unsigned long long* counter, BlockTotals* bt) {
    Lane<Cfg> L{};
    bool active = false, exhausted = false;
    while (true) {
        if (!active && !exhausted) {
            const long long k = claim_run(counter);
            if (k < a.n_runs) {
                lane_begin<Cfg>(L, a, a.run_order ? a.run_order[k] : k);
                active = true;
            } else {
                exhausted = true;
            }
        }
        if (!__any_sync(0xffffffffu, active)) break;
        if (active) {
            if (lane_iterate<Cfg>(L, a)) {
                lane_end<Cfg>(L, a, bt);
                active = false;
            }
        }
    }
}

template <int I, class... Cs>
struct FamilyDispatch;

template <int I, class C0, class... Cs>
struct FamilyDispatch<I, C0, Cs...> {
    static __device__ __forceinline__ void drain(int f, const cbx_hetero_args& h, BlockTotals* bt) {
        if (f == I) {
            drain_family<C0>(h.family[I], h.work_counter + I, bt + I);
            return;
        }
        if constexpr (sizeof...(Cs) > 0) FamilyDispatch<I + 1, Cs...>::drain(f, h, bt);
    }
};

template <class... Cs>
__device__ __forceinline__ void run_hetero(const cbx_hetero_args& h) {
    constexpr int F = int(sizeof...(Cs));
    static_assert(F <= CBX_MAX_FAMILIES, "too many families for cbx_hetero_args");
    __shared__ BlockTotals bt[F];
#ifndef CBX_HOST_EMULATION
    if (threadIdx.x < 4 * F) bt[threadIdx.x / 4].v[threadIdx.x % 4] = 0ull;
    __syncthreads();
#endif
    const int warp = int((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    for (int j = 0; j < F; ++j) {
        const int f = (warp + j) % F;
        FamilyDispatch<0, Cs...>::drain(f, h, bt);
    }
#ifndef CBX_HOST_EMULATION
    __syncthreads();
    if (threadIdx.x < 4 * F) {
        const int k = threadIdx.x / 4, q = threadIdx.x % 4;
        unsigned long long* dst = nullptr;
#pragma unroll
        for (int j = 0; j < F; ++j)
            if (j == k) dst = h.family[j].totals;
        if (dst && bt[k].v[q]) atomicAdd(dst + q, bt[k].v[q]);
    }
#endif
}

template <class... Cs>
struct FamilyCount {
    static constexpr int value = int(sizeof...(Cs));
};

}  // namespace cbx

// The size of cbx_hetero_probe tells the host how many families the
// module was generated for.
#define CBX_DEFINE_HETERO_KERNEL(BLOCK, ...)                                                          \
    __constant__ char cbx_hetero_probe[cbx::FamilyCount<__VA_ARGS__>::value];                         \
    extern "C" __global__ void __launch_bounds__(BLOCK) cbx_integrate_hetero(cbx_hetero_args h) {    \
        cbx::run_hetero<__VA_ARGS__>(h);                                                              \
    }
