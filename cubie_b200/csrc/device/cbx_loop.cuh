// Per-system integration loop and the two kernels built on it.
//
// The loop follows IVPLoop.loop_fn (src/cubie/integrators/loops/ode_loop.py
// :493-984): event-clamped adaptive stepping with float64 time, saves at a
// regular cadence or at the end, summary updates every sample interval and
// summary writes every ``samples_per_summary`` updates, status folding
// only on irrecoverable failure, stagnation after two stale time values.
//
// The loop is written as a per-run state machine (``Lane``) advanced one
// step attempt at a time.  The plain kernel gives each thread one run; the
// persistent kernel keeps a grid of resident warps whose lanes claim the
// next unstarted run the moment their own run finishes, so a lane never
// idles while its warp-mates integrate long runs.
#pragma once
#include "cbx_common.cuh"
#include "cbx_args.h"
#include "cbx_steps.cuh"
#include "cbx_control.cuh"

namespace cbx {

template <class Cfg>
struct Lane {
    using R = typename Cfg::R;
    using C = typename Cfg::C;
    using Step = typename Cfg::Step;
    using Ctl = Controller<Cfg>;
    static constexpr int N = Cfg::N, NP = Cfg::NP, ND = Cfg::ND, NO = Cfg::NO;
    static constexpr int SBUF_S = Cfg::N_SUMM_STATES * Cfg::Summ::BUF;
    static constexpr int SBUF_O = Cfg::N_SUMM_OBS * Cfg::Summ::BUF;

    long long run;
    double t;
    C tp;
    C t_end;
    double save_stop, summary_stop;
    C dt, dt_raw;
    C next_save, next_update;
    C tol_scale;
    typename Cfg::G ctl_ts;   // tol_scale in the gain precision (the error norm's)
    R y[N];
    R comp[N];
    R p[NP > 0 ? NP : 1];
    R drv[ND > 0 ? ND : 1];
    R obs[NO > 0 ? NO : 1];
    R sbuf_s[SBUF_S > 0 ? SBUF_S : 1];
    R sbuf_o[SBUF_O > 0 ? SBUF_O : 1];
    int counters[4];
    int save_idx, summary_idx, update_idx;
    int status, iteration_status, stagnant;
    bool first_step, prev_accepted, irrecoverable;
    // per-run totals, 32-bit (a run of more than 2^32 attempted steps would
    // wrap them; the launch totals are 64-bit)
    unsigned steps, rejections, newton, krylov;
    typename Ctl::State ctl;
    typename Step::Persist ps;
};

template <class Cfg>
__device__ __forceinline__ void save_row(const Lane<Cfg>& L, const cbx_solve_args a) {
    using R = typename Cfg::R;
    const int row = L.save_idx;
    if (row >= a.n_save_rows) return;
    const long long s = a.run_stride;
    if constexpr (Cfg::SAVE_STATE || Cfg::SAVE_TIME) {
        constexpr int W = Cfg::N_SAVED_STATES + (Cfg::SAVE_TIME ? 1 : 0);
        R* out = static_cast<R*>(a.state_out) + (long long)row * W * s + L.run;
        if constexpr (Cfg::SAVE_STATE) {
#pragma unroll
            for (int k = 0; k < Cfg::N_SAVED_STATES; ++k) out[k * s] = L.y[Cfg::Idx::saved_state(k)];
        }
        if constexpr (Cfg::SAVE_TIME) out[Cfg::N_SAVED_STATES * s] = R(L.tp);
    }
    if constexpr (Cfg::SAVE_OBS) {
        R* out = static_cast<R*>(a.obs_out) + (long long)row * Cfg::N_SAVED_OBS * s + L.run;
#pragma unroll
        for (int k = 0; k < Cfg::N_SAVED_OBS; ++k) out[k * s] = L.obs[Cfg::Idx::saved_obs(k)];
    }
    if constexpr (Cfg::SAVE_COUNTERS) {
        int* out = a.counters_out + (long long)row * 4 * s + L.run;
#pragma unroll
        for (int k = 0; k < 4; ++k) out[k * s] = L.counters[k];
    }
}

template <class Cfg>
__device__ __forceinline__ void update_summaries(Lane<Cfg>& L) {
    using Summ = typename Cfg::Summ;
#pragma unroll
    for (int k = 0; k < Cfg::N_SUMM_STATES; ++k)
        Summ::update(L.y[Cfg::Idx::summ_state(k)], L.sbuf_s + k * Summ::BUF, L.update_idx);
#pragma unroll
    for (int k = 0; k < Cfg::N_SUMM_OBS; ++k)
        Summ::update(L.obs[Cfg::Idx::summ_obs(k)], L.sbuf_o + k * Summ::BUF, L.update_idx);
}

template <class Cfg>
__device__ __forceinline__ void save_summaries(Lane<Cfg>& L, const cbx_solve_args a) {
    using R = typename Cfg::R;
    using Summ = typename Cfg::Summ;
    const int row = L.summary_idx;
    const bool in_range = row < a.n_summary_rows;
    const long long s = a.run_stride;
    R vals[Summ::OUT > 0 ? Summ::OUT : 1];
#pragma unroll
    for (int k = 0; k < Cfg::N_SUMM_STATES; ++k) {
        Summ::save(L.sbuf_s + k * Summ::BUF, vals, Cfg::SAMPLES_PER_SUMMARY);
        if (in_range) {
            R* out = static_cast<R*>(a.state_sum_out) +
                     ((long long)row * Cfg::N_SUMM_STATES * Summ::OUT + k * Summ::OUT) * s + L.run;
#pragma unroll
            for (int q = 0; q < Summ::OUT; ++q) out[q * s] = vals[q];
        }
    }
#pragma unroll
    for (int k = 0; k < Cfg::N_SUMM_OBS; ++k) {
        Summ::save(L.sbuf_o + k * Summ::BUF, vals, Cfg::SAMPLES_PER_SUMMARY);
        if (in_range) {
            R* out = static_cast<R*>(a.obs_sum_out) +
                     ((long long)row * Cfg::N_SUMM_OBS * Summ::OUT + k * Summ::OUT) * s + L.run;
#pragma unroll
            for (int q = 0; q < Summ::OUT; ++q) out[q * s] = vals[q];
        }
    }
}

// Seed a run: load inputs, evaluate drivers and observables at t0, save the
// initial row and reset the summary buffers (ode_loop.py:560-703).
template <class Cfg>
__device__ __forceinline__ void lane_begin(Lane<Cfg>& L, const cbx_solve_args a, long long run) {
    using R = typename Cfg::R;
    using C = typename Cfg::C;
    using Step = typename Cfg::Step;
    constexpr int N = Cfg::N, NP = Cfg::NP, NO = Cfg::NO;
    L.run = run;
    const double duration = a.durations ? a.durations[run] : a.duration;
    L.tol_scale = a.tol_scale ? C(a.tol_scale[run]) : C(1);
    L.ctl_ts = typename Cfg::G(L.tol_scale);
    L.t = a.t0;
    L.tp = C(L.t);
    L.t_end = C(a.warmup + a.t0 + duration);
    if (a.durations) {
        L.save_stop = a.warmup + a.t0 + duration;
        L.summary_stop = a.warmup + a.t0 + duration;
    } else {
        L.save_stop = a.save_stop;
        L.summary_stop = a.summary_stop;
    }
    const R* inits = static_cast<const R*>(a.inits);
    const R* params = static_cast<const R*>(a.params);
#pragma unroll
    for (int k = 0; k < N; ++k) {
        L.y[k] = inits[k * a.run_stride + run];
        L.comp[k] = R(0);
    }
#pragma unroll
    for (int k = 0; k < NP; ++k) L.p[k] = params[k * a.run_stride + run];
#pragma unroll
    for (int k = 0; k < Lane<Cfg>::SBUF_S; ++k) L.sbuf_s[k] = R(0);
#pragma unroll
    for (int k = 0; k < Lane<Cfg>::SBUF_O; ++k) L.sbuf_o[k] = R(0);
    if constexpr (Cfg::ND > 0) Drivers<Cfg>::eval(R(L.tp), static_cast<const R*>(a.driver_coeffs), L.drv);
    if constexpr (NO > 0) Cfg::Sys::template observables<R>(L.y, L.p, L.drv, R(L.tp), L.obs);
    L.next_save = C(a.warmup + a.t0);
    L.next_update = C(a.warmup + a.t0);
    L.save_idx = 0;
    L.summary_idx = 0;
    L.update_idx = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) L.counters[k] = 0;
    if (a.warmup == 0.0) {
        if (Cfg::SAVE_REG) L.next_save = C(L.next_save + C(Cfg::SAVE_EVERY));
        if (Cfg::SUMM_REG) L.next_update = C(C(Cfg::SAMPLE_EVERY) + L.next_update);
        save_row<Cfg>(L, a);
        L.save_idx += 1;
        if (Cfg::SUMMARISE) save_summaries<Cfg>(L, a);
    }
    L.status = SUCCESS;
    L.iteration_status = 0;
    L.dt = C(Cfg::DT0);
    L.dt_raw = C(Cfg::DT0);
    L.stagnant = 0;
    L.first_step = true;
    L.prev_accepted = true;
    L.irrecoverable = false;
    L.steps = L.rejections = L.newton = L.krylov = 0;
    Controller<Cfg>::init(L.ctl);
    Step::init(L.ps);
}

// Accept a step's result: the state (compensated in the mixed-precision
// mode: y + (delta + carried rounding)) and the drivers at its end.
template <class Cfg>
__device__ __forceinline__ void commit_state(Lane<Cfg>& L, const typename Cfg::R* ynew,
                                             const typename Cfg::R* delta, const typename Cfg::R* drv_new) {
    using R = typename Cfg::R;
    constexpr int N = Cfg::N, ND = Cfg::ND;
    if (Cfg::MIXED) {
#pragma unroll
        for (int i = 0; i < N; ++i) {
            const R z = add_rn(delta[i], L.comp[i]);
            const R ys = L.y[i] + z;
            L.comp[i] = z - (ys - L.y[i]);
            L.y[i] = ys;
        }
    } else {
#pragma unroll
        for (int i = 0; i < N; ++i) L.y[i] = ynew[i];
    }
    if constexpr (ND > 0) {
#pragma unroll
        for (int q = 0; q < ND; ++q) L.drv[q] = drv_new[q];
    }
}

// Observer of accepted steps (the adjoint's segment recorder); the default
// observes nothing and compiles away.
struct NoHook {
    static constexpr bool ACTIVE = false;
};

// One pass of the main loop body.  Returns true when the run is finished.
// ``hook->accepted(L, dt_eff, row)`` sees every accepted step before the
// state is updated: ``L`` still holds the step's start (state, time, and the
// first-step and previous-attempt flags the step function received),
// ``dt_eff`` is the step size in the control precision (the step function
// received it rounded to the system precision), ``row`` the output row saved
// at its end (-1 if none).
template <class Cfg, class Hook = NoHook>
__device__ __forceinline__ bool lane_iterate(Lane<Cfg>& L, const cbx_solve_args a, Hook* hook = nullptr) {
    using R = typename Cfg::R;
    using C = typename Cfg::C;
    using Step = typename Cfg::Step;
    constexpr int N = Cfg::N, ND = Cfg::ND, NO = Cfg::NO;

    const C end_of_step = L.tp + L.dt_raw;
    bool finished;
    bool save_finished = false, summary_finished = false, at_end = false;
    if (Cfg::SAVE_REG || Cfg::SUMM_REG) {
        finished = true;
        if (Cfg::SAVE_REG) {
            save_finished = double(L.next_save) > L.save_stop;
            finished = finished && save_finished;
        }
        if (Cfg::SUMM_REG) {
            summary_finished = double(L.next_update) > L.summary_stop;
            finished = finished && summary_finished;
        }
    } else {
        finished = end_of_step >= L.t_end;
    }
    if (Cfg::SAVE_LAST) {
        at_end = (L.tp < L.t_end) && finished;
        finished = finished && !at_end;
    }
    finished = finished || L.irrecoverable;
    if (finished) return true;
    // Step budget and host abort request end the run with status bit 32
    // (reserved but unused in the reference, result_codes.py:57).  Written
    // as direct returns: folding them into ``irrecoverable`` ahead of the
    // finish test made NVRTC's optimiser drop the event clamp below.
    if (a.max_steps > 0 && (long long)L.steps >= a.max_steps) {
        L.status |= MAX_LOOP_ITERS_EXCEEDED;
        return true;
    }
    if (a.abort_flag && (L.steps & 255) == 0 && *a.abort_flag) {
        L.status |= MAX_LOOP_ITERS_EXCEEDED;
        return true;
    }

    bool do_save = Cfg::SAVE_REG ? ((end_of_step >= L.next_save) && !save_finished) : false;
    bool do_update = Cfg::SUMM_REG ? ((end_of_step >= L.next_update) && !summary_finished) : false;
    if (Cfg::SAVE_LAST) do_save = do_save || at_end;

    C dt_eff = L.dt_raw;
    bool truncated = false;
    if (do_save || do_update) {
        C next_event = L.t_end;
        if (do_save && Cfg::SAVE_REG) next_event = C(pymin(next_event, L.next_save));
        if (do_update && Cfg::SUMM_REG) next_event = C(pymin(next_event, L.next_update));
        const C gap = C(next_event - L.tp);
        dt_eff = gap > C(0) ? gap : L.dt_raw;
        truncated = dt_eff != L.dt_raw;
    }

    R ynew[N], delta[N], err[N];
    R drv_new[ND > 0 ? ND : 1];
    StepCtx<Cfg> ctx{L.p, static_cast<const R*>(a.driver_coeffs), L.tol_scale};
    Iters its;
    const int step_status = Step::step(ctx, L.y, ynew, delta, err, L.drv, drv_new, R(dt_eff), R(L.tp),
                                       L.first_step, L.prev_accepted, L.ps, its);
    // Rosenbrock steps report no Newton iterations: a constant here lets the
    // controller's iteration-dependent factor fold away
    const int nit = Cfg::ALGO == ALGO_ROSENBROCK ? 0 : its.nit, kit = its.kit;
    L.first_step = false;
    L.iteration_status |= step_status;
    const bool step_failed = step_status != SUCCESS;
    L.irrecoverable = L.irrecoverable || (!Cfg::ADAPTIVE && step_failed);
    if (step_failed) {
#pragma unroll
        for (int i = 0; i < N; ++i) err[i] = R(1e16);
    }
    bool accept;
    if constexpr (Cfg::ADAPTIVE) {
        bool ctl_accept = false;
        const int ctl_status =
            Controller<Cfg>::update(L.dt, ynew, L.y, err, nit, truncated, ctl_accept, L.ctl, L.ctl_ts);
        accept = ctl_accept && !step_failed;
        L.iteration_status |= ctl_status;
        L.irrecoverable = L.irrecoverable || ((ctl_status & STEP_TOO_SMALL) != 0);
    } else {
        accept = !step_failed;
    }
    L.dt_raw = L.dt;
    if (Cfg::SAVE_COUNTERS) {
        L.counters[0] += nit;
        L.counters[1] += kit;
        L.counters[2] += 1;
        if (!accept) L.counters[3] += 1;
    }
    L.steps += 1;
    L.rejections += accept ? 0 : 1;
    L.newton += its.nit_all;
    L.krylov += its.kit_all;

    const double t_proposal = L.t + double(dt_eff);
    L.stagnant = (t_proposal == L.t) ? L.stagnant + 1 : 0;
    const bool stagnant = L.stagnant >= 2;
    if (stagnant) L.iteration_status |= STAGNATION;
    L.irrecoverable = L.irrecoverable || stagnant;
    if (L.irrecoverable) L.status |= L.iteration_status;
    if (accept) L.iteration_status = 0;
    if (accept) {
        if constexpr (Hook::ACTIVE) hook->accepted(L, dt_eff, do_save ? L.save_idx : -1);
        L.t = t_proposal;
        L.tp = C(L.t);
        commit_state<Cfg>(L, ynew, delta, drv_new);
        if constexpr (NO > 0) Cfg::Sys::template observables<R>(L.y, L.p, L.drv, R(L.tp), L.obs);
    }
    L.prev_accepted = accept;
    do_save = do_save && accept;
    do_update = do_update && accept;
    if (do_save) {
        if (Cfg::SAVE_REG) L.next_save += C(Cfg::SAVE_EVERY);
        save_row<Cfg>(L, a);
        L.save_idx += 1;
        if (Cfg::SAVE_COUNTERS) {
#pragma unroll
            for (int k = 0; k < 4; ++k) L.counters[k] = 0;
        }
    }
    if (do_update) {
        if (Cfg::SUMM_REG) L.next_update += C(Cfg::SAMPLE_EVERY);
        if (Cfg::SUMMARISE) {
            update_summaries<Cfg>(L);
            L.update_idx += 1;
            if (L.update_idx % Cfg::SAMPLES_PER_SUMMARY == 0) {
                save_summaries<Cfg>(L, a);
                L.summary_idx += 1;
            }
        }
    }
    return false;
}

struct BlockTotals {
    unsigned long long v[4];
};

template <class Cfg>
__device__ __forceinline__ void lane_end(const Lane<Cfg>& L, const cbx_solve_args a, BlockTotals* bt) {
    a.status_out[L.run] = L.status;
    if (a.totals) {
#ifdef CBX_HOST_EMULATION
        // one emulated thread at a time: no block-level staging
        unsigned long long* dst = a.totals;
#else
        unsigned long long* dst = bt->v;
#endif
        atomicAdd(dst + 0, (unsigned long long)L.steps);
        atomicAdd(dst + 1, (unsigned long long)L.rejections);
        atomicAdd(dst + 2, (unsigned long long)L.newton);
        atomicAdd(dst + 3, (unsigned long long)L.krylov);
    }
}

__device__ __forceinline__ void totals_begin(BlockTotals* bt) {
#ifndef CBX_HOST_EMULATION
    if (threadIdx.x < 4) bt->v[threadIdx.x] = 0ull;
    __syncthreads();
#endif
}

__device__ __forceinline__ void totals_flush(BlockTotals* bt, const cbx_solve_args a) {
#ifndef CBX_HOST_EMULATION
    __syncthreads();
    if (a.totals && threadIdx.x < 4 && bt->v[threadIdx.x]) atomicAdd(a.totals + threadIdx.x, bt->v[threadIdx.x]);
#endif
}

// Plain kernel: one thread integrates one run to completion
// (BatchSolverKernel.py:947-998).
template <class Cfg>
__device__ __forceinline__ void run_plain(const cbx_solve_args a) {
    __shared__ BlockTotals bt;
    totals_begin(&bt);
    const long long run = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (run < a.n_runs) {
        Lane<Cfg> L;
        lane_begin<Cfg>(L, a, run);
        while (!lane_iterate<Cfg>(L, a)) {
        }
        lane_end<Cfg>(L, a, &bt);
    }
    totals_flush(&bt, a);
}

// Claim the next run for every lane of the calling (converged) subset with
// one atomic per warp.
__device__ __forceinline__ long long claim_run(unsigned long long* counter) {
    const unsigned mask = __activemask();
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    const int rank = __popc(mask & ((1u << lane) - 1u));
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(counter, (unsigned long long)__popc(mask));
    base = __shfl_sync(mask, base, leader);
    return (long long)(base + rank);
}

// Persistent work-stealing kernel: resident warps loop until the run
// counter is exhausted; a lane whose run finishes claims a new one at the
// top of the next iteration.  Claims follow ``run_order`` when given (the
// host orders runs longest first, so the last claims are the short runs
// and warps do not idle behind a few long ones at the end).  blockDim.x
// must be a multiple of 32.
template <class Cfg>
__device__ __forceinline__ void run_persistent(const cbx_solve_args a) {
    __shared__ BlockTotals bt;
    totals_begin(&bt);
    Lane<Cfg> L;
    bool active = false, exhausted = false;
    while (true) {
        if (!active && !exhausted) {
            const long long k = claim_run(a.work_counter);
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
                lane_end<Cfg>(L, a, &bt);
                active = false;
            }
        }
    }
    totals_flush(&bt, a);
}

}  // namespace cbx

// Launch bounds: the block size, plus a minimum of resident blocks per SM
// when the configuration asks for one (which caps registers per thread).
#ifndef CBX_LAUNCH_BOUNDS
#define CBX_LAUNCH_BOUNDS(CFG) __launch_bounds__(CFG::BLOCK)
#endif

#define CBX_DEFINE_KERNELS(CFG)                                                                     \
    extern "C" __global__ void CBX_LAUNCH_BOUNDS(CFG) cbx_integrate_plain(cbx_solve_args a) { \
        cbx::run_plain<CFG>(a);                                                                     \
    }                                                                                               \
    extern "C" __global__ void CBX_LAUNCH_BOUNDS(CFG) cbx_integrate_persistent(cbx_solve_args a) { \
        cbx::run_persistent<CFG>(a);                                                                \
    }
