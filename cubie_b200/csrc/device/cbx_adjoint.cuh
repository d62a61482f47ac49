// Discrete adjoint of the integration: gradients of a loss on the saved
// state rows with respect to every run's initial state and parameters.
//
// The reference has no adjoint.  The method differentiates the discrete map
// the forward integration applied, with the accepted step sizes held fixed
// (rejected attempts and the controller do not enter the map):
//
//   forward   ``cbx_adjoint_forward`` integrates exactly as the persistent
//             kernel does and additionally stores the complete per-run loop
//             state (``Lane``) every ``ckpt_every`` accepted steps;
//   reverse   ``cbx_adjoint_backward`` walks each run's checkpoints from
//             last to first.  From checkpoint s it replays the loop (same
//             code, same arithmetic, hence the same accepted steps) and
//             records the start state, start time and size of the next
//             ``ckpt_every`` accepted steps, then back-propagates
//             lambda = dL/dy through those steps in reverse order, adding
//             dL/d(saved row) where a row was saved.  Parameter gradients
//             accumulate in the control precision.
//
// Step adjoints:
//   ERK         y+ = y + h sum_i b_i k_i, k_i = f(Y_i), Y_i = y + h sum_j a_ij k_j
//               kbar_i = h (b_i lambda + sum_{j>i} a_ji Ybar_j), Ybar_i = J(Y_i)^T kbar_i,
//               ybar = lambda + sum_i Ybar_i, pbar += sum_i (df/dp)(Y_i)^T kbar_i.
//   Rosenbrock  (I - gamma h J) K_s = gamma h (f(Y_s) + sum_j C_sj K_j / h),
//               Y_s = y + sum_j a_sj K_j, J = J(y) (autonomous systems):
//               rbar_s = (I - gamma h J)^-T Kbar_s (transposed Krylov solve),
//               f(Y_s) gets gamma h rbar_s, K_j gets gamma C_sj rbar_s and
//               a_sj Ybar_s, and J(y) gets gamma h rbar_s K_s^T, which reaches
//               y and p through the generated second-derivative contractions
//               grad_y (v^T J(y) w) and grad_p (v^T J(y) w).
#pragma once
#include "cbx_loop.cuh"

namespace cbx {

// A checkpoint is the raw image of the per-run loop state, padded to whole
// 16-byte vectors and moved with 16-byte accesses.
template <class Cfg>
struct LaneImage {
    static constexpr int VECS = int((sizeof(Lane<Cfg>) + 15) / 16);
    static constexpr int WORDS = VECS * 4;
};

template <class Cfg>
__device__ __forceinline__ void store_lane(const Lane<Cfg>& L, unsigned* dst) {
    unsigned buf[LaneImage<Cfg>::WORDS];
    buf[LaneImage<Cfg>::WORDS - 1] = 0u;
    buf[LaneImage<Cfg>::WORDS - 2] = 0u;
    buf[LaneImage<Cfg>::WORDS - 3] = 0u;
    memcpy(buf, &L, sizeof(Lane<Cfg>));
#pragma unroll
    for (int k = 0; k < LaneImage<Cfg>::VECS; ++k)
        reinterpret_cast<uint4*>(dst)[k] = make_uint4(buf[4 * k], buf[4 * k + 1], buf[4 * k + 2], buf[4 * k + 3]);
}

template <class Cfg>
__device__ __forceinline__ void load_lane(Lane<Cfg>& L, const unsigned* src) {
    unsigned buf[LaneImage<Cfg>::WORDS];
#pragma unroll
    for (int k = 0; k < LaneImage<Cfg>::VECS; ++k) {
        const uint4 v = reinterpret_cast<const uint4*>(src)[k];
        buf[4 * k] = v.x;
        buf[4 * k + 1] = v.y;
        buf[4 * k + 2] = v.z;
        buf[4 * k + 3] = v.w;
    }
    memcpy(&L, buf, sizeof(Lane<Cfg>));
}

// One replayed step is one record of ``SegRecord<Cfg>::F`` values of the
// system precision, contiguous per run, ``[run][step][F]``: the start state,
// the start time, the step size and the saved output row (-1 if none; exact
// as a floating value), padded to whole 16-byte vectors.  Lanes of a warp are
// at different steps of different runs, so a record per lane moved with
// 16-byte vector accesses costs one or two sectors per lane per step.
template <class Cfg>
struct SegRecord {
    using R = typename Cfg::R;
    static constexpr int V = int(16 / sizeof(R));
    static constexpr int F = ((Cfg::N + 3 + V - 1) / V) * V;
    static __device__ __forceinline__ void store(R* dst, const R* rec) {
        if constexpr (sizeof(R) == 4) {
#pragma unroll
            for (int k = 0; k < F; k += 4)
                *reinterpret_cast<float4*>(dst + k) = make_float4(rec[k], rec[k + 1], rec[k + 2], rec[k + 3]);
        } else {
#pragma unroll
            for (int k = 0; k < F; k += 2)
                *reinterpret_cast<double2*>(dst + k) = make_double2(rec[k], rec[k + 1]);
        }
    }
    static __device__ __forceinline__ void load(const R* src, R* rec) {
        if constexpr (sizeof(R) == 4) {
#pragma unroll
            for (int k = 0; k < F; k += 4) {
                const float4 v = *reinterpret_cast<const float4*>(src + k);
                rec[k] = v.x;
                rec[k + 1] = v.y;
                rec[k + 2] = v.z;
                rec[k + 3] = v.w;
            }
        } else {
#pragma unroll
            for (int k = 0; k < F; k += 2) {
                const double2 v = *reinterpret_cast<const double2*>(src + k);
                rec[k] = v.x;
                rec[k + 1] = v.y;
            }
        }
    }
};

// Records the accepted steps of one replayed segment.
template <class Cfg>
struct SegRecorder {
    using R = typename Cfg::R;
    static constexpr bool ACTIVE = true;
    static constexpr int F = SegRecord<Cfg>::F;
    R* seg;        // this run's records
    int count;
    __device__ __forceinline__ void accepted(const Lane<Cfg>& L, R t, R h, int row) {
        R rec[F];
#pragma unroll
        for (int k = 0; k < Cfg::N; ++k) rec[k] = L.y[k];
        rec[Cfg::N] = t;
        rec[Cfg::N + 1] = h;
        rec[Cfg::N + 2] = R(row);
#pragma unroll
        for (int k = Cfg::N + 3; k < F; ++k) rec[k] = R(0);
        SegRecord<Cfg>::store(seg + (long long)count * F, rec);
        ++count;
    }
};

// ---------------------------------------------------------------------------
// Explicit Runge-Kutta step adjoint.
// ---------------------------------------------------------------------------
template <class Cfg>
struct ErkAdjoint {
    using R = typename Cfg::R;
    using C = typename Cfg::C;
    using Sys = typename Cfg::Sys;
    using Tab = typename Cfg::Tab;
    static constexpr int N = Cfg::N, S = Cfg::S, NP = Cfg::NP, ND = Cfg::ND;

    // Stage i influences y+ when b_i != 0 or a later stage reads it.
    static __host__ __device__ constexpr bool stage_used(int i) {
        bool used = Tab::b(i) != 0.0;
        for (int j = i + 1; j < S; ++j) used = used || (Tab::a(j, i) != 0.0);
        return used;
    }

    static __device__ __forceinline__ void reverse(const StepCtx<Cfg>& ctx, const R* y, R t, R h, R* lam,
                                                   C* pbar) {
        R Y[S][N];
        R k[S][N];
        R drv_stage[ND > 0 ? ND : 1];
#pragma unroll
        for (int i = 0; i < S; ++i) {
            if (!stage_used(i)) continue;
            const R stage_time = t + h * R(Tab::c(i));
#pragma unroll
            for (int q = 0; q < N; ++q) {
                R acc = R(0);
#pragma unroll
                for (int j = 0; j < S; ++j)
                    if (j < i && Tab::a(i, j) != 0.0) acc += R(Tab::a(i, j)) * k[j][q];
                Y[i][q] = (i == 0) ? y[q] : acc * h + y[q];
            }
            if constexpr (ND > 0) Drivers<Cfg>::eval(stage_time, ctx.coeffs, drv_stage);
            bool feeds_later = false;
#pragma unroll
            for (int j = 0; j < S; ++j)
                if (j > i && Tab::a(j, i) != 0.0) feeds_later = true;
            if (feeds_later) Sys::template dxdt<R>(Y[i], ctx.p, drv_stage, stage_time, k[i]);
        }
        R Ybar[S][N];
        R lam_out[N];
#pragma unroll
        for (int q = 0; q < N; ++q) lam_out[q] = lam[q];
#pragma unroll
        for (int i = S - 1; i >= 0; --i) {
            if (!stage_used(i)) continue;
            R kbar[N];
#pragma unroll
            for (int q = 0; q < N; ++q) {
                R acc = R(Tab::b(i)) * lam[q];
#pragma unroll
                for (int j = 0; j < S; ++j)
                    if (j > i && Tab::a(j, i) != 0.0 && stage_used(j)) acc += R(Tab::a(j, i)) * Ybar[j][q];
                kbar[q] = h * acc;
            }
            const R stage_time = t + h * R(Tab::c(i));
            if constexpr (ND > 0) Drivers<Cfg>::eval(stage_time, ctx.coeffs, drv_stage);
            R J[Sys::NJ];
            Sys::template jac<R>(Y[i], ctx.p, drv_stage, stage_time, J);
            Sys::template jtmv<R>(J, kbar, Ybar[i]);
#pragma unroll
            for (int q = 0; q < N; ++q) lam_out[q] += Ybar[i][q];
            if constexpr (NP > 0) {
                R P[Sys::NPJ > 0 ? Sys::NPJ : 1];
                R pb[NP];
                Sys::template pjac<R>(Y[i], ctx.p, drv_stage, stage_time, P);
                Sys::template ptmv<R>(P, kbar, pb);
#pragma unroll
                for (int q = 0; q < NP; ++q) pbar[q] += C(pb[q]);
            }
        }
#pragma unroll
        for (int q = 0; q < N; ++q) lam[q] = lam_out[q];
    }
};

// ---------------------------------------------------------------------------
// Rosenbrock-W step adjoint (autonomous systems without drivers).
// ---------------------------------------------------------------------------
// A^T v = v - s J^T v and its truncated Neumann preconditioner, with the
// tolerance weights of the forward operator.
template <class Cfg>
struct TransposedStageOp {
    using R = typename Cfg::R;
    using C = typename Cfg::C;
    using Sys = typename Cfg::Sys;
    static constexpr int K = Cfg::N;
    const R* J;
    R s;
    const R* ref;
    C scale;
    __device__ __forceinline__ void apply(const R* v, R* out) const {
        R jv[K];
        Sys::template jtmv<R>(J, v, jv);
#pragma unroll
        for (int i = 0; i < K; ++i) out[i] = v[i] - s * jv[i];
    }
    __device__ __forceinline__ void precond(const R* v, R* out, R* scratch) const {
#pragma unroll
        for (int i = 0; i < K; ++i) out[i] = v[i];
#pragma unroll 1
        for (int k = 0; k < Cfg::PRECOND_ORDER; ++k) {
            Sys::template jtmv<R>(J, out, scratch);
#pragma unroll
            for (int i = 0; i < K; ++i) out[i] = v[i] + s * scratch[i];
        }
    }
    __device__ __forceinline__ C tol(int i) const { return krylov_tol<Cfg>(i, ref[i], scale); }
    __device__ __forceinline__ C wnorm2(const R* v) const { return weighted_norm2<Cfg, K>(v, ref, scale); }
    template <class T> __device__ __forceinline__ T reduce(T partial) const { return partial; }
    static constexpr int KT = K;
};

template <class Cfg>
struct RosenbrockAdjoint {
    using R = typename Cfg::R;
    using C = typename Cfg::C;
    using Sys = typename Cfg::Sys;
    using Tab = typename Cfg::Tab;
    static constexpr int N = Cfg::N, S = Cfg::S, NP = Cfg::NP, ND = Cfg::ND;

    static __device__ __forceinline__ void reverse(const StepCtx<Cfg>& ctx, const R* y, R t, R h, R* lam,
                                                   C* pbar) {
        const R gamma = R(Tab::GAMMA);
        const R inv_dt = R(1) / h;
        const R* drv = nullptr;  // no drivers on this path
        R J[Sys::NJ];
        Sys::template jac<R>(y, ctx.p, drv, t, J);
        // Recompute the stage increments as the forward step did.
        R K[S][N], Y[S][N];
        SingleStageOp<Cfg> op{J, gamma * h, y, ctx.tol_scale};
        R guess[N];
#pragma unroll
        for (int i = 0; i < N; ++i) guess[i] = R(0);
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const R stage_time = t + h * R(Tab::c(s));
            R corr[N], f[N], rhs[N];
#pragma unroll
            for (int i = 0; i < N; ++i) {
                R v = y[i], c = R(0);
#pragma unroll
                for (int j = 0; j < S; ++j) {
                    if (j < s && Tab::a(s, j) != 0.0) v += R(Tab::a(s, j)) * K[j][i];
                    if (j < s && Tab::Cm(s, j) != 0.0) c += R(Tab::Cm(s, j)) * K[j][i];
                }
                Y[s][i] = v;
                corr[i] = c;
            }
            Sys::template dxdt<R>(Y[s], ctx.p, drv, stage_time, f);
#pragma unroll
            for (int i = 0; i < N; ++i) {
                const R rv = (s > 0) ? f[i] + corr[i] * inv_dt : f[i];
                rhs[i] = rv * h * gamma;
            }
            int it = 0;
            linear_solve<Cfg>(op, rhs, guess, it);
#pragma unroll
            for (int i = 0; i < N; ++i) K[s][i] = guess[i];
        }
        // Reverse through the stages.
        R Kbar[S][N], rbar[S][N], ybar[N];
#pragma unroll
        for (int s = 0; s < S; ++s)
#pragma unroll
            for (int i = 0; i < N; ++i) Kbar[s][i] = R(Tab::b(s)) * lam[i];
#pragma unroll
        for (int i = 0; i < N; ++i) ybar[i] = lam[i];
        TransposedStageOp<Cfg> opT{J, gamma * h, y, ctx.tol_scale};
#pragma unroll
        for (int s = S - 1; s >= 0; --s) {
            R rhs[N];
#pragma unroll
            for (int i = 0; i < N; ++i) {
                rhs[i] = Kbar[s][i];
                rbar[s][i] = R(0);
            }
            int it = 0;
            linear_solve<Cfg>(opT, rhs, rbar[s], it);
            R fbar[N], Ybar[N];
#pragma unroll
            for (int i = 0; i < N; ++i) fbar[i] = h * gamma * rbar[s][i];
            const R stage_time = t + h * R(Tab::c(s));
            if (s == 0) {
                Sys::template jtmv<R>(J, fbar, Ybar);
            } else {
                R Js[Sys::NJ];
                Sys::template jac<R>(Y[s], ctx.p, drv, stage_time, Js);
                Sys::template jtmv<R>(Js, fbar, Ybar);
            }
            if constexpr (NP > 0) {
                R P[Sys::NPJ > 0 ? Sys::NPJ : 1];
                R pb[NP];
                Sys::template pjac<R>(Y[s], ctx.p, drv, stage_time, P);
                Sys::template ptmv<R>(P, fbar, pb);
#pragma unroll
                for (int q = 0; q < NP; ++q) pbar[q] += C(pb[q]);
            }
#pragma unroll
            for (int i = 0; i < N; ++i) {
                ybar[i] += Ybar[i];
#pragma unroll
                for (int j = 0; j < S; ++j) {
                    if (j < s && Tab::a(s, j) != 0.0) Kbar[j][i] += R(Tab::a(s, j)) * Ybar[i];
                    if (j < s && Tab::Cm(s, j) != 0.0) Kbar[j][i] += gamma * R(Tab::Cm(s, j)) * rbar[s][i];
                }
            }
        }
        // J(y) enters every stage matrix: Jbar = gamma h sum_s rbar_s K_s^T.
#pragma unroll
        for (int s = 0; s < S; ++s) {
            R gy[N];
            Sys::template hvpy<R>(y, ctx.p, drv, t, K[s], rbar[s], gy);
#pragma unroll
            for (int i = 0; i < N; ++i) ybar[i] += gamma * h * gy[i];
            if constexpr (NP > 0) {
                R gp[NP];
                Sys::template hvpp<R>(y, ctx.p, drv, t, K[s], rbar[s], gp);
#pragma unroll
                for (int q = 0; q < NP; ++q) pbar[q] += C(gamma * h * gp[q]);
            }
        }
#pragma unroll
        for (int i = 0; i < N; ++i) lam[i] = ybar[i];
    }
};

template <class Cfg, int ALGO>
struct StepAdjoint;
template <class Cfg>
struct StepAdjoint<Cfg, ALGO_ERK> : ErkAdjoint<Cfg> {};
template <class Cfg>
struct StepAdjoint<Cfg, ALGO_ROSENBROCK> : RosenbrockAdjoint<Cfg> {};

// Forward integration with checkpoints (persistent work stealing, as
// run_persistent).  A run that needs more than ``max_ckpts`` checkpoints
// stops with status bit 32, like an exhausted step budget.
template <class Cfg>
__device__ __forceinline__ void run_adjoint_forward(const cbx_solve_args a, const cbx_adjoint_args g) {
    __shared__ BlockTotals bt;
    totals_begin(&bt);
    Lane<Cfg> L;
    bool active = false, exhausted = false;
    int nck = 0;
    long long next_ck = 0;
    constexpr int W = LaneImage<Cfg>::WORDS;
    while (true) {
        if (!active && !exhausted) {
            const long long run = claim_run(a.work_counter);
            if (run < a.n_runs) {
                lane_begin<Cfg>(L, a, run);
                active = true;
                nck = 0;
                next_ck = 0;
            } else {
                exhausted = true;
            }
        }
        if (!__any_sync(0xffffffffu, active)) break;
        if (active) {
            bool done = false;
            if (L.steps - L.rejections == next_ck) {
                if (nck < g.max_ckpts) {
                    store_lane<Cfg>(L, static_cast<unsigned*>(g.ckpt) + (L.run * g.max_ckpts + nck) * (long long)W);
                    ++nck;
                    next_ck += g.ckpt_every;
                } else {
                    L.status |= MAX_LOOP_ITERS_EXCEEDED;
                    done = true;
                }
            }
            if (!done) done = lane_iterate<Cfg>(L, a);
            if (done) {
                lane_end<Cfg>(L, a, &bt);
                g.ckpt_count[L.run] = nck;
                active = false;
            }
        }
    }
    totals_flush(&bt, a);
}

template <class Cfg>
__device__ __forceinline__ void add_row_grad(typename Cfg::R* lam, const cbx_solve_args a,
                                             const cbx_adjoint_args g, int row, long long run) {
    using R = typename Cfg::R;
    if (row < 0 || row >= a.n_save_rows || !g.grad_state) return;
    if constexpr (Cfg::SAVE_STATE) {
        constexpr int W = Cfg::N_SAVED_STATES + (Cfg::SAVE_TIME ? 1 : 0);
        const R* gr = static_cast<const R*>(g.grad_state) + (long long)row * W * a.run_stride + run;
#pragma unroll
        for (int k = 0; k < Cfg::N_SAVED_STATES; ++k) lam[Cfg::Idx::saved_state(k)] += gr[k * a.run_stride];
    }
}

// Reverse sweep.  Every lane works on its own run, but a warp moves through
// the phases together: all lanes replay their current segment (each until it
// holds ``ckpt_every`` records or its run ends), then all lanes
// back-propagate through their records, then each lane steps back to its
// previous checkpoint or, when its run is done, writes the gradients and
// claims the next run.  Phases are warp-uniform, so the replay and the
// reverse code never diverge against each other; lanes wait only for the
// longest segment of the warp.
template <class Cfg>
__device__ __forceinline__ void run_adjoint_backward(const cbx_solve_args a, const cbx_adjoint_args g) {
    using R = typename Cfg::R;
    using C = typename Cfg::C;
    using Adj = StepAdjoint<Cfg, Cfg::ALGO>;
    constexpr int N = Cfg::N, NP = Cfg::NP, F = SegRecord<Cfg>::F;
    constexpr int W = LaneImage<Cfg>::WORDS;
    constexpr unsigned FULL = 0xffffffffu;
    const long long s = a.run_stride;
    cbx_solve_args replay = a;
    replay.n_save_rows = 0;      // the replay writes no outputs
    replay.n_summary_rows = 0;
    R* seg = static_cast<R*>(g.seg);
    const unsigned* ckpt = static_cast<const unsigned*>(g.ckpt);
    Lane<Cfg> L;
    SegRecorder<Cfg> rec{seg, 0};
    R lam[N];
    C pbar[NP > 0 ? NP : 1];
    long long run = -1;
    int ck = -1;              // checkpoint of the segment in hand; -1: no run
    bool exhausted = false;
    while (true) {
        if (ck < 0 && !exhausted) {
            run = claim_run(a.work_counter);
            if (run < a.n_runs) {
#pragma unroll
                for (int q = 0; q < N; ++q) lam[q] = R(0);
#pragma unroll
                for (int q = 0; q < (NP > 0 ? NP : 1); ++q) pbar[q] = C(0);
                ck = g.ckpt_count[run] - 1;
                if (ck >= 0) load_lane<Cfg>(L, ckpt + (run * g.max_ckpts + ck) * (long long)W);
                rec.seg = seg + run * (long long)g.ckpt_every * F;
                rec.count = 0;
            } else {
                exhausted = true;
            }
        }
        const bool busy = ck >= 0;
        if (!__any_sync(FULL, busy)) break;
        // replay
        bool replaying = busy;
        while (__any_sync(FULL, replaying)) {
            if (replaying) {
                const bool done = lane_iterate<Cfg, SegRecorder<Cfg>>(L, replay, &rec);
                if (done || rec.count >= g.ckpt_every) replaying = false;
            }
        }
        // reverse
        int j = busy ? rec.count - 1 : -1;
        while (__any_sync(FULL, j >= 0)) {
            if (j >= 0) {
                R rec_j[F];
                SegRecord<Cfg>::load(rec.seg + (long long)j * F, rec_j);
                add_row_grad<Cfg>(lam, a, g, int(rec_j[N + 2]), run);
                StepCtx<Cfg> ctx{L.p, static_cast<const R*>(a.driver_coeffs), L.tol_scale};
                Adj::reverse(ctx, rec_j, rec_j[N], rec_j[N + 1], lam, pbar);
                --j;
            }
        }
        // previous checkpoint, or finish the run
        if (busy) {
            if (ck > 0) {
                --ck;
                load_lane<Cfg>(L, ckpt + (run * g.max_ckpts + ck) * (long long)W);
                rec.count = 0;
            } else {
                if (a.warmup == 0.0) add_row_grad<Cfg>(lam, a, g, 0, run);
                R* gi = static_cast<R*>(g.grad_inits);
#pragma unroll
                for (int q = 0; q < N; ++q) gi[q * s + run] = lam[q];
                if constexpr (NP > 0) {
                    R* gp = static_cast<R*>(g.grad_params);
                    if (gp) {
#pragma unroll
                        for (int q = 0; q < NP; ++q) gp[q * s + run] = R(pbar[q]);
                    }
                }
                ck = -1;
            }
        }
    }
}

}  // namespace cbx

#define CBX_DEFINE_ADJOINT_KERNELS(CFG)                                                              \
    __constant__ char cbx_lane_probe[4 * cbx::LaneImage<CFG>::WORDS];                                         \
    __constant__ char cbx_seg_record_probe[sizeof(CFG::R) * cbx::SegRecord<CFG>::F];         \
    extern "C" __global__ void CBX_LAUNCH_BOUNDS(CFG) cbx_adjoint_forward(cbx_solve_args a,           \
                                                                         cbx_adjoint_args g) {       \
        cbx::run_adjoint_forward<CFG>(a, g);                                                          \
    }                                                                                                 \
    extern "C" __global__ void CBX_LAUNCH_BOUNDS(CFG) cbx_adjoint_backward(cbx_solve_args a,          \
                                                                          cbx_adjoint_args g) {      \
        cbx::run_adjoint_backward<CFG>(a, g);                                                         \
    }
