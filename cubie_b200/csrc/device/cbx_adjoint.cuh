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
//             last to first.  From checkpoint s it replays the next
//             ``ckpt_every`` accepted steps bit for bit (explicit tableaus:
//             the step function driven by the forward's step-size tape;
//             Rosenbrock: the whole loop) and records each step's start
//             state, start time and size, then back-propagates
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
// the start time (only when the right-hand side depends on time, directly or
// through drivers) and the step size, negated when the step ends on a saved
// output row, padded to whole 16-byte vectors.  Saved rows are consecutive,
// so the reverse sweep recovers each row index by counting down from the
// row count at the segment's end.  Lanes of a warp are at different steps
// of different runs, so a record per lane moved with 16-byte vector
// accesses costs one sector per lane per step for systems of up to three
// states; the records of all resident lanes then stay within L2.
template <class Cfg>
struct SegRecord {
    using R = typename Cfg::R;
    static constexpr bool TIMED = Cfg::ND > 0 || Cfg::Sys::HAS_DFDT;
    static constexpr int T_AT = Cfg::N;                    // start time (TIMED only)
    static constexpr int H_AT = Cfg::N + (TIMED ? 1 : 0);  // signed step size
    static constexpr int V = int(16 / sizeof(R));
    static constexpr int F = ((H_AT + 1 + V - 1) / V) * V;
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
    using C = typename Cfg::C;
    static constexpr bool ACTIVE = true;
    static constexpr int F = SegRecord<Cfg>::F;
    using Rec = SegRecord<Cfg>;
    R* seg;        // this run's records
    int count;
    __device__ __forceinline__ void record(const R* y, R t, R h, bool saved) {
        R rec[F];
#pragma unroll
        for (int k = 0; k < Cfg::N; ++k) rec[k] = y[k];
        if constexpr (Rec::TIMED) rec[Rec::T_AT] = t;
        rec[Rec::H_AT] = saved ? -h : h;
#pragma unroll
        for (int k = Rec::H_AT + 1; k < F; ++k) rec[k] = R(0);
        SegRecord<Cfg>::store(seg + (long long)count * F, rec);
        ++count;
    }
    __device__ __forceinline__ void accepted(const Lane<Cfg>& L, C dt_eff, int row) {
        record(L.y, R(L.tp), R(dt_eff), row >= 0);
    }
};

// Step-size tape of the explicit Runge-Kutta adjoint.  For every accepted
// step k of a run the checkpointing forward stores
//   tape[run][k]        the step size as the loop advanced time with it
//                       (control precision when the right-hand side depends
//                       on time, else as the step function received it),
//                       negated when the step ended on a saved output row;
//   tape_flags[run][k / 32], bit k % 32: the attempt before it was rejected
//                       (an FSAL tableau then re-evaluated its first stage
//                       instead of reusing the last one);
//   step_count[run]     the number of accepted steps.
// Rows hold ``tape_row_entries(cap)`` entries and ``tape_flag_words(cap)``
// words for cap = max_ckpts * ckpt_every.  Lanes of a warp are at different
// steps of different runs, so the forward buffers entries in registers and
// writes whole 16-byte vectors.  The reverse sweep replays a segment from its
// checkpoint by calling the step function with those sizes, so the
// controller, the event logic and the rejected attempts are not repeated.
// An explicit step's result depends only on the start state, the step size,
// the time and the two flags, so the replay is bit-identical to the forward.
template <class Cfg>
struct Tape {
    using T = typename Pick<SegRecord<Cfg>::TIMED, typename Cfg::C, typename Cfg::R>::type;
    static constexpr int V = int(16 / sizeof(T));   // entries per vector
    static __host__ __device__ long long row_entries(long long cap) { return (cap + V - 1) / V * V; }
    static __host__ __device__ long long flag_words(long long cap) { return (cap + 31) / 32; }
    static __device__ __forceinline__ void store_vec(T* dst, const T* v) {
        if constexpr (sizeof(T) == 4) {
            *reinterpret_cast<float4*>(dst) = make_float4(v[0], v[1], v[2], v[3]);
        } else {
            *reinterpret_cast<double2*>(dst) = make_double2(v[0], v[1]);
        }
    }
};

// Explicit tableaus replay from the step-size tape; the others repeat the
// loop (a Rosenbrock step's Krylov start depends on rejected attempts).
template <class Cfg>
struct UsesTape {
    static constexpr bool VALUE = Cfg::ALGO == ALGO_ERK;
};
// Bytes of one tape entry, or 1 when the configuration keeps no tape (the
// size of the module's ``cbx_tape_probe`` symbol).
template <class Cfg>
struct TapeBytes {
    static constexpr int VALUE = UsesTape<Cfg>::VALUE ? int(sizeof(typename Tape<Cfg>::T)) : 1;
};

// Writes a run's tape from the forward loop's accepted steps.
template <class Cfg>
struct TapeRecorder {
    using C = typename Cfg::C;
    using T = typename Tape<Cfg>::T;
    static constexpr int V = Tape<Cfg>::V;
    static constexpr bool ACTIVE = true;
    T* row;            // this run's entries
    unsigned* flags;   // this run's rejected-attempt bits
    T buf[V];          // entries of the current vector, newest last
    unsigned rmask;    // bits of the current flag word
    __device__ __forceinline__ void begin(T* r, unsigned* f) {
        row = r;
        flags = f;
        rmask = 0u;
#pragma unroll
        for (int j = 0; j < V; ++j) buf[j] = T(0);
    }
    __device__ __forceinline__ void push(T v) {
#pragma unroll
        for (int j = 0; j < V - 1; ++j) buf[j] = buf[j + 1];
        buf[V - 1] = v;
    }
    __device__ __forceinline__ void accepted(const Lane<Cfg>& L, C dt_eff, int saved_row) {
        const int k = int(L.steps - L.rejections) - 1;   // below max_ckpts * ckpt_every
        const T v = T(dt_eff);
        push(saved_row >= 0 ? -v : v);
        if (!L.prev_accepted) rmask |= 1u << (k & 31);
        if ((k & (V - 1)) == V - 1) Tape<Cfg>::store_vec(row + (k - (V - 1)), buf);
        if ((k & 31) == 31) {
            flags[k >> 5] = rmask;
            rmask = 0u;
        }
    }
    // After the run's last accepted step (n in total): the partial vector
    // and flag word.
    __device__ __forceinline__ void finish(long long n) {
        const int r = int(n % V);
        if (r != 0) {
            for (int j = r; j < V; ++j) push(T(0));
            Tape<Cfg>::store_vec(row + (n - r), buf);
        }
        if ((n & 31) != 0) flags[n >> 5] = rmask;
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

    // Stage i influences y+ when b_i != 0 or a later stage that influences
    // y+ reads it (bit i of USED, filled from the last stage down).
    static __host__ __device__ constexpr unsigned used_mask() {
        unsigned m = 0u;
        for (int i = S - 1; i >= 0; --i) {
            bool used = Tab::b(i) != 0.0;
            for (int j = i + 1; j < S; ++j) used = used || (Tab::a(j, i) != 0.0 && ((m >> j) & 1u));
            if (used) m |= 1u << i;
        }
        return m;
    }
    static constexpr unsigned USED = used_mask();
    static __host__ __device__ constexpr bool stage_used(int i) { return (USED >> i) & 1u; }
    // k_i must be recomputed when a later stage that itself matters reads it
    // (Dormand-Prince's last stage only feeds the error estimate, so the
    // stage before it needs no derivative here).
    static __host__ __device__ constexpr unsigned feeds_mask() {
        unsigned m = 0u;
        for (int i = 0; i < S; ++i)
            for (int j = i + 1; j < S; ++j)
                if (Tab::a(j, i) != 0.0 && ((USED >> j) & 1u)) m |= 1u << i;
        return m;
    }
    static constexpr unsigned FEEDS = feeds_mask();
    static __host__ __device__ constexpr bool stage_feeds_used(int i) { return (FEEDS >> i) & 1u; }

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
            if (stage_feeds_used(i)) {
                if constexpr (ND > 0) Drivers<Cfg>::eval(stage_time, ctx.coeffs, drv_stage);
                Sys::template dxdt<R>(Y[i], ctx.p, drv_stage, stage_time, k[i]);
            }
        }
        R Ybar[S][N];
        R lam_out[N];
        // this step's parameter sensitivity, summed over the stages in the
        // working precision and added to the control-precision total once
        R pstep[NP > 0 ? NP : 1];
#pragma unroll
        for (int q = 0; q < (NP > 0 ? NP : 1); ++q) pstep[q] = R(0);
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
                for (int q = 0; q < NP; ++q) pstep[q] += pb[q];
            }
        }
#pragma unroll
        for (int q = 0; q < N; ++q) lam[q] = lam_out[q];
        if constexpr (NP > 0) {
#pragma unroll
            for (int q = 0; q < NP; ++q) pbar[q] += C(pstep[q]);
        }
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
        using Rhs = RosenbrockRhs<Cfg>;
        const R gamma = R(Tab::GAMMA);
        const R inv_dt = Rhs::FOLDED ? R(0) : R(1) / h;
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
            for (int i = 0; i < N; ++i) rhs[i] = Rhs::value(f[i], corr[i], s == 0, h, inv_dt, gamma * h, R(0));
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
    using T = typename Tape<Cfg>::T;
    __shared__ BlockTotals bt;
    totals_begin(&bt);
    Lane<Cfg> L;
    bool active = false, exhausted = false;
    int nck = 0;
    long long next_ck = 0;
    constexpr int W = LaneImage<Cfg>::WORDS;
    const long long tape_cap = (long long)g.max_ckpts * g.ckpt_every;
    TapeRecorder<Cfg> tr;
    while (true) {
        if (!active && !exhausted) {
            const long long run = claim_run(a.work_counter);
            if (run < a.n_runs) {
                lane_begin<Cfg>(L, a, run);
                active = true;
                nck = 0;
                next_ck = 0;
                if constexpr (UsesTape<Cfg>::VALUE)
                    tr.begin(static_cast<T*>(g.tape) + run * Tape<Cfg>::row_entries(tape_cap),
                             g.tape_flags + run * Tape<Cfg>::flag_words(tape_cap));
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
            if (!done) {
                if constexpr (UsesTape<Cfg>::VALUE) done = lane_iterate<Cfg, TapeRecorder<Cfg>>(L, a, &tr);
                else done = lane_iterate<Cfg>(L, a);
            }
            if (done) {
                if constexpr (UsesTape<Cfg>::VALUE) {
                    const long long n = L.steps - L.rejections;
                    tr.finish(n);
                    g.step_count[L.run] = int(n);
                }
                lane_end<Cfg>(L, a, &bt);
                g.ckpt_count[L.run] = nck;
                active = false;
            }
        }
    }
    totals_flush(&bt, a);
}

// One accepted step replayed from the tape: the step function with the
// recorded size and flag, then the loop's own state commit and clock
// update, recorded for the reverse pass.
template <class Cfg>
__device__ __forceinline__ void tape_step(Lane<Cfg>& L, typename Tape<Cfg>::T entry, bool prev_rejected,
                                          SegRecorder<Cfg>& rec, const typename Cfg::R* coeffs) {
    using R = typename Cfg::R;
    using C = typename Cfg::C;
    using T = typename Tape<Cfg>::T;
    constexpr int N = Cfg::N, ND = Cfg::ND;
    const bool saved = entry < T(0);
    const T dt = saved ? -entry : entry;
    const R h = R(dt);
    rec.record(L.y, R(L.tp), h, saved);
    L.save_idx += saved ? 1 : 0;   // rows are counted as the loop counts them
    R ynew[N], delta[N], err[N];
    R drv_new[ND > 0 ? ND : 1];
    StepCtx<Cfg> ctx{L.p, coeffs, L.tol_scale};
    Iters its;
    Cfg::Step::step(ctx, L.y, ynew, delta, err, L.drv, drv_new, h, R(L.tp), L.first_step, !prev_rejected, L.ps,
                    its);
    L.first_step = false;
    if constexpr (SegRecord<Cfg>::TIMED) {
        L.t = L.t + double(dt);
        L.tp = C(L.t);
    }
    commit_state<Cfg>(L, ynew, delta, drv_new);
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

// dL/d(saved state) of one output row (zeros outside the saved rows), loaded
// ahead of the reverse step that adds it.
template <class Cfg>
struct RowGrad {
    using R = typename Cfg::R;
    static constexpr int NS = Cfg::SAVE_STATE ? Cfg::N_SAVED_STATES : 0;
    R v[NS > 0 ? NS : 1];
    __device__ __forceinline__ void load(const cbx_solve_args& a, const cbx_adjoint_args& g, int row,
                                         long long run) {
        const bool in = row >= 0 && row < a.n_save_rows && g.grad_state;
        if constexpr (NS > 0) {
            constexpr int W = Cfg::N_SAVED_STATES + (Cfg::SAVE_TIME ? 1 : 0);
            const R* gr = static_cast<const R*>(g.grad_state) + (long long)(in ? row : 0) * W * a.run_stride + run;
#pragma unroll
            for (int k = 0; k < NS; ++k) v[k] = in ? gr[k * a.run_stride] : R(0);
        }
    }
    __device__ __forceinline__ void add_to(R* lam) const {
#pragma unroll
        for (int k = 0; k < NS; ++k) lam[Cfg::Idx::saved_state(k)] += v[k];
    }
};

// Reverse sweep.  Every lane works on its own run, but a warp moves through
// the phases together: all lanes replay their current segment (each until it
// holds ``ckpt_every`` records or its run ends), then all lanes
// back-propagate through their records, then each lane steps back to its
// previous checkpoint or, when its run is done, writes the gradients and
// claims the next run.  Phases are warp-uniform, so the replay and the
// reverse code never diverge against each other; lanes wait only for the
// longest segment of the warp.  The loop state lives only inside one pass
// (loaded from the checkpoint, replayed, dead once the records exist), so
// the replay and the reverse step do not hold registers for each other.
template <class Cfg>
__device__ __forceinline__ void run_adjoint_backward(const cbx_solve_args a, const cbx_adjoint_args g) {
    using R = typename Cfg::R;
    using C = typename Cfg::C;
    using Adj = StepAdjoint<Cfg, Cfg::ALGO>;
    using Rec = SegRecord<Cfg>;
    using T = typename Tape<Cfg>::T;
    constexpr int N = Cfg::N, NP = Cfg::NP, F = Rec::F;
    constexpr int W = LaneImage<Cfg>::WORDS;
    constexpr unsigned FULL = 0xffffffffu;
    const long long s = a.run_stride;
    const long long tape_cap = (long long)g.max_ckpts * g.ckpt_every;
    cbx_solve_args replay = a;
    replay.n_save_rows = 0;      // the replay writes no outputs
    replay.n_summary_rows = 0;
    R* seg = static_cast<R*>(g.seg);
    const unsigned* ckpt = static_cast<const unsigned*>(g.ckpt);
    constexpr int NPP = NP > 0 ? NP : 1;
    R lam[N];
    C pbar[NPP];
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
                for (int q = 0; q < NPP; ++q) pbar[q] = C(0);
                ck = g.ckpt_count[run] - 1;
            } else {
                exhausted = true;
            }
        }
        const bool busy = ck >= 0;
        if (!__any_sync(FULL, busy)) break;
        R* const run_seg = seg + (busy ? run : 0) * (long long)g.ckpt_every * F;
        R p[Cfg::NP > 0 ? Cfg::NP : 1];
        C tol_scale;
        int count, rows_end;
        {
            // replay
            Lane<Cfg> L;
            if (busy) load_lane<Cfg>(L, ckpt + (run * g.max_ckpts + ck) * (long long)W);
            SegRecorder<Cfg> rec{run_seg, 0};
            bool replaying = busy;
            if constexpr (UsesTape<Cfg>::VALUE) {
                // the segment's accepted steps from the tape, next entry in flight
                const T* trow = static_cast<const T*>(g.tape) + (busy ? run : 0) * Tape<Cfg>::row_entries(tape_cap);
                const unsigned* frow = g.tape_flags + (busy ? run : 0) * Tape<Cfg>::flag_words(tape_cap);
                long long k = (long long)(busy ? ck : 0) * g.ckpt_every;
                long long kend = 0;
                if (busy) {
                    const long long n = g.step_count[run];
                    kend = k + g.ckpt_every < n ? k + g.ckpt_every : n;
                }
                T nxt = T(0);
                unsigned word = 0u;
                if (k < kend) {
                    nxt = trow[k];
                    word = frow[k >> 5];
                }
                while (__any_sync(FULL, replaying)) {
                    if (replaying) {
                        if (k >= kend) {
                            replaying = false;
                        } else {
                            const T cur = nxt;
                            const bool rej = ((word >> (k & 31)) & 1u) != 0u;
                            if (k + 1 < kend) {
                                nxt = trow[k + 1];
                                if (((k + 1) & 31) == 0) word = frow[(k + 1) >> 5];
                            }
                            tape_step<Cfg>(L, cur, rej, rec, static_cast<const R*>(a.driver_coeffs));
                            ++k;
                        }
                    }
                }
            } else {
                while (__any_sync(FULL, replaying)) {
                    if (replaying) {
                        const bool done = lane_iterate<Cfg, SegRecorder<Cfg>>(L, replay, &rec);
                        if (done || rec.count >= g.ckpt_every) replaying = false;
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < (Cfg::NP > 0 ? Cfg::NP : 1); ++q) p[q] = busy ? L.p[q] : R(0);
            tol_scale = busy ? L.tol_scale : C(1);
            count = busy ? rec.count : 0;
            rows_end = busy ? L.save_idx : 0;   // rows saved up to the segment's end
        }
        // reverse, with the next (earlier) record and the next saved row's
        // loss gradient (rows are met in decreasing order) in flight
        int j = count - 1;
        R nxt[F];
        RowGrad<Cfg> row_next;
        if (j >= 0) {
            Rec::load(run_seg + (long long)j * F, nxt);
            row_next.load(a, g, rows_end - 1, run);
        }
        while (__any_sync(FULL, j >= 0)) {
            if (j >= 0) {
                R rec_j[F];
#pragma unroll
                for (int k = 0; k < F; ++k) rec_j[k] = nxt[k];
                if (j > 0) Rec::load(run_seg + (long long)(j - 1) * F, nxt);
                const R hs = rec_j[Rec::H_AT];
                if (hs < R(0)) {
                    row_next.add_to(lam);
                    --rows_end;
                    if (j > 0) row_next.load(a, g, rows_end - 1, run);
                }
                const R t = Rec::TIMED ? rec_j[Rec::T_AT] : R(0);
                StepCtx<Cfg> ctx{p, static_cast<const R*>(a.driver_coeffs), tol_scale};
                Adj::reverse(ctx, rec_j, t, fabs(hs), lam, pbar);
                --j;
            }
        }
        // previous checkpoint, or finish the run
        if (busy) {
            if (ck > 0) {
                --ck;
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
    __constant__ char cbx_tape_probe[cbx::TapeBytes<CFG>::VALUE];                                     \
    extern "C" __global__ void CBX_LAUNCH_BOUNDS(CFG) cbx_adjoint_forward(cbx_solve_args a,           \
                                                                         cbx_adjoint_args g) {       \
        cbx::run_adjoint_forward<CFG>(a, g);                                                          \
    }                                                                                                 \
    extern "C" __global__ void CBX_LAUNCH_BOUNDS(CFG) cbx_adjoint_backward(cbx_solve_args a,          \
                                                                          cbx_adjoint_args g) {      \
        cbx::run_adjoint_backward<CFG>(a, g);                                                         \
    }
