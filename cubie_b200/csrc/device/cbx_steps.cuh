// Tableau-driven step functions: explicit RK, Rosenbrock-W, fully implicit
// RK and diagonally implicit RK.  One system per thread.
//
// Every step receives the accepted state ``y`` at time ``t`` and returns
//   ynew   the proposed state (as the reference forms it),
//   delta  the increment ynew - y before it is added to y (used for the
//          compensated state update of the mixed-precision path),
//   err    the embedded error estimate (adaptive tableaus),
//   drv_new / obs_new  drivers and observables at the proposed time,
// plus the Newton and Krylov iteration counts of the attempt.
#pragma once
#include "cbx_common.cuh"
#include "cbx_newton.cuh"

namespace cbx {

// ---------------------------------------------------------------------------
// Drivers: piecewise polynomials sampled on a uniform grid, evaluated with
// Horner's rule; wrap or clamp at the ends (array_interpolator.py:463-550).
// ---------------------------------------------------------------------------
template <class Cfg>
struct Drivers {
    using R = typename Cfg::R;
    static constexpr int ND = Cfg::ND;
    static __device__ __forceinline__ void locate(R time, int& seg, R& tau, bool& in_range) {
        const R start = R(Cfg::DRV_EVAL_START);
        const R inv_res = R(Cfg::DRV_INV_RESOLUTION);
        const R scaled = (time - start) * inv_res;
        const R fl = floor(scaled);
        int idx = int(fl);
        if (Cfg::DRV_WRAP) {
            int m = idx % Cfg::DRV_NSEG;
            seg = m < 0 ? m + Cfg::DRV_NSEG : m;
            tau = scaled - fl;
            in_range = true;
        } else {
            in_range = (scaled >= R(0)) && (scaled <= R(Cfg::DRV_NSEG));
            seg = idx < 0 ? 0 : idx;
            seg = seg >= Cfg::DRV_NSEG ? Cfg::DRV_NSEG - 1 : seg;
            tau = scaled - R(seg);
        }
    }
    static __device__ __forceinline__ void eval(R time, const R* __restrict__ coeffs, R* out) {
        if constexpr (ND > 0) {
            int seg;
            R tau;
            bool in_range;
            locate(time, seg, tau, in_range);
#pragma unroll
            for (int k = 0; k < ND; ++k) {
                const R* c = coeffs + (size_t(seg) * ND + k) * (Cfg::DRV_ORDER + 1);
                R acc = R(0);
#pragma unroll
                for (int q = Cfg::DRV_ORDER; q >= 0; --q) acc = acc * tau + __ldg(c + q);
                out[k] = in_range ? acc : R(0);
            }
        }
    }
    static __device__ __forceinline__ void deriv(R time, const R* __restrict__ coeffs, R* out) {
        if constexpr (ND > 0) {
            int seg;
            R tau;
            bool in_range;
            locate(time, seg, tau, in_range);
#pragma unroll
            for (int k = 0; k < ND; ++k) {
                const R* c = coeffs + (size_t(seg) * ND + k) * (Cfg::DRV_ORDER + 1);
                R acc = R(0);
#pragma unroll
                for (int q = Cfg::DRV_ORDER; q >= 1; --q) acc = acc * tau + R(q) * __ldg(c + q);
                out[k] = in_range ? acc * R(Cfg::DRV_INV_RESOLUTION) : R(0);
            }
        }
    }
};

// Iteration counts of one step attempt.  ``nit``/``kit`` are what the
// reference reports to its counters output and to the Gustafsson
// controller: zero for Rosenbrock steps (its linear solver count never
// reaches the step's counters) and the last implicit stage's Newton solve
// for DIRK steps (each stage's solve overwrites the counters,
// generic_dirk.py:640-652 with newton_krylov.py:514-515).  ``*_all`` are
// the true totals over the attempt, used for throughput accounting.
struct Iters {
    int nit = 0, kit = 0, nit_all = 0, kit_all = 0;
};

template <class Cfg>
struct StepCtx {
    using R = typename Cfg::R;
    using C = typename Cfg::C;
    const R* p;        // parameters of this run
    const R* coeffs;   // driver coefficients
    C tol_scale;       // per-run tolerance scale (1 when uniform)
};

// ---------------------------------------------------------------------------
// Explicit RK (generic_erk.py:359-577).  Streams stage contributions into
// per-successor accumulators; reuses the last stage derivative of an
// accepted first-same-as-last step.
// ---------------------------------------------------------------------------
template <class Cfg>
struct ErkStep {
    using R = typename Cfg::R;
    using C = typename Cfg::C;
    using Sys = typename Cfg::Sys;
    using Tab = typename Cfg::Tab;
    static constexpr int N = Cfg::N, S = Cfg::S, ND = Cfg::ND;
    struct Persist {
        R k[N];
    };
    static __device__ __forceinline__ void init(Persist& ps) {
#pragma unroll
        for (int i = 0; i < N; ++i) ps.k[i] = R(0);
    }
    static __device__ __forceinline__ int step(const StepCtx<Cfg>& ctx, const R* y, R* ynew, R* delta, R* err,
                                               const R* drv, R* drv_new, R dt, R t, bool first_step,
                                               bool prev_accepted, Persist& ps, Iters& its) {
        its = Iters{};
        R outacc[N], erracc[N];
        R acc[(S > 1 ? S - 1 : 1)][N];
#pragma unroll
        for (int i = 0; i < N; ++i) {
            outacc[i] = R(0);
            erracc[i] = R(0);
        }
        const bool use_cached = Tab::FSAL && (S > 1) && !first_step && prev_accepted;
        if (!use_cached) Sys::template dxdt<R>(y, ctx.p, drv, t, ps.k);
#pragma unroll
        for (int i = 0; i < N; ++i) {
            if (Tab::ACC_OUT) outacc[i] += R(Tab::b(0)) * ps.k[i];
            if (Tab::HAS_ERR && Tab::ACC_ERR) erracc[i] += R(Tab::d(0)) * ps.k[i];
        }
#pragma unroll
        for (int r = 0; r < S - 1; ++r)
#pragma unroll
            for (int i = 0; i < N; ++i) acc[r][i] = R(0);
        R drv_stage[ND > 0 ? ND : 1];
#pragma unroll
        for (int prev = 0; prev < S - 1; ++prev) {
            const int stage = prev + 1;
#pragma unroll
            for (int succ = 0; succ < S - 1; ++succ) {
                const double coeff = Tab::a(succ + 1, prev);
                if (coeff != 0.0) {
#pragma unroll
                    for (int i = 0; i < N; ++i) acc[succ][i] += R(coeff) * ps.k[i];
                }
            }
            const R stage_time = t + dt * R(Tab::c(stage));
#pragma unroll
            for (int i = 0; i < N; ++i) {
                const R scaled = acc[prev][i] * dt;
                if (stage == Tab::B_ROW) delta[i] = scaled;
                acc[prev][i] = scaled + y[i];
            }
            if constexpr (ND > 0) Drivers<Cfg>::eval(stage_time, ctx.coeffs, drv_stage);
            Sys::template dxdt<R>(acc[prev], ctx.p, drv_stage, stage_time, ps.k);
#pragma unroll
            for (int i = 0; i < N; ++i) {
                if (Tab::ACC_OUT) outacc[i] += R(Tab::b(stage)) * ps.k[i];
                if (Tab::HAS_ERR && Tab::ACC_ERR) erracc[i] += R(Tab::d(stage)) * ps.k[i];
            }
        }
#pragma unroll
        for (int i = 0; i < N; ++i) {
            if constexpr (Tab::ACC_OUT) {
                delta[i] = outacc[i] * dt;
                ynew[i] = delta[i] + y[i];
            } else {
                ynew[i] = acc[(Tab::B_ROW > 0 ? Tab::B_ROW : 1) - 1][i];
            }
            if constexpr (Tab::HAS_ERR) {
                if constexpr (Tab::ACC_ERR) err[i] = erracc[i] * dt;
                else err[i] = ynew[i] - acc[(Tab::BHAT_ROW > 0 ? Tab::BHAT_ROW : 1) - 1][i];
            }
        }
        if constexpr (ND > 0) Drivers<Cfg>::eval(t + dt, ctx.coeffs, drv_new);
        return SUCCESS;
    }
};

// ---------------------------------------------------------------------------
// Rosenbrock-W (generic_rosenbrock_w.py:459-759).  Stage solves of
// (I - gamma h J) K_i = gamma h (f(Y_i) + sum_j C_ij K_j / h + gamma_i h f_t)
// with Y_i = y + sum_j a_ij K_j and the Jacobian frozen at the step start.
// ---------------------------------------------------------------------------
// The right-hand side of a Rosenbrock stage's linear system is
// h gamma (f_s + sum_j C_sj K_j / h + gs_s h f_t)
// (generic_rosenbrock_w.py:682-698).  Written in that order it costs a
// division per step and two multiplies per component beyond the sums;
// distributed, h gamma f_s + gamma sum_j C_sj K_j (+ gs_s h gamma (h f_t)),
// it costs one multiply and one multiply-add per component and no
// division.  The distributed form is used wherever no reference result is
// compared bit for bit (the mixed-precision mode and direct stage solves);
// elsewhere the reference's order is kept.  gamma stays a separate factor:
// folding it into the C coefficients would save the multiply, but the
// products gamma C_sj rounded to FP32 perturb the method's coefficients
// against the gamma of the stage matrix, and over the thousands of steps of
// a tight-tolerance run in the mixed-precision mode that coherent error
// doubled the 90th-percentile global error.
template <class Cfg>
struct RosenbrockRhs {
    using R = typename Cfg::R;
    using Tab = typename Cfg::Tab;
    static constexpr bool FOLDED = Cfg::MIXED || Cfg::LIN == LIN_DIRECT;
    // one component: f the stage derivative, corr = sum_j C_sj K_j (times M
    // for a mass-matrix system), hg = gamma h, gs_tdv = gs_s (h f_t) or 0
    static __device__ __forceinline__ R value(R f, R corr, bool first, R h, R inv_h, R hg, R gs_tdv) {
        constexpr bool T = Cfg::Sys::HAS_DFDT;
        if constexpr (FOLDED) {
            R v = first ? f * hg : f * hg + R(Tab::GAMMA) * corr;
            if constexpr (T) v = v + gs_tdv * hg;
            return v;
        } else {
            R rv = first ? f : f + corr * inv_h;
            if constexpr (T) rv = rv + gs_tdv;
            return rv * h * R(Tab::GAMMA);
        }
    }
};

template <class Cfg>
struct RosenbrockStep {
    using R = typename Cfg::R;
    using C = typename Cfg::C;
    using Sys = typename Cfg::Sys;
    using Tab = typename Cfg::Tab;
    using Rhs = RosenbrockRhs<Cfg>;
    static constexpr int N = Cfg::N, S = Cfg::S, ND = Cfg::ND;
    // In the mixed-precision mode the proposed state only sizes the error
    // tolerance (the state update is the compensated y + delta), so it is
    // formed once from delta instead of accumulated beside it.
    static constexpr bool YNEW_FROM_DELTA = Cfg::MIXED && Tab::ACC_OUT;
    struct Persist {
        R guess[N];   // last solved stage increment: first-stage initial guess
    };
    static __device__ __forceinline__ void init(Persist& ps) {
#pragma unroll
        for (int i = 0; i < N; ++i) ps.guess[i] = R(0);
    }
    static __device__ __forceinline__ int step(const StepCtx<Cfg>& ctx, const R* y, R* ynew, R* delta, R* err,
                                               const R* drv, R* drv_new, R dt, R t, bool, bool, Persist& ps,
                                               Iters& its) {
        its = Iters{};
        const R gamma = R(Tab::GAMMA);
        const R inv_dt = Rhs::FOLDED ? R(0) : R(1) / dt;
        const R hg = gamma * dt;
        R J[Sys::NJ];
        Sys::template jac<R>(y, ctx.p, drv, t, J);
        // h times the time derivative of f (explicit t and driver chain
        // rule); skipped for systems where it is identically zero
        R tdv[N];
        if constexpr (Sys::HAS_DFDT) {
            R dd[ND > 0 ? ND : 1];
            if constexpr (ND > 0) Drivers<Cfg>::deriv(t, ctx.coeffs, dd);
            else dd[0] = R(0);
            Sys::template dfdt<R>(y, ctx.p, drv, dd, t, tdv);
        }
        // The proposed state starts from y and takes each stage's weighted
        // increment in turn (or is the stage state whose row of a equals b);
        // the error likewise, in the reference's order of operations.
        // ``delta`` (sum of the weighted increments) feeds the compensated
        // update of the mixed-precision mode.
#pragma unroll
        for (int i = 0; i < N; ++i) {
            if constexpr (Sys::HAS_DFDT) tdv[i] *= dt;
            delta[i] = R(0);
            ynew[i] = y[i];
            if (Tab::HAS_ERR) err[i] = R(0);
        }
        R K[S][N];
        R f[N], rhs[N], Y[N];
        R drv_stage[ND > 0 ? ND : 1];
        int status = SUCCESS;
        SingleStageOp<Cfg> op{J, hg, y, ctx.tol_scale};
        // direct solves: one factorisation of I - gamma h J serves every stage
        DenseLU<R, N> lu;
        if constexpr (Cfg::LIN == LIN_DIRECT) {
            lu.factor(op);
            if (!lu.ok) status |= MAX_LINEAR_ITERATIONS_EXCEEDED;
        }
        // One loop over the stages with a single call site of the linear
        // solver keeps one copy of it in the instruction stream.  The stage
        // index is a run-time value here, so tableau entries and the stored
        // stage increments are picked with compile-time-unrolled selects
        // (the increments stay in registers).  The initial guess of every
        // stage is the solution of the one before it (the first stage uses
        // the previous step's last increment), which is what ``ps.guess``
        // already holds when the solve starts.  With direct solves the
        // solve is a few multiply-adds, so the loop is unrolled and every
        // select folds to a constant.
        constexpr int STAGE_UNROLL = (Cfg::LIN == LIN_DIRECT) ? S : 1;
#pragma unroll (STAGE_UNROLL)
        for (int stage = 0; stage < S; ++stage) {
            R c_s = R(0), gs_s = R(0), b_s = R(0), d_s = R(0);
#pragma unroll
            for (int q = 0; q < S; ++q) {
                if (q == stage) {
                    c_s = R(Tab::c(q));
                    gs_s = R(Tab::gs(q));
                    b_s = R(Tab::b(q));
                    d_s = R(Tab::d(q));
                }
            }
            const R stage_time = t + dt * c_s;
#pragma unroll
            for (int i = 0; i < N; ++i) {
                R v = y[i];
                R corr = R(0);
#pragma unroll
                for (int j = 0; j < S - 1; ++j) {
                    R a_sj = R(0), c_sj = R(0);
#pragma unroll
                    for (int q = 1; q < S; ++q) {
                        if (q == stage) {
                            a_sj = R(Tab::a(q, j));
                            c_sj = R(Tab::Cm(q, j));
                        }
                    }
                    if (j < stage) {
                        if (a_sj != R(0)) v += a_sj * K[j][i];
                        if (c_sj != R(0)) corr += c_sj * K[j][i];
                    }
                }
                Y[i] = v;
                rhs[i] = corr;
                if (!Tab::ACC_OUT && stage == Tab::B_ROW) ynew[i] = v;
                if (Tab::HAS_ERR && !Tab::ACC_ERR && stage == Tab::BHAT_ROW) err[i] = v;
            }
            if constexpr (Sys::HAS_MASS) {
                // the C_ij K_j / h term of a mass-matrix system is
                // M (C_ij K_j) / h (Hairer & Wanner, Solving ODEs II, VI.4;
                // the reference leaves M out, generic_rosenbrock_w.py:682-698,
                // and fails on every non-identity M tried)
                R mc[N];
                Sys::template mass_mv<R>(rhs, mc);
#pragma unroll
                for (int i = 0; i < N; ++i) rhs[i] = mc[i];
            }
            if constexpr (ND > 0) {
                if (stage == 0) {
#pragma unroll
                    for (int k = 0; k < ND; ++k) drv_stage[k] = drv[k];
                } else {
                    Drivers<Cfg>::eval(stage_time, ctx.coeffs, drv_stage);
                }
            }
            Sys::template dxdt<R>(Y, ctx.p, ND > 0 ? drv_stage : drv, stage_time, f);
#pragma unroll
            for (int i = 0; i < N; ++i) {
                R gs_tdv = R(0);
                if constexpr (Sys::HAS_DFDT) gs_tdv = gs_s * tdv[i];
                rhs[i] = Rhs::value(f[i], rhs[i], stage == 0, dt, inv_dt, hg, gs_tdv);
            }
            int it = 0;
            if constexpr (Cfg::LIN == LIN_DIRECT) {
                lu.solve(rhs, ps.guess);
                it = 1;
            } else {
                status |= linear_solve<Cfg>(op, rhs, ps.guess, it);
            }
            its.kit_all += it;
#pragma unroll
            for (int i = 0; i < N; ++i) {
                const R k = ps.guess[i];
#pragma unroll
                for (int j = 0; j < S; ++j)
                    if (j == stage) K[j][i] = k;
                delta[i] += b_s * k;
                if (Tab::ACC_OUT && !YNEW_FROM_DELTA) ynew[i] += b_s * k;
                if (Tab::HAS_ERR && Tab::ACC_ERR) err[i] += d_s * k;
            }
        }
        if constexpr (YNEW_FROM_DELTA) {
#pragma unroll
            for (int i = 0; i < N; ++i) ynew[i] = y[i] + delta[i];
        }
        if (Tab::HAS_ERR && !Tab::ACC_ERR) {
#pragma unroll
            for (int i = 0; i < N; ++i) err[i] = ynew[i] - err[i];
        }
        if constexpr (ND > 0) Drivers<Cfg>::eval(t + dt, ctx.coeffs, drv_new);
        return status;
    }
};

// ---------------------------------------------------------------------------
// Fully implicit RK (generic_firk.py:508-701): one coupled Newton solve over
// the S*N scaled stage derivatives u_i = h f(t + c_i h, y + sum_j a_ij u_j),
// warm-started by dense prediction of the previous step's stage curve
// (stage_predictors.py:345-548); Kahan-summed output and error.
// ---------------------------------------------------------------------------
template <class Cfg>
struct FirkProblem {
    using R = typename Cfg::R;
    using C = typename Cfg::C;
    using Sys = typename Cfg::Sys;
    using Tab = typename Cfg::Tab;
    static constexpr int N = Cfg::N, S = Cfg::S, ND = Cfg::ND;
    static constexpr int K = S * N;
    const StepCtx<Cfg>* ctx;
    const R* base;              // step-start state
    const R (*drv)[ND > 0 ? ND : 1];
    R t, h;
    R J[S][Sys::NJ];
    __device__ __forceinline__ void stage_state(const R* u, int i, R* Y) const {
#pragma unroll
        for (int k = 0; k < N; ++k) {
            R v = base[k];
#pragma unroll
            for (int j = 0; j < S; ++j)
                if (Tab::a(i, j) != 0.0) v += R(Tab::a(i, j)) * u[j * N + k];
            Y[k] = v;
        }
    }
    __device__ __forceinline__ void residual(const R* u, R* out) const {
#pragma unroll
        for (int i = 0; i < S; ++i) {
            R Y[N], f[N];
            stage_state(u, i, Y);
            Sys::template dxdt<R>(Y, ctx->p, drv[i], t + h * R(Tab::c(i)), f);
#pragma unroll
            for (int k = 0; k < N; ++k) out[i * N + k] = u[i * N + k] - h * f[k];
            if constexpr (Sys::HAS_MASS) {
                // M u_i - h f(Y_i) (nonlinear_residuals.py:324-345)
                R mu[N];
                Sys::template mass_mv<R>(u + i * N, mu);
#pragma unroll
                for (int k = 0; k < N; ++k) out[i * N + k] = mu[k] - h * f[k];
            }
        }
    }
    __device__ __forceinline__ void linearize(const R* u) {
#pragma unroll
        for (int i = 0; i < S; ++i) {
            R Y[N];
            stage_state(u, i, Y);
            Sys::template jac<R>(Y, ctx->p, drv[i], t + h * R(Tab::c(i)), J[i]);
        }
    }
    __device__ __forceinline__ CoupledOp<Cfg> op() const { return CoupledOp<Cfg>{J, h, base, ctx->tol_scale}; }
    // FIRK correction norm (norms.py:377-435): stage values against the
    // step start, Newton atol/rtol.
    __device__ __forceinline__ C corr_norm2(const R* delta, const R* u) const {
        C nrm2 = C(0);
#pragma unroll
        for (int i = 0; i < S; ++i) {
            R Y[N];
            stage_state(u, i, Y);
#pragma unroll
            for (int k = 0; k < N; ++k) {
                const R ref = pymax(absv(Y[k]), absv(base[k]));
                const C ratio = tol_ratio<Cfg>(delta[i * N + k], ref, Cfg::natol(k), Cfg::nrtol(k), ctx->tol_scale);
                nrm2 += ratio * ratio;
            }
        }
        return nrm2 * (C(1) / C(K));
    }
};

template <class Cfg>
struct FirkStep {
    using R = typename Cfg::R;
    using C = typename Cfg::C;
    using Sys = typename Cfg::Sys;
    using Tab = typename Cfg::Tab;
    static constexpr int N = Cfg::N, S = Cfg::S, ND = Cfg::ND;
    struct Persist {
        R u[S * N];
        R prev_dt;
        C theta;
    };
    static __device__ __forceinline__ void init(Persist& ps) {
#pragma unroll
        for (int i = 0; i < S * N; ++i) ps.u[i] = R(0);
        ps.prev_dt = R(0);
        ps.theta = C(0);
    }
    // In-place read-ahead of the stage curve (stage_predictors.py:474-548):
    // each transform entry is a polynomial in the step ratio, highest power
    // first; the commit is a predicated select.
    static __device__ __forceinline__ void predict(R* u, R ratio, bool apply) {
        constexpr int F = Tab::PRED_FIRST;
        constexpr int P = Tab::PRED_POWERS;
        R T[(S - F) > 0 ? (S - F) : 1][S];
#pragma unroll
        for (int r = 0; r < S - F; ++r)
#pragma unroll
            for (int c = 0; c < S; ++c) {
                R acc = R(0);
#pragma unroll
                for (int q = P - 1; q >= 0; --q) acc = acc * ratio + R(Tab::pred(q, r + F, c));
                T[r][c] = acc * ratio;
            }
#pragma unroll
        for (int k = 0; k < N; ++k) {
            R prev[S];
#pragma unroll
            for (int c = 0; c < S; ++c) prev[c] = u[c * N + k];
#pragma unroll
            for (int r = 0; r < S - F; ++r) {
                R acc = R(0);
#pragma unroll
                for (int c = 0; c < S; ++c) acc += T[r][c] * prev[c];
                u[(r + F) * N + k] = apply ? acc : u[(r + F) * N + k];
            }
        }
    }
    static __device__ __forceinline__ int step(const StepCtx<Cfg>& ctx, const R* y, R* ynew, R* delta, R* err,
                                               const R*, R* drv_new, R dt, R t, bool first_step,
                                               bool prev_accepted, Persist& ps, Iters& its) {
        its = Iters{};
        if (Tab::DENSE_PRED) {
            const R previous_dt = ps.prev_dt;
            ps.prev_dt = dt;
            const R safe_prev = previous_dt > R(0) ? previous_dt : dt;
            const R ratio = dt / safe_prev;
            const bool apply = !first_step && prev_accepted && (ratio <= R(Tab::PRED_RATIO_LIMIT));
            predict(ps.u, ratio, apply);
        }
        R drv_stack[S][ND > 0 ? ND : 1];
        if constexpr (ND > 0) {
#pragma unroll
            for (int i = 0; i < S; ++i) Drivers<Cfg>::eval(t + dt * R(Tab::c(i)), ctx.coeffs, drv_stack[i]);
        }
        FirkProblem<Cfg> prob;
        prob.ctx = &ctx;
        prob.base = y;
        prob.drv = drv_stack;
        prob.t = t;
        prob.h = dt;
        const int status = newton_solve<Cfg>(prob, ps.u, ps.theta, its.nit, its.kit);
        its.nit_all = its.nit;
        its.kit_all = its.kit;
        if (!Tab::ACC_OUT) {
            // output equals a stage state: y + sum_j a_{row,j} u_j
#pragma unroll
            for (int k = 0; k < N; ++k) {
                R v = R(0);
                R yv = y[k];
#pragma unroll
                for (int j = 0; j < S; ++j)
                    if (Tab::a(Tab::B_ROW, j) != 0.0) {
                        v += R(Tab::a(Tab::B_ROW, j)) * ps.u[j * N + k];
                        yv += R(Tab::a(Tab::B_ROW, j)) * ps.u[j * N + k];
                    }
                delta[k] = v;
                ynew[k] = yv;
            }
        } else {
#pragma unroll
            for (int k = 0; k < N; ++k) {
                Kahan<R> acc;
#pragma unroll
                for (int j = 0; j < S; ++j) acc.add(R(Tab::b(j)) * ps.u[j * N + k]);
                delta[k] = acc.sum;
                ynew[k] = y[k] + acc.sum;
            }
        }
        if (Tab::HAS_ERR) {
#pragma unroll
            for (int k = 0; k < N; ++k) {
                if (Tab::ACC_ERR) {
                    Kahan<R> acc;
#pragma unroll
                    for (int j = 0; j < S; ++j) acc.add(R(Tab::d(j)) * ps.u[j * N + k]);
                    err[k] = acc.sum;
                } else {
                    R yv = y[k];
#pragma unroll
                    for (int j = 0; j < S; ++j)
                        if (Tab::a(Tab::BHAT_ROW, j) != 0.0) yv += R(Tab::a(Tab::BHAT_ROW, j)) * ps.u[j * N + k];
                    err[k] = ynew[k] - yv;
                }
            }
        }
        if constexpr (ND > 0) {
            if (Tab::c(S - 1) == 1.0) {
#pragma unroll
                for (int q = 0; q < ND; ++q) drv_new[q] = drv_stack[S - 1][q];
            } else {
                Drivers<Cfg>::eval(t + dt, ctx.coeffs, drv_new);
            }
        }
        return status;
    }
};

// ---------------------------------------------------------------------------
// Diagonally implicit RK (generic_dirk.py:515-855): per-stage Newton solves
// of z = h f(t_i, base_i + a_ii z) with explicit accumulation of earlier
// stage derivatives into the stage bases.
// ---------------------------------------------------------------------------
template <class Cfg>
struct DirkProblem {
    using R = typename Cfg::R;
    using C = typename Cfg::C;
    using Sys = typename Cfg::Sys;
    static constexpr int N = Cfg::N, ND = Cfg::ND;
    static constexpr int K = N;
    const StepCtx<Cfg>* ctx;
    const R* base;
    const R* step_start;
    const R* drv;
    R t, h, a;
    R J[Sys::NJ];
    __device__ __forceinline__ void residual(const R* z, R* out) const {
        R Y[N], f[N];
#pragma unroll
        for (int k = 0; k < N; ++k) Y[k] = base[k] + a * z[k];
        Sys::template dxdt<R>(Y, ctx->p, drv, t, f);
        if constexpr (Sys::HAS_MASS) {
            // M z - h f(base + a z) (nonlinear_residuals.py:59-130)
            R mz[N];
            Sys::template mass_mv<R>(z, mz);
#pragma unroll
            for (int k = 0; k < N; ++k) out[k] = mz[k] - h * f[k];
        } else {
#pragma unroll
            for (int k = 0; k < N; ++k) out[k] = z[k] - h * f[k];
        }
    }
    __device__ __forceinline__ void linearize(const R* z) {
        R Y[N];
#pragma unroll
        for (int k = 0; k < N; ++k) Y[k] = base[k] + a * z[k];
        Sys::template jac<R>(Y, ctx->p, drv, t, J);
    }
    __device__ __forceinline__ SingleStageOp<Cfg> op() const {
        return SingleStageOp<Cfg>{J, a * h, base, ctx->tol_scale};
    }
    // DIRK correction norm (norms.py:337-375).
    __device__ __forceinline__ C corr_norm2(const R* delta, const R* z) const {
        C nrm2 = C(0);
#pragma unroll
        for (int k = 0; k < N; ++k) {
            const R sv = base[k] + a * z[k];
            const R ref = pymax(absv(sv), absv(step_start[k]));
            const C ratio = tol_ratio<Cfg>(delta[k], ref, Cfg::natol(k), Cfg::nrtol(k), ctx->tol_scale);
            nrm2 += ratio * ratio;
        }
        return nrm2 * (C(1) / C(K));
    }
};

template <class Cfg>
struct DirkStep {
    using R = typename Cfg::R;
    using C = typename Cfg::C;
    using Sys = typename Cfg::Sys;
    using Tab = typename Cfg::Tab;
    static constexpr int N = Cfg::N, S = Cfg::S, ND = Cfg::ND;
    static constexpr int H = Tab::DENSE_PRED ? S * N : 1;
    struct Persist {
        R z[N];          // stage increment, carried across stages and steps
        R rhs[N];        // last stage derivative (first-same-as-last reuse)
        R hist[H];       // dense-prediction history
        R prev_dt;
        C theta;
    };
    static __device__ __forceinline__ void init(Persist& ps) {
#pragma unroll
        for (int i = 0; i < N; ++i) {
            ps.z[i] = R(0);
            ps.rhs[i] = R(0);
        }
#pragma unroll
        for (int i = 0; i < H; ++i) ps.hist[i] = R(0);
        ps.prev_dt = R(0);
        ps.theta = C(0);
    }
    static __device__ __forceinline__ int step(const StepCtx<Cfg>& ctx, const R* y, R* ynew, R* delta, R* err,
                                               const R* drv, R* drv_new, R dt, R t, bool first_step,
                                               bool prev_accepted, Persist& ps, Iters& its) {
        its = Iters{};
        int status = SUCCESS;
        if (Tab::DENSE_PRED) {
            const R previous_dt = ps.prev_dt;
            ps.prev_dt = dt;
            const R safe_prev = previous_dt > R(0) ? previous_dt : dt;
            const R ratio = dt / safe_prev;
            const bool apply = !first_step && prev_accepted && (ratio <= R(Tab::PRED_RATIO_LIMIT));
            FirkStep<Cfg>::predict(ps.hist, ratio, apply);
        }
        const bool use_cached = Tab::FSAL && (S > 1) && !first_step && prev_accepted;
        R base[N], outacc[N], erracc[N];
        R acc[(S > 1 ? S - 1 : 1)][N];
        R drv_stage[ND > 0 ? ND : 1];
#pragma unroll
        for (int i = 0; i < N; ++i) {
            base[i] = y[i];
            outacc[i] = R(0);
            erracc[i] = R(0);
        }
#pragma unroll
        for (int r = 0; r < S - 1; ++r)
#pragma unroll
            for (int i = 0; i < N; ++i) acc[r][i] = R(0);
        R stage_time = t + dt * R(Tab::c(0));
        if (!use_cached) {
            if constexpr (ND > 0) {
                if (Tab::c(0) == 0.0) {
#pragma unroll
                    for (int q = 0; q < ND; ++q) drv_stage[q] = drv[q];
                } else {
                    Drivers<Cfg>::eval(stage_time, ctx.coeffs, drv_stage);
                }
            }
            if (Tab::a(0, 0) != 0.0) {
                if (Tab::DENSE_PRED) {
#pragma unroll
                    for (int i = 0; i < N; ++i) ps.z[i] = ps.hist[i];
                }
                DirkProblem<Cfg> prob;
                prob.ctx = &ctx; prob.base = base; prob.step_start = y; prob.drv = drv_stage;
                prob.t = stage_time; prob.h = dt; prob.a = R(Tab::a(0, 0));
                int ni = 0, ki = 0;
                status |= newton_solve<Cfg>(prob, ps.z, ps.theta, ni, ki);
                its.nit = ni;
                its.kit = ki;
                its.nit_all += ni;
                its.kit_all += ki;
                if (Tab::DENSE_PRED) {
#pragma unroll
                    for (int i = 0; i < N; ++i) ps.hist[i] = ps.z[i];
                }
#pragma unroll
                for (int i = 0; i < N; ++i) base[i] += R(Tab::a(0, 0)) * ps.z[i];
            }
            if (Tab::need_f(0)) Sys::template dxdt<R>(base, ctx.p, drv_stage, stage_time, ps.rhs);
        }
        if (Tab::DENSE_PRED && Tab::a(0, 0) == 0.0) {
#pragma unroll
            for (int i = 0; i < N; ++i) ps.hist[i] = dt * ps.rhs[i];
        }
#pragma unroll
        for (int i = 0; i < N; ++i) {
            if (Tab::ACC_OUT) {
                if (Tab::b(0) != 0.0) outacc[i] += R(Tab::b(0)) * ps.rhs[i];
            } else if (Tab::B_ROW == 0) ynew[i] = base[i];
            if (Tab::HAS_ERR) {
                if (Tab::ACC_ERR) {
                    if (Tab::d(0) != 0.0) erracc[i] += R(Tab::d(0)) * ps.rhs[i];
                }
                else if (Tab::BHAT_ROW == 0) err[i] = base[i];
            }
        }
#pragma unroll
        for (int prev = 0; prev < S - 1; ++prev) {
            const int stage = prev + 1;
#pragma unroll
            for (int succ = 0; succ < S - 1; ++succ) {
                const double coeff = (succ + 1 > prev) ? Tab::a(succ + 1, prev) : 0.0;
                if (coeff != 0.0) {
#pragma unroll
                    for (int i = 0; i < N; ++i) acc[succ][i] += R(coeff) * ps.rhs[i];
                }
            }
            stage_time = t + dt * R(Tab::c(stage));
            if constexpr (ND > 0) Drivers<Cfg>::eval(stage_time, ctx.coeffs, drv_stage);
            R stage_delta[N];
#pragma unroll
            for (int i = 0; i < N; ++i) {
                stage_delta[i] = acc[prev][i] * dt;
                base[i] = stage_delta[i] + y[i];
            }
            if (Tab::a(stage, stage) != 0.0) {
                if (Tab::DENSE_PRED) {
#pragma unroll
                    for (int i = 0; i < N; ++i) ps.z[i] = ps.hist[Tab::pred_source(stage) * N + i];
                } else if (Tab::EULER_GUESS && Tab::a(prev, prev) == 0.0) {
#pragma unroll
                    for (int i = 0; i < N; ++i) ps.z[i] = dt * ps.rhs[i];
                }
                DirkProblem<Cfg> prob;
                prob.ctx = &ctx; prob.base = base; prob.step_start = y; prob.drv = drv_stage;
                prob.t = stage_time; prob.h = dt; prob.a = R(Tab::a(stage, stage));
                int ni = 0, ki = 0;
                status |= newton_solve<Cfg>(prob, ps.z, ps.theta, ni, ki);
                its.nit = ni;
                its.kit = ki;
                its.nit_all += ni;
                its.kit_all += ki;
                if (Tab::DENSE_PRED) {
#pragma unroll
                    for (int i = 0; i < N; ++i) ps.hist[stage * N + i] = ps.z[i];
                }
#pragma unroll
                for (int i = 0; i < N; ++i) {
                    base[i] += R(Tab::a(stage, stage)) * ps.z[i];
                    stage_delta[i] += R(Tab::a(stage, stage)) * ps.z[i];
                }
            }
            if (Tab::need_f(stage)) Sys::template dxdt<R>(base, ctx.p, drv_stage, stage_time, ps.rhs);
            if (Tab::DENSE_PRED && Tab::HAS_LATER_EXPLICIT && Tab::a(stage, stage) == 0.0) {
#pragma unroll
                for (int i = 0; i < N; ++i) ps.hist[stage * N + i] = dt * ps.rhs[i];
            }
#pragma unroll
            for (int i = 0; i < N; ++i) {
                if (Tab::ACC_OUT) {
                    if (Tab::b(stage) != 0.0) outacc[i] += R(Tab::b(stage)) * ps.rhs[i];
                } else if (Tab::B_ROW == stage) {
                    ynew[i] = base[i];
                    delta[i] = stage_delta[i];
                }
                if (Tab::HAS_ERR) {
                    if (Tab::ACC_ERR) {
                        if (Tab::d(stage) != 0.0) erracc[i] += R(Tab::d(stage)) * ps.rhs[i];
                    }
                    else if (Tab::BHAT_ROW == stage) err[i] = base[i];
                }
            }
        }
#pragma unroll
        for (int i = 0; i < N; ++i) {
            if (Tab::ACC_OUT) {
                delta[i] = outacc[i] * dt;
                ynew[i] = delta[i] + y[i];
            } else if (Tab::B_ROW == 0) {
                delta[i] = ynew[i] - y[i];
            }
            if (Tab::HAS_ERR) {
                if (Tab::ACC_ERR) err[i] = erracc[i] * dt;
                else err[i] = ynew[i] - err[i];
            }
        }
        if constexpr (ND > 0) Drivers<Cfg>::eval(t + dt, ctx.coeffs, drv_new);
        return status;
    }
};

}  // namespace cbx
