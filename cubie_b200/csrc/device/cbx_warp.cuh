// Warp-per-system integration for large systems (one warp integrates one
// run; the reference runs every system on one thread with its vectors in
// local memory).
//
// Layout: lane l of the warp holds components l, l + 32, l + 64, ... of
// every state-sized vector (L = ceil(N / 32) values per lane, padded with
// zeros).  The right-hand side and the Jacobian-vector product are
// evaluated by the whole warp from copies in shared memory, through the
// class-grouped generated functions (``WSys::dxdt_lanes`` /
// ``WSys::jmv_lanes``; cubie_b200/warpgen.py).  Dot products and norms are
// lane partials summed with shuffles and then broadcast from lane 0, so
// every lane holds bit-identical scalars and all control flow (accept or
// reject, Newton and Krylov convergence, the event schedule) is uniform
// across the warp.  The Krylov solvers and the Newton iteration are the
// shared ones (cbx_linear.cuh, cbx_newton.cuh) instantiated on the warp
// operators below.
//
// Scope: diagonally implicit RK tableaus (Newton + MR/SD/BiCGSTAB/GMRES),
// every step-size controller, drivers, saved states/time/counters and
// state summaries; no observables and no dense stage prediction.
#pragma once
#include "cbx_loop.cuh"

namespace cbx {

constexpr unsigned kWarpFull = 0xffffffffu;

// Sum over the warp, then lane 0's value everywhere (the butterfly alone
// may round differently on different lanes).
template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kWarpFull, v, o);
    return __shfl_sync(kWarpFull, v, 0);
}

// Per-warp shared memory.  With a cached Jacobian (WSys::NNZ > 0) the
// linearisation stores J's nonzero coefficients in ``jac`` and every J v
// reads them back; otherwise J v is re-derived from the linearisation
// point ``ylin``.  With Cfg::SHARED_SCRATCH the stage solve's base state,
// the step's start state and BiCGSTAB's shadow residual live here too
// ("shared" placement); otherwise they stay in the calling thread's
// registers or local memory ("local" placement).
template <class Cfg>
struct WarpMem {
    using R = typename Cfg::R;
    static constexpr int N = Cfg::N;
    static constexpr bool CACHED = Cfg::WSys::NNZ > 0;
    static constexpr int SH = Cfg::SHARED_SCRATCH ? N : 1;
    R ys[N];                              // state of a right-hand-side evaluation
    R vs[N];                              // operand of J v
    R out[N];                             // class outputs
    R kw[N];                              // Krylov weights 1 / tol_i of the current stage solve
    R jac[CACHED ? Cfg::WSys::NNZ : 1];   // cached Jacobian coefficients
    R ylin[CACHED ? 1 : N];               // linearisation point (matrix-free J v)
    R sbase[SH];                          // stage base state (shared placement)
    R sstart[SH];                         // step start state (shared placement)
    R r0[Cfg::SHARED_SCRATCH ? 32 * ((N + 31) / 32) : 1];  // BiCGSTAB shadow residual (shared placement)
    R sz[Cfg::SHARED_SCRATCH ? 32 * ((N + 31) / 32) : 1];  // stage increment in and out of the solve
    R p[Cfg::NP > 0 ? Cfg::NP : 1];
    R d[Cfg::ND > 0 ? Cfg::ND : 1];       // drivers of the evaluation
    R dlin[Cfg::ND > 0 ? Cfg::ND : 1];    // drivers at the linearisation point
};

template <class Cfg>
struct WarpCtx {
    using R = typename Cfg::R;
    using C = typename Cfg::C;
    static constexpr int N = Cfg::N, ND = Cfg::ND, L = (Cfg::N + 31) / 32;
    static constexpr bool CACHED = WarpMem<Cfg>::CACHED;
    WarpMem<Cfg>* m;
    int lane;
    const R* coeffs;
    C tol_scale;
    mutable R tlin;

    // every slot is a component when N is a multiple of 32 (the check then
    // folds away from every per-lane loop)
    __device__ __forceinline__ bool valid(int k) const { return (N % 32 == 0) || lane + 32 * k < N; }
    __device__ __forceinline__ void put(R* dst, const R* loc) const {
#pragma unroll
        for (int k = 0; k < L; ++k)
            if (valid(k)) dst[lane + 32 * k] = loc[k];
    }
    __device__ __forceinline__ void get(const R* src, R* loc) const {
#pragma unroll
        for (int k = 0; k < L; ++k) loc[k] = valid(k) ? src[lane + 32 * k] : R(0);
    }
    __device__ __forceinline__ void put_drivers(R* dst, const R* drv) const {
#pragma unroll
        for (int q = 0; q < ND; ++q)
            if (lane == q) dst[q] = drv[q];
    }
    // f(t, y): y and f local.  Every exchange is put -> sync -> class code
    // -> sync -> get: the second sync already orders every lane's reads of
    // the inputs before any later put, and every write of ``out`` comes after
    // the next exchange's first sync, so no sync follows the get.
    __device__ __forceinline__ void rhs(const R* yloc, R t, const R* drv, R* floc) const {
        put(m->ys, yloc);
        put_drivers(m->d, drv);
        __syncwarp();
        Cfg::WSys::template dxdt_lanes<R>(m->ys, m->p, m->d, t, m->out, lane);
        __syncwarp();
        get(m->out, floc);
    }
    __device__ __forceinline__ void linearize(const R* Yloc, R t, const R* drv) const {
        if constexpr (CACHED) {
            R scratch[L];
            rhs_linearize(Yloc, t, drv, scratch);
        } else {
            put(m->ylin, Yloc);
            put_drivers(m->dlin, drv);
            tlin = t;
            __syncwarp();
        }
    }
    // f(t, Y) and the linearisation at Y in one pass: with a cached
    // Jacobian, f and J's coefficients share their subexpressions (the
    // exponentials of a gating rate appear in both).
    __device__ __forceinline__ void rhs_linearize(const R* Yloc, R t, const R* drv, R* floc) const {
        if constexpr (CACHED) {
            put(m->ys, Yloc);
            put_drivers(m->d, drv);
            __syncwarp();
            Cfg::WSys::template fj_lanes<R>(m->ys, m->p, m->d, t, m->out, m->jac, lane);
            __syncwarp();
            get(m->out, floc);
        } else {
            rhs(Yloc, t, drv, floc);
            linearize(Yloc, t, drv);
        }
    }
    // J(y_lin) v: v and the result local.
    __device__ __forceinline__ void jmv(const R* vloc, R* outloc) const {
        put(m->vs, vloc);
        __syncwarp();
        if constexpr (CACHED) {
            Cfg::WSys::template jmv_cached<R>(m->vs, m->jac, m->out, lane);
        } else {
            Cfg::WSys::template jmv_lanes<R>(m->ylin, m->vs, m->p, m->dlin, tlin, m->out, lane);
        }
        __syncwarp();
        get(m->out, outloc);
    }
};

// v - s J(y_lin) v over the warp, with the truncated Neumann preconditioner.
// Its weighted norm reads the Krylov weights 1 / tol_i that the stage solve
// formed once from the stage base (the base is fixed for the whole solve),
// in the working precision.
template <class Cfg>
struct WarpStageOp {
    using R = typename Cfg::R;
    using C = typename Cfg::C;
    static constexpr int K = WarpCtx<Cfg>::L;
    static constexpr int KT = Cfg::N;
    static constexpr bool SHADOW_SHARED = Cfg::SHARED_SCRATCH;
    WarpCtx<Cfg> w;   // by value: no address of the solve's state is taken
    R s;
    __device__ __forceinline__ void apply(const R* v, R* out) const {
        R jv[K];
        w.jmv(v, jv);
#pragma unroll
        for (int i = 0; i < K; ++i) out[i] = v[i] - s * jv[i];
    }
    __device__ __forceinline__ void precond(const R* v, R* out, R* scratch) const {
#pragma unroll
        for (int i = 0; i < K; ++i) out[i] = v[i];
#pragma unroll 1
        for (int k = 0; k < Cfg::PRECOND_ORDER; ++k) {
            w.jmv(out, scratch);
#pragma unroll
            for (int i = 0; i < K; ++i) out[i] = v[i] + s * scratch[i];
        }
    }
    __device__ __forceinline__ C tol(int i) const {
        const int c = w.lane + 32 * i;
        return w.valid(i) ? C(R(1) / w.m->kw[c]) : C(1);
    }
    __device__ __forceinline__ C wnorm2(const R* v) const {
        R s2 = R(0);
#pragma unroll
        for (int i = 0; i < K; ++i) {
            if (w.valid(i)) {
                const R ratio = v[i] * w.m->kw[w.lane + 32 * i];
                s2 += ratio * ratio;
            }
        }
        return C(warp_sum(s2) * (R(1) / R(Cfg::N)));
    }
    // BiCGSTAB's shadow residual in shared memory (shared placement)
    __device__ __forceinline__ R* shadow() const { return w.m->r0; }
    __device__ __forceinline__ int slot(int i) const { return w.lane + 32 * i; }
    template <class T>
    __device__ __forceinline__ T reduce(T partial) const { return warp_sum(partial); }
};

// The per-lane vectors a stage solve starts from, passed by value into the
// out-of-line solve ("registers" placement): no address of the caller's
// arrays crosses the call, so neither they nor the Newton loop's reads of
// them go to local memory, at the price of more live registers around the
// call.
template <class Cfg>
struct WarpStageIn {
    using R = typename Cfg::R;
    static constexpr int L = WarpCtx<Cfg>::L, ND = Cfg::ND;
    R base[L];                    // stage base state
    R start[L];                   // step start state
    R z[L];                       // initial guess of the stage increment
    R drv[ND > 0 ? ND : 1];       // drivers at the stage time
};
template <class Cfg>
struct WarpStageOut {
    using R = typename Cfg::R;
    using C = typename Cfg::C;
    R z[WarpCtx<Cfg>::L];
    C theta;
    int status, newton, krylov;
};

// z = h f(t, base + a z) solved by Newton over the warp (DirkProblem).  The
// base and step-start states are read through ``b(k)`` / ``y0(k)``: from
// shared memory with the "shared" placement, from the problem's own copies
// with "registers", from the caller's arrays (local memory) with "local".
template <class Cfg>
struct WarpDirkProblem {
    using R = typename Cfg::R;
    using C = typename Cfg::C;
    static constexpr int K = WarpCtx<Cfg>::L;
    static constexpr int ND = Cfg::ND;
    static constexpr int KL = Cfg::REG_SCRATCH ? K : 1;
    static constexpr bool FUSED = true;
    WarpCtx<Cfg> w;   // by value: no address of the solve's state is taken
    const R* base_p;
    const R* start_p;
    R base_v[KL];
    R start_v[KL];
    R drv[ND > 0 ? ND : 1];
    R t, h, a;
    __device__ __forceinline__ R b(int k) const {
        if constexpr (Cfg::SHARED_SCRATCH) return w.valid(k) ? w.m->sbase[w.lane + 32 * k] : R(0);
        else if constexpr (Cfg::REG_SCRATCH) return base_v[k];
        else return base_p[k];
    }
    __device__ __forceinline__ R y0(int k) const {
        if constexpr (Cfg::SHARED_SCRATCH) return w.valid(k) ? w.m->sstart[w.lane + 32 * k] : R(0);
        else if constexpr (Cfg::REG_SCRATCH) return start_v[k];
        else return start_p[k];
    }
    __device__ __forceinline__ void residual(const R* z, R* out) const {
        R Y[K], f[K];
#pragma unroll
        for (int k = 0; k < K; ++k) Y[k] = b(k) + a * z[k];
        w.rhs(Y, t, drv, f);
#pragma unroll
        for (int k = 0; k < K; ++k) out[k] = w.valid(k) ? z[k] - h * f[k] : R(0);
    }
    __device__ __forceinline__ void linearize(const R* z) {
        R Y[K];
#pragma unroll
        for (int k = 0; k < K; ++k) Y[k] = b(k) + a * z[k];
        w.linearize(Y, t, drv);
    }
    // residual and linearisation at the same iterate (the Newton loop
    // evaluates both at every iteration)
    __device__ __forceinline__ void residual_linearize(const R* z, R* out) {
        R Y[K], f[K];
#pragma unroll
        for (int k = 0; k < K; ++k) Y[k] = b(k) + a * z[k];
        w.rhs_linearize(Y, t, drv, f);
#pragma unroll
        for (int k = 0; k < K; ++k) out[k] = w.valid(k) ? z[k] - h * f[k] : R(0);
    }
    __device__ __forceinline__ WarpStageOp<Cfg> op() const { return WarpStageOp<Cfg>{w, a * h}; }
    // Krylov weights 1 / max(katol + krtol * scale * |base|, 1e-16), once per
    // stage solve
    __device__ __forceinline__ void form_weights() const {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if (!w.valid(k)) continue;
            const int c = w.lane + 32 * k;
            if constexpr (Cfg::MIXED)
                w.m->kw[c] = R(1) / pymax(R(Cfg::katol(c)) + R(Cfg::krtol(c)) * R(w.tol_scale) * absv(b(k)),
                                          R(1e-16));
            else
                w.m->kw[c] = R(C(1) / krylov_tol<Cfg>(c, b(k), w.tol_scale));
        }
        __syncwarp();
    }
    __device__ __forceinline__ C corr_norm2(const R* delta, const R* z) const {
        C nrm2 = C(0);
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if (!w.valid(k)) continue;
            const int c = w.lane + 32 * k;
            const R sv = b(k) + a * z[k];
            const R ref = pymax(absv(sv), absv(y0(k)));
            const C ratio = tol_ratio<Cfg>(delta[k], ref, Cfg::natol(c), Cfg::nrtol(c), w.tol_scale);
            nrm2 += ratio * ratio;
        }
        return warp_sum(nrm2) * (C(1) / C(Cfg::N));
    }
};

// DIRK step over the warp (DirkStep without dense stage prediction).
template <class Cfg>
struct WarpDirkStep {
    using R = typename Cfg::R;
    using C = typename Cfg::C;
    using Tab = typename Cfg::Tab;
    static constexpr int L = WarpCtx<Cfg>::L, S = Cfg::S, ND = Cfg::ND;
    struct Persist {
        R z[L];
        R rhs[L];
        C theta;
    };
    static __device__ __forceinline__ void init(Persist& ps) {
#pragma unroll
        for (int i = 0; i < L; ++i) {
            ps.z[i] = R(0);
            ps.rhs[i] = R(0);
        }
        ps.theta = C(0);
    }
    // Out of line: one copy of Newton + the Krylov solver serves every stage.
    // Inlined into each unrolled stage, with the class-grouped f and J v
    // bodies inlined at every call site, the 64-compartment cable's kernel
    // held 246 KB of code and instruction fetch bounded it (the same time
    // at 8 and at 12 resident warps per SM); as calls it holds 137 KB and
    // runs 24 % faster.  Moving the operator and norm helpers out of line
    // as well (98 KB) was slower again: their calls pass the per-lane
    // vectors through the stack.
    // The context comes by value: passing the caller's context by reference
    // kept it in local memory, reloaded after every shared-memory store.
    // The stage base, step start and increment cross the call through
    // shared memory ("shared" placement), by address from the caller's
    // arrays ("local": they live in local memory, cached in L1, and the
    // kernel body keeps few registers), or by value with the increment,
    // theta and counts returned by value ("registers": no local memory for
    // them, more live registers around the call).  The autotuner picks.
    static __device__ CBX_NOINLINE int stage_solve(WarpCtx<Cfg> w, const R* base, const R* y, const R* drv_stage,
                                                      R stage_time, R dt, R a, R* z_io, C& theta, int2& iters) {
        WarpDirkProblem<Cfg> prob{w, base, y, {}, {}, {}, stage_time, dt, a};
#pragma unroll
        for (int q = 0; q < ND; ++q) prob.drv[q] = drv_stage[q];
        prob.form_weights();
        R u[L];
#pragma unroll
        for (int k = 0; k < L; ++k) {
            if constexpr (Cfg::SHARED_SCRATCH) u[k] = w.m->sz[w.lane + 32 * k];
            else u[k] = z_io[k];
        }
        C th = theta;
        int ni = 0, ki = 0;
        const int st = newton_solve<Cfg>(prob, u, th, ni, ki);
        theta = th;
#pragma unroll
        for (int k = 0; k < L; ++k) {
            if constexpr (Cfg::SHARED_SCRATCH) w.m->sz[w.lane + 32 * k] = u[k];
            else z_io[k] = u[k];
        }
        iters = make_int2(ni, ki);
        return st;
    }
    static __device__ CBX_NOINLINE WarpStageOut<Cfg> stage_solve_regs(WarpCtx<Cfg> w, WarpStageIn<Cfg> in,
                                                                       R stage_time, R dt, R a, C theta) {
        WarpDirkProblem<Cfg> prob{w, nullptr, nullptr, {}, {}, {}, stage_time, dt, a};
#pragma unroll
        for (int k = 0; k < L; ++k) {
            prob.base_v[k] = in.base[k];
            prob.start_v[k] = in.start[k];
        }
#pragma unroll
        for (int q = 0; q < ND; ++q) prob.drv[q] = in.drv[q];
        prob.form_weights();
        WarpStageOut<Cfg> out;
#pragma unroll
        for (int k = 0; k < L; ++k) out.z[k] = in.z[k];
        out.theta = theta;
        out.newton = 0;
        out.krylov = 0;
        out.status = newton_solve<Cfg>(prob, out.z, out.theta, out.newton, out.krylov);
        return out;
    }
    static __device__ __forceinline__ int solve_stage(WarpCtx<Cfg>& w, const R* base, const R* y,
                                                      const R* drv_stage, R stage_time, R dt, R a, Persist& ps,
                                                      Iters& its) {
        int ni, ki, st;
        if constexpr (Cfg::REG_SCRATCH) {
            WarpStageIn<Cfg> in;
#pragma unroll
            for (int k = 0; k < L; ++k) {
                in.base[k] = base[k];
                in.start[k] = y[k];
                in.z[k] = ps.z[k];
            }
#pragma unroll
            for (int q = 0; q < ND; ++q) in.drv[q] = drv_stage[q];
            const WarpStageOut<Cfg> out = stage_solve_regs(w, in, stage_time, dt, a, ps.theta);
#pragma unroll
            for (int k = 0; k < L; ++k) ps.z[k] = out.z[k];
            ps.theta = out.theta;
            st = out.status;
            ni = out.newton;
            ki = out.krylov;
        } else {
            int2 it2;
            if constexpr (Cfg::SHARED_SCRATCH) {
                w.put(w.m->sbase, base);
                w.put(w.m->sz, ps.z);
                st = stage_solve(w, nullptr, nullptr, drv_stage, stage_time, dt, a, nullptr, ps.theta, it2);
                w.get(w.m->sz, ps.z);
            } else {
                st = stage_solve(w, base, y, drv_stage, stage_time, dt, a, ps.z, ps.theta, it2);
            }
            ni = it2.x;
            ki = it2.y;
        }
        its.nit = ni;
        its.kit = ki;
        its.nit_all += ni;
        its.kit_all += ki;
        return st;
    }
    static __device__ __forceinline__ int step(WarpCtx<Cfg>& w, const R* y, R* ynew, R* delta, R* err,
                                               const R* drv, R* drv_new, R dt, R t, bool first_step,
                                               bool prev_accepted, Persist& ps, Iters& its) {
        its = Iters{};
        int status = SUCCESS;
        const bool use_cached = Tab::FSAL && (S > 1) && !first_step && prev_accepted;
        if constexpr (Cfg::SHARED_SCRATCH) w.put(w.m->sstart, y);
        R base[L], outacc[L], erracc[L];
        R acc[(S > 1 ? S - 1 : 1)][L];
        R drv_stage[ND > 0 ? ND : 1];
#pragma unroll
        for (int i = 0; i < L; ++i) {
            base[i] = y[i];
            outacc[i] = R(0);
            erracc[i] = R(0);
        }
#pragma unroll
        for (int r = 0; r < S - 1; ++r)
#pragma unroll
            for (int i = 0; i < L; ++i) acc[r][i] = R(0);
        R stage_time = t + dt * R(Tab::c(0));
        if (!use_cached) {
            if constexpr (ND > 0) {
                if (Tab::c(0) == 0.0) {
#pragma unroll
                    for (int q = 0; q < ND; ++q) drv_stage[q] = drv[q];
                } else {
                    Drivers<Cfg>::eval(stage_time, w.coeffs, drv_stage);
                }
            }
            if (Tab::a(0, 0) != 0.0) {
                status |= solve_stage(w, base, y, drv_stage, stage_time, dt, R(Tab::a(0, 0)), ps, its);
#pragma unroll
                for (int i = 0; i < L; ++i) base[i] += R(Tab::a(0, 0)) * ps.z[i];
            }
            if (Tab::need_f(0)) w.rhs(base, stage_time, drv_stage, ps.rhs);
        }
#pragma unroll
        for (int i = 0; i < L; ++i) {
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
                    for (int i = 0; i < L; ++i) acc[succ][i] += R(coeff) * ps.rhs[i];
                }
            }
            stage_time = t + dt * R(Tab::c(stage));
            if constexpr (ND > 0) Drivers<Cfg>::eval(stage_time, w.coeffs, drv_stage);
            R stage_delta[L];
#pragma unroll
            for (int i = 0; i < L; ++i) {
                stage_delta[i] = acc[prev][i] * dt;
                base[i] = stage_delta[i] + y[i];
            }
            if (Tab::a(stage, stage) != 0.0) {
                if (Tab::EULER_GUESS && Tab::a(prev, prev) == 0.0) {
#pragma unroll
                    for (int i = 0; i < L; ++i) ps.z[i] = dt * ps.rhs[i];
                }
                status |= solve_stage(w, base, y, drv_stage, stage_time, dt, R(Tab::a(stage, stage)), ps, its);
#pragma unroll
                for (int i = 0; i < L; ++i) {
                    base[i] += R(Tab::a(stage, stage)) * ps.z[i];
                    stage_delta[i] += R(Tab::a(stage, stage)) * ps.z[i];
                }
            }
            if (Tab::need_f(stage)) w.rhs(base, stage_time, drv_stage, ps.rhs);
#pragma unroll
            for (int i = 0; i < L; ++i) {
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
        for (int i = 0; i < L; ++i) {
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
            if (!w.valid(i)) {
                ynew[i] = R(0);
                delta[i] = R(0);
                err[i] = R(0);
            }
        }
        if constexpr (ND > 0) Drivers<Cfg>::eval(t + dt, w.coeffs, drv_new);
        return status;
    }
};

template <class Cfg>
struct WarpLane {
    using R = typename Cfg::R;
    using C = typename Cfg::C;
    using Ctl = Controller<Cfg>;
    static constexpr int L = WarpCtx<Cfg>::L, ND = Cfg::ND;
    static constexpr int SK = (Cfg::N_SUMM_STATES + 31) / 32;  // summarised variables per lane
    static constexpr int SB = SK * Cfg::Summ::BUF;
    long long run;
    double t;
    C tp, t_end;
    double save_stop, summary_stop;
    C dt, dt_raw, next_save, next_update;
    R y[L];
    R comp[L];
    R drv[ND > 0 ? ND : 1];
    R sbuf[SB > 0 ? SB : 1];
    int counters[4];
    int save_idx, summary_idx, update_idx;
    int status, iteration_status, stagnant;
    bool first_step, prev_accepted, irrecoverable;
    long long steps, rejections, newton, krylov;
    typename Ctl::State ctl;
    typename WarpDirkStep<Cfg>::Persist ps;
};

template <class Cfg>
__device__ __forceinline__ void warp_save_row(const WarpLane<Cfg>& L, WarpCtx<Cfg>& w, const cbx_solve_args& a) {
    using R = typename Cfg::R;
    const int row = L.save_idx;
    if (row >= a.n_save_rows) return;
    const long long s = a.run_stride;
    if constexpr (Cfg::SAVE_STATE || Cfg::SAVE_TIME) {
        constexpr int W = Cfg::N_SAVED_STATES + (Cfg::SAVE_TIME ? 1 : 0);
        R* out = static_cast<R*>(a.state_out) + (long long)row * W * s + L.run;
        if constexpr (Cfg::SAVE_STATE) {
            w.put(w.m->ys, L.y);
            __syncwarp();
            for (int k = w.lane; k < Cfg::N_SAVED_STATES; k += 32) out[k * s] = w.m->ys[Cfg::Idx::saved_state(k)];
            __syncwarp();
        }
        if constexpr (Cfg::SAVE_TIME) {
            if (w.lane == 0) out[Cfg::N_SAVED_STATES * s] = R(L.tp);
        }
    }
    if constexpr (Cfg::SAVE_COUNTERS) {
        int* out = a.counters_out + (long long)row * 4 * s + L.run;
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (w.lane == k) out[k * s] = L.counters[k];
    }
}

template <class Cfg>
__device__ __forceinline__ void warp_update_summaries(WarpLane<Cfg>& L, WarpCtx<Cfg>& w) {
    using Summ = typename Cfg::Summ;
    w.put(w.m->ys, L.y);
    __syncwarp();
#pragma unroll
    for (int kk = 0; kk < WarpLane<Cfg>::SK; ++kk) {
        const int sv = w.lane + 32 * kk;
        if (Cfg::N_SUMM_STATES % 32 == 0 || sv < Cfg::N_SUMM_STATES)
            Summ::update(w.m->ys[Cfg::Idx::summ_state(sv)], L.sbuf + kk * Summ::BUF, L.update_idx);
    }
    __syncwarp();
}

template <class Cfg>
__device__ __forceinline__ void warp_save_summaries(WarpLane<Cfg>& L, WarpCtx<Cfg>& w, const cbx_solve_args& a) {
    using R = typename Cfg::R;
    using Summ = typename Cfg::Summ;
    const int row = L.summary_idx;
    const bool in_range = row < a.n_summary_rows;
    const long long s = a.run_stride;
    R vals[Summ::OUT > 0 ? Summ::OUT : 1];
#pragma unroll
    for (int kk = 0; kk < WarpLane<Cfg>::SK; ++kk) {
        const int sv = w.lane + 32 * kk;
        if (Cfg::N_SUMM_STATES % 32 == 0 || sv < Cfg::N_SUMM_STATES) {
            Summ::save(L.sbuf + kk * Summ::BUF, vals, Cfg::SAMPLES_PER_SUMMARY);
            if (in_range) {
                R* out = static_cast<R*>(a.state_sum_out) +
                         ((long long)row * Cfg::N_SUMM_STATES * Summ::OUT + sv * Summ::OUT) * s + L.run;
#pragma unroll
                for (int q = 0; q < Summ::OUT; ++q) out[q * s] = vals[q];
            }
        }
    }
}

template <class Cfg>
__device__ __forceinline__ void warp_begin(WarpLane<Cfg>& L, WarpCtx<Cfg>& w, const cbx_solve_args& a,
                                           long long run) {
    using R = typename Cfg::R;
    using C = typename Cfg::C;
    constexpr int NL = WarpCtx<Cfg>::L, NP = Cfg::NP;
    L.run = run;
    const double duration = a.durations ? a.durations[run] : a.duration;
    w.tol_scale = a.tol_scale ? C(a.tol_scale[run]) : C(1);
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
    for (int k = 0; k < NL; ++k) {
        const int c = w.lane + 32 * k;
        L.y[k] = c < Cfg::N ? inits[c * a.run_stride + run] : R(0);
        L.comp[k] = R(0);
    }
#pragma unroll
    for (int q = 0; q < NP; ++q)
        if (w.lane == q) w.m->p[q] = params[q * a.run_stride + run];
    __syncwarp();
#pragma unroll
    for (int k = 0; k < WarpLane<Cfg>::SB; ++k) L.sbuf[k] = R(0);
    if constexpr (Cfg::ND > 0) Drivers<Cfg>::eval(R(L.tp), w.coeffs, L.drv);
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
        warp_save_row<Cfg>(L, w, a);
        L.save_idx += 1;
        if (Cfg::SUMMARISE) warp_save_summaries<Cfg>(L, w, a);
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
    WarpDirkStep<Cfg>::init(L.ps);
}

// One step attempt of the warp's run (lane_iterate over the warp).  Returns
// true when the run is finished.
template <class Cfg>
__device__ __forceinline__ bool warp_iterate(WarpLane<Cfg>& L, WarpCtx<Cfg>& w, const cbx_solve_args& a) {
    using R = typename Cfg::R;
    using C = typename Cfg::C;
    constexpr int NL = WarpCtx<Cfg>::L, ND = Cfg::ND;

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
    if (a.max_steps > 0 && L.steps >= a.max_steps) {
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

    R ynew[NL], delta[NL], err[NL];
    R drv_new[ND > 0 ? ND : 1];
    Iters its;
    const int step_status = WarpDirkStep<Cfg>::step(w, L.y, ynew, delta, err, L.drv, drv_new, R(dt_eff), R(L.tp),
                                                    L.first_step, L.prev_accepted, L.ps, its);
    const int nit = its.nit, kit = its.kit;
    L.first_step = false;
    L.iteration_status |= step_status;
    const bool step_failed = step_status != SUCCESS;
    L.irrecoverable = L.irrecoverable || (!Cfg::ADAPTIVE && step_failed);
    bool accept;
    if constexpr (Cfg::ADAPTIVE) {
        // error norm over the warp (Controller::error_norm2): ratios in the
        // gain precision G, their squares summed in the control precision
        using G = typename Cfg::G;
        using Ctl = Controller<Cfg>;
        C nrm2 = C(0);
        const G ts = G(w.tol_scale);
#pragma unroll
        for (int i = 0; i < NL; ++i) {
            if (!w.valid(i)) continue;
            const int c = w.lane + 32 * i;
            const R e = step_failed ? R(1e16) : err[i];
            const C ratio = C(Ctl::error_ratio(e, ynew[i], L.y[i], G(Cfg::atol(c)), G(Cfg::rtol(c)), ts));
            nrm2 += ratio * ratio;
        }
        nrm2 = warp_sum(nrm2) * C(Cfg::CTL_INV_N);
        bool ctl_accept = false;
        const int ctl_status = Controller<Cfg>::update_with_norm(L.dt, nrm2, nit, truncated, ctl_accept, L.ctl);
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
        L.t = t_proposal;
        L.tp = C(L.t);
        if (Cfg::MIXED) {
#pragma unroll
            for (int i = 0; i < NL; ++i) {
                const R z = delta[i] + L.comp[i];
                const R ys = L.y[i] + z;
                L.comp[i] = z - (ys - L.y[i]);
                L.y[i] = ys;
            }
        } else {
#pragma unroll
            for (int i = 0; i < NL; ++i) L.y[i] = ynew[i];
        }
        if constexpr (ND > 0) {
#pragma unroll
            for (int q = 0; q < ND; ++q) L.drv[q] = drv_new[q];
        }
    }
    L.prev_accepted = accept;
    do_save = do_save && accept;
    do_update = do_update && accept;
    if (do_save) {
        if (Cfg::SAVE_REG) L.next_save += C(Cfg::SAVE_EVERY);
        warp_save_row<Cfg>(L, w, a);
        L.save_idx += 1;
        if (Cfg::SAVE_COUNTERS) {
#pragma unroll
            for (int k = 0; k < 4; ++k) L.counters[k] = 0;
        }
    }
    if (do_update) {
        if (Cfg::SUMM_REG) L.next_update += C(Cfg::SAMPLE_EVERY);
        if (Cfg::SUMMARISE) {
            warp_update_summaries<Cfg>(L, w);
            L.update_idx += 1;
            if (L.update_idx % Cfg::SAMPLES_PER_SUMMARY == 0) {
                warp_save_summaries<Cfg>(L, w, a);
                L.summary_idx += 1;
            }
        }
    }
    return false;
}

// Persistent warp-per-run kernel: every warp claims one run at a time.
template <class Cfg>
__device__ __forceinline__ void run_warp(const cbx_solve_args& a) {
    using R = typename Cfg::R;
    // the warps' WarpMem records live in dynamic shared memory (their size,
    // BLOCK / 32 records, is published as the size of cbx_warp_smem_probe
    // and passed by the launch), so large records are not held to the
    // 48 KB limit of static shared memory
    extern __shared__ __align__(16) unsigned char cbx_dyn_smem[];
    WarpMem<Cfg>* mem = reinterpret_cast<WarpMem<Cfg>*>(cbx_dyn_smem);
    __shared__ BlockTotals bt;
    totals_begin(&bt);
    const int lane = threadIdx.x & 31;
    WarpCtx<Cfg> w{&mem[threadIdx.x >> 5], lane, static_cast<const R*>(a.driver_coeffs), typename Cfg::C(1), R(0)};
    while (true) {
        unsigned long long r = 0;
        if (lane == 0) r = atomicAdd(a.work_counter, 1ull);
        r = __shfl_sync(kWarpFull, r, 0);
        if ((long long)r >= a.n_runs) break;
        WarpLane<Cfg> L;
        warp_begin<Cfg>(L, w, a, a.run_order ? a.run_order[r] : (long long)r);
        while (!warp_iterate<Cfg>(L, w, a)) {
        }
        if (lane == 0) {
            a.status_out[L.run] = L.status;
            if (a.totals) {
                atomicAdd(bt.v + 0, (unsigned long long)L.steps);
                atomicAdd(bt.v + 1, (unsigned long long)L.rejections);
                atomicAdd(bt.v + 2, (unsigned long long)L.newton);
                atomicAdd(bt.v + 3, (unsigned long long)L.krylov);
            }
        }
    }
    totals_flush(&bt, a);
}

}  // namespace cbx

#define CBX_DEFINE_WARP_KERNEL(CFG)                                                                  \
    extern "C" __device__ char cbx_warp_smem_probe[sizeof(cbx::WarpMem<CFG>) * (CFG::BLOCK / 32)];      \
    extern "C" __global__ void __launch_bounds__(CFG::BLOCK) cbx_integrate_warp(cbx_solve_args a) {    \
        cbx::run_warp<CFG>(a);                                                                         \
    }
