// Operators, preconditioners, norms and the damped Newton iteration used by
// the implicit steps.  One system per thread; vectors live in registers.
#pragma once
#include "cbx_common.cuh"
#include "cbx_linear.cuh"

namespace cbx {

// Tolerance helpers over the generated __constant__ arrays.  Solver vectors
// of width S*N reuse the per-state entries stage by stage (the reference
// broadcasts tolerance arrays to the solver width, norms.py:275-324).
template <class Cfg>
__device__ __forceinline__ typename Cfg::C krylov_tol(int i, typename Cfg::R ref, typename Cfg::C scale) {
    using C = typename Cfg::C;
    const int k = i % Cfg::N;
    C t = C(Cfg::katol(k)) + C(Cfg::krtol(k)) * scale * C(absv(ref));
    return pymax(t, C(1e-16));
}

// One component's ratio v / max(atol + rtol scale |ref|, 1e-16) of a
// tolerance-weighted norm; the caller sums the squares in the control
// precision C.  On the mixed-precision path the ratio is formed in FP32:
// v and ref are FP32 values, so the ratio carries no more information in
// FP64, and an FP64 division per component costs more issue slots (and
// code) than the rest of the norm.  Otherwise it is formed in C, in the
// reference's order of operations.
template <class Cfg>
__device__ __forceinline__ typename Cfg::C tol_ratio(typename Cfg::R v, typename Cfg::R ref, double atol,
                                                     double rtol, typename Cfg::C scale) {
    using R = typename Cfg::R;
    using C = typename Cfg::C;
    if constexpr (Cfg::MIXED) {
        const R tol = pymax(R(atol) + R(rtol) * R(scale) * absv(ref), R(1e-16));
        return C(v / tol);
    } else {
        C tol = C(atol) + C(rtol) * scale * C(absv(ref));
        tol = pymax(tol, C(1e-16));
        return C(v) / tol;
    }
}

template <class Cfg, int K>
__device__ __forceinline__ typename Cfg::C weighted_norm2(const typename Cfg::R* v, const typename Cfg::R* ref,
                                                          typename Cfg::C scale) {
    using C = typename Cfg::C;
    C nrm2 = C(0);
#pragma unroll
    for (int i = 0; i < K; ++i) {
        const int k = i % Cfg::N;
        const C ratio = tol_ratio<Cfg>(absv(v[i]), ref[k], Cfg::katol(k), Cfg::krtol(k), scale);
        nrm2 += ratio * ratio;
    }
    return nrm2 * (C(1) / C(K));
}

template <class Cfg, class Op>
__device__ __forceinline__ int linear_solve(const Op& op, typename Cfg::R* rhs, typename Cfg::R* x, int& iters) {
    if constexpr (Cfg::LIN == LIN_BICGSTAB) {
        return solve_bicgstab<Cfg, Op>(op, rhs, x, iters);
    } else if constexpr (Cfg::LIN == LIN_GMRES) {
        return solve_gmres<Cfg, Op>(op, rhs, x, iters);
    } else if constexpr (Cfg::LIN == LIN_DIRECT) {
        return solve_direct<Cfg, Op>(op, rhs, x, iters);
    } else {
        return solve_mr<Cfg, Op, Cfg::LIN == LIN_SD>(op, rhs, x, iters);
    }
}

// Single-stage operator A v = M v - s J v with a Jacobian fixed for the solve
// (Rosenbrock: J at the step start and s = gamma h; DIRK Newton: J at
// base + a_ii z and s = a_ii h).  Matches the generated operator
// beta M v - gamma a_ij h J v with beta = 1, M the system's constant mass
// matrix or the identity (codegen/linear_operators.py:80-177) and the
// truncated Neumann
// preconditioner out <- v + s J out repeated ``order`` times
// (codegen/preconditioners.py:85-200).
template <class Cfg>
struct SingleStageOp {
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
        Sys::template jmv<R>(J, v, jv);
        if constexpr (Sys::HAS_MASS) {
            R mv[K];
            Sys::template mass_mv<R>(v, mv);
#pragma unroll
            for (int i = 0; i < K; ++i) out[i] = mv[i] - s * jv[i];
        } else {
#pragma unroll
            for (int i = 0; i < K; ++i) out[i] = v[i] - s * jv[i];
        }
    }
    __device__ __forceinline__ void precond(const R* v, R* out, R* scratch) const {
#pragma unroll
        for (int i = 0; i < K; ++i) out[i] = v[i];
#pragma unroll 1
        for (int k = 0; k < Cfg::PRECOND_ORDER; ++k) {
            Sys::template jmv<R>(J, out, scratch);
#pragma unroll
            for (int i = 0; i < K; ++i) out[i] = v[i] + s * scratch[i];
        }
    }
    __device__ __forceinline__ C tol(int i) const { return krylov_tol<Cfg>(i, ref[i], scale); }
    __device__ __forceinline__ C wnorm2(const R* v) const { return weighted_norm2<Cfg, K>(v, ref, scale); }
    template <class T> __device__ __forceinline__ T reduce(T partial) const { return partial; }
    static constexpr int KT = K;
};

// Coupled S-stage operator (A v)_i = v_i - h J_i sum_j a_ij v_j with J_i the
// Jacobian at stage state i (codegen/linear_operators.py:600-700 n-stage
// operator) and its Neumann preconditioner with h_eff = h
// (codegen/preconditioners.py:187-235).
template <class Cfg>
struct CoupledOp {
    using R = typename Cfg::R;
    using C = typename Cfg::C;
    using Sys = typename Cfg::Sys;
    static constexpr int N = Cfg::N;
    static constexpr int S = Cfg::S;
    static constexpr int K = S * N;
    const R (*J)[Sys::NJ];
    R h;
    const R* ref;
    C scale;
    __device__ __forceinline__ void couple_jv(const R* v, R* out) const {
#pragma unroll
        for (int i = 0; i < S; ++i) {
            R w[N];
#pragma unroll
            for (int k = 0; k < N; ++k) {
                R acc = R(0);
#pragma unroll
                for (int j = 0; j < S; ++j)
                    if (Cfg::Tab::a(i, j) != 0.0) acc += R(Cfg::Tab::a(i, j)) * v[j * N + k];
                w[k] = acc;
            }
            Sys::template jmv<R>(J[i], w, out + i * N);
        }
    }
    __device__ __forceinline__ void apply(const R* v, R* out) const {
        R jv[K];
        couple_jv(v, jv);
        if constexpr (Sys::HAS_MASS) {
            // M v_i - h J_i sum_j a_ij v_j per stage block
            // (linear_operators.py:708-735)
#pragma unroll
            for (int i = 0; i < S; ++i) {
                R mv[N];
                Sys::template mass_mv<R>(v + i * N, mv);
#pragma unroll
                for (int k = 0; k < N; ++k) out[i * N + k] = mv[k] - h * jv[i * N + k];
            }
        } else {
#pragma unroll
            for (int i = 0; i < K; ++i) out[i] = v[i] - h * jv[i];
        }
    }
    __device__ __forceinline__ void precond(const R* v, R* out, R* scratch) const {
#pragma unroll
        for (int i = 0; i < K; ++i) out[i] = v[i];
#pragma unroll 1
        for (int k = 0; k < Cfg::PRECOND_ORDER; ++k) {
            couple_jv(out, scratch);
#pragma unroll
            for (int i = 0; i < K; ++i) out[i] = v[i] + h * scratch[i];
        }
    }
    __device__ __forceinline__ C tol(int i) const { return krylov_tol<Cfg>(i, ref[i % N], scale); }
    __device__ __forceinline__ C wnorm2(const R* v) const { return weighted_norm2<Cfg, K>(v, ref, scale); }
    template <class T> __device__ __forceinline__ T reduce(T partial) const { return partial; }
    static constexpr int KT = K;
};

// Problems whose residual and linearisation share work at one iterate
// (``FUSED``) provide residual_linearize(u, out) in place of the two calls.
template <class P, class = void> struct HasFused { static constexpr bool value = false; };
template <class P> struct HasFused<P, decltype(void(P::FUSED))> { static constexpr bool value = P::FUSED; };

// Damped Newton iteration with NLNewton-style acceptance
// (newton_krylov.py:340-517): contraction estimate theta carried between
// solves, acceptance eta*||dz|| < kappa (kappa = 0.01), a first-iteration
// bound ||dz|| < 1e-5, divergence when theta > 2 or the update norm is not
// finite, and a stagnation band |theta - 1| <= 100 sqrt(eps).
//
// ``Prob`` supplies: K, residual(u, out) (out = u - h f(...)),
// linearize(u) (fixes the Jacobians for the linear solve), op(), and
// corr_norm2(delta, u) (the correction norm).
template <class Cfg, class Prob>
__device__ __forceinline__ int newton_solve(Prob& prob, typename Cfg::R* u, typename Cfg::C& prev_theta_store,
                                            int& newton_iters, int& krylov_iters) {
    using R = typename Cfg::R;
    using C = typename Cfg::C;
    constexpr int K = Prob::K;
    const C kappa = C(0.01);
    const C first_bound = C(1.0e-5);
    const C theta_decay = C(0.3);
    const C theta_div = C(2.0);
    const C stag_eps = C(100.0) * sqrt_t(C(Limits<R>::eps()));
    const C huge = C(Limits<R>::huge());
    C prev_theta = (prev_theta_store > C(0)) ? prev_theta_store : C(1);
    C ndz_prev = C(0);
    bool converged = false, failed = false;
    int last_lin = SUCCESS;
    int iters = 0, total_k = 0;
    R res[K], delta[K];
    for (int it = 0; it < Cfg::NEWTON_MAX_ITERS; ++it) {
        if (converged || failed) break;
        if constexpr (HasFused<Prob>::value) prob.residual_linearize(u, res);
        else prob.residual(u, res);
#pragma unroll
        for (int i = 0; i < K; ++i) {
            res[i] = -res[i];
            delta[i] = R(0);
        }
        if constexpr (!HasFused<Prob>::value) prob.linearize(u);
        int kit = 0;
        const int lin = linear_solve<Cfg>(prob.op(), res, delta, kit);
        total_k += kit;
        last_lin = lin;
        ++iters;
        const C norm2_dz = prob.corr_norm2(delta, u);
        const C ndz = sqrt_t(norm2_dz);
        const bool judged = (lin == SUCCESS);
        const bool history = ndz_prev > C(0);
        const C ndz_prev_safe = history ? ndz_prev : C(1);
        const C theta = history ? pymax(theta_decay * prev_theta, ndz / ndz_prev_safe) : prev_theta;
        const bool small_first = (iters == 1) && (ndz < first_bound);
        const bool eta_accept = (theta < C(1)) && (theta * ndz < kappa * (C(1) - theta));
        const bool nonfinite = !(norm2_dz <= huge);
        const bool stagnant = judged && history && (absv(theta - C(1)) <= stag_eps);
        const bool diverging = judged && ((history && theta > theta_div) || nonfinite);
        const bool converged_stagnant = stagnant && (ndz <= C(1)) && !diverging;
        const bool failed_now = diverging || (stagnant && ndz > C(1));
        failed = failed || failed_now;
        const bool commit = judged && !failed_now && !converged_stagnant;
        if (commit) {
#pragma unroll
            for (int i = 0; i < K; ++i) u[i] = u[i] + delta[i];
        }
        converged = converged || converged_stagnant || (commit && (eta_accept || small_first));
        ndz_prev = commit ? ndz : C(0);
        prev_theta = (judged && history) ? theta : prev_theta;
    }
    prev_theta_store = converged ? prev_theta : C(1);
    int fail_bits = failed ? NEWTON_DIVERGENCE : MAX_NEWTON_ITERATIONS_EXCEEDED;
    if (last_lin != SUCCESS) fail_bits |= last_lin;
    newton_iters = iters;
    krylov_iters = total_k;
    return converged ? SUCCESS : fail_bits;
}

}  // namespace cbx
