// Matrix-free Krylov solvers for one system per thread.
//
// Each solver works on an operator object ``Op`` that provides
//   static constexpr int K;                       // solver width
//   void apply(const R* v, R* out) const;         // out = A v
//   void precond(const R* v, R* out, R* scratch) const;  // out ~= A^-1 v
//   C    wnorm2(const R* v) const;                // weighted mean-square norm
//   C    tol(int i) const;                        // weight denominator of wnorm2
//   T    reduce(T partial) const;                 // sum of a per-holder partial
//   static constexpr int KT;                      // total width (K summed over holders)
// where an operator held by one thread has K = system width and an
// identity ``reduce``, and an operator whose vectors are spread over a warp
// has K = components per lane and sums the lanes' partials.
// where wnorm2(v) = mean_i (|v_i| / tol(i))^2 is the reference's scaled
// norm (src/cubie/integrators/norms.py:165-196) with the Krylov atol/rtol.
//
// Stopping rule of every solver: ||r|| <= floor + reduction * ||b|| in that
// norm, fixed against the untouched right-hand side
// (src/cubie/integrators/matrix_free_solvers/linear_solver.py:291-298).
#pragma once
#include "cbx_common.cuh"

namespace cbx {

// Preconditioned minimal-residual / steepest-descent iteration.
// Follows MRLinearSolver (linear_solver.py:220-385): one operator and one
// preconditioner application per iteration, x and r updated with
// alpha = <t,r>/<t,t> (MR) or <r,z>/<t,z> (SD).  ``rhs`` is overwritten
// with the running residual and ``x`` holds the initial guess on entry.
template <class Cfg, class Op, bool SD>
__device__ __forceinline__ int solve_mr(const Op& op, typename Cfg::R* rhs,
                                        typename Cfg::R* x, int& iters) {
    using R = typename Cfg::R;
    using C = typename Cfg::C;
    constexpr int K = Op::K;
    const C rhs_norm2 = op.wnorm2(rhs);
    const C tol = C(Cfg::KRYLOV_FLOOR) + C(Cfg::KRYLOV_REDUCTION) * sqrt_t(rhs_norm2);
    const C tol2 = tol * tol;
    R z[K];
    R tmp[K];
    op.apply(x, tmp);
#pragma unroll
    for (int i = 0; i < K; ++i) rhs[i] = rhs[i] - tmp[i];
    C acc = op.wnorm2(rhs);
    bool converged = acc <= tol2;
    int it = 0;
    for (int k = 0; k < Cfg::KRYLOV_MAX_ITERS; ++k) {
        if (converged) break;
        ++it;
        if (Cfg::PRECONDITIONED) {
            op.precond(rhs, z, tmp);
        } else {
#pragma unroll
            for (int i = 0; i < K; ++i) z[i] = rhs[i];
        }
        op.apply(z, tmp);
        C num = C(0), den = C(0);
#pragma unroll
        for (int i = 0; i < K; ++i) {
            if (SD) {
                num += C(rhs[i]) * C(z[i]);
                den += C(tmp[i]) * C(z[i]);
            } else {
                num += C(tmp[i]) * C(rhs[i]);
                den += C(tmp[i]) * C(tmp[i]);
            }
        }
        num = op.reduce(num);
        den = op.reduce(den);
        const R alpha = (den != C(0)) ? R(num / den) : R(0);
#pragma unroll
        for (int i = 0; i < K; ++i) {
            x[i] += alpha * z[i];
            rhs[i] -= alpha * tmp[i];
        }
        acc = op.wnorm2(rhs);
        converged = converged || (acc <= tol2);
    }
    iters = it;
    return converged ? SUCCESS : MAX_LINEAR_ITERATIONS_EXCEEDED;
}

// Operators may keep BiCGSTAB's shadow residual in shared memory
// (``SHADOW_SHARED``, with ``shadow()`` and ``slot(i)`` giving its storage);
// by default it is a register array.
template <class Op, class = void> struct ShadowShared { static constexpr bool value = false; };
template <class Op> struct ShadowShared<Op, decltype(void(Op::SHADOW_SHARED))> {
    static constexpr bool value = Op::SHADOW_SHARED;
};

template <class R> __device__ __forceinline__ R clampd(R v, R lim) {
    v = (v > lim) ? lim : v;
    return (v < -lim) ? -lim : v;
}

// Preconditioned BiCGSTAB with the reference's breakdown and overflow
// guards (bicgstab_solver.py:367-663): clamps every vector element and
// product to +-dot_clamp, flags BICGSTAB_BREAKDOWN when rho or omega
// collapse (1e-30 in float32, 1e-200 in float64) or a recurrence quotient
// would leave the clamp budget.
template <class Cfg, class Op>
__device__ __forceinline__ int solve_bicgstab(const Op& op, typename Cfg::R* rhs,
                                              typename Cfg::R* x, int& iters) {
    using R = typename Cfg::R;
    using C = typename Cfg::C;
    constexpr int K = Op::K;
    constexpr bool F32 = sizeof(R) == 4;
    const R tiny = F32 ? R(1e-30) : R(1e-200);
    const R lim = F32 ? R(1e16) : R(1e150);
    constexpr bool SHS = ShadowShared<Op>::value;
    R r0[SHS ? 1 : K], p[K], v[K], tmp[K], sh[K];
    R* r0s = nullptr;
    if constexpr (SHS) r0s = op.shadow();
    auto shadow_at = [&](int i) -> R {
        if constexpr (SHS) return r0s[op.slot(i)];
        else return r0[i];
    };

    const C rhs_norm2 = op.wnorm2(rhs);
    const C tol = C(Cfg::KRYLOV_FLOOR) + C(Cfg::KRYLOV_REDUCTION) * sqrt_t(rhs_norm2);
    const C tol2 = tol * tol;
    op.apply(x, tmp);
    R rho_prev = R(0);
#pragma unroll
    for (int i = 0; i < K; ++i) {
        const R ax = clampd(tmp[i], lim);
        const R ri = rhs[i] - ax;
        rhs[i] = ri;
        if constexpr (SHS) r0s[op.slot(i)] = ri;
        else r0[i] = ri;
        p[i] = clampd(ri, lim);
        R sq = ri * ri;
        sq = (sq > lim) ? lim : sq;
        rho_prev += sq;
    }
    rho_prev = op.reduce(rho_prev);
    C acc = op.wnorm2(rhs);
    bool converged = acc <= tol2;
    bool broken = false;
    bool finished = converged;
    int it = 0;
    for (int k = 0; k < Cfg::KRYLOV_MAX_ITERS; ++k) {
        if (finished) break;
        ++it;
        if (Cfg::PRECONDITIONED) {
            op.precond(p, tmp, v);
#pragma unroll
            for (int i = 0; i < K; ++i) tmp[i] = clampd(tmp[i], lim);
        } else {
#pragma unroll
            for (int i = 0; i < K; ++i) tmp[i] = p[i];
        }
        op.apply(tmp, v);
        R dot_r0v = R(0);
#pragma unroll
        for (int i = 0; i < K; ++i) {
            v[i] = clampd(v[i], lim);
            dot_r0v += clampd(shadow_at(i) * v[i], lim);
        }
        dot_r0v = op.reduce(dot_r0v);
        const bool alpha_overflow = absv(rho_prev) > absv(dot_r0v) * lim;
        broken = broken || alpha_overflow;
        finished = converged || broken;
        const R alpha = (dot_r0v != R(0) && !alpha_overflow) ? rho_prev / dot_r0v : R(0);
        const R alpha_eff = finished ? R(0) : alpha;
#pragma unroll
        for (int i = 0; i < K; ++i) {
            x[i] = x[i] + alpha_eff * tmp[i];
            rhs[i] = rhs[i] - alpha_eff * v[i];
        }
        acc = op.wnorm2(rhs);
        converged = converged || (acc <= tol2);
        finished = converged || broken;
        if (Cfg::PRECONDITIONED) {
            op.precond(rhs, sh, tmp);
#pragma unroll
            for (int i = 0; i < K; ++i) sh[i] = clampd(sh[i], lim);
        } else {
#pragma unroll
            for (int i = 0; i < K; ++i) sh[i] = clampd(rhs[i], lim);
        }
        op.apply(sh, tmp);
        R dot_ts = R(0), dot_tt = R(0);
#pragma unroll
        for (int i = 0; i < K; ++i) {
            tmp[i] = clampd(tmp[i], lim);
            dot_ts += clampd(tmp[i] * rhs[i], lim);
            R sq = tmp[i] * tmp[i];
            dot_tt += (sq > lim) ? lim : sq;
        }
        dot_ts = op.reduce(dot_ts);
        dot_tt = op.reduce(dot_tt);
        const bool omega_overflow = absv(dot_ts) > dot_tt * lim;
        const R omega = (dot_tt != R(0) && !omega_overflow) ? dot_ts / dot_tt : R(0);
        const R omega_eff = finished ? R(0) : omega;
#pragma unroll
        for (int i = 0; i < K; ++i) {
            x[i] = x[i] + omega_eff * sh[i];
            rhs[i] = rhs[i] - omega_eff * tmp[i];
        }
        acc = op.wnorm2(rhs);
        converged = converged || (acc <= tol2);
        R rho_new = R(0);
#pragma unroll
        for (int i = 0; i < K; ++i) rho_new += clampd(shadow_at(i) * rhs[i], lim);
        rho_new = op.reduce(rho_new);
        const bool rho_bad = absv(rho_new) < tiny;
        const bool omega_bad = absv(omega) < tiny;
        broken = broken || (!converged && (rho_bad || omega_bad));
        finished = converged || broken;
        const bool beta_overflow = (absv(rho_new) > absv(rho_prev) * lim) ||
                                   (absv(alpha) > absv(omega) * lim);
        broken = broken || (!finished && beta_overflow);
        finished = converged || broken;
        const R beta = !finished ? (rho_new / rho_prev) * (alpha / omega) : R(0);
#pragma unroll
        for (int i = 0; i < K; ++i) {
            R pi = !finished ? rhs[i] + beta * (p[i] - omega * v[i]) : p[i];
            p[i] = clampd(pi, lim);
        }
        rho_prev = !finished ? rho_new : rho_prev;
    }
    iters = it;
    if (converged) return SUCCESS;
    return broken ? BICGSTAB_BREAKDOWN : MAX_LINEAR_ITERATIONS_EXCEEDED;
}

// Restarted GMRES(m) with right preconditioning and modified Gram-Schmidt.
//
// There is no GMRES in the reference; this solver uses its stopping rule.
// The system is scaled by W = diag(1 / (tol_i sqrt(K))), so the 2-norm of
// the scaled residual equals the reference's weighted RMS norm and the
// Givens-rotated residual estimate |g_{j+1}| is checked directly against
// floor + reduction * ||b||.  The weights are formed once per solve; the
// basis, inner products, Hessenberg matrix and rotations are kept in the
// working precision R (FP32 on the mixed-precision path, where the
// reduction is floored at 8 FP32 epsilons, so wider scalars would not
// change the answer and only cost FP64 and conversion issue slots).  One
// Arnoldi step (one operator and one preconditioner application) counts
// as one iteration.
template <class Cfg, class Op>
__device__ __forceinline__ int solve_gmres(const Op& op, typename Cfg::R* rhs,
                                           typename Cfg::R* x, int& iters) {
    using R = typename Cfg::R;
    constexpr int K = Op::K;
    constexpr int M = (Cfg::GMRES_RESTART < K) ? Cfg::GMRES_RESTART : K;
    R V[M + 1][K];
    R H[M][M];
    R g[M + 1], cs[M], sn[M], yv[M];
    R b[K], w[K], z[K];
    R wt[K], iwt[K];  // W and W^-1
    {
        const R sK = sqrt_t(R(Op::KT));  // total width: the weighted norm is a mean over every component
#pragma unroll
        for (int i = 0; i < K; ++i) {
            iwt[i] = R(op.tol(i)) * sK;
            wt[i] = R(1) / iwt[i];
        }
    }
    auto scaled_norm = [&](const R* v) {
        R s = R(0);
#pragma unroll
        for (int i = 0; i < K; ++i) {
            const R u = v[i] * wt[i];
            s += u * u;
        }
        return sqrt_t(op.reduce(s));
    };

    const R tol = R(Cfg::KRYLOV_FLOOR) + R(Cfg::KRYLOV_REDUCTION) * scaled_norm(rhs);
    op.apply(x, w);
#pragma unroll
    for (int i = 0; i < K; ++i) {
        b[i] = rhs[i];
        rhs[i] = rhs[i] - w[i];
    }
    R beta = scaled_norm(rhs);
    bool converged = beta <= tol;
    int it = 0;
    while (!converged && it < Cfg::KRYLOV_MAX_ITERS) {
        const R inv_beta = R(1) / beta;
#pragma unroll
        for (int i = 0; i < K; ++i) V[0][i] = rhs[i] * wt[i] * inv_beta;
        g[0] = beta;
#pragma unroll
        for (int j = 1; j <= M; ++j) g[j] = R(0);
        int jend = 0;
        bool cycle_converged = false;
#pragma unroll
        for (int j = 0; j < M; ++j) {
            if (it >= Cfg::KRYLOV_MAX_ITERS) break;
            ++it;
            // z = P^-1 W^-1 V_j ; w = W A z
#pragma unroll
            for (int i = 0; i < K; ++i) w[i] = V[j][i] * iwt[i];
            if (Cfg::PRECONDITIONED) {
                op.precond(w, z, V[M]);
            } else {
#pragma unroll
                for (int i = 0; i < K; ++i) z[i] = w[i];
            }
            op.apply(z, w);
#pragma unroll
            for (int i = 0; i < K; ++i) w[i] = w[i] * wt[i];
            R hcol[M + 1];
#pragma unroll
            for (int l = 0; l < M; ++l) {
                if (l <= j) {
                    R dot = R(0);
#pragma unroll
                    for (int i = 0; i < K; ++i) dot += w[i] * V[l][i];
                    dot = op.reduce(dot);
                    hcol[l] = dot;
#pragma unroll
                    for (int i = 0; i < K; ++i) w[i] = w[i] - dot * V[l][i];
                }
            }
            R hn = R(0);
#pragma unroll
            for (int i = 0; i < K; ++i) hn += w[i] * w[i];
            hn = sqrt_t(op.reduce(hn));
            {
                const R inv = (hn > R(0)) ? R(1) / hn : R(0);
#pragma unroll
                for (int i = 0; i < K; ++i) V[j + 1][i] = w[i] * inv;
            }
#pragma unroll
            for (int l = 0; l < M - 1; ++l) {
                if (l < j) {
                    const R a0 = hcol[l], a1 = hcol[l + 1];
                    hcol[l] = cs[l] * a0 + sn[l] * a1;
                    hcol[l + 1] = -sn[l] * a0 + cs[l] * a1;
                }
            }
            const R a = hcol[j];
            const R den = sqrt_t(a * a + hn * hn);
            const R inv_den = (den > R(0)) ? R(1) / den : R(0);
            const R c = (den > R(0)) ? a * inv_den : R(1);
            const R s = hn * inv_den;
            cs[j] = c;
            sn[j] = s;
            hcol[j] = den;
            g[j + 1] = -s * g[j];
            g[j] = c * g[j];
#pragma unroll
            for (int l = 0; l < M; ++l)
                if (l <= j) H[l][j] = hcol[l];
            jend = j + 1;
            if (absv(g[j + 1]) <= tol || hn == R(0)) {
                cycle_converged = true;
                break;
            }
        }
        if (jend == 0) break;
        // back substitution H y = g on the leading jend x jend block
#pragma unroll
        for (int l = M - 1; l >= 0; --l) {
            if (l < jend) {
                R s = g[l];
#pragma unroll
                for (int m = 0; m < M; ++m)
                    if (m > l && m < jend) s -= H[l][m] * yv[m];
                yv[l] = (H[l][l] != R(0)) ? s / H[l][l] : R(0);
            }
        }
        // x += P^-1 W^-1 sum_l y_l V_l
#pragma unroll
        for (int i = 0; i < K; ++i) {
            R u = R(0);
#pragma unroll
            for (int l = 0; l < M; ++l)
                if (l < jend) u += yv[l] * V[l][i];
            w[i] = u * iwt[i];
        }
        if (Cfg::PRECONDITIONED) {
            op.precond(w, z, V[M]);
        } else {
#pragma unroll
            for (int i = 0; i < K; ++i) z[i] = w[i];
        }
#pragma unroll
        for (int i = 0; i < K; ++i) x[i] += z[i];
        // Convergence is judged on the rotated residual estimate, as in
        // standard GMRES: the residual recomputed from the stored iterate
        // carries the rounding of the working precision (in FP32 it sits
        // above a floor measured against a 1e-6 absolute tolerance), so it
        // only seeds the next restart cycle.
        if (cycle_converged) {
            converged = true;
            break;
        }
        op.apply(x, w);
#pragma unroll
        for (int i = 0; i < K; ++i) rhs[i] = b[i] - w[i];
        beta = scaled_norm(rhs);
        converged = beta <= tol;
    }
    iters = it;
    return converged ? SUCCESS : MAX_LINEAR_ITERATIONS_EXCEEDED;
}

// Dense LU with partial pivoting, held in registers, for operators small
// enough to form (one system per thread, K <= a few dozen).  The matrix is
// built column by column from K operator applications, so it is exactly
// the operator the Krylov solvers see.  Row interchanges are done with
// compile-time-indexed selects (no runtime register indexing), and the
// inverse diagonal is kept so a solve costs K^2 multiply-adds.  A
// Rosenbrock step factors once and solves every stage with the factors,
// which is the reason W/Rosenbrock methods freeze their Jacobian.
//
// K = 2 is solved in closed form instead: m holds adj(A) / det(A), one
// reciprocal and no pivot search per factorisation, two multiplies and two
// multiply-adds per solve.  For 2 x 2 systems Cramer's rule is forward
// stable (Higham, Accuracy and Stability of Numerical Algorithms, 2nd ed.,
// sec. 1.10.1): its error is within a small multiple of cond(A) times the
// unit roundoff, the bound partial pivoting gives, which is what a stage
// increment needs.  A zero, non-finite or overflowing determinant fails
// the factorisation as a zero pivot does.
template <class R, int K>
struct DenseLU {
    R m[K][K];
    R rdiag[K];
    int piv[K];
    bool ok;
    template <class Op>
    __device__ __forceinline__ void factor(const Op& op) {
#pragma unroll
        for (int j = 0; j < K; ++j) {
            R e[K], col[K];
#pragma unroll
            for (int i = 0; i < K; ++i) e[i] = (i == j) ? R(1) : R(0);
            op.apply(e, col);
#pragma unroll
            for (int i = 0; i < K; ++i) m[i][j] = col[i];
        }
        if constexpr (K == 2) {
            const R a00 = m[0][0], a01 = m[0][1], a10 = m[1][0], a11 = m[1][1];
            const R det = a00 * a11 - a01 * a10;
            const R inv = R(1) / det;
            ok = is_finite(det) && is_finite(inv);
            m[0][0] = a11 * inv;
            m[0][1] = -a01 * inv;
            m[1][0] = -a10 * inv;
            m[1][1] = a00 * inv;
            return;
        }
        ok = true;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            int p = k;
            R best = absv(m[k][k]);
#pragma unroll
            for (int i = k + 1; i < K; ++i) {
                const R a = absv(m[i][k]);
                if (a > best) {
                    best = a;
                    p = i;
                }
            }
            piv[k] = p;
            ok = ok && (best > R(0)) && is_finite(best);
#pragma unroll
            for (int i = k + 1; i < K; ++i) {
                const bool sw = (i == p);
#pragma unroll
                for (int c = 0; c < K; ++c) {
                    const R t = m[k][c];
                    m[k][c] = sw ? m[i][c] : t;
                    m[i][c] = sw ? t : m[i][c];
                }
            }
            const R inv = R(1) / m[k][k];
            rdiag[k] = inv;
#pragma unroll
            for (int i = k + 1; i < K; ++i) {
                const R l = m[i][k] * inv;
                m[i][k] = l;
#pragma unroll
                for (int c = k + 1; c < K; ++c) m[i][c] -= l * m[k][c];
            }
        }
    }
    // x = A^-1 b (b is left untouched).
    __device__ __forceinline__ void solve(const R* b, R* x) const {
        if constexpr (K == 2) {
            const R b0 = b[0], b1 = b[1];
            x[0] = m[0][0] * b0 + m[0][1] * b1;
            x[1] = m[1][0] * b0 + m[1][1] * b1;
            return;
        }
        R y[K];
#pragma unroll
        for (int i = 0; i < K; ++i) y[i] = b[i];
#pragma unroll
        for (int k = 0; k < K; ++k) {
#pragma unroll
            for (int i = k + 1; i < K; ++i) {
                const bool sw = (i == piv[k]);
                const R t = y[k];
                y[k] = sw ? y[i] : t;
                y[i] = sw ? t : y[i];
            }
        }
#pragma unroll
        for (int i = 1; i < K; ++i)
#pragma unroll
            for (int c = 0; c < i; ++c) y[i] -= m[i][c] * y[c];
#pragma unroll
        for (int i = K - 1; i >= 0; --i) {
#pragma unroll
            for (int c = i + 1; c < K; ++c) y[i] -= m[i][c] * y[c];
            y[i] *= rdiag[i];
        }
#pragma unroll
        for (int i = 0; i < K; ++i) x[i] = y[i];
    }
};

// The direct solve behind ``linear_solve`` for Newton iterations (the
// operator changes with every iterate, so it is formed and factored per
// call).  ``rhs`` holds b on entry and is left as the (zero) residual;
// ``iters`` is 1.
template <class Cfg, class Op>
__device__ __forceinline__ int solve_direct(const Op& op, typename Cfg::R* rhs, typename Cfg::R* x, int& iters) {
    using R = typename Cfg::R;
    DenseLU<R, Op::K> lu;
    lu.factor(op);
    lu.solve(rhs, x);
#pragma unroll
    for (int i = 0; i < Op::K; ++i) rhs[i] = R(0);
    iters = 1;
    return lu.ok ? SUCCESS : MAX_LINEAR_ITERATIONS_EXCEEDED;
}

}  // namespace cbx
