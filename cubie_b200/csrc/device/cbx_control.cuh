// Step-size controllers (fixed, I, PI, PID, Gustafsson).
//
// All adaptive controllers share the error measure of the reference
// (adaptive_PI_controller.py:222-233):
//   nrm2 = mean_i (max(|e_i|, 1e-16) / (atol_i + rtol_i max(|y_new_i|, |y_i|)))^2
// with non-finite values mapped to 1e16 and acceptance nrm2 <= 1.  The
// exponents are halved because nrm2 is a mean square.  Gains are clamped to
// [min_gain, max_gain], a deadband maps gains inside it to 1, a rejected
// step caps the gain at the safety factor, and an accepted step that was
// truncated onto an output event keeps dt (freeze) and leaves the history
// untouched.  STEP_TOO_SMALL is returned when dt * gain <= dt_min.
// Precision on the mixed-precision path: the step size, its clamp to
// [dt_min, dt_max], the STEP_TOO_SMALL test, the controller history of
// step sizes and the error norm's reduction (the sum of squared ratios and
// the acceptance test) run in the control precision C, FP64.  Each
// component's ratio e_i / tol_i and the gain's powers run in the gain
// precision G, FP32: e_i and y_i are FP32 values, so their ratio carries no
// more information in FP64, and the gain is a factor clamped to
// [min_gain, max_gain] before it scales the FP64 step size, so its last
// bits only nudge dt, while FP64 divisions and powers cost many issue slots
// per step.  Out-of-range arguments behave alike in both widths after the
// clamp (an FP32 overflow to inf gives a zero or infinite factor where FP64
// gives a tiny or huge one; non-finite norms map to 1e16 in both).  On the
// FP32 and FP64 paths G = C = the system precision, in the reference's
// order of operations.
#pragma once
#include "cbx_common.cuh"

namespace cbx {

template <class Cfg>
struct Controller {
    using R = typename Cfg::R;
    using C = typename Cfg::C;
    using G = typename Cfg::G;
    static constexpr int N = Cfg::N;
    struct State {
        G h0, h1;   // previous error norms (PI, PID); h1: previous norm (Gustafsson)
        C hdt;      // previous accepted step size (Gustafsson)
    };
    // On the mixed-precision path Gustafsson's controller works in the log2
    // domain: h1 holds log2(max(previous norm, 1e-16)) and h0 log2 of the
    // previous accepted step size, so both candidate gains come from one
    // log2 of the norm and one of the step size, and the smaller is raised
    // with a single exp2 (no reference counterpart, so no bit pattern to
    // keep).
    static constexpr bool LOG_GUS = Cfg::MIXED && Cfg::CTRL == CTRL_GUSTAFSSON;
    static constexpr double LOG2_1EM16 = -53.150849518197795;   // log2(1e-16)
    static __device__ __forceinline__ void init(State& st) {
        st.h0 = LOG_GUS ? G(-1e30) : G(0);   // no accepted step yet
        st.h1 = LOG_GUS ? G(LOG2_1EM16) : G(0);
        st.hdt = C(0);
    }
    static __device__ __forceinline__ G gpow(G a, G b) { return pow_t(a, b); }
    // One component's ratio max(|e|, 1e-16) / (atol + rtol s max(|y_new|, |y|)).
    static __device__ __forceinline__ G error_ratio(R e_i, R ynew_i, R y_i, G atol, G rtol, G ts) {
        const G e = pymax(G(absv(e_i)), G(1e-16));
        const G tol = atol + rtol * ts * pymax(G(absv(ynew_i)), G(absv(y_i)));
        return e / tol;
    }
    static __device__ __forceinline__ C error_norm2(const R* ynew, const R* y, const R* err, G ts) {
        C nrm2 = C(0);
#pragma unroll
        for (int i = 0; i < N; ++i) {
            const C ratio = C(error_ratio(err[i], ynew[i], y[i], G(Cfg::atol(i)), G(Cfg::rtol(i)), ts));
            nrm2 += ratio * ratio;
        }
        // non-finite norms map to 1e16 in update_with_norm
        return nrm2 * C(Cfg::CTL_INV_N);
    }
    static __device__ __forceinline__ G finish_gain(G gain, bool accept) {
        gain = clampv(gain, G(Cfg::CTL_MIN_GAIN), G(Cfg::CTL_MAX_GAIN));
        if (!(Cfg::CTL_DEADBAND_MIN == 1.0 && Cfg::CTL_DEADBAND_MAX == 1.0)) {
            const bool within = (gain >= G(Cfg::CTL_DEADBAND_MIN)) && (gain <= G(Cfg::CTL_DEADBAND_MAX));
            gain = within ? G(1) : gain;
        }
        return accept ? gain : pymin(gain, G(Cfg::CTL_SAFETY));
    }
    // Returns the controller status bits; updates dt, accept and history.
    // ``ts``: the run's tolerance scale in the gain precision
    static __device__ __forceinline__ int update(C& dt, const R* ynew, const R* y, const R* err, int niters,
                                                 bool truncated, bool& accept, State& st, G ts) {
        if constexpr (Cfg::CTRL == CTRL_FIXED) {
            accept = true;
            return SUCCESS;
        } else {
            return update_with_norm(dt, error_norm2(ynew, y, err, ts), niters, truncated, accept, st);
        }
    }
    // The same decision from an error norm computed elsewhere (the
    // warp-per-system path reduces it over the lanes).
    static __device__ __forceinline__ int update_with_norm(C& dt, C nrm2_c, int niters, bool truncated, bool& accept,
                                                           State& st) {
        if constexpr (Cfg::CTRL == CTRL_FIXED) {
            accept = true;
            return SUCCESS;
        } else {
            // a NaN or infinite norm rejects the step; the gain sees 1e16
            accept = nrm2_c <= C(1);
            G nrm2 = G(nrm2_c);
            if (!is_finite(nrm2)) nrm2 = G(1e16);
            const G safety = G(Cfg::CTL_SAFETY);
            G gain;
            bool commit_history = accept && !truncated;
            const C current_dt = dt;
            if constexpr (Cfg::CTRL == CTRL_I) {
                gain = G(safety * gpow(nrm2, -G(Cfg::CTL_E1)));
            } else if constexpr (Cfg::CTRL == CTRL_PI) {
                const G err_prev = st.h0;
                const G pgain = gpow(nrm2, -G(Cfg::CTL_E1));
                const G src = err_prev > G(0) ? err_prev : nrm2;
                const G igain = gpow(src, -G(Cfg::CTL_E2));
                gain = safety * pgain * igain;
                st.h0 = commit_history ? nrm2 : err_prev;
            } else if constexpr (Cfg::CTRL == CTRL_PID) {
                const G err_prev = st.h0, err_prev_prev = st.h1;
                const G eps = err_prev > G(0) ? err_prev : nrm2;
                const G epps = err_prev_prev > G(0) ? err_prev_prev : eps;
                gain = G(safety * gpow(nrm2, -G(Cfg::CTL_E1)) * gpow(eps, -G(Cfg::CTL_E2)) *
                         gpow(epps, -G(Cfg::CTL_E3)));
                st.h1 = commit_history ? err_prev : err_prev_prev;
                st.h0 = commit_history ? nrm2 : err_prev;
            } else {  // Gustafsson (gustafsson_controller.py:236-283)
                const G expo = G(Cfg::CTL_E1);
                const C dt_prev = pymax(st.hdt, C(1e-16));
                const G gain_numerator = G(1 + 2 * Cfg::CTL_NEWTON_TARGET) * safety;
                const G denom = G(niters + 2 * Cfg::CTL_NEWTON_TARGET);
                const G tmp = gain_numerator / denom;
                const G fac = safety < tmp ? safety : tmp;
                if constexpr (LOG_GUS) {
                    // gain_basic = fac nrm2^-e and gain_gus = safety (dt /
                    // dt_prev) (nrm2^2 / prev)^-e, both fac 2^x: the smaller
                    // exponent is raised once.  log2(safety / fac) is zero
                    // unless the Newton count lowered fac (a constant fold
                    // when the step reports no Newton iterations).
                    const G l2 = log2_t(nrm2);
                    const G ldt = log2_t(G(current_dt));
                    const G lprev = pymax(st.h1, G(LOG2_1EM16));
                    const G lsf = safety < tmp ? G(0) : log2_t(safety / tmp);
                    const G x_basic = -expo * l2;
                    const G x_gus = lsf + (ldt - st.h0) - expo * (G(2) * l2 - lprev);
                    const bool use_gus = accept && st.h0 > G(LOG2_1EM16);
                    gain = fac * exp2_t(use_gus && x_gus < x_basic ? x_gus : x_basic);
                    st.h1 = commit_history ? l2 : st.h1;
                    st.h0 = commit_history ? ldt : st.h0;
                } else {
                    const G err_prev = pymax(st.h1, G(1e-16));
                    const G gain_basic = G(fac * gpow(nrm2, -expo));
                    const G ratio = nrm2 * nrm2 / err_prev;
                    const G gain_gus = G(safety * G(dt / dt_prev) * gpow(ratio, -expo));
                    gain = gain_gus < gain_basic ? gain_gus : gain_basic;
                    gain = (accept && dt_prev > C(1e-16)) ? gain : gain_basic;
                    st.h1 = commit_history ? nrm2 : st.h1;
                }
                st.hdt = commit_history ? current_dt : st.hdt;
            }
            gain = finish_gain(gain, accept);
            const bool freeze = accept && truncated;
            const C dt_new_raw = current_dt * C(gain);
            dt = freeze ? current_dt : clampv(dt_new_raw, C(Cfg::DT_MIN), C(Cfg::DT_MAX));
            return (freeze || dt_new_raw > C(Cfg::DT_MIN)) ? SUCCESS : STEP_TOO_SMALL;
        }
    }
};

}  // namespace cbx
