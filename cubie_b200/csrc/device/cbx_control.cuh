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
// Everything is computed in the control precision C (FP64 on the
// mixed-precision path) except the exponentiations of the gain there,
// which run in FP32: the gain is clamped to [min_gain, max_gain] before it
// scales the FP64 step size, so its 24-bit value gives the same step
// sequence to within that rounding, and an FP64 pow costs far more issue
// slots than the rest of the step update.  Out-of-range arguments behave
// alike in both widths after the clamp (an FP32 overflow to inf gives a
// zero or infinite factor where FP64 gives a tiny or huge one).
#pragma once
#include "cbx_common.cuh"

namespace cbx {

template <class Cfg>
struct Controller {
    using R = typename Cfg::R;
    using C = typename Cfg::C;
    static constexpr int N = Cfg::N;
    struct State {
        C h0, h1;
    };
    static __device__ __forceinline__ void init(State& st) {
        st.h0 = C(0);
        st.h1 = C(0);
    }
    static __device__ __forceinline__ C cpow(C a, C b) {
        if constexpr (Cfg::MIXED) return C(pow_t(float(a), float(b)));
        else return pow_t(a, b);
    }
    static __device__ __forceinline__ C error_norm2(const R* ynew, const R* y, const R* err, C tol_scale) {
        C nrm2 = C(0);
#pragma unroll
        for (int i = 0; i < N; ++i) {
            const C e = pymax(C(absv(err[i])), C(1e-16));
            const C tol = C(Cfg::atol(i)) + C(Cfg::rtol(i)) * tol_scale * pymax(C(absv(ynew[i])), C(absv(y[i])));
            const C ratio = e / tol;
            nrm2 += ratio * ratio;
        }
        nrm2 = nrm2 * C(Cfg::CTL_INV_N);
        if (is_nan(nrm2) || !is_finite(nrm2)) nrm2 = C(1e16);
        return nrm2;
    }
    static __device__ __forceinline__ C finish_gain(C gain, bool accept) {
        gain = clampv(gain, C(Cfg::CTL_MIN_GAIN), C(Cfg::CTL_MAX_GAIN));
        if (!(Cfg::CTL_DEADBAND_MIN == 1.0 && Cfg::CTL_DEADBAND_MAX == 1.0)) {
            const bool within = (gain >= C(Cfg::CTL_DEADBAND_MIN)) && (gain <= C(Cfg::CTL_DEADBAND_MAX));
            gain = within ? C(1) : gain;
        }
        return accept ? gain : pymin(gain, C(Cfg::CTL_SAFETY));
    }
    // Returns the controller status bits; updates dt, accept and history.
    static __device__ __forceinline__ int update(C& dt, const R* ynew, const R* y, const R* err, int niters,
                                                 bool truncated, bool& accept, State& st, C tol_scale) {
        if constexpr (Cfg::CTRL == CTRL_FIXED) {
            accept = true;
            return SUCCESS;
        } else {
            return update_with_norm(dt, error_norm2(ynew, y, err, tol_scale), niters, truncated, accept, st);
        }
    }
    // The same decision from an error norm computed elsewhere (the
    // warp-per-system path reduces it over the lanes).
    static __device__ __forceinline__ int update_with_norm(C& dt, C nrm2, int niters, bool truncated, bool& accept,
                                                           State& st) {
        if constexpr (Cfg::CTRL == CTRL_FIXED) {
            accept = true;
            return SUCCESS;
        } else {
            if (is_nan(nrm2) || !is_finite(nrm2)) nrm2 = C(1e16);
            accept = nrm2 <= C(1);
            const C safety = C(Cfg::CTL_SAFETY);
            C gain;
            bool commit_history = accept && !truncated;
            const C current_dt = dt;
            if constexpr (Cfg::CTRL == CTRL_I) {
                gain = C(safety * cpow(nrm2, -C(Cfg::CTL_E1)));
            } else if constexpr (Cfg::CTRL == CTRL_PI) {
                const C err_prev = st.h0;
                const C pgain = cpow(nrm2, -C(Cfg::CTL_E1));
                const C src = err_prev > C(0) ? err_prev : nrm2;
                const C igain = cpow(src, -C(Cfg::CTL_E2));
                gain = safety * pgain * igain;
                st.h0 = commit_history ? nrm2 : err_prev;
            } else if constexpr (Cfg::CTRL == CTRL_PID) {
                const C err_prev = st.h0, err_prev_prev = st.h1;
                const C eps = err_prev > C(0) ? err_prev : nrm2;
                const C epps = err_prev_prev > C(0) ? err_prev_prev : eps;
                gain = C(safety * cpow(nrm2, -C(Cfg::CTL_E1)) * cpow(eps, -C(Cfg::CTL_E2)) *
                         cpow(epps, -C(Cfg::CTL_E3)));
                st.h1 = commit_history ? err_prev : err_prev_prev;
                st.h0 = commit_history ? nrm2 : err_prev;
            } else {  // Gustafsson (gustafsson_controller.py:236-283)
                const C expo = C(Cfg::CTL_E1);
                const C dt_prev = pymax(st.h0, C(1e-16));
                const C err_prev = pymax(st.h1, C(1e-16));
                const C gain_numerator = C(1 + 2 * Cfg::CTL_NEWTON_TARGET) * safety;
                const C denom = C(niters + 2 * Cfg::CTL_NEWTON_TARGET);
                const C tmp = gain_numerator / denom;
                const C fac = safety < tmp ? safety : tmp;
                const C gain_basic = C(fac * cpow(nrm2, -expo));
                const C ratio = nrm2 * nrm2 / err_prev;
                const C gain_gus = C(safety * (dt / dt_prev) * cpow(ratio, -expo));
                gain = gain_gus < gain_basic ? gain_gus : gain_basic;
                gain = (accept && dt_prev > C(1e-16)) ? gain : gain_basic;
                st.h0 = commit_history ? current_dt : st.h0;
                st.h1 = commit_history ? nrm2 : st.h1;
            }
            gain = finish_gain(gain, accept);
            const bool freeze = accept && truncated;
            const C dt_new_raw = current_dt * gain;
            dt = freeze ? current_dt : clampv(dt_new_raw, C(Cfg::DT_MIN), C(Cfg::DT_MAX));
            return (freeze || dt_new_raw > C(Cfg::DT_MIN)) ? SUCCESS : STEP_TOO_SMALL;
        }
    }
};

}  // namespace cbx
