/* Launch arguments of the integration kernels.
 *
 * One definition shared by the host library (C ABI) and the NVRTC-compiled
 * device code, so the struct layout cannot drift between the two sides.
 * Only pointer, 64-bit and 32-bit fields are used, in an order that needs
 * no padding differences between compilers.
 *
 * Array layouts follow the reference (BatchSolverKernel.py:964-965 and
 * output_sizes.py:284-380): the run index is the fastest axis, so
 *   inits[k * run_stride + run], params[k * run_stride + run],
 *   state_out[(row * width + k) * run_stride + run], and so on.
 */
#ifndef CBX_ARGS_H
#define CBX_ARGS_H

typedef struct cbx_solve_args {
    /* inputs (device pointers, system precision) */
    const void* inits;          /* [n_states][run_stride] */
    const void* params;         /* [n_params][run_stride] */
    const void* driver_coeffs;  /* [n_segments][n_drivers][order + 1] */
    /* outputs (device pointers; NULL when the output is not compiled in) */
    void* state_out;            /* [n_save_rows][n_saved_states + save_time][run_stride] */
    void* obs_out;              /* [n_save_rows][n_saved_observables][run_stride] */
    void* state_sum_out;        /* [n_summary_rows][n_summarised_states * per_var][run_stride] */
    void* obs_sum_out;          /* [n_summary_rows][n_summarised_obs * per_var][run_stride] */
    int* counters_out;          /* [n_save_rows][4][run_stride] int32 */
    int* status_out;            /* [run_stride] int32 */
    /* optional per-run arrays (NULL = uniform) */
    const double* durations;    /* per-run integration duration */
    const double* tol_scale;    /* per-run multiplier on every rtol */
    /* scheduling and statistics */
    unsigned long long* work_counter; /* persistent launch: next run to claim */
    unsigned long long* totals;       /* [4]: steps, rejections, newton, krylov */
    const volatile int* abort_flag;   /* host-visible abort request, or NULL */
    const long long* run_order; /* persistent launch: claim k integrates run
                                   run_order[k] (NULL: run k); a permutation
                                   of [0, n_runs) */
    /* sizes */
    long long n_runs;
    long long run_stride;
    long long max_steps;        /* per-run step budget, 0 = unlimited */
    /* timing (float64, as the reference's kernel scalars) */
    double duration;
    double warmup;
    double t0;
    double save_stop;
    double summary_stop;
    int n_save_rows;
    int n_summary_rows;
} cbx_solve_args;

/* Extra arguments of the discrete-adjoint kernels (forward with
 * checkpoints, then the reverse sweep).  The reference has no adjoint.
 *
 *   ckpt        [run][slot][lane_bytes / 4] 32-bit words: the complete
 *               per-run loop state at every ckpt_every-th accepted step
 *               (slot 0 = the state after the run is seeded);
 *   ckpt_count  [run] int32: slots written by the forward launch;
 *   seg         [run][ckpt_every][record_bytes]: one record per accepted
 *               step of the segment being replayed (start state, start
 *               time when f depends on time, step size negated on steps
 *               that end on a saved row), system precision;
 *   grad_state  [n_save_rows][n_saved_states + save_time][run_stride]:
 *               dL/d(saved state), same layout as state_out;
 *   grad_inits  [n_states][run_stride], grad_params [n_params][run_stride]:
 *               results (written, not accumulated);
 *   tape, tape_flags, step_count: explicit Runge-Kutta modules only
 *               (cbx_adjoint_tape_bytes > 0), NULL otherwise; written by the
 *               forward launch and read by the reverse sweep.  With
 *               cap = max_ckpts * ckpt_every, e = cbx_adjoint_tape_bytes and
 *               v = 16 / e: tape [run][ceil(cap / v) * v] entries of e bytes
 *               (each accepted step's size, negated when it ended on a saved
 *               row), tape_flags [run][ceil(cap / 32)] 32-bit words (bit set:
 *               the attempt before that step was rejected), step_count [run]
 *               int32 (accepted steps).
 */
typedef struct cbx_adjoint_args {
    void* ckpt;
    int* ckpt_count;
    void* seg;
    const void* grad_state;
    void* grad_inits;
    void* grad_params;
    long long lane_words;       /* lane_bytes / 4 as reported by the module (a multiple of 4) */
    int ckpt_every;
    int max_ckpts;
    void* tape;
    unsigned* tape_flags;
    int* step_count;
} cbx_adjoint_args;

/* Several configurations ("families") in one persistent launch.  Global
 * run r belongs to family k when first_run[k] <= r < first_run[k + 1] and is
 * run r - first_run[k] of family[k] (that family's own inputs, outputs,
 * status words and, when non-NULL, iteration totals).  The families'
 * work_counter fields are unused: ``work_counter`` points at
 * CBX_MAX_FAMILIES zeroed 64-bit counters, one per family.
 * first_run[n_families] is the total number of runs. */
#define CBX_MAX_FAMILIES 8
typedef struct cbx_hetero_args {
    cbx_solve_args family[CBX_MAX_FAMILIES];
    long long first_run[CBX_MAX_FAMILIES + 1];
    unsigned long long* work_counter; /* [CBX_MAX_FAMILIES] */
    int n_families;
    int reserved;
} cbx_hetero_args;

#endif /* CBX_ARGS_H */
