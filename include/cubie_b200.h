/* cubie_b200 C ABI: compile, load and launch batch ODE integration kernels.
 *
 * The reference (ccam80/cubie) has no native boundary: its Python
 * BatchSolverKernel.run (src/cubie/batchsolving/BatchSolverKernel.py:525-604)
 * JIT-compiles one Numba kernel per configuration (build_kernel, :851-1011)
 * and launches it once per chunk (_execute_run, :741-762).  This library is
 * the seam that call now crosses: the Python layer (or any other host)
 * generates CUDA C++ for a configuration, compiles it here with NVRTC for
 * sm_100a, and launches the plain or persistent integration kernel with
 * caller-owned device buffers.
 *
 * Conventions: every function returns 0 on success and a negative code on
 * failure; cbx_last_error() then describes the failure for the calling
 * thread.  The library never frees caller memory.  Streams are CUstream /
 * cudaStream_t handles passed as void*.
 */
#ifndef CUBIE_B200_H
#define CUBIE_B200_H

#include <stddef.h>
#include "../cubie_b200/csrc/device/cbx_args.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cbx_module cbx_module;

enum cbx_kernel_kind { CBX_KERNEL_PLAIN = 0, CBX_KERNEL_PERSISTENT = 1, CBX_KERNEL_HETERO = 2, CBX_KERNEL_WARP = 3 };

enum cbx_error {
    CBX_OK = 0,
    CBX_ERR_ARGUMENT = -1,
    CBX_ERR_NVRTC = -2,
    CBX_ERR_DRIVER = -3,
    CBX_ERR_RUNTIME = -4,
    CBX_ERR_NO_DEVICE = -5
};

/* Library version (major * 10000 + minor * 100 + patch). */
int cbx_version(void);

/* Thread-local description of the last failure (replaces the Python
 * exceptions the reference raises, e.g. limit_blocksize's ValueError,
 * BatchSolverKernel.py:823-830). */
const char* cbx_last_error(void);

/* NVRTC version linked into the library. */
int cbx_nvrtc_version(int* major, int* minor);

/* Compile CUDA C++ source to an sm_100a cubin with NVRTC.  No GPU needed.
 * *cubin is malloc'ed; release it with cbx_free.  ``log`` receives the
 * compiler log (truncated to log_len, always NUL-terminated when
 * log_len > 0).  Replaces the Numba compile that reading
 * BatchSolverKernel.kernel triggers (CUDAFactory.get_cached_output). */
int cbx_compile(const char* source, const char* name, const char* const* options, int n_options,
                void** cubin, size_t* cubin_size, char* log, size_t log_len);
void cbx_free(void* p);

/* Load a cubin on ``device`` (primary context) and resolve whichever of
 * the integration kernels cbx_integrate_plain, cbx_integrate_persistent,
 * cbx_integrate_hetero and cbx_integrate_warp it defines (at least one). */
int cbx_module_load(const void* cubin, size_t cubin_size, int device, cbx_module** module);

/* cbx_compile + cbx_module_load. */
int cbx_module_create(const char* source, const char* const* options, int n_options, int device,
                      cbx_module** module, char* log, size_t log_len);

int cbx_module_destroy(cbx_module* module);

/* Resource use of a kernel (registers per thread, local bytes per thread,
 * max threads per block, static shared bytes). */
int cbx_kernel_info(cbx_module* module, int kernel, int* registers, int* local_bytes,
                    int* max_threads, int* shared_bytes);

/* Resident blocks per SM for ``block`` threads. */
int cbx_occupancy(cbx_module* module, int kernel, int block, int* blocks_per_sm);

/* Launch the integration kernel: the replacement for the reference's
 * kernel launch (BatchSolverKernel.py:741-762).  ``args`` holds caller
 * device pointers (layouts in cbx_args.h).  grid = 0 picks
 * ceil(n_runs / block) for the plain kernel and a resident grid for the
 * persistent kernel and for the warp-per-run kernel of large systems
 * (CBX_KERNEL_WARP; both also require args->work_counter to point at a
 * zeroed device counter).  Asynchronous on ``stream``. */
int cbx_solve(cbx_module* module, const cbx_solve_args* args, int kernel, int block, int grid,
              void* stream);

/* Several configurations in one persistent work-stealing launch (module
 * generated for a list of families; layout in cbx_args.h).  No counterpart
 * in the reference, which launches one kernel per system.  Requires
 * args->work_counter to point at CBX_MAX_FAMILIES zeroed 64-bit counters;
 * grid = 0 picks a resident grid.  Asynchronous on ``stream``. */
int cbx_solve_hetero(cbx_module* module, const cbx_hetero_args* args, int block, int grid, void* stream);

/* Device facts used for launch geometry. */
int cbx_device_info(int device, int* sm_count, int* cc_major, int* cc_minor);

/* FP32 fused multiply-add throughput probe: launches a fixed FMA loop
 * (nvcc-compiled for sm_100a) and returns the elapsed milliseconds for
 * ``flops`` floating-point operations.  Used to state the FP32 roofline
 * denominator next to the integrator's achieved FLOP rate. */
int cbx_fp32_peak_probe(int device, double* flops, float* milliseconds);

/* Overwrite ``bytes`` of device memory at ``buffer`` on ``stream`` (L2
 * flush between timed launches). */
int cbx_flush_l2(void* buffer, size_t bytes, void* stream);

/* Discrete adjoint (no counterpart in the reference, which cannot
 * differentiate its integrations).  For a module generated with the
 * adjoint kernels (explicit Runge-Kutta and Rosenbrock tableaus):
 *
 * cbx_adjoint_info reports the size of one per-run checkpoint image and of
 * one replay record (both multiples of 16 bytes); size adj->ckpt as
 * n_runs * max_ckpts * lane_bytes and adj->seg as
 * n_runs * ckpt_every * record_bytes, both 16-byte aligned, and pass
 * adj->lane_words = lane_bytes / 4.
 *
 * cbx_adjoint_tape_bytes reports the size of one step-size tape entry:
 * 4 or 8 for explicit Runge-Kutta modules, which then need adj->tape,
 * adj->tape_flags and adj->step_count (sizes in cbx_args.h, 16-byte
 * aligned), and 0 for the others (those three unused).
 *
 * cbx_adjoint_launch with phase 0 integrates like cbx_solve's persistent
 * kernel (same outputs) and stores a checkpoint every adj->ckpt_every
 * accepted steps (and, with a tape, every accepted step's size); a run
 * needing more than adj->max_ckpts checkpoints stops with status bit 32.
 * Phase 1, with the same args, the checkpoints (and tape) of phase 0,
 * dL/d(saved state) in adj->grad_state and args->work_counter zeroed
 * again, writes dL/d(initial state) and dL/d(parameters) for every run,
 * holding the accepted step sizes fixed.  Both are asynchronous on
 * ``stream``; grid = 0 picks a resident grid. */
int cbx_adjoint_info(cbx_module* module, long long* lane_bytes, long long* record_bytes);
int cbx_adjoint_tape_bytes(cbx_module* module, long long* entry_bytes);
int cbx_adjoint_launch(cbx_module* module, const cbx_solve_args* args, const cbx_adjoint_args* adj,
                       int phase, int block, int grid, void* stream);

/* Size of the device scratch array behind cbx_solve_noalloc.  Every device
 * that loads this library holds it until the process exits. */
#define CBX_NOALLOC_SCRATCH_BYTES 256

/* The persistent launch of cbx_solve for hosts that cannot allocate device
 * memory while they run: a custom call or plugin inside another framework
 * that hands it only that framework's input and output buffers, or a loop
 * whose device memory is fixed at start-up.  No counterpart in the
 * reference (its kernels allocate nothing themselves; Numba's launch does).
 *
 * Same arguments and meaning as cbx_solve with kernel = persistent, except
 * that args->work_counter is ignored: the work counter lives in a static
 * device array of CBX_NOALLOC_SCRATCH_BYTES bytes (a call needs 40 of them
 * for any batch size), and the four iteration totals go there too when
 * args->totals is NULL (to args->totals, which the caller zeroes, when it
 * is not).  The call clears the scratch words it uses, in stream order,
 * before the launch; the array keeps the last call's values afterwards.
 * Calls that overlap on the GPU (on different streams, or from several
 * threads) share the array and race: serialise them.  Rejects device
 * ordinals of 64 and above, and modules loaded while a context other than
 * the device's primary context was current (the array's address belongs to
 * the primary context).  Every argument check comes before the clear, so a
 * rejected call touches nothing on the device.  Calls no cudaMalloc or
 * cudaFree.
 *
 * The first call on a device looks up the array's device address with
 * cudaGetSymbolAddress, with the module's (primary) context current, which
 * loads this library's device code into that context: make that first
 * call before any stream capture. */
int cbx_solve_noalloc(cbx_module* module, const cbx_solve_args* args, int block, int grid,
                      void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CUBIE_B200_H */
