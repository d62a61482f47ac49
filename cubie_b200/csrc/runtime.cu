// C-ABI implementation: NVRTC compilation, module management and launches.
//
// Host code uses the CUDA driver API for modules and launches (so cubins
// produced at run time load into whatever primary context the caller, e.g.
// PyTorch, already holds) and the runtime API only for the two fixed
// utility kernels defined at the bottom of this file, which nvcc compiles
// for sm_100a with the library itself.
#include <cuda.h>
#include <cuda_runtime.h>
#include <nvrtc.h>

#include <dlfcn.h>

#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/cubie_b200.h"

struct cbx_module {
    CUmodule module;
    CUcontext context;
    CUfunction fn[4];  // plain, persistent, hetero, warp (NULL when the module has none)
    int device;
    int sm_count;
    // discrete-adjoint kernels, resolved on first use (modules generated
    // without them have neither)
    CUfunction adj[2];
    size_t lane_bytes;
    size_t record_bytes;
    size_t tape_bytes;
    bool adj_resolved;
    int n_families;  // families of the heterogeneous kernel (0 without one)
    int primary;     // 1: context is the device's primary context, 0: it is not, -1: not yet checked
    size_t warp_smem;  // dynamic shared memory of the warp kernel's launch (bytes)
};

namespace {

thread_local std::string g_error;

// The driver API is resolved with dlopen at first use, so the library loads
// (and NVRTC compiles) on hosts without a GPU driver.
struct DriverApi {
    bool loaded = false;
    bool failed = false;
#define CBX_DRV(name) decltype(&::name) name = nullptr;
    CBX_DRV(cuInit)
    CBX_DRV(cuDeviceGet)
    CBX_DRV(cuCtxGetCurrent)
    CBX_DRV(cuCtxGetDevice)
    CBX_DRV(cuDevicePrimaryCtxRetain)
    CBX_DRV(cuDevicePrimaryCtxRelease)
    CBX_DRV(cuCtxSetCurrent)
    CBX_DRV(cuModuleLoadData)
    CBX_DRV(cuModuleGetFunction)
    CBX_DRV(cuModuleUnload)
    CBX_DRV(cuDeviceGetAttribute)
    CBX_DRV(cuFuncGetAttribute)
    CBX_DRV(cuFuncSetAttribute)
    CBX_DRV(cuOccupancyMaxActiveBlocksPerMultiprocessor)
    CBX_DRV(cuLaunchKernel)
    CBX_DRV(cuGetErrorName)
    CBX_DRV(cuGetErrorString)
    CBX_DRV(cuModuleGetGlobal)
#undef CBX_DRV
};

DriverApi g_drv;

bool load_driver() {
    if (g_drv.loaded) return true;
    if (g_drv.failed) return false;
    void* h = dlopen("libcuda.so.1", RTLD_NOW | RTLD_LOCAL);
    if (!h) h = dlopen("libcuda.so", RTLD_NOW | RTLD_LOCAL);
    if (!h) {
        g_drv.failed = true;
        return false;
    }
#define CBX_SYM(name)                                                          \
    g_drv.name = reinterpret_cast<decltype(g_drv.name)>(dlsym(h, #name));     \
    if (!g_drv.name) {                                                         \
        g_drv.failed = true;                                                   \
        return false;                                                          \
    }
    CBX_SYM(cuInit)
    CBX_SYM(cuDeviceGet)
    CBX_SYM(cuCtxGetCurrent)
    CBX_SYM(cuCtxGetDevice)
    CBX_SYM(cuDevicePrimaryCtxRetain)
    CBX_SYM(cuCtxSetCurrent)
    CBX_SYM(cuModuleLoadData)
    CBX_SYM(cuModuleGetFunction)
    CBX_SYM(cuModuleUnload)
    CBX_SYM(cuDeviceGetAttribute)
    CBX_SYM(cuFuncGetAttribute)
    CBX_SYM(cuFuncSetAttribute)
    CBX_SYM(cuOccupancyMaxActiveBlocksPerMultiprocessor)
    CBX_SYM(cuLaunchKernel)
    CBX_SYM(cuGetErrorName)
    CBX_SYM(cuGetErrorString)
#undef CBX_SYM
    // versioned entry points behind cuda.h's macros
    g_drv.cuDevicePrimaryCtxRelease =
        reinterpret_cast<decltype(g_drv.cuDevicePrimaryCtxRelease)>(dlsym(h, "cuDevicePrimaryCtxRelease_v2"));
    if (!g_drv.cuDevicePrimaryCtxRelease) {
        g_drv.failed = true;
        return false;
    }
    g_drv.cuModuleGetGlobal = reinterpret_cast<decltype(g_drv.cuModuleGetGlobal)>(dlsym(h, "cuModuleGetGlobal_v2"));
    if (!g_drv.cuModuleGetGlobal) {
        g_drv.failed = true;
        return false;
    }
    g_drv.loaded = true;
    return true;
}

int fail(int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_error = buf;
    return code;
}

int check_cu(CUresult r, const char* what) {
    if (r == CUDA_SUCCESS) return CBX_OK;
    const char* name = nullptr;
    const char* msg = nullptr;
    g_drv.cuGetErrorName(r, &name);
    g_drv.cuGetErrorString(r, &msg);
    return fail(CBX_ERR_DRIVER, "%s failed: %s (%s)", what, name ? name : "?", msg ? msg : "?");
}

void copy_log(const std::string& s, char* log, size_t log_len) {
    if (!log || log_len == 0) return;
    size_t n = s.size() < log_len - 1 ? s.size() : log_len - 1;
    memcpy(log, s.data(), n);
    log[n] = '\0';
}

int require_driver() {
    if (!load_driver()) return fail(CBX_ERR_NO_DEVICE, "CUDA driver library (libcuda.so.1) is not available");
    return CBX_OK;
}

int ensure_context(int device, CUcontext* out) {
    int rc = require_driver();
    if (rc) return rc;
    rc = check_cu(g_drv.cuInit(0), "cuInit");
    if (rc) return rc;
    CUcontext ctx = nullptr;
    CUdevice dev;
    rc = check_cu(g_drv.cuDeviceGet(&dev, device), "cuDeviceGet");
    if (rc) return rc;
    rc = check_cu(g_drv.cuCtxGetCurrent(&ctx), "cuCtxGetCurrent");
    if (rc) return rc;
    CUdevice cur_dev = -1;
    if (ctx) {
        if (g_drv.cuCtxGetDevice(&cur_dev) != CUDA_SUCCESS) cur_dev = -1;
    }
    if (!ctx || cur_dev != dev) {
        rc = check_cu(g_drv.cuDevicePrimaryCtxRetain(&ctx, dev), "cuDevicePrimaryCtxRetain");
        if (rc) return rc;
        rc = check_cu(g_drv.cuCtxSetCurrent(ctx), "cuCtxSetCurrent");
        if (rc) return rc;
    }
    *out = ctx;
    return CBX_OK;
}

}  // namespace

extern "C" {

int cbx_version(void) { return 1 * 10000 + 0 * 100 + 0; }

const char* cbx_last_error(void) { return g_error.c_str(); }

int cbx_nvrtc_version(int* major, int* minor) {
    if (!major || !minor) return fail(CBX_ERR_ARGUMENT, "null output pointer");
    if (nvrtcVersion(major, minor) != NVRTC_SUCCESS) return fail(CBX_ERR_NVRTC, "nvrtcVersion failed");
    return CBX_OK;
}

int cbx_compile(const char* source, const char* name, const char* const* options, int n_options,
                void** cubin, size_t* cubin_size, char* log, size_t log_len) {
    if (!source || !cubin || !cubin_size) return fail(CBX_ERR_ARGUMENT, "null argument to cbx_compile");
    if (n_options < 0 || (n_options > 0 && !options)) return fail(CBX_ERR_ARGUMENT, "bad option list");
    nvrtcProgram prog;
    nvrtcResult r = nvrtcCreateProgram(&prog, source, name ? name : "cbx_kernel.cu", 0, nullptr, nullptr);
    if (r != NVRTC_SUCCESS) return fail(CBX_ERR_NVRTC, "nvrtcCreateProgram: %s", nvrtcGetErrorString(r));
    r = nvrtcCompileProgram(prog, n_options, options);
    size_t lsz = 0;
    std::string logs;
    if (nvrtcGetProgramLogSize(prog, &lsz) == NVRTC_SUCCESS && lsz > 1) {
        logs.resize(lsz);
        nvrtcGetProgramLog(prog, &logs[0]);
        while (!logs.empty() && logs.back() == '\0') logs.pop_back();
    }
    copy_log(logs, log, log_len);
    if (r != NVRTC_SUCCESS) {
        nvrtcDestroyProgram(&prog);
        return fail(CBX_ERR_NVRTC, "NVRTC compilation failed: %s\n%s", nvrtcGetErrorString(r),
                    logs.substr(0, 800).c_str());
    }
    size_t sz = 0;
    r = nvrtcGetCUBINSize(prog, &sz);
    if (r != NVRTC_SUCCESS || sz == 0) {
        nvrtcDestroyProgram(&prog);
        return fail(CBX_ERR_NVRTC, "nvrtcGetCUBINSize: %s (compile for a real sm_ target)",
                    nvrtcGetErrorString(r));
    }
    void* buf = malloc(sz);
    if (!buf) {
        nvrtcDestroyProgram(&prog);
        return fail(CBX_ERR_RUNTIME, "out of host memory");
    }
    r = nvrtcGetCUBIN(prog, static_cast<char*>(buf));
    nvrtcDestroyProgram(&prog);
    if (r != NVRTC_SUCCESS) {
        free(buf);
        return fail(CBX_ERR_NVRTC, "nvrtcGetCUBIN: %s", nvrtcGetErrorString(r));
    }
    *cubin = buf;
    *cubin_size = sz;
    return CBX_OK;
}

void cbx_free(void* p) { free(p); }

int cbx_module_load(const void* cubin, size_t cubin_size, int device, cbx_module** module) {
    if (!cubin || cubin_size == 0 || !module) return fail(CBX_ERR_ARGUMENT, "null argument to cbx_module_load");
    CUcontext ctx;
    int rc = ensure_context(device, &ctx);
    if (rc) return rc;
    cbx_module* m = new cbx_module();
    m->context = ctx;
    m->device = device;
    m->primary = -1;
    rc = check_cu(g_drv.cuModuleLoadData(&m->module, cubin), "cuModuleLoadData");
    if (rc) {
        delete m;
        return rc;
    }
    const char* names[4] = {"cbx_integrate_plain", "cbx_integrate_persistent", "cbx_integrate_hetero",
                            "cbx_integrate_warp"};
    int found = 0;
    for (int k = 0; k < 4; ++k) {
        if (g_drv.cuModuleGetFunction(&m->fn[k], m->module, names[k]) != CUDA_SUCCESS) m->fn[k] = nullptr;
        else ++found;
    }
    if (!found) {
        g_drv.cuModuleUnload(m->module);
        delete m;
        return fail(CBX_ERR_ARGUMENT, "the cubin defines none of the integration kernels");
    }
    if (m->fn[CBX_KERNEL_WARP]) {
        // the warp kernel's per-warp records: dynamic shared memory sized by
        // its probe symbol, opted in above the default 48 KB
        CUdeviceptr probe = 0;
        size_t bytes = 0;
        if (g_drv.cuModuleGetGlobal(&probe, &bytes, m->module, "cbx_warp_smem_probe") == CUDA_SUCCESS) {
            m->warp_smem = bytes;
            if (bytes > 48 * 1024) {
                int rc2 = check_cu(g_drv.cuFuncSetAttribute(m->fn[CBX_KERNEL_WARP],
                                                            CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES,
                                                            (int)bytes), "cuFuncSetAttribute");
                if (rc2) {
                    g_drv.cuModuleUnload(m->module);
                    delete m;
                    return rc2;
                }
            }
        }
    }
    if (m->fn[CBX_KERNEL_HETERO]) {
        CUdeviceptr probe = 0;
        size_t fams = 0;
        if (g_drv.cuModuleGetGlobal(&probe, &fams, m->module, "cbx_hetero_probe") == CUDA_SUCCESS)
            m->n_families = (int)fams;
    }
    CUdevice dev;
    g_drv.cuDeviceGet(&dev, device);
    g_drv.cuDeviceGetAttribute(&m->sm_count, CU_DEVICE_ATTRIBUTE_MULTIPROCESSOR_COUNT, dev);
    *module = m;
    return CBX_OK;
}

int cbx_module_create(const char* source, const char* const* options, int n_options, int device,
                      cbx_module** module, char* log, size_t log_len) {
    void* cubin = nullptr;
    size_t sz = 0;
    int rc = cbx_compile(source, "cbx_kernel.cu", options, n_options, &cubin, &sz, log, log_len);
    if (rc) return rc;
    rc = cbx_module_load(cubin, sz, device, module);
    free(cubin);
    return rc;
}

int cbx_module_destroy(cbx_module* module) {
    if (!module) return CBX_OK;
    if (!load_driver()) return fail(CBX_ERR_NO_DEVICE, "CUDA driver library is not available");
    CUcontext ctx;
    if (g_drv.cuCtxGetCurrent(&ctx) == CUDA_SUCCESS && ctx != module->context) g_drv.cuCtxSetCurrent(module->context);
    g_drv.cuModuleUnload(module->module);
    delete module;
    return CBX_OK;
}

int cbx_kernel_info(cbx_module* module, int kernel, int* registers, int* local_bytes, int* max_threads,
                    int* shared_bytes) {
    if (!module || kernel < 0 || kernel > 3 || !module->fn[kernel])
        return fail(CBX_ERR_ARGUMENT, "bad module or kernel index (or the module has no such kernel)");
    CUfunction f = module->fn[kernel];
    int v = 0;
    if (registers && !g_drv.cuFuncGetAttribute(&v, CU_FUNC_ATTRIBUTE_NUM_REGS, f)) *registers = v;
    if (local_bytes && !g_drv.cuFuncGetAttribute(&v, CU_FUNC_ATTRIBUTE_LOCAL_SIZE_BYTES, f)) *local_bytes = v;
    if (max_threads && !g_drv.cuFuncGetAttribute(&v, CU_FUNC_ATTRIBUTE_MAX_THREADS_PER_BLOCK, f)) *max_threads = v;
    if (shared_bytes && !g_drv.cuFuncGetAttribute(&v, CU_FUNC_ATTRIBUTE_SHARED_SIZE_BYTES, f)) *shared_bytes = v;
    return CBX_OK;
}

int cbx_occupancy(cbx_module* module, int kernel, int block, int* blocks_per_sm) {
    if (!module || kernel < 0 || kernel > 3 || !module->fn[kernel] || block <= 0 || !blocks_per_sm)
        return fail(CBX_ERR_ARGUMENT, "bad occupancy query");
    const size_t smem = kernel == CBX_KERNEL_WARP ? module->warp_smem : 0;
    return check_cu(g_drv.cuOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, module->fn[kernel], block,
                                                                      smem),
                    "cuOccupancyMaxActiveBlocksPerMultiprocessor");
}

}  // extern "C"

namespace {
// Argument checks of cbx_solve; ``need_counter`` = false for callers that
// supply the work counter themselves.
int validate_solve(const cbx_module* module, const cbx_solve_args* args, int kernel, int block, bool need_counter) {
    if (!module || !args) return fail(CBX_ERR_ARGUMENT, "null module or args");
    if (kernel != CBX_KERNEL_PLAIN && kernel != CBX_KERNEL_PERSISTENT && kernel != CBX_KERNEL_WARP)
        return fail(CBX_ERR_ARGUMENT, "unknown kernel kind %d", kernel);
    if (!module->fn[kernel]) return fail(CBX_ERR_ARGUMENT, "the module has no kernel of kind %d", kernel);
    if (block <= 0 || block > 1024 || (block % 32) != 0)
        return fail(CBX_ERR_ARGUMENT, "block size %d must be a positive multiple of 32 <= 1024", block);
    if (args->n_runs < 0 || args->run_stride < args->n_runs)
        return fail(CBX_ERR_ARGUMENT, "run_stride (%lld) must be >= n_runs (%lld)", args->run_stride,
                    args->n_runs);
    if (!args->inits || !args->status_out) return fail(CBX_ERR_ARGUMENT, "inits and status_out are required");
    if (need_counter && (kernel == CBX_KERNEL_PERSISTENT || kernel == CBX_KERNEL_WARP) && !args->work_counter)
        return fail(CBX_ERR_ARGUMENT, "the persistent and warp kernels need a zeroed work_counter");
    return CBX_OK;
}
}  // namespace

extern "C" {

int cbx_solve(cbx_module* module, const cbx_solve_args* args, int kernel, int block, int grid, void* stream) {
    int vrc = validate_solve(module, args, kernel, block, true);
    if (vrc) return vrc;
    if (args->n_runs == 0) return CBX_OK;
    CUcontext cur = nullptr;
    g_drv.cuCtxGetCurrent(&cur);
    if (cur != module->context) {
        int rc = check_cu(g_drv.cuCtxSetCurrent(module->context), "cuCtxSetCurrent");
        if (rc) return rc;
    }
    long long g = grid;
    if (g <= 0) {
        if (kernel == CBX_KERNEL_PLAIN) {
            g = (args->n_runs + block - 1) / block;
        } else {
            int per_sm = 0;
            const size_t smem = kernel == CBX_KERNEL_WARP ? module->warp_smem : 0;
            if (g_drv.cuOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, module->fn[kernel], block, smem) !=
                    CUDA_SUCCESS || per_sm <= 0)
                per_sm = 1;
            g = (long long)per_sm * module->sm_count;
            const long long runs_per_block = kernel == CBX_KERNEL_WARP ? block / 32 : block;
            long long needed = (args->n_runs + runs_per_block - 1) / runs_per_block;
            if (g > needed) g = needed;
        }
    }
    if (g > 2147483647LL) return fail(CBX_ERR_ARGUMENT, "grid too large");
    if (kernel == CBX_KERNEL_WARP && module->warp_smem == 0)
        return fail(CBX_ERR_ARGUMENT, "the warp kernel's module publishes no shared-memory size");
    const unsigned smem = kernel == CBX_KERNEL_WARP ? (unsigned)module->warp_smem : 0u;
    cbx_solve_args local = *args;
    void* params[] = {&local};
    return check_cu(g_drv.cuLaunchKernel(module->fn[kernel], (unsigned)g, 1, 1, (unsigned)block, 1, 1, smem,
                                   static_cast<CUstream>(stream), params, nullptr),
                    "cuLaunchKernel");
}

int cbx_device_info(int device, int* sm_count, int* cc_major, int* cc_minor) {
    int rc = require_driver();
    if (rc) return rc;
    rc = check_cu(g_drv.cuInit(0), "cuInit");
    if (rc) return rc;
    CUdevice dev;
    rc = check_cu(g_drv.cuDeviceGet(&dev, device), "cuDeviceGet");
    if (rc) return rc;
    if (sm_count) g_drv.cuDeviceGetAttribute(sm_count, CU_DEVICE_ATTRIBUTE_MULTIPROCESSOR_COUNT, dev);
    if (cc_major) g_drv.cuDeviceGetAttribute(cc_major, CU_DEVICE_ATTRIBUTE_COMPUTE_CAPABILITY_MAJOR, dev);
    if (cc_minor) g_drv.cuDeviceGetAttribute(cc_minor, CU_DEVICE_ATTRIBUTE_COMPUTE_CAPABILITY_MINOR, dev);
    return CBX_OK;
}

}  // extern "C"

extern "C" int cbx_solve_hetero(cbx_module* module, const cbx_hetero_args* args, int block, int grid,
                                void* stream) {
    if (!module || !args) return fail(CBX_ERR_ARGUMENT, "null module or args");
    if (!module->fn[CBX_KERNEL_HETERO]) return fail(CBX_ERR_ARGUMENT, "the module has no heterogeneous kernel");
    if (block <= 0 || block > 1024 || (block % 32) != 0)
        return fail(CBX_ERR_ARGUMENT, "block size %d must be a positive multiple of 32 <= 1024", block);
    if (args->n_families != module->n_families)
        return fail(CBX_ERR_ARGUMENT, "the module was generated for %d families, args has %d", module->n_families,
                    args->n_families);
    if (!args->work_counter) return fail(CBX_ERR_ARGUMENT, "a zeroed work_counter is required");
    if (args->first_run[0] != 0) return fail(CBX_ERR_ARGUMENT, "first_run[0] must be 0");
    for (int k = 0; k < args->n_families; ++k) {
        const cbx_solve_args& f = args->family[k];
        const long long n = args->first_run[k + 1] - args->first_run[k];
        if (n < 0) return fail(CBX_ERR_ARGUMENT, "first_run must be non-decreasing (family %d)", k);
        if (f.n_runs != n || f.run_stride < n)
            return fail(CBX_ERR_ARGUMENT, "family %d: n_runs (%lld) must equal its run range (%lld) and run_stride "
                        "must cover it", k, f.n_runs, n);
        if (n > 0 && (!f.inits || !f.status_out))
            return fail(CBX_ERR_ARGUMENT, "family %d: inits and status_out are required", k);
    }
    const long long total = args->first_run[args->n_families];
    if (total == 0) return CBX_OK;
    CUcontext cur = nullptr;
    g_drv.cuCtxGetCurrent(&cur);
    if (cur != module->context) {
        int rc = check_cu(g_drv.cuCtxSetCurrent(module->context), "cuCtxSetCurrent");
        if (rc) return rc;
    }
    long long g = grid;
    if (g <= 0) {
        int per_sm = 0;
        if (g_drv.cuOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, module->fn[CBX_KERNEL_HETERO], block, 0) !=
                CUDA_SUCCESS || per_sm <= 0)
            per_sm = 1;
        g = (long long)per_sm * module->sm_count;
        const long long needed = (total + block - 1) / block;
        if (g > needed) g = needed;
    }
    if (g > 2147483647LL) return fail(CBX_ERR_ARGUMENT, "grid too large");
    cbx_hetero_args local = *args;
    // the kernel reads first_run[F] for its own family count F
    for (int k = args->n_families + 1; k <= CBX_MAX_FAMILIES; ++k) local.first_run[k] = total;
    void* params[] = {&local};
    return check_cu(g_drv.cuLaunchKernel(module->fn[CBX_KERNEL_HETERO], (unsigned)g, 1, 1, (unsigned)block, 1, 1, 0,
                                         static_cast<CUstream>(stream), params, nullptr),
                    "cuLaunchKernel");
}

// ---------------------------------------------------------------------------
// Discrete adjoint launches.
// ---------------------------------------------------------------------------
namespace {
int resolve_adjoint(cbx_module* m) {
    if (m->adj_resolved) return CBX_OK;
    CUdeviceptr probe = 0;
    size_t bytes = 0;
    if (g_drv.cuModuleGetGlobal(&probe, &bytes, m->module, "cbx_lane_probe") != CUDA_SUCCESS)
        return fail(CBX_ERR_ARGUMENT, "module was generated without the adjoint kernels");
    CUdeviceptr probe2 = 0;
    size_t rbytes = 0;
    if (g_drv.cuModuleGetGlobal(&probe2, &rbytes, m->module, "cbx_seg_record_probe") != CUDA_SUCCESS)
        return fail(CBX_ERR_ARGUMENT, "module was generated without the adjoint kernels");
    const char* names[2] = {"cbx_adjoint_forward", "cbx_adjoint_backward"};
    for (int k = 0; k < 2; ++k) {
        int rc = check_cu(g_drv.cuModuleGetFunction(&m->adj[k], m->module, names[k]), names[k]);
        if (rc) return rc;
    }
    // a module without the probe keeps no tape
    CUdeviceptr probe3 = 0;
    size_t tbytes = 0;
    if (g_drv.cuModuleGetGlobal(&probe3, &tbytes, m->module, "cbx_tape_probe") != CUDA_SUCCESS) tbytes = 0;
    m->lane_bytes = bytes;
    m->record_bytes = rbytes;
    m->tape_bytes = tbytes > 1 ? tbytes : 0;
    m->adj_resolved = true;
    return CBX_OK;
}
}  // namespace

extern "C" int cbx_adjoint_info(cbx_module* module, long long* lane_bytes, long long* record_bytes) {
    if (!module || !lane_bytes || !record_bytes) return fail(CBX_ERR_ARGUMENT, "null module or output pointer");
    if (!load_driver()) return fail(CBX_ERR_NO_DEVICE, "CUDA driver library is not available");
    int rc = resolve_adjoint(module);
    if (rc) return rc;
    *lane_bytes = (long long)module->lane_bytes;
    *record_bytes = (long long)module->record_bytes;
    return CBX_OK;
}

extern "C" int cbx_adjoint_tape_bytes(cbx_module* module, long long* entry_bytes) {
    if (!module || !entry_bytes) return fail(CBX_ERR_ARGUMENT, "null module or output pointer");
    if (!load_driver()) return fail(CBX_ERR_NO_DEVICE, "CUDA driver library is not available");
    int rc = resolve_adjoint(module);
    if (rc) return rc;
    *entry_bytes = (long long)module->tape_bytes;
    return CBX_OK;
}

extern "C" int cbx_adjoint_launch(cbx_module* module, const cbx_solve_args* args, const cbx_adjoint_args* adj,
                                  int phase, int block, int grid, void* stream) {
    if (!module || !args || !adj) return fail(CBX_ERR_ARGUMENT, "null module, args or adjoint args");
    if (phase != 0 && phase != 1) return fail(CBX_ERR_ARGUMENT, "phase must be 0 (forward) or 1 (backward)");
    if (block <= 0 || block > 1024 || (block % 32) != 0)
        return fail(CBX_ERR_ARGUMENT, "block size %d must be a positive multiple of 32 <= 1024", block);
    if (args->n_runs < 0 || args->run_stride < args->n_runs)
        return fail(CBX_ERR_ARGUMENT, "run_stride (%lld) must be >= n_runs (%lld)", args->run_stride, args->n_runs);
    if (!args->inits || !args->work_counter)
        return fail(CBX_ERR_ARGUMENT, "inits and a zeroed work_counter are required");
    if (!adj->ckpt || !adj->ckpt_count || adj->ckpt_every < 1 || adj->max_ckpts < 1)
        return fail(CBX_ERR_ARGUMENT, "checkpoint buffers, ckpt_every >= 1 and max_ckpts >= 1 are required");
    if (phase == 0 && !args->status_out) return fail(CBX_ERR_ARGUMENT, "status_out is required");
    if (phase == 1 && (!adj->seg || !adj->grad_inits))
        return fail(CBX_ERR_ARGUMENT, "seg and grad_inits are required for the backward sweep");
    if (!load_driver()) return fail(CBX_ERR_NO_DEVICE, "CUDA driver library is not available");
    CUcontext cur = nullptr;
    g_drv.cuCtxGetCurrent(&cur);
    if (cur != module->context) {
        int rc = check_cu(g_drv.cuCtxSetCurrent(module->context), "cuCtxSetCurrent");
        if (rc) return rc;
    }
    int rc = resolve_adjoint(module);
    if (rc) return rc;
    if (module->tape_bytes > 0 && (!adj->tape || !adj->tape_flags || !adj->step_count))
        return fail(CBX_ERR_ARGUMENT, "this module's adjoint needs a step-size tape, its flag words and step "
                    "counts (%zu bytes per entry)", module->tape_bytes);
    if ((size_t)adj->lane_words * 4 < module->lane_bytes)
        return fail(CBX_ERR_ARGUMENT, "lane_words (%lld) is smaller than the module's lane image (%zu bytes)",
                    adj->lane_words, module->lane_bytes);
    if (args->n_runs == 0) return CBX_OK;
    CUfunction f = module->adj[phase];
    long long g = grid;
    if (g <= 0) {
        int per_sm = 0;
        if (g_drv.cuOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f, block, 0) != CUDA_SUCCESS || per_sm <= 0)
            per_sm = 1;
        g = (long long)per_sm * module->sm_count;
        long long needed = (args->n_runs + block - 1) / block;
        if (g > needed) g = needed;
    }
    if (g > 2147483647LL) return fail(CBX_ERR_ARGUMENT, "grid too large");
    cbx_solve_args la = *args;
    cbx_adjoint_args lg = *adj;
    void* params[] = {&la, &lg};
    return check_cu(g_drv.cuLaunchKernel(f, (unsigned)g, 1, 1, (unsigned)block, 1, 1, 0,
                                         static_cast<CUstream>(stream), params, nullptr),
                    "cuLaunchKernel");
}

// ---------------------------------------------------------------------------
// Fixed utility kernels (compiled by nvcc for sm_100a with the library).
// ---------------------------------------------------------------------------
namespace {
constexpr int kProbeIters = 4096;
constexpr int kProbeChains = 8;

// Eight independent FMA chains per thread keep the FP32 pipes full; the
// result is written so the work cannot be removed.
__global__ void __launch_bounds__(256) fp32_probe_kernel(float* out, float a, float b) {
    float x[kProbeChains];
#pragma unroll
    for (int c = 0; c < kProbeChains; ++c) x[c] = float(threadIdx.x + c);
#pragma unroll 16
    for (int i = 0; i < kProbeIters; ++i) {
#pragma unroll
        for (int c = 0; c < kProbeChains; ++c) x[c] = fmaf(x[c], a, b);
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < kProbeChains; ++c) s += x[c];
    if (s == 1.2345f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void flush_kernel(uint4* buf, size_t n16) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    size_t stride = (size_t)gridDim.x * blockDim.x;
    for (; i < n16; i += stride) buf[i] = make_uint4((unsigned)i, 0u, 0u, 1u);
}
}  // namespace

extern "C" int cbx_fp32_peak_probe(int device, double* flops, float* milliseconds) {
    if (!flops || !milliseconds) return fail(CBX_ERR_ARGUMENT, "null output pointer");
    if (cudaSetDevice(device) != cudaSuccess) return fail(CBX_ERR_RUNTIME, "cudaSetDevice failed");
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int block = 256;
    const int grid = sms * 8;
    float* out = nullptr;
    if (cudaMalloc(&out, sizeof(float) * block * grid) != cudaSuccess)
        return fail(CBX_ERR_RUNTIME, "cudaMalloc failed");
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    fp32_probe_kernel<<<grid, block>>>(out, 0.999f, 0.001f);  // warm-up
    cudaEventRecord(e0);
    fp32_probe_kernel<<<grid, block>>>(out, 0.999f, 0.001f);
    cudaEventRecord(e1);
    cudaError_t err = cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (err != cudaSuccess) return fail(CBX_ERR_RUNTIME, "probe failed: %s", cudaGetErrorString(err));
    *flops = 2.0 * kProbeIters * kProbeChains * double(block) * double(grid);
    *milliseconds = ms;
    return CBX_OK;
}

extern "C" int cbx_flush_l2(void* buffer, size_t bytes, void* stream) {
    if (!buffer || bytes < 16) return fail(CBX_ERR_ARGUMENT, "bad flush buffer");
    size_t n16 = bytes / 16;
    flush_kernel<<<1184, 256, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<uint4*>(buffer), n16);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(CBX_ERR_RUNTIME, "flush launch: %s", cudaGetErrorString(e));
    return CBX_OK;
}

// ---------------------------------------------------------------------------
// cbx_solve_noalloc: the persistent launch with its scratch in a static array.
//
// Some hosts cannot call cudaMalloc while they integrate: a custom call or
// plugin inside another framework receives only the input and output
// buffers that framework allocated (allocating behind its memory pool would
// break its accounting or a graph it is capturing), and a real-time loop
// fixes its device memory at start-up.  Besides inputs and outputs, the
// persistent kernel needs a work counter that starts at zero and a place
// for its four iteration totals.  For those hosts both live in the array
// below.  The driver creates it when it loads this library's device code on
// a device, and every device that loads it keeps its 256 bytes until the
// process exits.  The record a call uses has the same size for any batch.
// ---------------------------------------------------------------------------
namespace {
constexpr int kNoAllocWords = CBX_NOALLOC_SCRATCH_BYTES / 8;
constexpr int kNoAllocCounterWords = 1;                        // word 0: work counter
constexpr int kNoAllocRecordWords = kNoAllocCounterWords + 4;  // words 1-4: totals
static_assert(kNoAllocRecordWords <= kNoAllocWords, "scratch record larger than the scratch array");
static __device__ __align__(256) unsigned long long g_noalloc_scratch[kNoAllocWords];

constexpr int kNoAllocMaxDevices = 64;
unsigned long long* g_noalloc_addr[kNoAllocMaxDevices] = {};
std::mutex g_noalloc_mutex;

// 0 when the module lives in its device's primary context (the one the
// CUDA runtime, and so the address of the static array, belongs to).
int require_primary_context(cbx_module* m) {
    if (m->primary < 0) {
        CUdevice dev;
        int rc = check_cu(g_drv.cuDeviceGet(&dev, m->device), "cuDeviceGet");
        if (rc) return rc;
        CUcontext prim = nullptr;
        rc = check_cu(g_drv.cuDevicePrimaryCtxRetain(&prim, dev), "cuDevicePrimaryCtxRetain");
        if (rc) return rc;
        m->primary = prim == m->context ? 1 : 0;
        g_drv.cuDevicePrimaryCtxRelease(dev);
    }
    if (m->primary != 1)
        return fail(CBX_ERR_ARGUMENT, "cbx_solve_noalloc needs a module loaded in device %d's primary context "
                    "(the module was loaded while another context was current)", m->device);
    return CBX_OK;
}

// Device address of the scratch array on the module's device.  The module's
// (primary) context must be current.  The first call for a device asks the
// runtime for the address, which loads this library's device code into the
// primary context; later calls reuse the address.
int noalloc_scratch(int device, unsigned long long** out) {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (g_noalloc_addr[device]) {
        *out = g_noalloc_addr[device];
        return CBX_OK;
    }
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
        return fail(CBX_ERR_RUNTIME, "cudaGetSymbolAddress of the no-alloc scratch on device %d: %s", device,
                    cudaGetErrorString(e));
    g_noalloc_addr[device] = static_cast<unsigned long long*>(p);
    *out = g_noalloc_addr[device];
    return CBX_OK;
}
}  // namespace

extern "C" int cbx_solve_noalloc(cbx_module* module, const cbx_solve_args* args, int block, int grid,
                                 void* stream) {
    // every check that cbx_solve makes comes first: a rejected call leaves
    // the shared array untouched
    int rc = validate_solve(module, args, CBX_KERNEL_PERSISTENT, block, false);
    if (rc) return rc;
    if (module->device < 0 || module->device >= kNoAllocMaxDevices)
        return fail(CBX_ERR_ARGUMENT, "cbx_solve_noalloc supports device ordinals 0-%d, got %d",
                    kNoAllocMaxDevices - 1, module->device);
    if (!load_driver()) return fail(CBX_ERR_NO_DEVICE, "CUDA driver library is not available");
    rc = require_primary_context(module);
    if (rc) return rc;
    if (args->n_runs == 0) return CBX_OK;
    CUcontext cur = nullptr;
    g_drv.cuCtxGetCurrent(&cur);
    if (cur != module->context) {
        rc = check_cu(g_drv.cuCtxSetCurrent(module->context), "cuCtxSetCurrent");
        if (rc) return rc;
    }
    unsigned long long* scratch = nullptr;
    rc = noalloc_scratch(module->device, &scratch);
    if (rc) return rc;
    cbx_solve_args local = *args;
    local.work_counter = scratch;
    const bool scratch_totals = local.totals == nullptr;
    if (scratch_totals) local.totals = scratch + kNoAllocCounterWords;
    // The array keeps the previous call's counter and totals: clear the
    // words this call reads before it starts, in stream order.
    const size_t clear = sizeof(unsigned long long) * (scratch_totals ? kNoAllocRecordWords : kNoAllocCounterWords);
    cudaError_t e = cudaMemsetAsync(scratch, 0, clear, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return fail(CBX_ERR_RUNTIME, "clearing the no-alloc scratch: %s", cudaGetErrorString(e));
    return cbx_solve(module, &local, CBX_KERNEL_PERSISTENT, block, grid, stream);
}
