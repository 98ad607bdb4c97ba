/* Launch shim for the reference's own GPU kernels (test and baseline
 * infrastructure only; nothing here is shipped).
 *
 * The reference builds blond/gpu/kernels.cu into a cubin
 * (blond/compile.py:167-169,422-490: --cubin -O3 --use_fast_math
 * -maxrregcount 32 -arch sm_XX) and launches it through CuPy RawModule with
 * 2 x SM-count blocks of MaxThreadsPerBlock threads (blond/gpu/__init__.py:
 * 46-52), choosing sm_histogram when 4 * n_slices < MaxSharedMemoryPerBlock
 * and hybrid_histogram otherwise (blond/gpu/butils_wrap_cupy.py:257-309).
 * CuPy is not installed, so this shim loads the same cubin with the CUDA
 * driver API into the current (primary) context and launches with the same
 * geometry and arguments.  All arrays are device pointers. */
#include <cuda.h>
#include <stdint.h>
#include <stdio.h>

static CUmodule mod;
static CUfunction f_kick, f_drift, f_sm_hist, f_hyb_hist, f_lik_copy, f_lik_comp;
static int grid, block, max_smem;
static char err_msg[256];

const char* refgpu_error(void) { return err_msg; }

static int check(CUresult r, const char* what) {
    if (r == CUDA_SUCCESS) return 0;
    const char* s = NULL;
    cuGetErrorString(r, &s);
    snprintf(err_msg, sizeof err_msg, "%s: %s", what, s ? s : "?");
    return (int)r;
}

int refgpu_load(const char* cubin) {
    CUdevice dev;
    CUcontext ctx;
    int rc, sms;
    if ((rc = check(cuCtxGetCurrent(&ctx), "cuCtxGetCurrent"))) return rc;
    if (!ctx) {
        snprintf(err_msg, sizeof err_msg, "no current CUDA context");
        return -1;
    }
    if ((rc = check(cuCtxGetDevice(&dev), "cuCtxGetDevice"))) return rc;
    if ((rc = check(cuModuleLoad(&mod, cubin), "cuModuleLoad"))) return rc;
    if ((rc = check(cuModuleGetFunction(&f_kick, mod, "simple_kick"), "simple_kick"))) return rc;
    if ((rc = check(cuModuleGetFunction(&f_drift, mod, "drift"), "drift"))) return rc;
    if ((rc = check(cuModuleGetFunction(&f_sm_hist, mod, "sm_histogram"), "sm_histogram"))) return rc;
    if ((rc = check(cuModuleGetFunction(&f_hyb_hist, mod, "hybrid_histogram"), "hybrid"))) return rc;
    if ((rc = check(cuModuleGetFunction(&f_lik_copy, mod, "lik_only_gm_copy"), "lik copy"))) return rc;
    if ((rc = check(cuModuleGetFunction(&f_lik_comp, mod, "lik_only_gm_comp"), "lik comp"))) return rc;
    cuDeviceGetAttribute(&sms, CU_DEVICE_ATTRIBUTE_MULTIPROCESSOR_COUNT, dev);
    cuDeviceGetAttribute(&block, CU_DEVICE_ATTRIBUTE_MAX_THREADS_PER_BLOCK, dev);
    cuDeviceGetAttribute(&max_smem, CU_DEVICE_ATTRIBUTE_MAX_SHARED_MEMORY_PER_BLOCK, dev);
    grid = 2 * sms;
    return 0;
}

static int launch(CUfunction f, unsigned smem, CUstream s, void** args, const char* what) {
    return check(cuLaunchKernel(f, grid, 1, 1, block, 1, 1, smem, s, args, NULL), what);
}

int refgpu_kick(double* dt, double* dE, int n_rf, double charge, const double* V,
                const double* om, const double* ph, int n, double acc, void* stream) {
    void* a[] = {&dt, &dE, &n_rf, &charge, &V, &om, &ph, &n, &acc};
    return launch(f_kick, 0, (CUstream)stream, a, "simple_kick");
}

int refgpu_drift(double* dt, double* dE, int solver, double T0, double length_ratio,
                 double alpha_order, double eta0, double eta1, double eta2, double a0,
                 double a1, double a2, double beta, double energy, int n, void* stream) {
    void* a[] = {&dt, &dE, &solver, &T0, &length_ratio, &alpha_order, &eta0, &eta1, &eta2,
                 &a0, &a1, &a2, &beta, &energy, &n};
    return launch(f_drift, 0, (CUstream)stream, a, "drift");
}

/* profile must be zeroed by the caller (the reference fills it with 0) */
int refgpu_slice(const double* dt, double* profile, double cut_left, double cut_right,
                 unsigned n_slices, int n, void* stream) {
    unsigned nm = (unsigned)n;
    if (4ull * n_slices < (unsigned long long)max_smem) {
        void* a[] = {&dt, &profile, &cut_left, &cut_right, &n_slices, &nm};
        return launch(f_sm_hist, 4 * n_slices, (CUstream)stream, a, "sm_histogram");
    }
    int capacity = max_smem / 4;
    void* a[] = {&dt, &profile, &cut_left, &cut_right, &n_slices, &nm, &capacity};
    return launch(f_hyb_hist, (unsigned)max_smem, (CUstream)stream, a, "hybrid_histogram");
}

/* factor: 2 * (n_slices - 1) doubles of scratch (the reference allocates it
 * per call with cp.empty) */
int refgpu_lik(double* dt, double* dE, const double* V, const double* bc, double charge,
               int n_slices, int n, double acc, double* factor, void* stream) {
    void* a[] = {&dt, &dE, &V, &bc, &charge, &n_slices, &n, &acc, &factor};
    int rc = launch(f_lik_copy, 0, (CUstream)stream, a, "lik_only_gm_copy");
    if (rc) return rc;
    return launch(f_lik_comp, 0, (CUstream)stream, a, "lik_only_gm_comp");
}
