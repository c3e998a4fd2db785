// noalloc.cu -- ductgpu_solve_fields_dev_noalloc: the batched FP64 solve of
// ductgpu_solve_fields_dev for callers that must not allocate device
// memory.  Some host codes reserve the whole device up front with their
// own pool allocator and have nothing left for a library's cudaMalloc;
// others drive several streams at once and cannot afford cudaFree, which
// waits for the whole device.  This entry point keeps its scratch (the two
// intermediate fields of the four GEMM passes and the per-plane lambda)
// in a fixed array that lives in this file, so it calls no cudaMalloc,
// cudaFree or other allocating routine.
//
// Limits and rules for callers:
//  * scratch is kScratchBytes (32 MiB) per GPU, held by every GPU that
//    loads this library until the process exits; a call needs
//    2 * planes * 2 * my * my doubles of it (planes = sum of nmodes) and at
//    most kLamSlots planes -- larger calls are rejected with DUCTGPU_EARG;
//  * the array is shared by every call on a GPU and keeps the last call's
//    contents; calls whose work overlaps on one GPU (two contexts, or two
//    streams) race on it and give wrong results -- serialise them;
//  * nothing in it needs to start at zero: each call writes every scratch
//    element (lambda copy, intermediate interiors) before reading it;
//  * the array's device address is taken with cudaGetSymbolAddress when
//    the first context is created on a GPU (ductgpu_create calls
//    noalloc_reserve); under CUDA's default lazy module loading that is
//    also when the 32 MiB is taken, under eager loading
//    (CUDA_MODULE_LOADING=EAGER) it is taken when the library's code is
//    loaded on the GPU.  Create the context before a pool allocator
//    reserves the device, and before any stream capture.  If the look-up
//    fails there it is retried by the first call, which then reports it;
//  * the solve's own kernels are loaded on their first launch under lazy
//    loading, which takes device memory for their code: a caller whose
//    pool will hold the whole device sets CUDA_MODULE_LOADING=EAGER or makes
//    one call of this entry before its pool reserves the device.
#include <mutex>

#include "internal.h"

static constexpr size_t kScratchBytes = 32u << 20;
static constexpr size_t kScratchDoubles = kScratchBytes / sizeof(double);
static constexpr int kLamSlots = 4096;        // planes per call (lambda slots)
static constexpr int kMaxDevices = 64;

// The scratch itself.  In host code this name is only a stand-in for the
// device array: kernels get the address from cudaGetSymbolAddress.  No
// device code here names it, so it is marked used to stay in the image.
static __device__ __align__(256) __attribute__((used)) double g_scratch[kScratchDoubles];

namespace {

// Per-device address of g_scratch, filled once per device.
double *g_scratch_dev[kMaxDevices] = {};
std::mutex g_setup_mutex;
// Host staging of the per-plane lambda (a plain array: no host allocation
// either); shared like the device array.
double g_lam_host[kMaxDevices][kLamSlots];

int scratch_for_device(ductgpu_ctx ctx, double **out)
{
    if (ctx->device < 0 || ctx->device >= kMaxDevices)
        return duct::set_error(ctx, DUCTGPU_EARG, "noalloc: device %d beyond %d", ctx->device, kMaxDevices);
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_dev[ctx->device]) {
        int prev = 0;
        cudaError_t e = cudaGetDevice(&prev);
        if (e != cudaSuccess) return duct::check_cuda(ctx, e, "noalloc: cudaGetDevice");
        if ((e = cudaSetDevice(ctx->device)) != cudaSuccess)
            return duct::check_cuda(ctx, e, "noalloc: cudaSetDevice");
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_scratch);
        cudaSetDevice(prev);   // the caller's current device is left as it was
        if (e != cudaSuccess) return duct::check_cuda(ctx, e, "noalloc: cudaGetSymbolAddress");
        g_scratch_dev[ctx->device] = static_cast<double *>(p);
    }
    *out = g_scratch_dev[ctx->device];
    return DUCTGPU_OK;
}

}  // namespace

namespace duct {

// Called by ductgpu_create: takes the scratch's address on the context's
// GPU up front.  A failure here is not the context's: it is cleared, and
// the first call of the entry point retries and reports it.
void noalloc_reserve(ductgpu_ctx ctx)
{
    double *p = nullptr;
    if (scratch_for_device(ctx, &p) != DUCTGPU_OK) {
        ctx->err[0] = 0;
        cudaGetLastError();
    }
}

}  // namespace duct

extern "C" int ductgpu_solve_fields_dev_noalloc(ductgpu_ctx ctx, const ductgpu_field *fields, int nfields)
{
    if (!ctx) return DUCTGPU_EARG;
    if (!ctx->ready) return duct::set_error(ctx, DUCTGPU_ESTATE, "operators not set up (call ductgpu_pseudomat)");
    if (!fields || nfields < 1 || nfields > duct::kMaxFields)
        return duct::set_error(ctx, DUCTGPU_EARG, "nfields=%d (1..%d)", nfields, duct::kMaxFields);
    long long planes = 0;
    for (int i = 0; i < nfields; ++i) {
        if (fields[i].nmodes < 1) return duct::set_error(ctx, DUCTGPU_EARG, "nmodes=%d", fields[i].nmodes);
        planes += fields[i].nmodes;
    }
    const size_t ps = 2ull * ctx->my * ctx->my;   // doubles per complex plane
    const size_t work_doubles = kScratchDoubles - kLamSlots;
    if (planes > kLamSlots || 2ull * (size_t)planes * ps > work_doubles)
        return duct::set_error(ctx, DUCTGPU_EARG,
                               "noalloc: %lld planes of %dx%d need %.1f MiB of scratch; the fixed scratch "
                               "holds %.1f MiB and %d planes (use ductgpu_solve_fields_dev)",
                               planes, ctx->my, ctx->my, 2.0 * planes * ps * 8.0 / (1 << 20),
                               work_doubles * 8.0 / (1 << 20), kLamSlots);
    double *scratch = nullptr;
    int rc = scratch_for_device(ctx, &scratch);
    if (rc) return rc;

    // Run the ordinary batched solve with the context's workspace, lambda
    // array and its staging pointed at the fixed scratch; sized as above,
    // nothing in that path needs to grow them, so it allocates nothing.
    const duct::Workspace work_saved = ctx->work;
    double *const lam_saved = ctx->lam, *const lam_host_saved = ctx->lam_host;
    const int lam_cap_saved = ctx->lam_cap;
    ctx->lam = scratch;                                   // [kLamSlots], 256-byte aligned
    ctx->lam_host = g_lam_host[ctx->device];
    ctx->lam_cap = kLamSlots;
    ctx->work.buf = scratch + kLamSlots;                  // 32 KB in: still 256-byte aligned
    ctx->work.bytes = work_doubles * sizeof(double);
    // the queued flip-symmetric passes keep device counters: the same
    // passes one launch each instead
    int variant_saved[3];
    for (int c = 0; c < 3; ++c) {
        variant_saved[c] = ctx->pass_variant[c];
        if (ctx->pass_variant[c] == DUCTGPU_PASS_PARITY_QUEUE) ctx->pass_variant[c] = DUCTGPU_PASS_PARITY;
    }
    rc = ductgpu_solve_fields_dev(ctx, fields, nfields, DUCTGPU_PREC_FP64);
    for (int c = 0; c < 3; ++c) ctx->pass_variant[c] = variant_saved[c];
    ctx->work = work_saved;
    ctx->lam = lam_saved;
    ctx->lam_host = lam_host_saved;
    ctx->lam_cap = lam_cap_saved;
    return rc;
}
