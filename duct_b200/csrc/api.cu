// api.cu -- the extern "C" entry points of libductgpu (declared in
// include/ductgpu.h).  Host-side argument checking, buffer management and
// the helm3d drop-in live here; the numerics are in setup.cu and
// solve_*.cu.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "internal.h"

namespace duct {

int set_error(ductgpu_ctx ctx, int code, const char *fmt, ...)
{
    if (ctx) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(ctx->err, sizeof(ctx->err), fmt, ap);
        va_end(ap);
    }
    return code;
}

int check_cuda(ductgpu_ctx ctx, cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return DUCTGPU_OK;
    return set_error(ctx, e == cudaErrorMemoryAllocation ? DUCTGPU_EALLOC : DUCTGPU_ECUDA,
                     "%s: %s", what, cudaGetErrorString(e));
}

int ensure(ductgpu_ctx ctx, Workspace &w, size_t bytes)
{
    if (w.bytes >= bytes) return DUCTGPU_OK;
    if (w.buf) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(w.buf);
        w.buf = nullptr;
        w.bytes = 0;
    }
    cudaError_t e = cudaMalloc(&w.buf, bytes);
    if (e != cudaSuccess) return check_cuda(ctx, e, "workspace");
    w.bytes = bytes;
    return DUCTGPU_OK;
}

static int ensure_lam(ductgpu_ctx ctx, int planes)
{
    if (ctx->lam_cap >= planes) return DUCTGPU_OK;
    cudaStreamSynchronize(ctx->stream);
    cudaFree(ctx->lam);
    cudaFreeHost(ctx->lam_host);
    ctx->lam = nullptr;
    ctx->lam_host = nullptr;
    ctx->lam_cap = 0;
    const int cap = planes < 256 ? 256 : planes;
    DUCT_CUDA(ctx, cudaMalloc(&ctx->lam, cap * sizeof(double)));
    DUCT_CUDA(ctx, cudaMallocHost(&ctx->lam_host, cap * sizeof(double)));
    ctx->lam_cap = cap;
    return DUCTGPU_OK;
}

static int validate_field(ductgpu_ctx ctx, const ductgpu_field &f)
{
    if (!f.rhs || !f.sol || (!f.xalp && f.nmodes > 0))
        return set_error(ctx, DUCTGPU_EARG, "null field pointer");
    if (f.bound != 'd' && f.bound != 'n')
        return set_error(ctx, DUCTGPU_EARG, "bound '%c' is neither 'd' nor 'n'", f.bound);
    if (f.nmodes < 1 || f.ib < 0)
        return set_error(ctx, DUCTGPU_EARG, "nmodes=%d ib=%d", f.nmodes, f.ib);
    if (((uintptr_t)f.rhs | (uintptr_t)f.sol) & 15)
        return set_error(ctx, DUCTGPU_EARG, "field arrays must be 16-byte aligned");
    return DUCTGPU_OK;
}

// Fill ctx->lam with lambda = alambda + xalp^2 (src/helm3d.f90:67) for every
// plane of the fields and build the task list.
static int prepare(ductgpu_ctx ctx, const ductgpu_field *fields, int nfields, FieldTask *tasks)
{
    int planes = 0;
    for (int i = 0; i < nfields; ++i) planes += fields[i].nmodes;
    int rc = ensure_lam(ctx, planes);
    if (rc) return rc;
    // the pinned staging buffer may still be read by an earlier copy
    if (!ctx->capturing) DUCT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    int p = 0;
    for (int i = 0; i < nfields; ++i) {
        const ductgpu_field &f = fields[i];
        tasks[i].rhs = f.rhs;
        tasks[i].sol = f.sol;
        tasks[i].nmodes = f.nmodes;
        tasks[i].mode0 = (f.ib == 0);
        tasks[i].bound = f.bound;
        tasks[i].plane0 = p;
        // refinement steps from the spectral condition number of the worst
        // plane: (2 max|E| + lam) / (2 min|E| + lam); well-conditioned
        // fields (e.g. the implicit viscous step, lam = 2/(nu dt)) converge
        // in one step, Poisson-like fields get the configured maximum.
        const BoundOps &b = (f.bound == 'n') ? ctx->neu : ctx->dir;
        double kappa = 0.0;
        for (int k = 0; k < f.nmodes; ++k) {
            const double lam = f.alambda + f.xalp[k] * f.xalp[k];
            ctx->lam_host[p + k] = lam;
            const double lo = 2.0 * b.emin + lam;
            kappa = fmax(kappa, lo > 0.0 ? (2.0 * b.emax + lam) / lo : 1e300);
        }
        tasks[i].refine = (kappa <= 1.0e3 && ctx->refine_steps > 0) ? 1 : ctx->refine_steps;
        p += f.nmodes;
    }
    if (!ctx->capturing)
        DUCT_CUDA(ctx, cudaMemcpyAsync(ctx->lam, ctx->lam_host, planes * sizeof(double),
                                       cudaMemcpyHostToDevice, ctx->stream));
    return DUCTGPU_OK;
}

LaunchScope::LaunchScope(ductgpu_ctx ctx, int kind) : c(ctx)
{
    c->launches += 1;
    if (!c->prof_on || c->capturing) return;
    if (c->prof_used >= ductgpu_ctx_s::kProfSlots) profile_drain(c);
    slot = c->prof_used++;
    c->prof_kind[slot] = kind;
    cudaEventRecord(c->prof_ev[2 * slot], c->stream);
}

LaunchScope::~LaunchScope()
{
    if (slot >= 0) cudaEventRecord(c->prof_ev[2 * slot + 1], c->stream);
}

void profile_drain(ductgpu_ctx c)
{
    if (!c->prof_used) return;
    cudaEventSynchronize(c->prof_ev[2 * (c->prof_used - 1) + 1]);
    for (int i = 0; i < c->prof_used; ++i) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, c->prof_ev[2 * i], c->prof_ev[2 * i + 1]) == cudaSuccess) {
            c->prof_ms[c->prof_kind[i]] += ms;
            c->prof_n[c->prof_kind[i]] += 1;
        }
    }
    c->prof_used = 0;
}

}  // namespace duct

using namespace duct;

extern "C" {

int ductgpu_create(int device, ductgpu_ctx *out)
{
    if (!out) return DUCTGPU_EARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
        return DUCTGPU_ECUDA;
    if (cudaSetDevice(device) != cudaSuccess) return DUCTGPU_ECUDA;
    ductgpu_ctx c = new (std::nothrow) ductgpu_ctx_s();
    if (!c) return DUCTGPU_EALLOC;
    c->device = device;
    cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (c->num_sms < 1) c->num_sms = 1;
    if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return DUCTGPU_ECUDA;
    }
    c->stream = c->own_stream;
    if (cusolverDnCreate(&c->solver) != CUSOLVER_STATUS_SUCCESS ||
        cusolverDnSetStream(c->solver, c->stream) != CUSOLVER_STATUS_SUCCESS) {
        cudaStreamDestroy(c->own_stream);
        delete c;
        return DUCTGPU_ESOLVER;
    }
    for (int i = 0; i < kNumEvents; ++i) cudaEventCreate(&c->ev[i]);
    if (cudaMalloc(&c->dev_err, sizeof(int)) != cudaSuccess || cudaMemset(c->dev_err, 0, sizeof(int)) != cudaSuccess) {
        cusolverDnDestroy(c->solver);
        cudaStreamDestroy(c->own_stream);
        delete c;
        return DUCTGPU_EALLOC;
    }
    noalloc_reserve(c);
    *out = c;
    return DUCTGPU_OK;
}

int ductgpu_destroy(ductgpu_ctx ctx)
{
    if (!ctx) return DUCTGPU_EARG;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    free_bound(ctx->dir);
    free_bound(ctx->neu);
    for (int i = 0; i < kMaxRect; ++i) free_rect(ctx->rect[i]);
    free_shen(ctx->shen_d);
    free_shen(ctx->shen_n);
    free_bound(ctx->pois);
    cudaFree(ctx->pois_r);
    cudaFree(ctx->mf_u);
    cudaFree(ctx->mf_f);
    cudaFree(ctx->mf_sum);
    for (int i = 0; i < ductgpu_ctx_s::kMaxGraphs; ++i)
        if (ctx->graph_exec[i]) { cudaGraphExecDestroy(ctx->graph_exec[i]); cudaFree(ctx->graph_lam[i]); }
    cudaFree(ctx->xcol); cudaFree(ctx->DC); cudaFree(ctx->D2); cudaFree(ctx->AM1); cudaFree(ctx->ccw);
    cudaFree(ctx->dcr); cudaFree(ctx->pin_cc);
    cudaFree(ctx->work.buf);
    cudaFree(ctx->io.buf);
    if (ctx->cp_in) {
        cudaStreamSynchronize(ctx->cp_in);
        cudaStreamSynchronize(ctx->cp_out);
        for (int i = 0; i < ductgpu_ctx_s::kPipeChunks; ++i) {
            cudaEventDestroy(ctx->ev_in[i]);
            cudaEventDestroy(ctx->ev_out[i]);
        }
        cudaStreamDestroy(ctx->cp_in);
        cudaStreamDestroy(ctx->cp_out);
    }
    for (int i = 0; i < ductgpu_ctx_s::kTwTables; ++i) cudaFree(ctx->tw_tab[i]);
    cudaFree(ctx->dev_err);
    cudaFree(ctx->pq_ctr);
    for (int i = 0; i < ductgpu_ctx_s::kSideStreams; ++i) {
        if (ctx->side[i]) {
            cudaStreamSynchronize(ctx->side[i]);
            cudaStreamDestroy(ctx->side[i]);
        }
        if (ctx->side_join[i]) cudaEventDestroy(ctx->side_join[i]);
    }
    if (ctx->side_fork) cudaEventDestroy(ctx->side_fork);
    free_dns_aux(ctx);
    free_dlines(ctx);
    cudaFree(ctx->lam);
    cudaFreeHost(ctx->lam_host);
    for (int i = 0; i < kNumEvents; ++i) cudaEventDestroy(ctx->ev[i]);
    if (ctx->prof_ev[0])
        for (int i = 0; i < 2 * ductgpu_ctx_s::kProfSlots; ++i) cudaEventDestroy(ctx->prof_ev[i]);
    if (ctx->solver) cusolverDnDestroy(ctx->solver);
    cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return DUCTGPU_OK;
}

int ductgpu_last_error(ductgpu_ctx ctx, char *buf, int len)
{
    if (!ctx || !buf || len < 1) return DUCTGPU_EARG;
    strncpy(buf, ctx->err, (size_t)len - 1);
    buf[len - 1] = 0;
    return DUCTGPU_OK;
}

int ductgpu_set_stream(ductgpu_ctx ctx, void *cuda_stream)
{
    if (!ctx) return DUCTGPU_EARG;
    ctx->stream = cuda_stream ? (cudaStream_t)cuda_stream : ctx->own_stream;
    if (cusolverDnSetStream(ctx->solver, ctx->stream) != CUSOLVER_STATUS_SUCCESS)
        return set_error(ctx, DUCTGPU_ESOLVER, "cusolverDnSetStream");
    return DUCTGPU_OK;
}

void *ductgpu_get_stream(ductgpu_ctx ctx) { return ctx ? (void *)ctx->stream : nullptr; }

// Reads and clears the device error word set by bounded waits in kernels.
static int device_status(ductgpu_ctx ctx)
{
    int h = 0;
    DUCT_CUDA(ctx, cudaMemcpyAsync(&h, ctx->dev_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    DUCT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (h) {
        cudaMemsetAsync(ctx->dev_err, 0, sizeof(int), ctx->stream);
        if (h == 2)
            return set_error(ctx, DUCTGPU_ECUDA, "a tcgen05 pass kernel found its shared memory base misaligned "
                                                 "(not on 1024 bytes) and did nothing");
        return set_error(ctx, DUCTGPU_ETIMEOUT, "a bounded device-side wait ran out (code %d)", h);
    }
    return DUCTGPU_OK;
}

int ductgpu_synchronize(ductgpu_ctx ctx)
{
    if (!ctx) return DUCTGPU_EARG;
    int rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "synchronize");
    return rc ? rc : device_status(ctx);
}

int ductgpu_selftest_wait_timeout(ductgpu_ctx ctx, unsigned polls)
{
    if (!ctx) return DUCTGPU_EARG;
    cudaSetDevice(ctx->device);
    if (polls < 1) polls = 1;
    if (polls > (1u << 20)) polls = 1u << 20;
    return check_cuda(ctx, wait_selftest(ctx, polls), "k_wait_selftest");
}

int ductgpu_pseudomat(ductgpu_ctx ctx, int my, int mz)
{
    if (!ctx) return DUCTGPU_EARG;
    if (my != mz)
        return set_error(ctx, DUCTGPU_EARG, "IN HELM3D: MY.NE.MZ (NOT IMPLEMENTED): my=%d mz=%d", my, mz);
    cudaSetDevice(ctx->device);
    return pseudomat_gpu(ctx, my, true);
}

int ductgpu_pseudomat_ex(ductgpu_ctx ctx, int my, int mz, int flags)
{
    if (!ctx) return DUCTGPU_EARG;
    if (my != mz)
        return set_error(ctx, DUCTGPU_EARG, "IN HELM3D: MY.NE.MZ (NOT IMPLEMENTED): my=%d mz=%d", my, mz);
    if (flags & ~DUCTGPU_SETUP_NO_EIGEN) return set_error(ctx, DUCTGPU_EARG, "setup flags 0x%x", flags);
    cudaSetDevice(ctx->device);
    return pseudomat_gpu(ctx, my, !(flags & DUCTGPU_SETUP_NO_EIGEN));
}

int ductgpu_set_gauge_point(ductgpu_ctx ctx, int iofzero)
{
    if (!ctx) return DUCTGPU_EARG;
    if (!ctx->grid_ready) return set_error(ctx, DUCTGPU_ESTATE, "call ductgpu_pseudomat first");
    if (iofzero < 0 || iofzero > ctx->my - 2)
        return set_error(ctx, DUCTGPU_EARG, "gauge point %d outside 0..%d", iofzero, ctx->my - 2);
    ctx->pin_point = iofzero;
    return DUCTGPU_OK;
}

int ductgpu_get_operators(ductgpu_ctx ctx, char bound, double *E, double *P, double *PM1, int *iofzero)
{
    if (!ctx) return DUCTGPU_EARG;
    if (bound == 'p' ? !ctx->pois_m : !ctx->ready) return set_error(ctx, DUCTGPU_ESTATE, "operators not set up");
    if (bound != 'd' && bound != 'n' && bound != 'p') return set_error(ctx, DUCTGPU_EARG, "bound '%c'", bound);
    const BoundOps &b = (bound == 'p') ? ctx->pois : (bound == 'n') ? ctx->neu : ctx->dir;
    const size_t nn = (size_t)b.n * b.n;
    if (E) DUCT_CUDA(ctx, cudaMemcpyAsync(E, b.E, b.n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (P) DUCT_CUDA(ctx, cudaMemcpyAsync(P, b.P, nn * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (PM1) DUCT_CUDA(ctx, cudaMemcpyAsync(PM1, b.PM1, nn * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    DUCT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (iofzero) *iofzero = b.iofzero;
    return DUCTGPU_OK;
}

int ductgpu_set_operators(ductgpu_ctx ctx, char bound, const double *E, const double *P, const double *PM1, int iofzero)
{
    if (!ctx) return DUCTGPU_EARG;
    if (bound == 'p' ? !ctx->pois_m : !ctx->grid_ready)
        return set_error(ctx, DUCTGPU_ESTATE, bound == 'p' ? "call ductgpu_pseudopois first" : "call ductgpu_pseudomat first");
    if (bound != 'd' && bound != 'n' && bound != 'p') return set_error(ctx, DUCTGPU_EARG, "bound '%c'", bound);
    if (!E || !P || !PM1) return set_error(ctx, DUCTGPU_EARG, "null operator");
    BoundOps &b = (bound == 'p') ? ctx->pois : (bound == 'n') ? ctx->neu : ctx->dir;
    const size_t nn = (size_t)b.n * b.n;
    DUCT_CUDA(ctx, cudaMemcpyAsync(b.E, E, b.n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    DUCT_CUDA(ctx, cudaMemcpyAsync(b.P, P, nn * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    DUCT_CUDA(ctx, cudaMemcpyAsync(b.PM1, PM1, nn * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    {
        double emin = 1e300, emax = 0.0;
        for (int i = 0; i < b.n; ++i) { emin = fmin(emin, fabs(E[i])); emax = fmax(emax, fabs(E[i])); }
        b.emin = emin;
        b.emax = emax;
    }
    if (bound != 'd') {
        if (iofzero <= 0) {
            double eigmin = 1.0e6;
            iofzero = 0;
            for (int i = 0; i < b.n; ++i) {
                const double e = fmin(eigmin, fabs(E[i]));
                if (e != eigmin) { iofzero = i + 1; eigmin = e; }
            }
        }
        if (iofzero > b.n) return set_error(ctx, DUCTGPU_EARG, "iofzero %d > n", iofzero);
        b.iofzero = iofzero;
    }
    int rc = pack_operators(ctx, b);
    if (rc) return rc;
    // Imported operators are applied as given, on the full passes.  Their
    // half blocks cannot be read off them: the eigenvectors of a block built
    // in floating point are even or odd only to the block's own asymmetry
    // (~1e-12 relative), and dropping that part moves the solve ~1e-11 away
    // from the imported decomposition's.
    cudaFree(b.Pfold);
    cudaFree(b.Qfold);
    cudaFree(b.PfoldT);
    cudaFree(b.QfoldT);
    cudaFree(b.Eperm);
    b.Pfold = b.Qfold = b.PfoldT = b.QfoldT = b.Eperm = nullptr;
    b.fold_ok = false;
    if ((rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "set_operators"))) return rc;
    if (bound != 'p') {
        ctx->ops_set |= (bound == 'd') ? 1 : 2;
        ctx->ready = ctx->grid_ready && ctx->ops_set == 3;
    }
    return DUCTGPU_OK;
}

int ductgpu_get_fold(ductgpu_ctx ctx, char bound, int *folded)
{
    if (!ctx || !folded) return DUCTGPU_EARG;
    if (bound != 'd' && bound != 'n') return set_error(ctx, DUCTGPU_EARG, "bound '%c'", bound);
    *folded = ((bound == 'n') ? ctx->neu : ctx->dir).fold_ok ? 1 : 0;
    return DUCTGPU_OK;
}

int ductgpu_set_gauge(ductgpu_ctx ctx, int gauge)
{
    if (!ctx) return DUCTGPU_EARG;
    if (gauge != DUCTGPU_GAUGE_POINT && gauge != DUCTGPU_GAUGE_MEAN)
        return set_error(ctx, DUCTGPU_EARG, "gauge %d", gauge);
    ctx->gauge = gauge;
    return DUCTGPU_OK;
}

int ductgpu_set_refinement(ductgpu_ctx ctx, int steps)
{
    if (!ctx) return DUCTGPU_EARG;
    if (steps < 0 || steps > 4) return set_error(ctx, DUCTGPU_EARG, "refinement steps %d (0..4)", steps);
    ctx->refine_steps = steps;
    return DUCTGPU_OK;
}

int ductgpu_set_pass_kernel(ductgpu_ctx ctx, int size_class, int kernel)
{
    if (!ctx) return DUCTGPU_EARG;
    if (kernel < -1 || kernel > DUCTGPU_PASS_PARITY_QUEUE)
        return set_error(ctx, DUCTGPU_EARG, "pass kernel %d", kernel);
    if (size_class < -1 || size_class > 2) return set_error(ctx, DUCTGPU_EARG, "size class %d", size_class);
    for (int c = 0; c < 3; ++c)
        if (size_class < 0 || size_class == c) ctx->pass_variant[c] = (kernel < 0) ? kPassDefault[c] : kernel;
    return DUCTGPU_OK;
}

int ductgpu_set_line_kernel(ductgpu_ctx ctx, int kernel)
{
    if (!ctx || kernel < 0 || kernel > 2) return DUCTGPU_EARG;
    ctx->dlines = kernel;
    return DUCTGPU_OK;
}

int ductgpu_set_rect_fold(ductgpu_ctx ctx, int on)
{
    if (!ctx) return DUCTGPU_EARG;
    if (on < 0 || on > 2) return set_error(ctx, DUCTGPU_EARG, "rect fold %d (0, 1, 2)", on);
    ctx->rect_fold = on;
    return DUCTGPU_OK;
}

int ductgpu_autotune(ductgpu_ctx ctx, const ductgpu_field *fields, int nfields, int reps, int *chosen)
{
    if (!ctx) return DUCTGPU_EARG;
    if (!ctx->ready) return set_error(ctx, DUCTGPU_ESTATE, "operators not set up (call ductgpu_pseudomat)");
    if (ctx->capturing) return set_error(ctx, DUCTGPU_ESTATE, "autotune during graph capture");
    if (reps < 1) reps = 5;
    const int cls = (ctx->my - 2 + 63) / 64 - 1;
    if (cls < 0 || cls > 2) return set_error(ctx, DUCTGPU_EARG, "grid %d", ctx->my);
    const int variants[6] = {DUCTGPU_PASS_STAGED, DUCTGPU_PASS_STAGED16, DUCTGPU_PASS_REGISTER, DUCTGPU_PASS_PERSIST,
                             DUCTGPU_PASS_PARITY, DUCTGPU_PASS_PARITY_QUEUE};
    const int saved = ctx->pass_variant[cls];
    const bool prof = ctx->prof_on;
    ctx->prof_on = false;
    float best_ms = 1e30f;
    int best = saved, rc = DUCTGPU_OK;
    for (int v : variants) {
        ctx->pass_variant[cls] = v;
        if ((rc = ductgpu_solve_fields_dev(ctx, fields, nfields, DUCTGPU_PREC_FP64))) break;   // warm-up
        if ((rc = check_cuda(ctx, cudaEventRecord(ctx->ev[kNumEvents - 2], ctx->stream), "autotune"))) break;
        for (int r = 0; r < reps && !rc; ++r) rc = ductgpu_solve_fields_dev(ctx, fields, nfields, DUCTGPU_PREC_FP64);
        if (rc) break;
        if ((rc = check_cuda(ctx, cudaEventRecord(ctx->ev[kNumEvents - 1], ctx->stream), "autotune"))) break;
        if ((rc = check_cuda(ctx, cudaEventSynchronize(ctx->ev[kNumEvents - 1]), "autotune"))) break;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev[kNumEvents - 2], ctx->ev[kNumEvents - 1]);
        if (ms < best_ms) { best_ms = ms; best = v; }
    }
    ctx->prof_on = prof;
    ctx->pass_variant[cls] = rc ? saved : best;
    if (chosen) *chosen = ctx->pass_variant[cls];
    return rc;
}

int ductgpu_solve_fields_dev(ductgpu_ctx ctx, const ductgpu_field *fields, int nfields, int precision)
{
    if (!ctx) return DUCTGPU_EARG;
    if (!ctx->ready) return set_error(ctx, DUCTGPU_ESTATE, "operators not set up (call ductgpu_pseudomat)");
    if (!fields || nfields < 1 || nfields > kMaxFields)
        return set_error(ctx, DUCTGPU_EARG, "nfields=%d (1..%d)", nfields, kMaxFields);
    if (precision != DUCTGPU_PREC_FP64 && precision != DUCTGPU_PREC_MIXED && precision != DUCTGPU_PREC_INT8)
        return set_error(ctx, DUCTGPU_EARG, "precision %d", precision);
    for (int i = 0; i < nfields; ++i) {
        int rc = validate_field(ctx, fields[i]);
        if (rc) return rc;
    }
    cudaSetDevice(ctx->device);
    FieldTask tasks[kMaxFields];
    int rc = prepare(ctx, fields, nfields, tasks);
    if (rc) return rc;
    if (precision == DUCTGPU_PREC_MIXED) return solve_mixed(ctx, tasks, nfields);
    if (precision == DUCTGPU_PREC_INT8) {
        if (ctx->my - 2 > 127)
            return set_error(ctx, DUCTGPU_EARG, "int8-emulated solve: my=%d (at most 129)", ctx->my);
        return solve_fp64_ex(ctx, tasks, nfields, true);
    }
    return solve_fp64(ctx, tasks, nfields);
}

int ductgpu_helm3d(ductgpu_ctx ctx, double *rhs, double *sol, int ipro, char bound, double alambda,
                   int my, int mz, int ib, int ie, const double *xalp, int precision)
{
    if (!ctx) return DUCTGPU_EARG;
    if (ipro <= 0) {
        int rc = ductgpu_pseudomat(ctx, my, mz);
        if (rc) return rc;
        if (ipro == -1) return DUCTGPU_OK;
    }
    if (!ctx->ready) return set_error(ctx, DUCTGPU_ESTATE, "operators not set up (call with ipro<=0)");
    if (my != ctx->my || mz != ctx->mz)
        return set_error(ctx, DUCTGPU_EARG, "grid %dx%d differs from the set-up %dx%d", my, mz, ctx->my, ctx->mz);
    if (!rhs || !sol || !xalp) return set_error(ctx, DUCTGPU_EARG, "null pointer");
    if (bound != 'd' && bound != 'n')
        return set_error(ctx, DUCTGPU_EARG, "in solvediag error in BC: bound '%c'", bound);
    if (ie < ib || ib < 0) return set_error(ctx, DUCTGPU_EARG, "ib=%d ie=%d", ib, ie);
    cudaSetDevice(ctx->device);
    const int nm = ie - ib + 1;
    const size_t bytes = (size_t)2 * my * mz * nm * sizeof(double);
    // helm3d zeroes the Dirichlet walls of rhs in place (src/helm3d.f90:48-60)
    if (bound == 'd') {
        for (int i = 0; i < nm; ++i) {
            double *r = rhs + (size_t)2 * my * mz * i;
            for (int j = 0; j < my; ++j) {
                r[2 * j] = r[2 * j + 1] = 0.0;
                r[2 * (j + (size_t)my * (mz - 1))] = r[2 * (j + (size_t)my * (mz - 1)) + 1] = 0.0;
            }
            for (int k = 0; k < mz; ++k) {
                r[2 * ((size_t)my * k)] = r[2 * ((size_t)my * k) + 1] = 0.0;
                r[2 * (my - 1 + (size_t)my * k)] = r[2 * (my - 1 + (size_t)my * k) + 1] = 0.0;
            }
        }
    }
    int rc = ensure(ctx, ctx->io, 2 * bytes);
    if (rc) return rc;
    double *drhs = ctx->io.buf, *dsol = ctx->io.buf + bytes / sizeof(double);
    ductgpu_field f;
    f.rhs = drhs;
    f.sol = dsol;
    f.xalp = xalp;
    f.alambda = alambda;
    f.ib = ib;
    f.nmodes = nm;
    f.bound = bound;
    DUCT_CUDA(ctx, cudaMemcpyAsync(drhs, rhs, bytes, cudaMemcpyHostToDevice, ctx->stream));
    rc = ductgpu_solve_fields_dev(ctx, &f, 1, precision);
    if (rc) return rc;
    DUCT_CUDA(ctx, cudaMemcpyAsync(sol, dsol, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "helm3d");
    return rc ? rc : device_status(ctx);
}

// Several fields of one substep on host arrays (u, v, w and p of
// src/main1.f90:617-619, 643), with the host<->device copies overlapped:
// a piece (a field, or a mode range of the first or last field) is copied
// in on one stream while the previous piece is solved on the context stream
// and the one before copied back on a third.  From pinned host memory
// (ductgpu_host_alloc) the copies run asynchronously; pageable memory gives
// the same results.
// Mode ranges per field in ductgpu_helm3d_batch: the first and the last
// field go through in two, the others whole.  Only the head (the first
// upload, before any download can start) and the tail (the last solve and
// download, after the uploads end) use one direction of the host link, so
// halving those two pieces is what pays; splitting every field adds solves
// of small batches (0.06 ms of launches each) between the copies and was
// slower.  cfg1 (4 fields of 64 modes, pinned host arrays): one piece per
// field 1.94 ms a call, first and last in two 1.87 ms, every field in two
// 2.08 ms, in four 2.40 ms.  The first field's first piece is a quarter of
// its modes (the upload before anything else can run), the last field's
// last piece too: 1.847 against 1.866 ms for halves.
static int batch_pieces(int i, int nfields) { return (i == 0 || i == nfields - 1) ? 2 : 1; }
// first mode of piece q of field i (q = 0 .. pieces)
static int batch_cut(int i, int q, int pieces, int nm)
{
    if (pieces != 2 || q != 1) return nm * q / pieces;
    const int quarter = nm / 4 > 1 ? nm / 4 : 1;   // pieces == 2 only when nm >= 2
    return (i == 0) ? quarter : nm - quarter;
}

int ductgpu_helm3d_batch(ductgpu_ctx ctx, int nfields, double *const *rhs, double *const *sol, const char *bounds,
                         const double *alambdas, int my, int mz, int ib, int ie, const double *xalp, int precision)
{
    if (!ctx) return DUCTGPU_EARG;
    if (!ctx->ready) return set_error(ctx, DUCTGPU_ESTATE, "operators not set up (call ductgpu_pseudomat)");
    if (nfields < 1 || nfields > kMaxFields || !rhs || !sol || !bounds || !alambdas || !xalp)
        return set_error(ctx, DUCTGPU_EARG, "helm3d_batch: nfields=%d or null argument", nfields);
    if (my != ctx->my || mz != ctx->mz)
        return set_error(ctx, DUCTGPU_EARG, "grid %dx%d differs from the set-up %dx%d", my, mz, ctx->my, ctx->mz);
    if (ie < ib || ib < 0) return set_error(ctx, DUCTGPU_EARG, "ib=%d ie=%d", ib, ie);
    if (precision != DUCTGPU_PREC_FP64 && precision != DUCTGPU_PREC_INT8 && precision != DUCTGPU_PREC_MIXED)
        return set_error(ctx, DUCTGPU_EARG, "precision %d", precision);
    if (precision == DUCTGPU_PREC_INT8 && ctx->my - 2 > 127)
        return set_error(ctx, DUCTGPU_EARG, "int8-emulated solve: my=%d (at most 129)", ctx->my);
    for (int i = 0; i < nfields; ++i) {
        if (!rhs[i] || !sol[i]) return set_error(ctx, DUCTGPU_EARG, "null field %d", i);
        if (bounds[i] != 'd' && bounds[i] != 'n') return set_error(ctx, DUCTGPU_EARG, "bound '%c'", bounds[i]);
    }
    cudaSetDevice(ctx->device);
    if (!ctx->cp_in) {
        DUCT_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->cp_in, cudaStreamNonBlocking));
        DUCT_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->cp_out, cudaStreamNonBlocking));
        for (int i = 0; i < ductgpu_ctx_s::kPipeChunks; ++i) {
            DUCT_CUDA(ctx, cudaEventCreateWithFlags(&ctx->ev_in[i], cudaEventDisableTiming));
            DUCT_CUDA(ctx, cudaEventCreateWithFlags(&ctx->ev_out[i], cudaEventDisableTiming));
        }
    }
    const int nm = ie - ib + 1;
    const size_t doubles = (size_t)2 * my * mz * nm, bytes = doubles * sizeof(double);
    int rc = ensure(ctx, ctx->io, 2 * bytes * nfields);
    if (rc) return rc;
    ductgpu_field f[kMaxFields];
    for (int i = 0; i < nfields; ++i) {
        f[i].rhs = ctx->io.buf + 2 * doubles * i;
        f[i].sol = f[i].rhs + doubles;
        f[i].xalp = xalp;
        f[i].alambda = alambdas[i];
        f[i].ib = ib;
        f[i].nmodes = nm;
        f[i].bound = bounds[i];
    }
    // lambda of every plane of the batch staged and uploaded once, before the
    // first field copy is queued (a per-solve upload would wait behind the
    // field copies on the copy engines, and the per-call staging sync would
    // hold the host until the previous solve ended)
    FieldTask tasks[kMaxFields];
    if ((rc = prepare(ctx, f, nfields, tasks))) return rc;
    // Each field goes through in batch_pieces mode ranges: piece j is copied
    // in while piece j-1 is solved and piece j-2 copied back, so both
    // directions of the host link run at once for all but the first and the
    // last piece.  Events are reused round-robin: every wait on an event is
    // enqueued before the event is recorded again.
    const size_t plane = (size_t)2 * my * mz;
    int e = 0;
    for (int i = 0; i < nfields; ++i)
        for (int p = 0, pieces = nm < batch_pieces(i, nfields) ? nm : batch_pieces(i, nfields); p < pieces; ++p, ++e) {
            const int k0 = batch_cut(i, p, pieces, nm), k1 = batch_cut(i, p + 1, pieces, nm);
            FieldTask t = tasks[i];
            t.rhs = f[i].rhs + plane * k0;
            t.sol = f[i].sol + plane * k0;
            t.nmodes = k1 - k0;
            t.mode0 = (ib + k0 == 0);
            t.plane0 = tasks[i].plane0 + k0;
            const size_t pb = plane * (k1 - k0) * sizeof(double);
            cudaEvent_t ein = ctx->ev_in[e % ductgpu_ctx_s::kPipeChunks];
            cudaEvent_t eout = ctx->ev_out[e % ductgpu_ctx_s::kPipeChunks];
            DUCT_CUDA(ctx, cudaMemcpyAsync(t.rhs, rhs[i] + plane * k0, pb, cudaMemcpyHostToDevice, ctx->cp_in));
            DUCT_CUDA(ctx, cudaEventRecord(ein, ctx->cp_in));
            DUCT_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ein, 0));
            rc = (precision == DUCTGPU_PREC_MIXED) ? solve_mixed(ctx, &t, 1)
                                                   : solve_fp64_ex(ctx, &t, 1, precision == DUCTGPU_PREC_INT8);
            if (rc) return rc;
            DUCT_CUDA(ctx, cudaEventRecord(eout, ctx->stream));
            DUCT_CUDA(ctx, cudaStreamWaitEvent(ctx->cp_out, eout, 0));
            DUCT_CUDA(ctx, cudaMemcpyAsync(sol[i] + plane * k0, t.sol, pb, cudaMemcpyDeviceToHost, ctx->cp_out));
        }
    // helm3d zeroes the Dirichlet walls of rhs in place (src/helm3d.f90:48-60).
    // Done here, while the copies and solves run: the solve reads only the
    // interior of rhs (the device copy's walls are zeroed on the device), so
    // whether a wall value reaches the device before or after it is zeroed
    // does not matter.
    for (int i = 0; i < nfields; ++i)
        if (bounds[i] == 'd')
            for (int k = 0; k < nm; ++k) {
                double *r = rhs[i] + (size_t)2 * my * mz * k;
                for (int j = 0; j < my; ++j) {
                    r[2 * j] = r[2 * j + 1] = 0.0;
                    r[2 * (j + (size_t)my * (mz - 1))] = r[2 * (j + (size_t)my * (mz - 1)) + 1] = 0.0;
                }
                for (int q = 0; q < mz; ++q) {
                    r[2 * ((size_t)my * q)] = r[2 * ((size_t)my * q) + 1] = 0.0;
                    r[2 * (my - 1 + (size_t)my * q)] = r[2 * (my - 1 + (size_t)my * q) + 1] = 0.0;
                }
            }
    DUCT_CUDA(ctx, cudaStreamSynchronize(ctx->cp_out));
    rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "helm3d_batch");
    return rc ? rc : device_status(ctx);
}

static int check_field(ductgpu_ctx ctx, const void *a, int my, int mz, int nmodes)
{
    if (!a) return set_error(ctx, DUCTGPU_EARG, "null field");
    if (my < 2 || mz < 2 || nmodes < 1) return set_error(ctx, DUCTGPU_EARG, "my=%d mz=%d nmodes=%d", my, mz, nmodes);
    if ((uintptr_t)a & 15) return set_error(ctx, DUCTGPU_EARG, "field must be 16-byte aligned");
    return DUCTGPU_OK;
}

int ductgpu_transyz_dev(ductgpu_ctx ctx, double *field, int my, int mz, int nmodes, char cdir, int iopt)
{
    if (!ctx) return DUCTGPU_EARG;
    int rc = check_field(ctx, field, my, mz, nmodes);
    if (rc) return rc;
    if (cdir != 'y' && cdir != 'z') return set_error(ctx, DUCTGPU_EARG, "err in transyz: cdir '%c'", cdir);
    cudaSetDevice(ctx->device);
    return transyz_dev(ctx, field, my, mz, nmodes, cdir, iopt);
}

// Host-array variant: copies through the context's io workspace.
static int host_roundtrip(ductgpu_ctx ctx, double *host, size_t bytes, double **dev)
{
    int rc = ensure(ctx, ctx->io, 2 * bytes);
    if (rc) return rc;
    *dev = ctx->io.buf;
    DUCT_CUDA(ctx, cudaMemcpyAsync(*dev, host, bytes, cudaMemcpyHostToDevice, ctx->stream));
    return DUCTGPU_OK;
}

int ductgpu_transyz(ductgpu_ctx ctx, double *field, int my, int mz, int nmodes, char cdir, int iopt)
{
    if (!ctx) return DUCTGPU_EARG;
    int rc = check_field(ctx, field, my, mz, nmodes);
    if (rc) return rc;
    cudaSetDevice(ctx->device);
    const size_t bytes = (size_t)2 * my * mz * nmodes * sizeof(double);
    double *d = nullptr;
    if ((rc = host_roundtrip(ctx, field, bytes, &d))) return rc;
    if ((rc = ductgpu_transyz_dev(ctx, d, my, mz, nmodes, cdir, iopt))) return rc;
    DUCT_CUDA(ctx, cudaMemcpyAsync(field, d, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    return check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "transyz");
}

int ductgpu_derivyz_dev(ductgpu_ctx ctx, const double *u, double *du, int my, int mz, int nmodes, char cdir,
                        int ider, double scal, char what, double aspect)
{
    if (!ctx) return DUCTGPU_EARG;
    int rc = check_field(ctx, u, my, mz, nmodes);
    if (rc || (rc = check_field(ctx, du, my, mz, nmodes))) return rc;
    if (cdir != 'y' && cdir != 'z') return set_error(ctx, DUCTGPU_EARG, "problem in derivyz: direction '%c'", cdir);
    if (ider != 1 && ider != 2) return set_error(ctx, DUCTGPU_EARG, "this order of deriv not implemented: %d", ider);
    if (u == du) return set_error(ctx, DUCTGPU_EARG, "derivyz: u and du must not overlap");
    cudaSetDevice(ctx->device);
    return derivyz_dev(ctx, u, du, my, mz, nmodes, cdir, ider, scal, what, aspect);
}

int ductgpu_derivyz(ductgpu_ctx ctx, const double *u, double *du, int my, int mz, int nmodes, char cdir,
                    int ider, double scal, char what, double aspect)
{
    if (!ctx) return DUCTGPU_EARG;
    int rc = check_field(ctx, u, my, mz, nmodes);
    if (rc || (rc = check_field(ctx, du, my, mz, nmodes))) return rc;
    cudaSetDevice(ctx->device);
    const size_t bytes = (size_t)2 * my * mz * nmodes * sizeof(double);
    if ((rc = ensure(ctx, ctx->io, 2 * bytes))) return rc;
    double *du_d = ctx->io.buf, *u_d = ctx->io.buf + bytes / sizeof(double);
    DUCT_CUDA(ctx, cudaMemcpyAsync(u_d, u, bytes, cudaMemcpyHostToDevice, ctx->stream));
    DUCT_CUDA(ctx, cudaMemcpyAsync(du_d, du, bytes, cudaMemcpyHostToDevice, ctx->stream));
    if ((rc = ductgpu_derivyz_dev(ctx, u_d, du_d, my, mz, nmodes, cdir, ider, scal, what, aspect))) return rc;
    DUCT_CUDA(ctx, cudaMemcpyAsync(du, du_d, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    return check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "derivyz");
}

int ductgpu_cxyz2yzx_dev(ductgpu_ctx ctx, const double *phys, double *phys2, int nmodes, int my, int nz)
{
    if (!ctx) return DUCTGPU_EARG;
    int rc = check_field(ctx, phys, my, nz, nmodes);
    if (rc || (rc = check_field(ctx, phys2, my, nz, nmodes))) return rc;
    cudaSetDevice(ctx->device);
    return transpose_dev(ctx, phys, phys2, nmodes, (long long)my * nz);
}

int ductgpu_cyzx2xyz_dev(ductgpu_ctx ctx, double *phys, const double *phys2, int nmodes, int my, int nz)
{
    if (!ctx) return DUCTGPU_EARG;
    int rc = check_field(ctx, phys, my, nz, nmodes);
    if (rc || (rc = check_field(ctx, phys2, my, nz, nmodes))) return rc;
    cudaSetDevice(ctx->device);
    return transpose_dev(ctx, phys2, phys, (long long)my * nz, nmodes);
}

int ductgpu_chx2z_dev(ductgpu_ctx ctx, double *xy, double *xz, int my, int mz, int nmodes)
{
    if (!ctx) return DUCTGPU_EARG;
    int rc = check_field(ctx, xy, my, mz, nmodes);
    if (rc || (rc = check_field(ctx, xz, my, mz, nmodes))) return rc;
    if (xy == xz) return set_error(ctx, DUCTGPU_EARG, "chx2z: xy and xz must differ");
    cudaSetDevice(ctx->device);
    const size_t bytes = (size_t)2 * my * mz * nmodes * sizeof(double);
    DUCT_CUDA(ctx, cudaMemcpyAsync(xz, xy, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    return transpose_dev(ctx, xz, xy, (long long)my * mz, nmodes);
}

int ductgpu_chz2x_dev(ductgpu_ctx ctx, double *xz, double *xy, int my, int mz, int nmodes)
{
    if (!ctx) return DUCTGPU_EARG;
    int rc = check_field(ctx, xy, my, mz, nmodes);
    if (rc || (rc = check_field(ctx, xz, my, mz, nmodes))) return rc;
    if (xy == xz) return set_error(ctx, DUCTGPU_EARG, "chz2x: xy and xz must differ");
    cudaSetDevice(ctx->device);
    if ((rc = transpose_dev(ctx, xz, xy, nmodes, (long long)my * mz))) return rc;
    const size_t bytes = (size_t)2 * my * mz * nmodes * sizeof(double);
    return check_cuda(ctx, cudaMemcpyAsync(xz, xy, bytes, cudaMemcpyDeviceToDevice, ctx->stream), "chz2x copy");
}

int ductgpu_pseudomat_temp(ductgpu_ctx ctx, int slot, int my, int mz, double sy, double sz,
                           char by1, char by2, char bz1, char bz2)
{
    if (!ctx) return DUCTGPU_EARG;
    cudaSetDevice(ctx->device);
    return rect_setup(ctx, slot, my, mz, sy, sz, by1, by2, bz1, bz2);
}

int ductgpu_solve_rect_fields_dev(ductgpu_ctx ctx, const ductgpu_rect_field *fields, int nfields)
{
    if (!ctx) return DUCTGPU_EARG;
    if (!fields || nfields < 1 || nfields > kMaxFields)
        return set_error(ctx, DUCTGPU_EARG, "nfields=%d (1..%d)", nfields, kMaxFields);
    int planes = 0;
    for (int i = 0; i < nfields; ++i) {
        const ductgpu_rect_field &f = fields[i];
        if (f.slot < 0 || f.slot >= kMaxRect || !ctx->rect[f.slot].ready)
            return set_error(ctx, DUCTGPU_ESTATE, "rectangular slot %d not set up", f.slot);
        if (!f.rhs || !f.sol || !f.xalp) return set_error(ctx, DUCTGPU_EARG, "null field pointer");
        if (f.nmodes < 1 || f.ib < 0) return set_error(ctx, DUCTGPU_EARG, "nmodes=%d ib=%d", f.nmodes, f.ib);
        if (((uintptr_t)f.rhs | (uintptr_t)f.sol) & 15) return set_error(ctx, DUCTGPU_EARG, "field arrays must be 16-byte aligned");
        planes += f.nmodes;
    }
    cudaSetDevice(ctx->device);
    int rc = ensure_lam(ctx, planes);
    if (rc) return rc;
    if (!ctx->capturing) DUCT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    RectTask tasks[kMaxFields];
    int p = 0;
    for (int i = 0; i < nfields; ++i) {
        const ductgpu_rect_field &f = fields[i];
        tasks[i].rhs = f.rhs;
        tasks[i].sol = f.sol;
        tasks[i].bcy = f.bcy;
        tasks[i].bcz = f.bcz;
        tasks[i].nmodes = f.nmodes;
        tasks[i].mode0 = (f.ib == 0);
        tasks[i].plane0 = p;
        tasks[i].slot = f.slot;
        for (int k = 0; k < f.nmodes; ++k) ctx->lam_host[p + k] = f.alambda + f.xalp[k] * f.xalp[k];
        p += f.nmodes;
    }
    if (!ctx->capturing)
        DUCT_CUDA(ctx, cudaMemcpyAsync(ctx->lam, ctx->lam_host, planes * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    return solve_rect(ctx, tasks, nfields);
}

int ductgpu_helm3d_temp(ductgpu_ctx ctx, double *rhs, double *sol, int ipro, double a, double b, double alambda,
                        int my, int mz, int ib, int ie, const double *xalp, const double *bcy, const double *bcz,
                        char by1, char by2, char bz1, char bz2)
{
    if (!ctx) return DUCTGPU_EARG;
    if (ipro <= 0) {
        int rc = ductgpu_pseudomat_temp(ctx, 0, my, mz, a, b, by1, by2, bz1, bz2);
        if (rc) return rc;
        if (ipro == -1) return DUCTGPU_OK;
    }
    const RectSlot &r = ctx->rect[0];
    if (!r.ready) return set_error(ctx, DUCTGPU_ESTATE, "operators not set up (call with ipro<=0)");
    if (my != r.my || mz != r.mz) return set_error(ctx, DUCTGPU_EARG, "grid %dx%d differs from the set-up %dx%d", my, mz, r.my, r.mz);
    if (!rhs || !sol || !xalp) return set_error(ctx, DUCTGPU_EARG, "null pointer");
    if (ie < ib || ib < 0) return set_error(ctx, DUCTGPU_EARG, "ib=%d ie=%d", ib, ie);
    cudaSetDevice(ctx->device);
    const int nm = ie - ib + 1;
    const size_t bytes = (size_t)2 * my * mz * nm * sizeof(double);
    const size_t by = bcy ? (size_t)2 * mz * nm * sizeof(double) : 0, bz = bcz ? (size_t)2 * my * nm * sizeof(double) : 0;
    int rc = ensure(ctx, ctx->io, 2 * bytes + by + bz);
    if (rc) return rc;
    double *drhs = ctx->io.buf, *dsol = drhs + bytes / sizeof(double);
    double *dby = dsol + bytes / sizeof(double), *dbz = dby + by / sizeof(double);
    DUCT_CUDA(ctx, cudaMemcpyAsync(drhs, rhs, bytes, cudaMemcpyHostToDevice, ctx->stream));
    if (bcy) DUCT_CUDA(ctx, cudaMemcpyAsync(dby, bcy, by, cudaMemcpyHostToDevice, ctx->stream));
    if (bcz) DUCT_CUDA(ctx, cudaMemcpyAsync(dbz, bcz, bz, cudaMemcpyHostToDevice, ctx->stream));
    ductgpu_rect_field f;
    f.rhs = drhs;
    f.sol = dsol;
    f.xalp = xalp;
    f.bcy = bcy ? dby : nullptr;
    f.bcz = bcz ? dbz : nullptr;
    f.alambda = alambda;
    f.ib = ib;
    f.nmodes = nm;
    f.slot = 0;
    if ((rc = ductgpu_solve_rect_fields_dev(ctx, &f, 1))) return rc;
    DUCT_CUDA(ctx, cudaMemcpyAsync(sol, dsol, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    return check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "helm3d_temp");
}

int ductgpu_solve_adjoint_fields_dev(ductgpu_ctx ctx, const ductgpu_field *fields, int nfields)
{
    if (!ctx) return DUCTGPU_EARG;
    if (!ctx->ready) return set_error(ctx, DUCTGPU_ESTATE, "operators not set up (call ductgpu_pseudomat)");
    if (!fields || nfields < 1 || nfields > kMaxFields)
        return set_error(ctx, DUCTGPU_EARG, "nfields=%d (1..%d)", nfields, kMaxFields);
    for (int i = 0; i < nfields; ++i) {
        int rc = validate_field(ctx, fields[i]);
        if (rc) return rc;
        if (fields[i].rhs == fields[i].sol)
            return set_error(ctx, DUCTGPU_EARG, "adjoint: input and output of field %d must differ", i);
    }
    cudaSetDevice(ctx->device);
    FieldTask tasks[kMaxFields];
    int rc = prepare(ctx, fields, nfields, tasks);
    if (rc) return rc;
    return solve_adjoint(ctx, tasks, nfields);
}

int ductgpu_helm3d_adjoint(ductgpu_ctx ctx, const double *gsol, double *grhs, char bound, double alambda, int my,
                           int mz, int ib, int ie, const double *xalp)
{
    if (!ctx) return DUCTGPU_EARG;
    if (!ctx->ready) return set_error(ctx, DUCTGPU_ESTATE, "operators not set up (call ductgpu_pseudomat)");
    if (my != ctx->my || mz != ctx->mz)
        return set_error(ctx, DUCTGPU_EARG, "grid %dx%d differs from the set-up %dx%d", my, mz, ctx->my, ctx->mz);
    if (!gsol || !grhs || !xalp) return set_error(ctx, DUCTGPU_EARG, "null pointer");
    if (ie < ib || ib < 0) return set_error(ctx, DUCTGPU_EARG, "ib=%d ie=%d", ib, ie);
    cudaSetDevice(ctx->device);
    const int nm = ie - ib + 1;
    const size_t bytes = (size_t)2 * my * mz * nm * sizeof(double);
    int rc = ensure(ctx, ctx->io, 2 * bytes);
    if (rc) return rc;
    double *dg = ctx->io.buf, *dout = ctx->io.buf + bytes / sizeof(double);
    DUCT_CUDA(ctx, cudaMemcpyAsync(dg, gsol, bytes, cudaMemcpyHostToDevice, ctx->stream));
    ductgpu_field f;
    f.rhs = dg;
    f.sol = dout;
    f.xalp = xalp;
    f.alambda = alambda;
    f.ib = ib;
    f.nmodes = nm;
    f.bound = bound;
    if ((rc = ductgpu_solve_adjoint_fields_dev(ctx, &f, 1))) return rc;
    DUCT_CUDA(ctx, cudaMemcpyAsync(grhs, dout, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    return check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "helm3d_adjoint");
}

int ductgpu_pseudopois(ductgpu_ctx ctx, int my)
{
    if (!ctx) return DUCTGPU_EARG;
    cudaSetDevice(ctx->device);
    return pois_setup(ctx, my);
}

int ductgpu_solve_pois_fields_dev(ductgpu_ctx ctx, const ductgpu_field *fields, int nfields)
{
    if (!ctx) return DUCTGPU_EARG;
    if (!ctx->pois_m) return set_error(ctx, DUCTGPU_ESTATE, "pseudopois not set up");
    if (!fields || nfields < 1 || nfields > kMaxFields)
        return set_error(ctx, DUCTGPU_EARG, "nfields=%d (1..%d)", nfields, kMaxFields);
    for (int i = 0; i < nfields; ++i) {
        int rc = validate_field(ctx, fields[i]);
        if (rc) return rc;
        if (fields[i].bound != 'n') return set_error(ctx, DUCTGPU_EARG, "solvepois is the Neumann solver (bound 'n')");
    }
    cudaSetDevice(ctx->device);
    FieldTask tasks[kMaxFields];
    int rc = prepare(ctx, fields, nfields, tasks);
    if (rc) return rc;
    return solve_pois(ctx, tasks, nfields);
}

int ductgpu_solvepois(ductgpu_ctx ctx, double *U, double xlambda, int my)
{
    if (!ctx) return DUCTGPU_EARG;
    if (!U) return set_error(ctx, DUCTGPU_EARG, "null pointer");
    if (!ctx->pois_m || my != ctx->pois_m)
        return set_error(ctx, DUCTGPU_ESTATE, "pseudopois not set up for my=%d", my);
    cudaSetDevice(ctx->device);
    const size_t plane = (size_t)my * my;
    std::vector<double> c(2 * plane, 0.0);
    for (size_t p = 0; p < plane; ++p) c[2 * p] = U[p];
    const size_t bytes = 2 * plane * sizeof(double);
    int rc = ensure(ctx, ctx->io, 2 * bytes);
    if (rc) return rc;
    double *drhs = ctx->io.buf, *dsol = drhs + 2 * plane;
    DUCT_CUDA(ctx, cudaMemcpyAsync(drhs, c.data(), bytes, cudaMemcpyHostToDevice, ctx->stream));
    const double zero = 0.0;
    ductgpu_field f;
    f.rhs = drhs;
    f.sol = dsol;
    f.xalp = &zero;
    f.alambda = xlambda;
    f.ib = 1;   // a real plane: no mode-0 rule needed, its imaginary part stays zero
    f.nmodes = 1;
    f.bound = 'n';
    if ((rc = ductgpu_solve_pois_fields_dev(ctx, &f, 1))) return rc;
    DUCT_CUDA(ctx, cudaMemcpyAsync(c.data(), dsol, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    if ((rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "solvepois"))) return rc;
    for (size_t p = 0; p < plane; ++p) U[p] = c[2 * p];
    return DUCTGPU_OK;
}

int ductgpu_preshen(ductgpu_ctx ctx, int my, char bound)
{
    if (!ctx) return DUCTGPU_EARG;
    if (bound != 'd' && bound != 'n') return set_error(ctx, DUCTGPU_EARG, "preshen: bound '%c'", bound);
    cudaSetDevice(ctx->device);
    return shen_setup(ctx, my, bound);
}

int ductgpu_solve_shen_fields_dev(ductgpu_ctx ctx, const ductgpu_field *fields, int nfields)
{
    if (!ctx) return DUCTGPU_EARG;
    if (!fields || nfields < 1 || nfields > kMaxFields)
        return set_error(ctx, DUCTGPU_EARG, "nfields=%d (1..%d)", nfields, kMaxFields);
    int planes = 0, m = 0;
    for (int i = 0; i < nfields; ++i) {
        int rc = validate_field(ctx, fields[i]);
        if (rc) return rc;
        const ShenOps &s = (fields[i].bound == 'n') ? ctx->shen_n : ctx->shen_d;
        if (!s.ready) return set_error(ctx, DUCTGPU_ESTATE, "preshen('%c') not set up", fields[i].bound);
        if (m && s.m != m) return set_error(ctx, DUCTGPU_EARG, "fields of one call need the same grid (%d vs %d)", s.m, m);
        m = s.m;
        planes += fields[i].nmodes;
    }
    cudaSetDevice(ctx->device);
    int rc = ensure_lam(ctx, planes);
    if (rc) return rc;
    // the pinned staging buffer may still be read by an earlier copy
    if (!ctx->capturing) DUCT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    ShenTask tasks[kMaxFields];
    int p = 0;
    for (int i = 0; i < nfields; ++i) {
        const ductgpu_field &f = fields[i];
        tasks[i].rhs = f.rhs;
        tasks[i].sol = f.sol;
        tasks[i].nmodes = f.nmodes;
        tasks[i].mode0 = (f.ib == 0);
        tasks[i].plane0 = p;
        tasks[i].bound = f.bound;
        // xlambda = alambda + xalp(imode)^2, src/helm_shen.f90:65
        for (int k = 0; k < f.nmodes; ++k) ctx->lam_host[p + k] = f.alambda + f.xalp[k] * f.xalp[k];
        p += f.nmodes;
    }
    if (!ctx->capturing)
        DUCT_CUDA(ctx, cudaMemcpyAsync(ctx->lam, ctx->lam_host, planes * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    return solve_shen(ctx, tasks, nfields);
}

int ductgpu_helm3d_shen(ductgpu_ctx ctx, double *rhs, double *sol, int ipro, char bound, double alambda,
                        int my, int mz, int ib, int ie, const double *xalp)
{
    if (!ctx) return DUCTGPU_EARG;
    if (bound != 'd' && bound != 'n') return set_error(ctx, DUCTGPU_EARG, "helm3d_shen: bound '%c'", bound);
    if (my != mz) return set_error(ctx, DUCTGPU_EARG, "helm3d_shen needs my == mz (%d, %d)", my, mz);
    if (ipro <= 0) {
        int rc = ductgpu_preshen(ctx, my, bound);
        if (rc) return rc;
        if (ipro == -1) return DUCTGPU_OK;
    }
    const ShenOps &s = (bound == 'n') ? ctx->shen_n : ctx->shen_d;
    if (!s.ready) return set_error(ctx, DUCTGPU_ESTATE, "preshen not set up (call with ipro<=0)");
    if (my != s.m) return set_error(ctx, DUCTGPU_EARG, "grid %d differs from the set-up %d", my, s.m);
    if (!rhs || !sol || !xalp) return set_error(ctx, DUCTGPU_EARG, "null pointer");
    if (ie < ib || ib < 0) return set_error(ctx, DUCTGPU_EARG, "ib=%d ie=%d", ib, ie);
    cudaSetDevice(ctx->device);
    const int nm = ie - ib + 1;
    const size_t bytes = (size_t)2 * my * mz * nm * sizeof(double);
    int rc = ensure(ctx, ctx->io, 2 * bytes);
    if (rc) return rc;
    double *drhs = ctx->io.buf, *dsol = ctx->io.buf + bytes / sizeof(double);
    DUCT_CUDA(ctx, cudaMemcpyAsync(drhs, rhs, bytes, cudaMemcpyHostToDevice, ctx->stream));
    ductgpu_field f;
    f.rhs = drhs;
    f.sol = dsol;
    f.xalp = xalp;
    f.alambda = alambda;
    f.ib = ib;
    f.nmodes = nm;
    f.bound = bound;
    if ((rc = ductgpu_solve_shen_fields_dev(ctx, &f, 1))) return rc;
    // rhs comes back as its Chebyshev coefficients, like the reference's
    DUCT_CUDA(ctx, cudaMemcpyAsync(rhs, drhs, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    DUCT_CUDA(ctx, cudaMemcpyAsync(sol, dsol, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    return check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "helm3d_shen");
}

static int run_solve(ductgpu_ctx ctx, int kind, const void *fields, int nfields, int precision)
{
    if (kind == 0)
        return ductgpu_solve_fields_dev(ctx, static_cast<const ductgpu_field *>(fields), nfields, precision);
    if (kind == 2)
        return ductgpu_solve_shen_fields_dev(ctx, static_cast<const ductgpu_field *>(fields), nfields);
    return ductgpu_solve_rect_fields_dev(ctx, static_cast<const ductgpu_rect_field *>(fields), nfields);
}

int ductgpu_graph_create(ductgpu_ctx ctx, int kind, const void *fields, int nfields, int precision, int *graph_id)
{
    if (!ctx || !fields || !graph_id || kind < 0 || kind > 2) return DUCTGPU_EARG;
    int id = -1;
    for (int i = 0; i < ductgpu_ctx_s::kMaxGraphs; ++i)
        if (!ctx->graph_exec[i]) { id = i; break; }
    if (id < 0) return set_error(ctx, DUCTGPU_EALLOC, "all %d graph slots in use", ductgpu_ctx_s::kMaxGraphs);
    cudaSetDevice(ctx->device);
    if (ctx->stream == (cudaStream_t)0)
        return set_error(ctx, DUCTGPU_EARG, "graph capture needs a non-default stream");
    // uncaptured run: sizes the workspaces and fills ctx->lam
    int rc = run_solve(ctx, kind, fields, nfields, precision);
    if (rc) return rc;
    int planes = 0;
    for (int i = 0; i < nfields; ++i)
        planes += (kind != 1) ? static_cast<const ductgpu_field *>(fields)[i].nmodes
                              : static_cast<const ductgpu_rect_field *>(fields)[i].nmodes;
    DUCT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    DUCT_CUDA(ctx, cudaMalloc(&ctx->graph_lam[id], planes * sizeof(double)));
    DUCT_CUDA(ctx, cudaMemcpy(ctx->graph_lam[id], ctx->lam, planes * sizeof(double), cudaMemcpyDeviceToDevice));
    double *lam_saved = ctx->lam;
    ctx->lam = ctx->graph_lam[id];
    ctx->capturing = true;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        rc = run_solve(ctx, kind, fields, nfields, precision);
        cudaError_t e2 = cudaStreamEndCapture(ctx->stream, &g);
        if (!rc && e2 != cudaSuccess) rc = check_cuda(ctx, e2, "cudaStreamEndCapture");
    } else {
        rc = check_cuda(ctx, e, "cudaStreamBeginCapture");
    }
    ctx->capturing = false;
    ctx->lam = lam_saved;
    if (!rc) rc = check_cuda(ctx, cudaGraphInstantiate(&ctx->graph_exec[id], g, 0), "cudaGraphInstantiate");
    if (g) cudaGraphDestroy(g);
    if (rc) {
        cudaFree(ctx->graph_lam[id]);
        ctx->graph_lam[id] = nullptr;
        ctx->graph_exec[id] = nullptr;
        return rc;
    }
    *graph_id = id;
    return DUCTGPU_OK;
}

int ductgpu_graph_launch(ductgpu_ctx ctx, int graph_id)
{
    if (!ctx || graph_id < 0 || graph_id >= ductgpu_ctx_s::kMaxGraphs || !ctx->graph_exec[graph_id])
        return DUCTGPU_EARG;
    ctx->launches += 1;
    return check_cuda(ctx, cudaGraphLaunch(ctx->graph_exec[graph_id], ctx->stream), "cudaGraphLaunch");
}

int ductgpu_graph_destroy(ductgpu_ctx ctx, int graph_id)
{
    if (!ctx || graph_id < 0 || graph_id >= ductgpu_ctx_s::kMaxGraphs || !ctx->graph_exec[graph_id])
        return DUCTGPU_EARG;
    cudaStreamSynchronize(ctx->stream);
    cudaGraphExecDestroy(ctx->graph_exec[graph_id]);
    cudaFree(ctx->graph_lam[graph_id]);
    ctx->graph_exec[graph_id] = nullptr;
    ctx->graph_lam[graph_id] = nullptr;
    return DUCTGPU_OK;
}

// ---- the reference's GPU entry points (src/mytranspose_cuda.cu:132-196) ----
__global__ void k_real_transpose(const double *A, double *C, int nx, int ny)
{
    __shared__ double tile[32][33];
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int r = ty; r < 32; r += 8)
        if (x0 + tx < nx && y0 + r < ny) tile[r][tx] = A[(x0 + tx) + (size_t)nx * (y0 + r)];
    __syncthreads();
    for (int r = ty; r < 32; r += 8)
        if (y0 + tx < ny && x0 + r < nx) C[(y0 + tx) + (size_t)ny * (x0 + r)] = tile[tx][r];
}

__global__ void k_invdiag(const double *F, const double *ED, double *C, long long n, double xlam)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        C[i] = F[i] / (ED[i] - xlam);
}

int transpose_gpu_(size_t *handle, const int *Nx, const int *Ny, const double *alpha, const size_t *devPtrA, size_t *devPtrC)
{
    (void)handle; (void)alpha;
    if (!Nx || !Ny || !devPtrA || !devPtrC || *Nx < 1 || *Ny < 1) return DUCTGPU_EARG;
    dim3 grid((*Nx + 31) / 32, (*Ny + 31) / 32);
    k_real_transpose<<<grid, 256>>>((const double *)(*devPtrA), (double *)(*devPtrC), *Nx, *Ny);
    return cudaGetLastError() == cudaSuccess ? DUCTGPU_OK : DUCTGPU_ECUDA;
}

int mat_invdiag_gpu_(size_t *handle, const int *Nx, const int *Ny, const double *xlam, const size_t *devPtrF,
                     const size_t *devPtrED, size_t *devPtrC)
{
    (void)handle;
    if (!Nx || !Ny || !xlam || !devPtrF || !devPtrED || !devPtrC || *Nx < 1 || *Ny < 1) return DUCTGPU_EARG;
    const long long n = (long long)(*Nx) * (*Ny);
    const int blocks = (int)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096);
    k_invdiag<<<blocks, 256>>>((const double *)(*devPtrF), (const double *)(*devPtrED), (double *)(*devPtrC), n, *xlam);
    return cudaGetLastError() == cudaSuccess ? DUCTGPU_OK : DUCTGPU_ECUDA;
}

int ductgpu_device_alloc(ductgpu_ctx ctx, size_t bytes, void **ptr)
{
    if (!ctx || !ptr) return DUCTGPU_EARG;
    cudaSetDevice(ctx->device);
    *ptr = nullptr;
    return check_cuda(ctx, cudaMalloc(ptr, bytes), "device_alloc");
}

int ductgpu_device_free(ductgpu_ctx ctx, void *ptr)
{
    if (!ctx) return DUCTGPU_EARG;
    cudaStreamSynchronize(ctx->stream);
    return check_cuda(ctx, cudaFree(ptr), "device_free");
}

int ductgpu_host_alloc(ductgpu_ctx ctx, size_t bytes, void **ptr)
{
    if (!ctx || !ptr) return DUCTGPU_EARG;
    *ptr = nullptr;
    return check_cuda(ctx, cudaMallocHost(ptr, bytes), "host_alloc");
}

int ductgpu_host_free(ductgpu_ctx ctx, void *ptr)
{
    if (!ctx) return DUCTGPU_EARG;
    cudaStreamSynchronize(ctx->stream);
    return check_cuda(ctx, cudaFreeHost(ptr), "host_free");
}

int ductgpu_copy(ductgpu_ctx ctx, void *dst, const void *src, size_t bytes, int kind)
{
    if (!ctx || (!dst && bytes) || (!src && bytes) || kind < 1 || kind > 3) return DUCTGPU_EARG;
    return check_cuda(ctx, cudaMemcpyAsync(dst, src, bytes, (cudaMemcpyKind)kind, ctx->stream), "copy");
}

int ductgpu_event_record(ductgpu_ctx ctx, int slot)
{
    if (!ctx || slot < 0 || slot >= kNumEvents) return DUCTGPU_EARG;
    return check_cuda(ctx, cudaEventRecord(ctx->ev[slot], ctx->stream), "event record");
}

int ductgpu_event_elapsed(ductgpu_ctx ctx, int s0, int s1, float *ms)
{
    if (!ctx || !ms || s0 < 0 || s1 < 0 || s0 >= kNumEvents || s1 >= kNumEvents) return DUCTGPU_EARG;
    DUCT_CUDA(ctx, cudaEventSynchronize(ctx->ev[s1]));
    return check_cuda(ctx, cudaEventElapsedTime(ms, ctx->ev[s0], ctx->ev[s1]), "event elapsed");
}

long long ductgpu_launch_count(ductgpu_ctx ctx) { return ctx ? ctx->launches : -1; }

int ductgpu_profile_enable(ductgpu_ctx ctx, int on)
{
    if (!ctx) return DUCTGPU_EARG;
    if (on && !ctx->prof_ev[0])
        for (int i = 0; i < 2 * ductgpu_ctx_s::kProfSlots; ++i)
            DUCT_CUDA(ctx, cudaEventCreate(&ctx->prof_ev[i]));
    if (!on) profile_drain(ctx);
    ctx->prof_on = on != 0;
    return DUCTGPU_OK;
}

int ductgpu_profile_reset(ductgpu_ctx ctx)
{
    if (!ctx) return DUCTGPU_EARG;
    profile_drain(ctx);
    for (int k = 0; k < DUCTGPU_K_COUNT; ++k) {
        ctx->prof_ms[k] = 0.0;
        ctx->prof_n[k] = 0;
        ctx->prof_bytes[k] = 0.0;
        ctx->prof_flops[k] = 0.0;
    }
    return DUCTGPU_OK;
}

int ductgpu_profile_read(ductgpu_ctx ctx, int kind, double *ms, long long *launches)
{
    if (!ctx || kind < 0 || kind >= DUCTGPU_K_COUNT) return DUCTGPU_EARG;
    profile_drain(ctx);
    if (ms) *ms = ctx->prof_ms[kind];
    if (launches) *launches = ctx->prof_n[kind];
    return DUCTGPU_OK;
}

int ductgpu_profile_bytes(ductgpu_ctx ctx, int kind, double *bytes)
{
    if (!ctx || kind < 0 || kind >= DUCTGPU_K_COUNT || !bytes) return DUCTGPU_EARG;
    *bytes = ctx->prof_bytes[kind];
    return DUCTGPU_OK;
}

int ductgpu_profile_flops(ductgpu_ctx ctx, int kind, double *flops)
{
    if (!ctx || kind < 0 || kind >= DUCTGPU_K_COUNT || !flops) return DUCTGPU_EARG;
    *flops = ctx->prof_flops[kind];
    return DUCTGPU_OK;
}

}  // extern "C"
