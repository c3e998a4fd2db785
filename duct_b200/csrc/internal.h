// internal.h -- context and shared declarations of libductgpu (not part of
// the C-ABI).  The context replaces the reference's module globals of the
// solver (fulldiagdir, fulldiagneu, chebystuff, gpudevice; src/mod.f90:
// 277-343, 409-483) with device-resident state owned by one handle.
#pragma once

#include <cuda_runtime.h>
#include <cusolverDn.h>
#include <stdarg.h>
#include <stdio.h>

#include <cstdint>

#include "../../include/ductgpu.h"

namespace duct {

constexpr int kMaxFields = 8;   // fields per batched launch
constexpr int kMaxN = 191;      // largest interior size (my-2) supported
constexpr int kNumEvents = 16;

// Interior operators of one boundary condition ('d' or 'n').
struct BoundOps {
    int n = 0;                 // interior points, my-2
    int kpad = 0;              // n rounded up to the K chunk (32)
    int mtiles = 0;            // 16-row tiles of the padded M extent
    double *E = nullptr;       // [n] eigenvalues
    double *P = nullptr;       // [n*n] eigenvectors, column-major
    double *PM1 = nullptr;     // [n*n] inverse
    double *Ppack = nullptr;   // P in DMMA A-fragment order, zero padded
    double *Qpack = nullptr;   // PM1 in DMMA A-fragment order
    double *pcol = nullptr;    // [n] column iofzero of P (Neumann pin)
    double *qrow = nullptr;    // [n] row iofzero of P^-1 (null-space projection)
    int iofzero = 0;           // 1-based, Neumann only
    double emin = 0.0, emax = 0.0;   // smallest / largest |eigenvalue| (host)
    double *D2B = nullptr;     // [n*n] the interior operator block itself
    double *Bpack = nullptr;   // D2B in DMMA A-fragment order (residual)
    uint8_t *Pslices = nullptr, *Qslices = nullptr;  // BF16 slices (mixed)
    int *Pexp = nullptr, *Qexp = nullptr;            // per-row exponents
};

struct Workspace {
    double *buf = nullptr;
    size_t bytes = 0;
};

}  // namespace duct

struct ductgpu_ctx_s {
    int device = 0;
    int num_sms = 148;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    cusolverDnHandle_t solver = nullptr;
    char err[512] = {0};

    int my = 0, mz = 0;
    bool ready = false;
    double *xcol = nullptr;    // [my]
    double *DC = nullptr;      // [my*my]
    double *D2 = nullptr;      // [my*my]
    double *AM1 = nullptr;     // [16] device copy
    double *ccw = nullptr;     // [my] Clenshaw-Curtis weights on the nodes
    double wanted = 0.0;
    int gauge = DUCTGPU_GAUGE_POINT;
    int refine_steps = 2;      // FP64 refinement steps of the split-precision path
    duct::BoundOps dir, neu;

    duct::Workspace work;      // pass intermediates
    duct::Workspace io;        // device copies for host entries
    int *dev_err = nullptr;    // device error word (bounded waits)
    double *lam = nullptr;     // per-plane lambda (device)
    double *lam_host = nullptr;// pinned staging
    int lam_cap = 0;

    cudaEvent_t ev[duct::kNumEvents] = {};
    long long launches = 0;

    // per-kernel profiling (events around launches)
    bool prof_on = false;
    static constexpr int kProfSlots = 4096;
    cudaEvent_t prof_ev[2 * kProfSlots] = {};
    int prof_kind[kProfSlots] = {};
    int prof_used = 0;
    double prof_ms[DUCTGPU_K_COUNT] = {};
    long long prof_n[DUCTGPU_K_COUNT] = {};
};

namespace duct {

int set_error(ductgpu_ctx ctx, int code, const char *fmt, ...);
int check_cuda(ductgpu_ctx ctx, cudaError_t e, const char *what);
int ensure(ductgpu_ctx ctx, Workspace &w, size_t bytes);

// Brackets one kernel launch with profiling events when enabled and
// counts it.  Use: { LaunchScope ls(ctx, DUCTGPU_K_...); kernel<<<>>>(); }
struct LaunchScope {
    ductgpu_ctx c;
    int slot = -1;
    LaunchScope(ductgpu_ctx ctx, int kind);
    ~LaunchScope();
};
void profile_drain(ductgpu_ctx ctx);

// setup.cu
int pseudomat_gpu(ductgpu_ctx ctx, int m);
int pack_operators(ductgpu_ctx ctx, BoundOps &b);
void free_bound(BoundOps &b);

// solve_fp64.cu
struct FieldTask {
    double *rhs;
    double *sol;
    int nmodes;
    int mode0;        // 1: first plane is Fourier mode 0
    char bound;
    int plane0;       // index of the first plane in ctx->lam
    int refine;       // FP64 refinement steps for the split-precision path
};
int solve_fp64(ductgpu_ctx ctx, const FieldTask *tasks, int ntasks);

// One batched FP64 GEMM pass (k_pass_fp64), usable by other solvers.
struct PassField {
    const double *src;
    double *dst;
    const double *A;     // packed operator
    const double *E;     // eigenvalues for the divide
    int nmodes;
    int mode0;
    int plane0;
    int sing_io;         // 0-based iofzero of a Neumann field, else -1
    // residual epilogue: dst = resF - resT - acc + lam * resU
    const double *resF, *resT, *resU;
};
struct PassParams {
    PassField f[kMaxFields];
    int cta_start[kMaxFields + 1];
    int nf;
    const double *lam;
    long long plane_stride;  // doubles per complex plane
    int n, kpad, nchunks;
    int sk, sl;              // complex strides of (k, line)
    int divide;
    int zero_im_mode0;
    int residual;
};
constexpr int kPassLines = 32;
int fp64_pass(ductgpu_ctx ctx, const PassParams &pp, int grid);

// solve_mixed.cu
int split_operator(ductgpu_ctx ctx, int n, const double *A, uint8_t **slices, int **rexp);
int solve_mixed(ductgpu_ctx ctx, const FieldTask *tasks, int ntasks);
int zero_walls(ductgpu_ctx ctx, const FieldTask *tasks, int ntasks);
int neumann_fill(ductgpu_ctx ctx, const FieldTask *tasks, int ntasks);

// transforms.cu
int transyz_dev(ductgpu_ctx ctx, double *f, int my, int mz, int nmodes, char cdir, int iopt);
int derivyz_dev(ductgpu_ctx ctx, const double *u, double *du, int my, int mz, int nmodes, char cdir,
                int ider, double scal, char what, double aspect);
int transpose_dev(ductgpu_ctx ctx, const double *in, double *out, long long A, long long Q);

}  // namespace duct

#define DUCT_CUDA(ctx, call)                                         \
    do {                                                             \
        cudaError_t e_ = (call);                                     \
        if (e_ != cudaSuccess) return duct::check_cuda(ctx, e_, #call); \
    } while (0)
