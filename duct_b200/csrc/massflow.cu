// massflow.cu -- constant mass-flow-rate forcing, the second caller of the
// square Dirichlet solve: precomp_mass_flow and impose_mass_flow
// (src/operators.F:2205-2344, square build).
//
// precomp: for each Runge-Kutta index k the particular solution of
//   (dyy + dzz) u - u / (alphak(k) dt nu) = 1,  u = 0 on the walls,
// and its flow rate, all RK indices in one batched solve.  impose: the flow
// rate of the real part of mode 0 and the correction u0 += fac premassfu(k),
// fac = (csum - flow)/premassf(k), on the device (a partial-sum kernel and
// an apply kernel), so the step needs no host round trip (iflag 1).
//
// The flow rate is the Clenshaw-Curtis quadrature of the physical values,
// sum_pq w_p w_q u_pq * aspect, which integrates the same Chebyshev
// interpolant exactly as the reference's transyz_plane + cheb2_integral
// (src/chebyshev.f90:542-595, 692-723); the two differ by round-off.
#include "internal.h"

namespace duct {

// rhs planes of precomp: 1 inside, 0 on the walls, zero imaginary part
__global__ void k_mf_rhs(double *rhs, int m, int planes)
{
    const long n = (long)m * m * planes;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const int p = (int)(i % m), q = (int)((i / m) % m);
        const bool wall = (p == 0 || q == 0 || p == m - 1 || q == m - 1);
        rhs[2 * i] = wall ? 0.0 : 1.0;
        rhs[2 * i + 1] = 0.0;
    }
}

// Block-wide deterministic sum (fixed order per launch configuration).
__device__ double block_sum(double v, double *red)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (warp == 0) {
        v = (lane < (int)(blockDim.x >> 5)) ? red[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[32] = v;
    }
    __syncthreads();
    const double r = red[32];
    __syncthreads();
    return r;
}

// One CTA per RK index: premassfu(:,k) = Re sol_k, premassf(k) = its flow.
__global__ void __launch_bounds__(1024) k_mf_store(const double *sol, double *pu, double *pf, const double *w,
                                                   int m, double aspect)
{
    __shared__ double red[33];
    const int k = blockIdx.x;
    const long plane = (long)m * m;
    const double *s = sol + 2 * plane * k;
    double acc = 0.0;
    for (long i = threadIdx.x; i < plane; i += blockDim.x) {
        const double v = s[2 * i];
        pu[plane * k + i] = v;
        acc += w[i % m] * w[i / m] * v;
    }
    acc = block_sum(acc, red);
    if (threadIdx.x == 0) pf[k] = acc * aspect;
}

// impose_mass_flow on the first (mode 0) plane of u in two kernels over
// kMfBlocks CTAs: per-CTA partial sums of the quadrature, then every CTA
// adds the partials in the same fixed order (so the result does not depend
// on scheduling), CTA 0 stores the flow rate, and with iflag 1 every CTA
// corrects its slice, u0.re += (csum - sum) / pf * pu.
constexpr int kMfBlocks = 64;
constexpr int kMfThreads = 256;

__global__ void __launch_bounds__(kMfThreads) k_mf_partial(const double *u, const double *w, int m, double *part)
{
    __shared__ double red[33];
    const long plane = (long)m * m, chunk = (plane + kMfBlocks - 1) / kMfBlocks;
    const long i0 = blockIdx.x * chunk, i1 = min(plane, i0 + chunk);
    double acc = 0.0;
    for (long i = i0 + threadIdx.x; i < i1; i += kMfThreads) acc += w[i % m] * w[i / m] * u[2 * i];
    acc = block_sum(acc, red);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

__global__ void __launch_bounds__(kMfThreads) k_mf_apply(double *u, double aspect, const double *pu,
                                                        const double *pf, double csum, int iflag, const double *part,
                                                        int m, double *sum_out)
{
    __shared__ double tot;
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int b = 0; b < kMfBlocks; ++b) s += part[b];
        tot = s * aspect;
        if (blockIdx.x == 0) *sum_out = tot;
    }
    __syncthreads();
    if (!iflag) return;
    const double fac = (csum - tot) / *pf;
    const long plane = (long)m * m, chunk = (plane + kMfBlocks - 1) / kMfBlocks;
    const long i0 = blockIdx.x * chunk, i1 = min(plane, i0 + chunk);
    for (long i = i0 + threadIdx.x; i < i1; i += kMfThreads) u[2 * i] += fac * pu[i];
}

}  // namespace duct

using namespace duct;

extern "C" int ductgpu_precomp_mass_flow(ductgpu_ctx ctx, double dtp, const double *alphak, int mrk, double fnu,
                                         double aspect, double *premassf, double *premassfu)
{
    if (!ctx) return DUCTGPU_EARG;
    if (!ctx->ready) return set_error(ctx, DUCTGPU_ESTATE, "operators not set up (call ductgpu_pseudomat)");
    if (!alphak || mrk < 1 || mrk > kMaxFields)
        return set_error(ctx, DUCTGPU_EARG, "precomp_mass_flow: mrk=%d (1..%d)", mrk, kMaxFields);
    if (!(dtp > 0.0) || !(fnu > 0.0)) return set_error(ctx, DUCTGPU_EARG, "precomp_mass_flow: dt=%g nu=%g", dtp, fnu);
    for (int k = 0; k < mrk; ++k)
        if (!(alphak[k] > 0.0)) return set_error(ctx, DUCTGPU_EARG, "precomp_mass_flow: alphak(%d)=%g", k + 1, alphak[k]);
    cudaSetDevice(ctx->device);
    const int m = ctx->my;
    const size_t plane = (size_t)m * m;
    DUCT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    cudaFree(ctx->mf_u);
    cudaFree(ctx->mf_f);
    cudaFree(ctx->mf_sum);
    ctx->mf_u = ctx->mf_f = ctx->mf_sum = nullptr;
    ctx->mf_mrk = 0;
    DUCT_CUDA(ctx, cudaMalloc(&ctx->mf_u, plane * mrk * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(&ctx->mf_f, mrk * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(&ctx->mf_sum, (1 + kMfBlocks) * sizeof(double)));   // the sum, then the partials
    int rc = ensure(ctx, ctx->io, 2 * 2 * plane * mrk * sizeof(double));
    if (rc) return rc;
    double *rhs = ctx->io.buf, *sol = rhs + 2 * plane * mrk;
    {
        LaunchScope ls(ctx, DUCTGPU_K_OTHER);
        k_mf_rhs<<<(unsigned)((plane * mrk + 255) / 256), 256, 0, ctx->stream>>>(rhs, m, mrk);
    }
    // flambda = -1/(alphak dt nu) as helco in main1.f90; the solve takes
    // xlambda = -flambda (src/operators.F:2243, 2274)
    const double zero = 0.0;
    ductgpu_field f[kMaxFields];
    for (int k = 0; k < mrk; ++k) {
        f[k].rhs = rhs + 2 * plane * k;
        f[k].sol = sol + 2 * plane * k;
        f[k].xalp = &zero;
        f[k].alambda = 1.0 / (alphak[k] * dtp * fnu);
        f[k].ib = 0;
        f[k].nmodes = 1;
        f[k].bound = 'd';
    }
    if ((rc = ductgpu_solve_fields_dev(ctx, f, mrk, DUCTGPU_PREC_FP64))) return rc;
    {
        LaunchScope ls(ctx, DUCTGPU_K_OTHER);
        k_mf_store<<<mrk, 1024, 0, ctx->stream>>>(sol, ctx->mf_u, ctx->mf_f, ctx->ccw, m, aspect);
    }
    DUCT_CUDA(ctx, cudaGetLastError());
    if (premassf) DUCT_CUDA(ctx, cudaMemcpyAsync(premassf, ctx->mf_f, mrk * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (premassfu)
        DUCT_CUDA(ctx, cudaMemcpyAsync(premassfu, ctx->mf_u, plane * mrk * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    DUCT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->mf_mrk = mrk;
    ctx->mf_my = m;
    ctx->mf_aspect = aspect;
    return DUCTGPU_OK;
}

extern "C" int ductgpu_impose_mass_flow_dev(ductgpu_ctx ctx, double *csum, int krk, double *u, int iflag)
{
    if (!ctx) return DUCTGPU_EARG;
    if (!csum || !u) return set_error(ctx, DUCTGPU_EARG, "impose_mass_flow: null pointer");
    if (iflag != 0 && iflag != 1) return set_error(ctx, DUCTGPU_EARG, "impose_mass_flow: iflag=%d", iflag);
    if (!ctx->mf_mrk || ctx->mf_my != ctx->my)
        return set_error(ctx, DUCTGPU_ESTATE, "impose_mass_flow: call ductgpu_precomp_mass_flow first");
    if (iflag && (krk < 1 || krk > ctx->mf_mrk))
        return set_error(ctx, DUCTGPU_EARG, "impose_mass_flow: krk=%d (1..%d)", krk, ctx->mf_mrk);
    if ((uintptr_t)u & 15) return set_error(ctx, DUCTGPU_EARG, "impose_mass_flow: u must be 16-byte aligned");
    cudaSetDevice(ctx->device);
    const int m = ctx->my;
    const int k = iflag ? krk - 1 : 0;
    {
        LaunchScope ls(ctx, DUCTGPU_K_OTHER);
        double *part = ctx->mf_sum + 1;
        k_mf_partial<<<kMfBlocks, kMfThreads, 0, ctx->stream>>>(u, ctx->ccw, m, part);
        k_mf_apply<<<kMfBlocks, kMfThreads, 0, ctx->stream>>>(u, ctx->mf_aspect, ctx->mf_u + (size_t)m * m * k,
                                                              ctx->mf_f + k, *csum, iflag, part, m, ctx->mf_sum);
        ctx->launches += 1;     // the scope counted the first of the two
    }
    DUCT_CUDA(ctx, cudaGetLastError());
    if (iflag) return DUCTGPU_OK;
    // iflag 0 returns the measured flow rate (src/operators.F:2329-2338)
    DUCT_CUDA(ctx, cudaMemcpyAsync(csum, ctx->mf_sum, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    return check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "impose_mass_flow");
}

extern "C" int ductgpu_impose_mass_flow(ductgpu_ctx ctx, double *csum, int krk, double *u, int iflag)
{
    if (!ctx) return DUCTGPU_EARG;
    if (!u || !csum) return set_error(ctx, DUCTGPU_EARG, "impose_mass_flow: null pointer");
    if (!ctx->mf_mrk) return set_error(ctx, DUCTGPU_ESTATE, "impose_mass_flow: call ductgpu_precomp_mass_flow first");
    cudaSetDevice(ctx->device);
    const size_t bytes = (size_t)2 * ctx->my * ctx->my * sizeof(double);   // mode 0 plane only
    int rc = ensure(ctx, ctx->io, bytes);
    if (rc) return rc;
    DUCT_CUDA(ctx, cudaMemcpyAsync(ctx->io.buf, u, bytes, cudaMemcpyHostToDevice, ctx->stream));
    if ((rc = ductgpu_impose_mass_flow_dev(ctx, csum, krk, ctx->io.buf, iflag))) return rc;
    if (iflag) DUCT_CUDA(ctx, cudaMemcpyAsync(u, ctx->io.buf, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    return check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "impose_mass_flow");
}
