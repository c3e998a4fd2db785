// shen.cu -- the Shen-Legendre Galerkin solver of the HELM_SHEN build:
// helm3d_shen -> int2d3d -> solveshen (src/helm_shen.f90:2-85,
// src/solveshen.f90:5-546, src/legendre.f90, src/preshen.f90).  It solves
//   -lap(u) + lambda u = f
// in the basis phi_k = L_k + b_k L_{k+2} (b_k = -1 Dirichlet,
// -k(k+1)/((k+2)(k+3)) Neumann), batched over fields and modes:
//
//   transyz y, z (rhs, in place)          k_dct
//   Chebyshev -> Legendre  A . A^T        2 DMMA passes (full planes)
//   Legendre -> Shen (Galerkin weights)   k_leg2shen (banded)
//   P^-1 S^-1 along y                     DMMA pass
//   SPD tridiagonals along z per y-eigen  k_shen_solv (batched LDL^T)
//   P along y                             DMMA pass
//   Shen -> Legendre                      k_shen2leg (banded)
//   Legendre -> Chebyshev B . B^T         2 DMMA passes
//   transyz y, z (sol)                    k_dct
//
// The reference splits every operator into even and odd halves and solves
// the tridiagonals with DPTSV; the full operators here give the same
// products (the parity halves decouple to round-off) and the elimination
// is the same LDL^T factorisation.  Set-up on the GPU: the generalized
// symmetric eigenproblem M x = rho S x (the reference's dsygv) is
// cuSOLVER's sygvd, inverses getrf/getrs.
#include <math.h>
#include <string.h>

#include <vector>

#include "internal.h"

namespace duct {

static int blocks(long n) { return (int)((n + 255) / 256 < 2048 ? (n + 255) / 256 : 2048); }

// leg_cheb_mat (src/legendre.f90:56-82): A upper triangular, one column
// after the other (column jj needs columns jj-1 and jj-2).  One CTA.
__global__ void k_leg_cheb(int m, double *A)
{
    for (int idx = threadIdx.x; idx < m * m; idx += blockDim.x) A[idx] = 0.0;
    __syncthreads();
    const int n = m - 1;
    if (threadIdx.x == 0) {
        A[0] = 1.0;
        A[1 + (size_t)m] = 1.0;
        for (int k = 2; k <= n; ++k)
            A[k + (size_t)m * k] = 2.0 * (double)k / (double)(2 * k - 1) * A[(k - 1) + (size_t)m * (k - 1)];
        for (int k = 2; k <= n; k += 2) A[(size_t)m * k] = -1.0 / (double)(k * k - 1);
    }
    __syncthreads();
    for (int j = 2; j <= n - 1; ++j) {   // 1-based j, column jj = j + 1
        const int jj = j + 1;
        for (int i = 1 + threadIdx.x; i <= j; i += blockDim.x) {
            const int ii = i + 1;
            const double c1 = (double)(2 * i + 2) / (double)(2 * i + 3);
            const double c2 = (double)(2 * i) / (double)(2 * i - 1);
            A[(ii - 1) + (size_t)m * jj] = c1 * A[ii + (size_t)m * (jj - 1)] + c2 * A[(ii - 2) + (size_t)m * (jj - 1)] -
                                          A[(ii - 1) + (size_t)m * (jj - 2)];
        }
        __syncthreads();
    }
}

__global__ void k_scale_cols(int n, double *A, const double *d)
{
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n * n; idx += gridDim.x * blockDim.x)
        A[idx] /= d[idx / n];
}

__global__ void k_identity_s(int n, double *I)
{
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n * n; idx += gridDim.x * blockDim.x)
        I[idx] = (idx % n == idx / n) ? 1.0 : 0.0;
}

// dst (n x n) = [1 0; 0 src (n1 x n1)]
__global__ void k_embed(int n, int n1, const double *src, double *dst)
{
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n * n; idx += gridDim.x * blockDim.x) {
        const int i = idx % n, j = idx / n;
        double v;
        if (i == 0 || j == 0) v = (i == j) ? 1.0 : 0.0;
        else v = src[(i - 1) + (size_t)n1 * (j - 1)];
        dst[idx] = v;
    }
}

__global__ void k_zero_imag(double *f, long n)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        f[2 * i + 1] = 0.0;
}

void free_shen(ShenOps &s)
{
    free_bound(s.leg);
    free_bound(s.eig);
    cudaFree(s.Md); cudaFree(s.Mo); cudaFree(s.Sm); cudaFree(s.bk);
    s = ShenOps();
}

// inverse of the n x n matrix A (device) into Ainv via getrf/getrs
int invert_dev(ductgpu_ctx ctx, int n, const double *A, double *Ainv)
{
    double *LU = nullptr, *work = nullptr;
    int *ipiv = nullptr, *dinfo = nullptr, lwork = 0, info = 0, rc = DUCTGPU_OK;
    if ((rc = check_cuda(ctx, cudaMalloc(&LU, (size_t)n * n * sizeof(double)), "inv LU"))) return rc;
    if ((rc = check_cuda(ctx, cudaMalloc(&ipiv, n * sizeof(int)), "inv ipiv"))) goto out;
    if ((rc = check_cuda(ctx, cudaMalloc(&dinfo, sizeof(int)), "inv info"))) goto out;
    if ((rc = check_cuda(ctx, cudaMemcpyAsync(LU, A, (size_t)n * n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream), "inv copy"))) goto out;
    if (cusolverDnDgetrf_bufferSize(ctx->solver, n, n, LU, n, &lwork) != CUSOLVER_STATUS_SUCCESS) { rc = set_error(ctx, DUCTGPU_ESOLVER, "getrf_bufferSize"); goto out; }
    if ((rc = check_cuda(ctx, cudaMalloc(&work, ((size_t)lwork + 16) * sizeof(double)), "inv work"))) goto out;
    k_identity_s<<<blocks((long)n * n), 256, 0, ctx->stream>>>(n, Ainv);
    ctx->launches += 1;
    if (cusolverDnDgetrf(ctx->solver, n, n, LU, n, work, ipiv, dinfo) != CUSOLVER_STATUS_SUCCESS ||
        cusolverDnDgetrs(ctx->solver, CUBLAS_OP_N, n, n, LU, n, ipiv, Ainv, n, dinfo) != CUSOLVER_STATUS_SUCCESS) {
        rc = set_error(ctx, DUCTGPU_ESOLVER, "getrf/getrs");
        goto out;
    }
    if ((rc = check_cuda(ctx, cudaMemcpyAsync(&info, dinfo, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream), "inv info"))) goto out;
    if ((rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "inv sync"))) goto out;
    if (info) rc = set_error(ctx, DUCTGPU_ESOLVER, "singular matrix (info %d)", info);
out:
    cudaFree(LU); cudaFree(work); cudaFree(ipiv); cudaFree(dinfo);
    return rc;
}

// generalized symmetric eigenproblem M x = rho S x (sygvd, itype 1,
// ascending rho, x^T S x = 1): M, S device n x n (destroyed; M -> x).
static int sygvd(ductgpu_ctx ctx, int n, double *M, double *S, double *w)
{
    int lwork = 0, info = 0, *dinfo = nullptr, rc = DUCTGPU_OK;
    double *work = nullptr;
    if (cusolverDnDsygvd_bufferSize(ctx->solver, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER,
                                    n, M, n, S, n, w, &lwork) != CUSOLVER_STATUS_SUCCESS)
        return set_error(ctx, DUCTGPU_ESOLVER, "sygvd_bufferSize");
    if ((rc = check_cuda(ctx, cudaMalloc(&work, ((size_t)lwork + 16) * sizeof(double)), "sygvd work"))) return rc;
    if ((rc = check_cuda(ctx, cudaMalloc(&dinfo, sizeof(int)), "sygvd info"))) goto out;
    if (cusolverDnDsygvd(ctx->solver, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, n, M, n, S,
                         n, w, work, lwork, dinfo) != CUSOLVER_STATUS_SUCCESS) {
        rc = set_error(ctx, DUCTGPU_ESOLVER, "sygvd");
        goto out;
    }
    if ((rc = check_cuda(ctx, cudaMemcpyAsync(&info, dinfo, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream), "sygvd info"))) goto out;
    if ((rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "sygvd sync"))) goto out;
    if (info) rc = set_error(ctx, DUCTGPU_ESOLVER, "sygvd info %d", info);
out:
    cudaFree(work); cudaFree(dinfo);
    return rc;
}

// preshen(bound) + leg_cheb_mat on the GPU (src/preshen.f90:2-535,
// src/legendre.f90:3-110).
int shen_setup(ductgpu_ctx ctx, int m, char bound)
{
    if (m < 5 || (m % 2) == 0 || m > kMaxN)
        return set_error(ctx, DUCTGPU_EARG, "preshen: my=%d must be odd in [5,%d]", m, kMaxN);
    ShenOps &s = (bound == 'n') ? ctx->shen_n : ctx->shen_d;
    cudaStreamSynchronize(ctx->stream);
    free_shen(s);
    const int n = m - 2;
    // makeMS / precomeigen coefficients (O(m) work, host)
    std::vector<double> b(m), Md(n), Mo(n, 0.0), Sm(n), M2((size_t)n * n, 0.0), S2((size_t)n * n, 0.0);
    for (int k = 0; k < m; ++k) b[k] = (bound == 'd') ? -1.0 : -(double)(k * (k + 1)) / (double)((k + 2) * (k + 3));
    for (int k = 0; k < n; ++k) {
        Sm[k] = -b[k] * (double)(4 * k + 6);
        Md[k] = 2.0 / (double)(2 * k + 1) + 2.0 * b[k] * b[k] / (double)(2 * k + 5);
        M2[k + (size_t)n * k] = Md[k];
        S2[k + (size_t)n * k] = Sm[k];
    }
    if (bound == 'n') S2[0] = 2.0;
    for (int k = 0; k < n - 2; ++k) {
        Mo[k] = b[k] * 2.0 / (double)(2 * k + 5);
        M2[k + (size_t)n * (k + 2)] = Mo[k];
        M2[(k + 2) + (size_t)n * k] = Mo[k];
    }
    std::vector<double> sdiag(n);
    for (int k = 0; k < n; ++k) sdiag[k] = S2[k + (size_t)n * k];
    // scratch of the set-up, freed on every return (s itself is released by
    // the next preshen or by ductgpu_destroy when a step fails)
    struct Tmp {
        double *p = nullptr;
        ~Tmp() { cudaFree(p); }
    } tM, tS, tsd;
    int rc = DUCTGPU_OK;
    s.m = m;
    s.bound = bound;
    s.eig.n = n;
    s.leg.n = m;
    DUCT_CUDA(ctx, cudaMalloc(&s.Md, n * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(&s.Mo, n * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(&s.Sm, n * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(&s.bk, m * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(&s.eig.E, n * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(&s.eig.P, (size_t)n * n * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(&s.eig.PM1, (size_t)n * n * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(&s.leg.P, (size_t)m * m * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(&s.leg.PM1, (size_t)m * m * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(&s.leg.E, m * sizeof(double)));
    DUCT_CUDA(ctx, cudaMemsetAsync(s.leg.E, 0, m * sizeof(double), ctx->stream));
    DUCT_CUDA(ctx, cudaMalloc(&tM.p, (size_t)n * n * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(&tS.p, (size_t)n * n * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(&tsd.p, n * sizeof(double)));
    double *dM = tM.p, *dS = tS.p, *dsd = tsd.p;
    DUCT_CUDA(ctx, cudaMemcpyAsync(s.Md, Md.data(), n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    DUCT_CUDA(ctx, cudaMemcpyAsync(s.Mo, Mo.data(), n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    DUCT_CUDA(ctx, cudaMemcpyAsync(s.Sm, Sm.data(), n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    DUCT_CUDA(ctx, cudaMemcpyAsync(s.bk, b.data(), m * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    DUCT_CUDA(ctx, cudaMemcpyAsync(dsd, sdiag.data(), n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    if (bound == 'd') {
        DUCT_CUDA(ctx, cudaMemcpyAsync(dM, M2.data(), (size_t)n * n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        DUCT_CUDA(ctx, cudaMemcpyAsync(dS, S2.data(), (size_t)n * n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        rc = sygvd(ctx, n, dM, dS, s.eig.E);
        if (!rc) rc = check_cuda(ctx, cudaMemcpyAsync(s.eig.P, dM, (size_t)n * n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream), "P");
    } else {
        // the constant mode is split off: eigenproblem of the (2..n) block
        // (src/preshen.f90:479-496), P(1,1) = 1, rho_1 = 1
        const int n1 = n - 1;
        std::vector<double> M1((size_t)n1 * n1), S1((size_t)n1 * n1);
        for (int j = 0; j < n1; ++j)
            for (int i = 0; i < n1; ++i) {
                M1[i + (size_t)n1 * j] = M2[(i + 1) + (size_t)n * (j + 1)];
                S1[i + (size_t)n1 * j] = S2[(i + 1) + (size_t)n * (j + 1)];
            }
        DUCT_CUDA(ctx, cudaMemcpyAsync(dM, M1.data(), (size_t)n1 * n1 * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        DUCT_CUDA(ctx, cudaMemcpyAsync(dS, S1.data(), (size_t)n1 * n1 * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        const double one = 1.0;
        DUCT_CUDA(ctx, cudaMemcpyAsync(s.eig.E, &one, sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        rc = sygvd(ctx, n1, dM, dS, s.eig.E + 1);
        if (!rc) {
            k_embed<<<blocks((long)n * n), 256, 0, ctx->stream>>>(n, n1, dM, s.eig.P);
            ctx->launches += 1;
        }
    }
    // PSM1 = P^-1 S~^-1 (src/preshen.f90:516-530)
    if (!rc) rc = invert_dev(ctx, n, s.eig.P, s.eig.PM1);
    if (!rc) {
        k_scale_cols<<<blocks((long)n * n), 256, 0, ctx->stream>>>(n, s.eig.PM1, dsd);
        k_leg_cheb<<<1, 256, 0, ctx->stream>>>(m, s.leg.P);
        ctx->launches += 2;
        rc = invert_dev(ctx, m, s.leg.P, s.leg.PM1);
    }
    if (!rc) rc = pack_operators(ctx, s.eig);
    if (!rc) rc = pack_operators(ctx, s.leg);
    if (!rc) rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "preshen");
    if (rc) { free_shen(s); return rc; }
    s.ready = true;
    return DUCTGPU_OK;
}

// ---------------------------------------------------------------------------
struct ShenKField {
    double *in, *out;
    int nmodes, mode0, plane0;
    const double *bk, *Md, *Mo, *Sm, *E;
    char bound;
};
struct ShenKParams {
    ShenKField f[kMaxFields];
    int cta_start[kMaxFields + 1];   // in planes
    int nf;
    const double *lam;
    int m;
    long long plane_stride;
};

__device__ __forceinline__ int shen_field(const ShenKParams &p, int plane)
{
    int fi = 0;
    while (fi + 1 < p.nf && plane >= p.cta_start[fi + 1]) ++fi;
    return fi;
}

// leg2shen_sweep2d (src/legendre.f90:562-589): s = T g T^T with
// T(i,i) = 2/(2i+1), T(i,i+2) = 2 b_i/(2i+5); one CTA per plane.
__global__ void __launch_bounds__(256) k_leg2shen(const __grid_constant__ ShenKParams p)
{
    const int fi = shen_field(p, blockIdx.x);
    const ShenKField &F = p.f[fi];
    const int plane = blockIdx.x - p.cta_start[fi];
    const int m = p.m, n = m - 2;
    const double2 *g = reinterpret_cast<const double2 *>(F.in + (long long)plane * p.plane_stride);
    double2 *s = reinterpret_cast<double2 *>(F.out + (long long)plane * p.plane_stride);
    for (int idx = threadIdx.x; idx < m * m; idx += blockDim.x) {
        const int ii = idx % m, jj = idx / m;
        double2 v = make_double2(0.0, 0.0);
        if (ii < n && jj < n) {
            const double ta = 2.0 / (double)(2 * jj + 1), tb = 2.0 * F.bk[jj] / (double)(2 * jj + 5);
            const double tc = 2.0 / (double)(2 * ii + 1), td = 2.0 * F.bk[ii] / (double)(2 * ii + 5);
            const double2 g00 = g[ii + (long long)m * jj], g20 = g[(ii + 2) + (long long)m * jj];
            const double2 g02 = g[ii + (long long)m * (jj + 2)], g22 = g[(ii + 2) + (long long)m * (jj + 2)];
            v.x = ta * (g00.x * tc + g20.x * td) + tb * (g02.x * tc + g22.x * td);
            v.y = ta * (g00.y * tc + g20.y * td) + tb * (g02.y * tc + g22.y * td);
        }
        s[idx] = v;
    }
}

// shen2leg_sweep2d (src/legendre.f90:627-660): g(i,j) = s(i,j) + b_{j-2}
// s(i,j-2) + b_{i-2} s(i-2,j) + b_{i-2} b_{j-2} s(i-2,j-2).
__global__ void __launch_bounds__(256) k_shen2leg(const __grid_constant__ ShenKParams p)
{
    const int fi = shen_field(p, blockIdx.x);
    const ShenKField &F = p.f[fi];
    const int plane = blockIdx.x - p.cta_start[fi];
    const int m = p.m, n = m - 2;
    const double2 *s = reinterpret_cast<const double2 *>(F.in + (long long)plane * p.plane_stride);
    double2 *g = reinterpret_cast<double2 *>(F.out + (long long)plane * p.plane_stride);
    for (int idx = threadIdx.x; idx < m * m; idx += blockDim.x) {
        const int ii = idx % m, jj = idx / m;
        const double bi = ii >= 2 ? F.bk[ii - 2] : 0.0, bj = jj >= 2 ? F.bk[jj - 2] : 0.0;
        auto S = [&](int i, int j) -> double2 {
            return (i >= 0 && j >= 0 && i < n && j < n) ? s[i + (long long)m * j] : make_double2(0.0, 0.0);
        };
        const double2 s00 = S(ii, jj), s01 = S(ii, jj - 2), s10 = S(ii - 2, jj), s11 = S(ii - 2, jj - 2);
        g[idx] = make_double2(s00.x + s01.x * bj + s10.x * bi + bi * bj * s11.x,
                              s00.y + s01.y * bj + s10.y * bi + bi * bj * s11.y);
    }
}

// solV + solevenodd (src/solveshen.f90:335-513): for each plane, y-eigen
// index ip and parity of the z index, the SPD tridiagonal system
//   [rho_ip (lambda M + S) + M] v = g      (Neumann ip = 0: lambda M + S)
// along z, solved in place by LDL^T elimination (DPTSV's factorisation);
// re and im share the matrix.  One thread per (ip, parity) of a plane.
constexpr int kMaxSolv = (kMaxN - 2 + 1) / 2;   // longest parity system
__global__ void __launch_bounds__(256) k_shen_solv(const __grid_constant__ ShenKParams p, int nplanes_total)
{
    const int m = p.m, n = m - 2;
    const long long gid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long per_plane = 2LL * n;
    if (gid >= per_plane * nplanes_total) return;
    const int pg = (int)(gid / per_plane);
    const int r = (int)(gid - (long long)pg * per_plane);
    const int ip = r % n, par = r / n;
    const int fi = shen_field(p, pg);
    const ShenKField &F = p.f[fi];
    const int plane = pg - p.cta_start[fi];
    const double lam = p.lam[F.plane0 + plane];
    double2 *W = reinterpret_cast<double2 *>(F.out + (long long)plane * p.plane_stride);
    const bool neu_first = (F.bound == 'n' && ip == 0);
    const double rho = F.E[ip];
    const double ra1 = neu_first ? lam : rho * lam + 1.0;
    const int len = (par == 0) ? (n + 1) / 2 : n / 2;
    double piv[kMaxSolv];
    double2 prev = make_double2(0.0, 0.0);
    double eprev = 0.0;
    for (int q = 0; q < len; ++q) {
        const int k = 2 * q + par;
        double d = neu_first ? (lam * F.Md[k] + F.Sm[k]) : (rho * (lam * F.Md[k] + F.Sm[k]) + F.Md[k]);
        double2 g = W[ip + (long long)m * k];
        if (neu_first && par == 0 && q == 0 && lam < 1.0e-10) {   // the intended pin of the constant mode
            d = 1.0;
            g = make_double2(0.0, 0.0);
        }
        if (q > 0) {
            const double l = eprev / piv[q - 1];
            d -= l * eprev;
            g = make_double2(g.x - l * prev.x, g.y - l * prev.y);
        }
        piv[q] = d;
        W[ip + (long long)m * k] = g;
        prev = g;
        eprev = (q < len - 1) ? ra1 * F.Mo[k] : 0.0;
    }
    double2 x = make_double2(0.0, 0.0);
    for (int q = len - 1; q >= 0; --q) {
        const int k = 2 * q + par;
        const double e = (q < len - 1) ? ra1 * F.Mo[k] : 0.0;
        const double2 g = W[ip + (long long)m * k];
        x = make_double2((g.x - e * x.x) / piv[q], (g.y - e * x.y) / piv[q]);
        W[ip + (long long)m * k] = x;
    }
}

int solve_shen(ductgpu_ctx ctx, const ShenTask *tasks, int ntasks)
{
    const ShenOps &ref = (tasks[0].bound == 'n') ? ctx->shen_n : ctx->shen_d;
    const int m = ref.m, n = m - 2;
    const long long ps = 2LL * m * m;
    int planes = 0;
    for (int i = 0; i < ntasks; ++i) planes += tasks[i].nmodes;
    int rc = ensure(ctx, ctx->work, (size_t)2 * planes * ps * sizeof(double));
    if (rc) return rc;
    double *w1 = ctx->work.buf, *w2 = w1 + (size_t)planes * ps;
    long long offs[kMaxFields];
    {
        long long o = 0;
        for (int i = 0; i < ntasks; ++i) { offs[i] = o * ps; o += tasks[i].nmodes; }
    }
    // physical -> Chebyshev, in place on rhs (the reference transforms rhs)
    for (int i = 0; i < ntasks; ++i) {
        if ((rc = transyz_dev(ctx, tasks[i].rhs, m, m, tasks[i].nmodes, 'y', -1))) return rc;
        if ((rc = transyz_dev(ctx, tasks[i].rhs, m, m, tasks[i].nmodes, 'z', -1))) return rc;
    }
    // one full-plane DMMA pass over all fields: the Legendre matrices
    // (which = 0, m points) or the eigen-operators (which = 1, m-2 points)
    // along y or z, P (useP) or its inverse
    auto pass = [&](int which, bool ypass, bool useP, int im0, double *const *src, double *const *dst) -> int {
        PassParams pp{};
        pp.lam = ctx->lam;
        int cta = 0;
        for (int i = 0; i < ntasks; ++i) {
            const ShenOps &s = (tasks[i].bound == 'n') ? ctx->shen_n : ctx->shen_d;
            const BoundOps &b = which ? s.eig : s.leg;
            PassField &f = pp.f[i];
            pass_geometry(f, b, b.E, which ? n : m, ypass ? 1 : m, ypass ? m : 1, ps);
            f.off = 0;
            f.nmodes = tasks[i].nmodes;
            f.mode0 = tasks[i].mode0;
            f.plane0 = tasks[i].plane0;
            f.sing_io = f.sing_l = -1;
            f.A = useP ? b.Ppack : b.Qpack;
            f.src = src[i];
            f.dst = dst[i];
            pp.cta_start[i] = cta;
            cta += tasks[i].nmodes * f.nchunks;
        }
        pp.cta_start[ntasks] = cta;
        pp.nf = ntasks;
        pp.zero_im_mode0 = im0;
        return fp64_pass(ctx, pp, cta);
    };
    double *A1[kMaxFields], *A2[kMaxFields], *R[kMaxFields], *S[kMaxFields];
    for (int i = 0; i < ntasks; ++i) {
        A1[i] = w1 + offs[i];
        A2[i] = w2 + offs[i];
        R[i] = tasks[i].rhs;
        S[i] = tasks[i].sol;
    }
    ShenKParams kp{};
    kp.nf = ntasks;
    kp.lam = ctx->lam;
    kp.m = m;
    kp.plane_stride = ps;
    int kcta = 0;
    for (int i = 0; i < ntasks; ++i) {
        const ShenOps &s = (tasks[i].bound == 'n') ? ctx->shen_n : ctx->shen_d;
        ShenKField &f = kp.f[i];
        f.nmodes = tasks[i].nmodes;
        f.mode0 = tasks[i].mode0;
        f.plane0 = tasks[i].plane0;
        f.bk = s.bk; f.Md = s.Md; f.Mo = s.Mo; f.Sm = s.Sm; f.E = s.eig.E;
        f.bound = tasks[i].bound;
        kp.cta_start[i] = kcta;
        kcta += tasks[i].nmodes;
    }
    kp.cta_start[ntasks] = kcta;
    auto set_io = [&](double *const *in, double *const *out) {
        for (int i = 0; i < ntasks; ++i) { kp.f[i].in = in[i]; kp.f[i].out = out[i]; }
    };
    // Chebyshev -> Legendre: A . A^T
    if ((rc = pass(0, true, true, 0, R, A1))) return rc;
    if ((rc = pass(0, false, true, 0, A1, A2))) return rc;
    // Legendre -> Shen
    set_io(A2, A1);
    { LaunchScope ls(ctx, DUCTGPU_K_OTHER); k_leg2shen<<<kcta, 256, 0, ctx->stream>>>(kp); }
    // P^-1 S^-1 along y, tridiagonals along z, P along y
    if ((rc = pass(1, true, false, 0, A1, A2))) return rc;
    set_io(A2, A2);
    {
        const long long threads = 2LL * n * kcta;
        LaunchScope ls(ctx, DUCTGPU_K_OTHER);
        k_shen_solv<<<(unsigned)((threads + 255) / 256), 256, 0, ctx->stream>>>(kp, kcta);
    }
    if ((rc = pass(1, true, true, 0, A2, A1))) return rc;
    // Shen -> Legendre -> Chebyshev (B . B^T)
    set_io(A1, A2);
    { LaunchScope ls(ctx, DUCTGPU_K_OTHER); k_shen2leg<<<kcta, 256, 0, ctx->stream>>>(kp); }
    if ((rc = check_cuda(ctx, cudaGetLastError(), "shen kernels"))) return rc;
    if ((rc = pass(0, true, false, 0, A2, A1))) return rc;
    if ((rc = pass(0, false, false, 0, A1, S))) return rc;
    for (int i = 0; i < ntasks; ++i) {
        if ((rc = transyz_dev(ctx, tasks[i].sol, m, m, tasks[i].nmodes, 'y', 1))) return rc;
        if ((rc = transyz_dev(ctx, tasks[i].sol, m, m, tasks[i].nmodes, 'z', 1))) return rc;
        // mode 0 is real (src/int2d3d.f90); the transform carries (re, im)
        // through one complex FFT, so the zero is set after it
        if (tasks[i].mode0) {
            LaunchScope ls(ctx, DUCTGPU_K_OTHER);
            k_zero_imag<<<blocks((long)m * m), 256, 0, ctx->stream>>>(tasks[i].sol, (long)m * m);
        }
    }
    return check_cuda(ctx, cudaGetLastError(), "solve_shen");
}

}  // namespace duct
