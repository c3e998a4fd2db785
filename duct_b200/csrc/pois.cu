// pois.cu -- the Galerkin-basis Neumann (pressure) solver: pseudopois and
// solvepois (src/pseudopois.f90:2-104, src/solvepois.f90:1-170).
//
// Basis phi_j = T_j - j^2/(j+2)^2 T_{j+2}, j = 0..my-3 (phi_j'(+-1) = 0).
// B(i,j) = phi_j(x_i), B2(i,j) = phi_j''(x_i) on the interior nodes; the
// Neumann operator is D = B2 B^-1 with eigen-pairs (EN, PN).  The interior
// solve is the diagonalisation solve of solve_fp64.cu with these operators
// (four batched DMMA passes, the kx=0 eigen-coefficient skipped and the
// point (iofzero+1, iofzero+1) pinned to wanted = 0).  The walls are the
// basis expansion evaluated at +-1: with the coefficients a = B^-1 U B^-T,
//   U(-1, z_j) = phi(-1)^T B^-1 U(:,j) = r_-^T U(:,j),  r_+- = B^-T phi(+-1),
// and the corners r_s^T U r_t -- the reference's coefficient GEMMs
// (src/solvepois.f90:104-169) collapse to these dot products, evaluated by
// one kernel per plane (k_pois_fill).
#include <math.h>

#include <vector>

#include "internal.h"

namespace duct {

static int blocks(long n) { return (int)((n + 255) / 256 < 2048 ? (n + 255) / 256 : 2048); }

// T_n(x) = cos(n acos x) and T_n''(x) = n (x sin(n t) - n cos(n t) sin t) /
// sin^3 t, t = acos x (interior nodes only, sin t > 0).
static double cheb_t(int n, double x) { return cos((double)n * acos(x)); }
static double cheb_t2(int n, double x)
{
    const double t = acos(x), s = sin(t);
    return (double)n * (x * sin((double)n * t) - (double)n * cos((double)n * t) * s) / (s * s * s);
}

__global__ void k_pois_matmul(int n, const double *A, const double *B, double *C)
{
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n * n; idx += gridDim.x * blockDim.x) {
        const int i = idx % n, j = idx / n;
        double s = 0.0;
        for (int k = 0; k < n; ++k) s = fma(A[i + (size_t)n * k], B[k + (size_t)n * j], s);
        C[idx] = s;
    }
}

// r_- (k) = sum_j Binv(j,k) phi_j(-1), r_+ (k) = sum_j Binv(j,k) phi_j(+1),
// phi_j(+1) = 4 (j+1)/(j+2)^2, phi_j(-1) = (-1)^j phi_j(+1).
__global__ void k_pois_rvec(int n, const double *Binv, double *r)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        double sm = 0.0, sp = 0.0;
        for (int j = 0; j < n; ++j) {
            const double v = 4.0 * (double)(j + 1) / ((double)(j + 2) * (double)(j + 2));
            const double b = Binv[j + (size_t)n * k];
            sp = fma(b, v, sp);
            sm = fma(b, (j & 1) ? -v : v, sm);
        }
        r[k] = sm;
        r[n + k] = sp;
    }
}

int pois_setup(ductgpu_ctx ctx, int m)
{
    if (m < 5 || m - 2 > kMaxN) return set_error(ctx, DUCTGPU_EARG, "pseudopois: my=%d (5..%d)", m, kMaxN + 2);
    cudaStreamSynchronize(ctx->stream);
    free_bound(ctx->pois);
    cudaFree(ctx->pois_r);
    ctx->pois_r = nullptr;
    ctx->pois_m = 0;
    const int n = m - 2;
    const double pi = 3.14159265358979323846;
    std::vector<double> B((size_t)n * n), B2((size_t)n * n);
    for (int i = 1; i < m - 1; ++i) {
        const double x = -cos(pi * (double)i / (double)(m - 1));
        for (int j = 0; j < n; ++j) {
            const double c = (double)j * (double)j / (((double)j + 2.0) * ((double)j + 2.0));
            B[(i - 1) + (size_t)n * j] = cheb_t(j, x) - c * cheb_t(j + 2, x);
            B2[(i - 1) + (size_t)n * j] = cheb_t2(j, x) - c * cheb_t2(j + 2, x);
        }
    }
    struct Tmp {
        double *p = nullptr;
        ~Tmp() { cudaFree(p); }
    } tB, tB2, tBi, tD;
    BoundOps &b = ctx->pois;
    b.n = n;
    DUCT_CUDA(ctx, cudaMalloc(&tB.p, (size_t)n * n * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(&tB2.p, (size_t)n * n * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(&tBi.p, (size_t)n * n * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(&tD.p, (size_t)n * n * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(&b.E, n * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(&b.P, (size_t)n * n * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(&b.PM1, (size_t)n * n * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(&ctx->pois_r, 2 * (size_t)n * sizeof(double)));
    DUCT_CUDA(ctx, cudaMemcpyAsync(tB.p, B.data(), (size_t)n * n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    DUCT_CUDA(ctx, cudaMemcpyAsync(tB2.p, B2.data(), (size_t)n * n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    // PNT = B^-1 (dgetrf/dgetri, src/pseudopois.f90:57-61), D = B2 B^-1 (:62)
    int rc = invert_dev(ctx, n, tB.p, tBi.p);
    if (!rc) {
        k_pois_matmul<<<blocks((long)n * n), 256, 0, ctx->stream>>>(n, tB2.p, tBi.p, tD.p);
        k_pois_rvec<<<1, 256, 0, ctx->stream>>>(n, tBi.p, ctx->pois_r);
        ctx->launches += 2;
        rc = check_cuda(ctx, cudaGetLastError(), "pseudopois");
    }
    // eigen-decomposition (dgeev), PNM1, iofzero (:64-80)
    if (!rc) rc = eigen_gpu(ctx, n, tD.p, b);
    if (!rc) rc = pack_operators(ctx, b);
    if (!rc) rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "pseudopois");
    if (rc) {
        free_bound(b);
        cudaFree(ctx->pois_r);
        ctx->pois_r = nullptr;
        return rc;
    }
    ctx->pois_m = m;
    return DUCTGPU_OK;
}

struct PoisFill {
    double *sol[kMaxFields];
    int plane0[kMaxFields];
    int cta_start[kMaxFields + 1];
    int nf;
    const double *pcol, *r, *lam;
    double wanted;
    int m, io;
    long long plane_stride;
};

// One CTA per complex plane: the kx=0 pin (src/solvepois.f90:38-86, in
// physical space: U += c p p^T, c = (wanted - U(io,io))/p_io^2), then the
// four wall lines and the corners from the basis (:104-169).
__global__ void __launch_bounds__(1024) k_pois_fill(const __grid_constant__ PoisFill p)
{
    extern __shared__ double2 edge[];   // y = -1, y = +1 (index j), z = -1, z = +1 (index i)
    int fi = 0;
    while (fi + 1 < p.nf && (int)blockIdx.x >= p.cta_start[fi + 1]) ++fi;
    const int plane = blockIdx.x - p.cta_start[fi];
    const int m = p.m, n = m - 2;
    double2 *U = reinterpret_cast<double2 *>(p.sol[fi] + (long long)plane * p.plane_stride);
    const double lam = p.lam[p.plane0[fi] + plane];
    if (fabs(lam) <= 1.0e-10 && p.io >= 0) {
        const int io = p.io;
        const double2 u0 = U[(io + 1) + (long long)m * (io + 1)];
        __syncthreads();
        const double pio = p.pcol[io];
        const double2 cc = make_double2((p.wanted - u0.x) / (pio * pio), (p.wanted - u0.y) / (pio * pio));
        for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
            const int i = idx % n, j = idx / n;
            const double w = p.pcol[i] * p.pcol[j];
            double2 &u = U[(i + 1) + (long long)m * (j + 1)];
            u = make_double2(u.x + w * cc.x, u.y + w * cc.y);
        }
        __syncthreads();
    }
    const double *rm = p.r, *rp = p.r + n;
    double2 *ey0 = edge, *eym = edge + n, *ez0 = edge + 2 * n, *ezm = edge + 3 * n;
    // y-walls, one warp per interior column j: r^T U(:, j)
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int j = warp; j < n; j += nw) {
        double a0 = 0, a1 = 0, b0 = 0, b1 = 0;
        for (int k = lane; k < n; k += 32) {
            const double2 v = U[(k + 1) + (long long)m * (j + 1)];
            a0 += rm[k] * v.x; a1 += rm[k] * v.y;
            b0 += rp[k] * v.x; b1 += rp[k] * v.y;
        }
        for (int o = 16; o > 0; o >>= 1) {
            a0 += __shfl_xor_sync(0xffffffffu, a0, o);
            a1 += __shfl_xor_sync(0xffffffffu, a1, o);
            b0 += __shfl_xor_sync(0xffffffffu, b0, o);
            b1 += __shfl_xor_sync(0xffffffffu, b1, o);
        }
        if (lane == 0) {
            ey0[j] = make_double2(a0, a1);
            eym[j] = make_double2(b0, b1);
        }
    }
    // z-walls, one thread per interior row i: U(i, :) r
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double a0 = 0, a1 = 0, b0 = 0, b1 = 0;
        for (int k = 0; k < n; ++k) {
            const double2 v = U[(i + 1) + (long long)m * (k + 1)];
            a0 += rm[k] * v.x; a1 += rm[k] * v.y;
            b0 += rp[k] * v.x; b1 += rp[k] * v.y;
        }
        ez0[i] = make_double2(a0, a1);
        ezm[i] = make_double2(b0, b1);
    }
    __syncthreads();
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        U[(long long)m * (j + 1)] = ey0[j];
        U[(m - 1) + (long long)m * (j + 1)] = eym[j];
        U[j + 1] = ez0[j];
        U[(j + 1) + (long long)m * (m - 1)] = ezm[j];
    }
    // corners: the y = -+1 edges contracted with r_-+ along z
    if (warp < 4) {
        const double2 *e = (warp & 1) ? eym : ey0;          // y = -1 (0, 2) or +1 (1, 3)
        const double *r = (warp & 2) ? rp : rm;             // z = -1 (0, 1) or +1 (2, 3)
        double a0 = 0, a1 = 0;
        for (int k = lane; k < n; k += 32) {
            a0 += r[k] * e[k].x;
            a1 += r[k] * e[k].y;
        }
        for (int o = 16; o > 0; o >>= 1) {
            a0 += __shfl_xor_sync(0xffffffffu, a0, o);
            a1 += __shfl_xor_sync(0xffffffffu, a1, o);
        }
        if (lane == 0) {
            const long long yi = (warp & 1) ? m - 1 : 0, zi = (warp & 2) ? m - 1 : 0;
            U[yi + (long long)m * zi] = make_double2(a0, a1);
        }
    }
}

int solve_pois(ductgpu_ctx ctx, const FieldTask *tasks, int ntasks)
{
    const int m = ctx->pois_m, n = m - 2;
    const long long ps = 2LL * m * m;
    int planes = 0;
    for (int i = 0; i < ntasks; ++i) planes += tasks[i].nmodes;
    int rc = ensure(ctx, ctx->work, (size_t)2 * planes * ps * sizeof(double));
    if (rc) return rc;
    double *w1 = ctx->work.buf, *w2 = w1 + (size_t)planes * ps;
    const BoundOps &b = ctx->pois;
    PassParams pp{};
    pp.lam = ctx->lam;
    // y: PNM1 -> w1 ; z: PNM1 + divide -> w2 ; z: PN -> w1 ; y: PN -> sol
    for (int pass = 0; pass < 4; ++pass) {
        long long off = 0;
        int cta = 0;
        const bool ypass = (pass == 0 || pass == 3);
        for (int i = 0; i < ntasks; ++i) {
            PassField &f = pp.f[i];
            double *a1 = w1 + off * ps, *a2 = w2 + off * ps;
            off += tasks[i].nmodes;
            pass_geometry(f, b, b.E, n, ypass ? 1 : m, ypass ? m : 1, ps);
            f.nmodes = tasks[i].nmodes;
            f.mode0 = tasks[i].mode0;
            f.plane0 = tasks[i].plane0;
            f.sing_io = f.sing_l = b.iofzero - 1;
            switch (pass) {
            case 0: f.src = tasks[i].rhs; f.dst = a1; f.A = b.Qpack; break;
            case 1: f.src = a1; f.dst = a2; f.A = b.Qpack; break;
            case 2: f.src = a2; f.dst = a1; f.A = b.Ppack; break;
            default: f.src = a1; f.dst = tasks[i].sol; f.A = b.Ppack; break;
            }
            pp.cta_start[i] = cta;
            cta += tasks[i].nmodes * f.nchunks;
        }
        pp.cta_start[ntasks] = cta;
        pp.nf = ntasks;
        pp.divide = (pass == 1);
        pp.zero_im_mode0 = (pass == 3);
        pp.residual = 0;
        if ((rc = fp64_pass(ctx, pp, cta))) return rc;
    }
    PoisFill fp{};
    int cta = 0;
    for (int i = 0; i < ntasks; ++i) {
        fp.sol[i] = tasks[i].sol;
        fp.plane0[i] = tasks[i].plane0;
        fp.cta_start[i] = cta;
        cta += tasks[i].nmodes;
    }
    fp.cta_start[ntasks] = cta;
    fp.nf = ntasks;
    fp.pcol = b.pcol;
    fp.r = ctx->pois_r;
    fp.lam = ctx->lam;
    fp.wanted = 0.0;   // src/pseudopois.f90:80
    fp.m = m;
    fp.io = b.pcol ? b.iofzero - 1 : -1;
    fp.plane_stride = ps;
    {
        LaunchScope ls(ctx, DUCTGPU_K_NEUMANN);
        k_pois_fill<<<cta, 1024, 4 * (size_t)n * sizeof(double2), ctx->stream>>>(fp);
    }
    return check_cuda(ctx, cudaGetLastError(), "solve_pois");
}

}  // namespace duct
