// transforms.cu -- Chebyshev transforms, derivatives and pencil transposes
// on complex (my, mz, nmodes) fields (FP64).
//
// transyz (src/chebyshev.f90:458-540 over tcheb_fftw, src/tchebw.f:62-192):
// the reference copies every line to a contiguous buffer and runs FFTW's
// REDFT00 (DCT-I) on the real and imaginary parts separately.  Here the
// complex line itself, extended evenly to length 2N (N = line length - 1),
// goes through one complex FFT in shared memory: the DFT of an even real
// sequence is real, so FFT(re + i im) = DCT(re) + i DCT(im) with no
// unpacking.  The FFT is a mixed radix-4/2/3 Stockham transform (N is 2^a 3^b
// in the reference, src/tchebw.f:11-12); every stage reads and writes shared
// memory only, so a pass costs one HBM read and one write of the field.
//
// derivyz (src/chebyshev.f90:1-295): the backward recurrence
// d_{k-1} = d_{k+1} + 2k c_k on Chebyshev coefficients, one thread per
// complex line, lines staged through shared memory when they are
// contiguous in memory (y) and read directly when they are strided (z).
//
// Pencil transposes (src/parallel.F:476-529): 32x32 tiles of complex
// elements through padded shared memory.
#include <math.h>

#include "internal.h"

namespace duct {

constexpr int kMaxStages = 16;

struct DctParams {
    double *f;            // complex field
    long long line_stride;   // complex elements between consecutive lines of a mode
    long long elem_stride;   // complex elements between points of a line
    long long mode_stride;   // complex elements between modes
    int lines_per_mode;
    int nlines;           // lines_per_mode * nmodes
    int nn;               // points per line
    int L;                // 2 (nn - 1)
    int lpb;              // lines per CTA
    int iopt;             // < 0 forward (phys -> cheb), >= 0 inverse
    int nstages;
    int radix[kMaxStages];
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// In-place DFT of R points (R = 2, 3, 4), forward sign exp(-2 pi i jk/R).
template <int R>
__device__ __forceinline__ void dft(double2 (&v)[4])
{
    if (R == 2) {
        const double2 a = v[0], b = v[1];
        v[0] = make_double2(a.x + b.x, a.y + b.y);
        v[1] = make_double2(a.x - b.x, a.y - b.y);
    } else if (R == 3) {
        const double s = 0.86602540378443864676;  // sqrt(3)/2
        const double2 a = v[0], b = v[1], c = v[2];
        const double2 t = make_double2(b.x + c.x, b.y + c.y);
        const double2 d = make_double2(b.x - c.x, b.y - c.y);
        v[0] = make_double2(a.x + t.x, a.y + t.y);
        const double2 m = make_double2(a.x - 0.5 * t.x, a.y - 0.5 * t.y);
        // -i s d
        v[1] = make_double2(m.x + s * d.y, m.y - s * d.x);
        v[2] = make_double2(m.x - s * d.y, m.y + s * d.x);
    } else {
        const double2 a = v[0], b = v[1], c = v[2], d = v[3];
        const double2 s0 = make_double2(a.x + c.x, a.y + c.y), s1 = make_double2(a.x - c.x, a.y - c.y);
        const double2 s2 = make_double2(b.x + d.x, b.y + d.y), s3 = make_double2(b.x - d.x, b.y - d.y);
        v[0] = make_double2(s0.x + s2.x, s0.y + s2.y);
        v[2] = make_double2(s0.x - s2.x, s0.y - s2.y);
        // s1 - i s3, s1 + i s3
        v[1] = make_double2(s1.x + s3.y, s1.y - s3.x);
        v[3] = make_double2(s1.x - s3.y, s1.y + s3.x);
    }
}

template <int R>
__device__ __forceinline__ void stockham_stage(const double2 *x, double2 *y, int L, int Ns, int lpb)
{
    const int nb = L / R;
    for (int idx = threadIdx.x; idx < nb * lpb; idx += blockDim.x) {
        const int l = idx / nb, j = idx - l * nb;
        const double2 *xl = x + l * L;
        double2 *yl = y + l * L;
        const int k = j % Ns;
        double2 v[4];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = xl[j + r * nb];
        if (Ns > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) {
                double sn, cs;
                sincospi(-2.0 * (double)(r * k) / (double)(Ns * R), &sn, &cs);
                v[r] = cmul(v[r], make_double2(cs, sn));
            }
        }
        dft<R>(v);
        const int d = (j / Ns) * Ns * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) yl[d + r * Ns] = v[r];
    }
}

__global__ void __launch_bounds__(256) k_dct(const __grid_constant__ DctParams p)
{
    extern __shared__ __align__(16) double2 buf[];
    double2 *x = buf, *y = buf + p.lpb * p.L;
    const int line0 = blockIdx.x * p.lpb;
    const int nl = min(p.lpb, p.nlines - line0);
    const int N = p.nn - 1, L = p.L;
    auto gaddr = [&](int l, int j) -> double2 * {
        const int line = line0 + l;
        const int mode = line / p.lines_per_mode, q = line - mode * p.lines_per_mode;
        return reinterpret_cast<double2 *>(p.f) + mode * p.mode_stride + q * p.line_stride + j * p.elem_stride;
    };
    // load + even extension; inverse: ends weighted 1, interior 1/2
    const bool contiguous = (p.elem_stride == 1);
    for (int idx = threadIdx.x; idx < p.lpb * p.nn; idx += blockDim.x) {
        int l, j;
        if (contiguous) { l = idx / p.nn; j = idx - l * p.nn; }
        else { j = idx / p.lpb; l = idx - j * p.lpb; }
        double2 v = make_double2(0.0, 0.0);
        if (l < nl) v = *gaddr(l, j);
        if (p.iopt >= 0 && j > 0 && j < N) v = make_double2(0.5 * v.x, 0.5 * v.y);
        x[l * L + j] = v;
        if (j > 0 && j < N) x[l * L + (L - j)] = v;
    }
    __syncthreads();
    int Ns = 1;
    for (int s = 0; s < p.nstages; ++s) {
        const int R = p.radix[s];
        if (R == 4) stockham_stage<4>(x, y, L, Ns, p.lpb);
        else if (R == 2) stockham_stage<2>(x, y, L, Ns, p.lpb);
        else stockham_stage<3>(x, y, L, Ns, p.lpb);
        Ns *= R;
        __syncthreads();
        double2 *t = x; x = y; y = t;
    }
    const double dn1 = 1.0 / (double)N, dn2 = 0.5 * dn1;
    for (int idx = threadIdx.x; idx < p.lpb * p.nn; idx += blockDim.x) {
        int l, j;
        if (contiguous) { l = idx / p.nn; j = idx - l * p.nn; }
        else { j = idx / p.lpb; l = idx - j * p.lpb; }
        if (l >= nl) continue;
        double2 v = x[l * L + j];
        if (p.iopt < 0) {
            const double sc = (j == 0 || j == N) ? dn2 : dn1;
            v = make_double2(sc * v.x, sc * v.y);
        }
        *gaddr(l, j) = v;
    }
}

// ---------------------------------------------------------------------------
struct DerivParams {
    const double *u;
    double *du;
    long long line_stride, elem_stride, mode_stride;
    int lines_per_mode, nlines, nn;
    int ider;
    int accumulate;
    double fac;           // scal (y) or scal/aspect^ider (z)
};

// out_k = -d_k fac (k >= 1), out_0 = -d_0 fac / 2, d_{k-1} = d_{k+1} + 2k c_k
// (the minus sign: the solver's coordinate is x = -cos, src/chebyshev.f90:44-58).
__device__ void deriv_rec(const double2 *c, long long cs, double2 *o, long long os, int nn, double fac, bool acc)
{
    double2 b = make_double2(0.0, 0.0), a = b, t = b;
    for (int kk = nn - 1; kk >= 1; --kk) {
        const double2 ck = c[kk * cs];
        const double2 cr = make_double2(b.x + 2.0 * kk * ck.x, b.y + 2.0 * kk * ck.y);
        const double2 val = make_double2(-t.x * fac, -t.y * fac);
        if (acc) o[kk * os] = make_double2(o[kk * os].x + val.x, o[kk * os].y + val.y);
        else o[kk * os] = val;
        b = a;
        t = cr;
        a = cr;
    }
    const double2 val = make_double2(-0.5 * t.x * fac, -0.5 * t.y * fac);
    if (acc) o[0] = make_double2(o[0].x + val.x, o[0].y + val.y);
    else o[0] = val;
}

constexpr int kDerivLines = 32;

__global__ void __launch_bounds__(256) k_deriv(const __grid_constant__ DerivParams p)
{
    extern __shared__ __align__(16) double2 sm[];
    const int line0 = blockIdx.x * kDerivLines;
    const int nl = min(kDerivLines, p.nlines - line0);
    auto base = [&](int l) -> long long {
        const int line = line0 + l;
        const int mode = line / p.lines_per_mode, q = line - mode * p.lines_per_mode;
        return mode * p.mode_stride + q * p.line_stride;
    };
    const double2 *U = reinterpret_cast<const double2 *>(p.u);
    double2 *DU = reinterpret_cast<double2 *>(p.du);
    const int nn = p.nn;
    if (p.elem_stride == 1) {
        // contiguous lines: stage (in, aux) through shared memory, padded rows
        const int ld = nn + 1;
        double2 *cin = sm, *aux = sm + kDerivLines * ld;
        for (int idx = threadIdx.x; idx < kDerivLines * nn; idx += blockDim.x) {
            const int l = idx / nn, j = idx - l * nn;
            if (l < nl) cin[l * ld + j] = U[base(l) + j];
        }
        __syncthreads();
        const int l = threadIdx.x;
        if (l < nl) {
            if (p.ider == 1) {
                deriv_rec(cin + l * ld, 1, aux + l * ld, 1, nn, p.fac, false);
            } else {
                deriv_rec(cin + l * ld, 1, aux + l * ld, 1, nn, 1.0, false);
                deriv_rec(aux + l * ld, 1, cin + l * ld, 1, nn, p.fac, false);
            }
        }
        __syncthreads();
        const double2 *res = (p.ider == 1) ? aux : cin;
        for (int idx = threadIdx.x; idx < kDerivLines * nn; idx += blockDim.x) {
            const int l2 = idx / nn, j = idx - l2 * nn;
            if (l2 >= nl) continue;
            const long long g = base(l2) + j;
            const double2 v = res[l2 * ld + j];
            DU[g] = p.accumulate ? make_double2(DU[g].x + v.x, DU[g].y + v.y) : v;
        }
    } else {
        // strided lines: neighbouring threads own neighbouring lines, so every
        // step of the recurrence is a coalesced access
        const int l = threadIdx.x;
        if (l >= nl) return;
        const long long b0 = base(l);
        if (p.ider == 1) {
            deriv_rec(U + b0, p.elem_stride, DU + b0, p.elem_stride, nn, p.fac, p.accumulate != 0);
        } else {
            // aux line in shared memory, column l
            double2 *aux = sm;
            deriv_rec(U + b0, p.elem_stride, aux + l, kDerivLines, nn, 1.0, false);
            deriv_rec(aux + l, kDerivLines, DU + b0, p.elem_stride, nn, p.fac, p.accumulate != 0);
        }
    }
}

// ---------------------------------------------------------------------------
// out(q, a) = in(a, q): transpose of an A x Q column-major matrix of complex
// elements (A fastest) into Q x A (Q fastest), 32x32 tiles.
__global__ void __launch_bounds__(256) k_transpose(const double2 *in, double2 *out, long long A, long long Q)
{
    __shared__ double2 tile[32][33];
    const long long a0 = (long long)blockIdx.x * 32, q0 = (long long)blockIdx.y * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int r = ty; r < 32; r += 8) {
        const long long a = a0 + tx, q = q0 + r;
        if (a < A && q < Q) tile[r][tx] = in[a + A * q];
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const long long q = q0 + tx, a = a0 + r;
        if (a < A && q < Q) out[q + Q * a] = tile[tx][r];
    }
}

// ---------------------------------------------------------------------------

static int plan_radices(int L, int *radix)
{
    int n = 0;
    while (L % 4 == 0 && n < kMaxStages) { radix[n++] = 4; L /= 4; }
    while (L % 2 == 0 && n < kMaxStages) { radix[n++] = 2; L /= 2; }
    while (L % 3 == 0 && n < kMaxStages) { radix[n++] = 3; L /= 3; }
    return L == 1 ? n : -1;
}

static void line_geometry(char cdir, int my, int mz, long long &ls, long long &es, long long &ms, int &lpm, int &nn)
{
    ms = (long long)my * mz;
    if (cdir == 'y') { ls = my; es = 1; lpm = mz; nn = my; }
    else { ls = 1; es = my; lpm = my; nn = mz; }
}

int transyz_dev(ductgpu_ctx ctx, double *f, int my, int mz, int nmodes, char cdir, int iopt)
{
    DctParams p{};
    p.f = f;
    line_geometry(cdir, my, mz, p.line_stride, p.elem_stride, p.mode_stride, p.lines_per_mode, p.nn);
    p.nlines = p.lines_per_mode * nmodes;
    p.L = 2 * (p.nn - 1);
    p.nstages = plan_radices(p.L, p.radix);
    if (p.nstages < 0)
        return set_error(ctx, DUCTGPU_EARG, "transyz: line length %d - 1 must be of the form 2^a 3^b", p.nn);
    p.lpb = 2048 / p.L;
    if (p.lpb < 1) p.lpb = 1;
    if (p.lpb > 32) p.lpb = 32;
    p.iopt = iopt;
    const size_t smem = 2 * (size_t)p.lpb * p.L * sizeof(double2);
    DUCT_CUDA(ctx, cudaFuncSetAttribute(k_dct, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int grid = (p.nlines + p.lpb - 1) / p.lpb;
    {
        LaunchScope ls(ctx, DUCTGPU_K_TRANSFORM);
        k_dct<<<grid, 256, smem, ctx->stream>>>(p);
    }
    return check_cuda(ctx, cudaGetLastError(), "k_dct");
}

int derivyz_dev(ductgpu_ctx ctx, const double *u, double *du, int my, int mz, int nmodes, char cdir,
                int ider, double scal, char what, double aspect)
{
    DerivParams p{};
    p.u = u;
    p.du = du;
    line_geometry(cdir, my, mz, p.line_stride, p.elem_stride, p.mode_stride, p.lines_per_mode, p.nn);
    p.nlines = p.lines_per_mode * nmodes;
    p.ider = ider;
    p.accumulate = (what != 'n');
    p.fac = scal;
    if (cdir == 'z') p.fac = (ider == 1) ? scal / aspect : scal / (aspect * aspect);
    size_t smem;
    if (p.elem_stride == 1) smem = 2 * (size_t)kDerivLines * (p.nn + 1) * sizeof(double2);
    else smem = (size_t)kDerivLines * p.nn * sizeof(double2);
    DUCT_CUDA(ctx, cudaFuncSetAttribute(k_deriv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int grid = (p.nlines + kDerivLines - 1) / kDerivLines;
    {
        LaunchScope ls(ctx, DUCTGPU_K_TRANSFORM);
        k_deriv<<<grid, (p.elem_stride == 1) ? 256 : kDerivLines, smem, ctx->stream>>>(p);
    }
    return check_cuda(ctx, cudaGetLastError(), "k_deriv");
}

int transpose_dev(ductgpu_ctx ctx, const double *in, double *out, long long A, long long Q)
{
    dim3 grid((unsigned)((A + 31) / 32), (unsigned)((Q + 31) / 32));
    if (grid.y > 65535) return set_error(ctx, DUCTGPU_EARG, "transpose: %lld columns too many", Q);
    {
        LaunchScope ls(ctx, DUCTGPU_K_TRANSPOSE);
        k_transpose<<<grid, 256, 0, ctx->stream>>>(reinterpret_cast<const double2 *>(in),
                                                    reinterpret_cast<double2 *>(out), A, Q);
    }
    return check_cuda(ctx, cudaGetLastError(), "k_transpose");
}

}  // namespace duct
