// dns.cu -- the DNS time step around the 2D solve (FP64): the x-direction
// Fourier products of the advection term with 2/3 de-aliasing, the
// operators of the fractional-step RK3/Crank-Nicolson substep, the
// statistics and wall diagnostics, and a device-resident stepper whose
// substeps are captured as CUDA graphs.
//
// Reference: advection3d (src/operators.F:9-276) with fourx / pack_fftw /
// fill (src/fourier.F:1-118), mult (src/mult.F:11-45) and the pencil
// transposes chx2z / chz2x (src/parallel.F:1-208); laplacian3d, grad3d,
// div3d, update_uvwp (src/operators.F:278-605); wallstressx
// (src/operators.F:676-710 -> src/chebyshev.f90:642-690), energy_fou
// (src/operators.F:907-973), statistics_fou / statistics_fou2
// (src/operators.F:1608-1765, 1957-2004), max_3din (src/operators.F:
// 2524-2550); the substep of src/main1.f90:384-723 (no temperature,
// DT_FIXED, icase 1 or CMASSFLOW).
//
// Layout: every field is x-cut complex (my, mz, nmodes), y fastest -- the
// reference's u(my,mz,ib:ie).  The reference's x transform works on z-cut
// pencils after chx2z; here the products are formed point by point straight
// from the x-cut layout (the modes of a point are a stride-(my mz) gather
// that is coalesced across consecutive points), so neither pencil
// transpose exists.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <initializer_list>
#include <new>
#include <vector>

#include "fft.cuh"
#include "internal.h"

namespace duct {

static const double kPi = 3.14159265358979323846;

// ---------------------------------------------------------------------------
// Advection products.  Per (y, z) point the three velocity spectra (modes
// 0..M-1, the rest of the mgalx-point spectrum zero: fill) go to physical
// space along x, the six products uu, vv, ww, uv, uw, vw are formed there
// and transformed back, modes 0..M-1 kept and scaled by 1/mgalx
// (pack_fftw).  Two real signals share one complex FFT: u + i v (inverse),
// w alone, and the products in pairs (uu + i vv, ww + i uv, uw + i vw),
// separated as A_k = (X_k + conj X_{N-k})/2, B_k = -i (X_k - conj X_{N-k})/2.
// The FFT is four-step with N = R^2: a thread per column holds R points
// in registers; after the inverse its registers hold the physical values
// at x = c + R k2, which are exactly the column-c inputs of the forward
// transform, so the products never leave registers.
// Outputs: adv1 = i kx UU, adv2 = i kx UV, adv3 = i kx UW (derivx of the
// diagonal products, src/operators.F advection3d steps (1), (4), (5)) and
// the five spectra uv, uw, vv, vw, ww that the y / z derivatives need.
struct AdvParams {
    const double2 *u, *v, *w;
    double2 *adv1, *adv2, *adv3;
    double2 *uv, *uw, *vv, *vw, *ww;
    double *stats2;        // [6][P] x-means of uu, vv, ww, uv, uw, vw (added), or null
    const double *xalp;    // device [M]
    long long P;           // points of a plane (my mz)
    int M;                 // Fourier modes kept (mx1 + 1)
    // determine_step / slip_velocity_3d (src/operators.F:608-672, 2552-2608)
    // on the physical velocities, or null: atomic maxima (order_key) of
    // max(|u| hx, |v|/dy, |w|/dz) into cfl[0] and cfl[2], of the velocity
    // components on the walls into cfl[1]
    unsigned long long *cfl;
    const double *rdyz;    // [my + mz]: 1/dy, 1/dz
    double hx;             // alp mgalx / (2 pi)
    int my, mz;
};

// A monotone map of doubles to unsigned integers (x < y <=> key(x) <
// key(y)), so that an integer atomic max keeps the largest double; key 0
// lies below every number.
__device__ __forceinline__ unsigned long long order_key(double x)
{
    const unsigned long long b = (unsigned long long)__double_as_longlong(x);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
static double order_key_value(unsigned long long k)
{
    const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
    double x;
    memcpy(&x, &b, sizeof x);
    return x;
}

// Step 2 of a four-step FFT over the CTA's points: thread (c, g) reads row
// c of point g from wk and returns X[c + R k2] in v.
template <int R, int TQ>
__device__ __forceinline__ void fft_step2(const double2 *wk, double2 (&v)[R], const double2 *tw, int c, int g)
{
#pragma unroll
    for (int n2 = 0; n2 < R; ++n2) v[n2] = wk[(c * R + n2) * TQ + g];
    reg_fft<R, 0, 1>(v, tw, R * R);
}

// Step 1: the R-point DFT of column c (already in v), twiddle W_N^(c k1),
// into wk for step 2.
template <int R, int TQ>
__device__ __forceinline__ void fft_step1(double2 (&v)[R], double2 *wk, const double2 *tw, int c, int g)
{
    reg_fft<R, 0, 1>(v, tw, R * R);
#pragma unroll
    for (int k1 = 0; k1 < R; ++k1) wk[(k1 * R + c) * TQ + g] = (k1 == 0) ? v[0] : cmul(v[k1], tw[c * k1]);
}

template <int R, int TQ, int MINB = 1, bool ALIAS = false>
__global__ void __launch_bounds__(R * TQ, MINB) k_advx(const __grid_constant__ AdvParams p, const double2 *__restrict__ twg)
{
    constexpr int N = R * R, NT = R * TQ;
    extern __shared__ __align__(16) double2 sm[];
    double2 *tw = sm;                // W_N^t
    double2 *wk = tw + N;            // [R][R][TQ] step buffer
    // [N][TQ] spectrum of a product pair; ALIAS: in the step buffer, once
    // every thread has read its step-2 column out of it
    double2 *xs = ALIAS ? wk : wk + N * TQ;
    const int c = threadIdx.x / TQ, g = threadIdx.x - c * TQ;
    const long long q0 = (long long)blockIdx.x * TQ;
    const long long q = q0 + g;
    const bool valid = q < p.P;
    const int M = p.M;
    const long long P = p.P;
    for (int t = threadIdx.x; t < N; t += NT) cp_async16(tw + t, twg + t);
    cp_async_wait_all();
    __syncthreads();

    // spectrum of mode k = R n1 + c of the Hermitian extension, conjugated
    // (the inverse transform is conj(DFT(conj Z)))
    double2 a[R];
#pragma unroll
    for (int n1 = 0; n1 < R; ++n1) {
        const int k = R * n1 + c;
        double2 z = make_double2(0.0, 0.0);
        if (valid && k < M) {
            const double2 uk = p.u[q + (long long)k * P], vk = p.v[q + (long long)k * P];
            // Z = U + i V; mode 0: imaginary parts ignored
            z = (k == 0) ? make_double2(uk.x, -vk.x) : make_double2(uk.x - vk.y, -(uk.y + vk.x));
        } else if (valid && k > N - M) {
            const long long kk = N - k;
            const double2 uk = p.u[q + kk * P], vk = p.v[q + kk * P];
            // Z_{N-k} = conj U_k + i conj V_k
            z = make_double2(uk.x + vk.y, -(vk.x - uk.y));
        }
        a[n1] = z;
    }
    fft_step1<R, TQ>(a, wk, tw, c, g);
    __syncthreads();
    fft_step2<R, TQ>(wk, a, tw, c, g);
    double uu[R], vv[R], ww[R];    // physical values at x = c + R k2
#pragma unroll
    for (int k2 = 0; k2 < R; ++k2) {
        uu[k2] = a[k2].x;
        vv[k2] = -a[k2].y;
    }
    // the time-step and slip checks of the step's first substep
    double eig = 0.0, slip = -1.0e308, rdz = 0.0;
    bool wall = false;
    if (p.cfl && valid) {
        const int j = (int)(q % p.my), kz = (int)(q / p.my);
        const double rdy = p.rdyz[j];
        rdz = p.rdyz[p.my + kz];
        wall = j == 0 || j == p.my - 1 || kz == 0 || kz == p.mz - 1;
#pragma unroll
        for (int k2 = 0; k2 < R; ++k2) {
            eig = fmax(eig, fmax(fabs(uu[k2]) * p.hx, fabs(vv[k2]) * rdy));
            if (wall) slip = fmax(slip, fmax(uu[k2], vv[k2]));
        }
    }
    __syncthreads();
#pragma unroll
    for (int n1 = 0; n1 < R; ++n1) {
        const int k = R * n1 + c;
        double2 z = make_double2(0.0, 0.0);
        if (valid && k < M) {
            const double2 wk0 = p.w[q + (long long)k * P];
            z = (k == 0) ? make_double2(wk0.x, 0.0) : make_double2(wk0.x, -wk0.y);
        } else if (valid && k > N - M) {
            const double2 wk0 = p.w[q + (long long)(N - k) * P];
            z = make_double2(wk0.x, wk0.y);
        }
        a[n1] = z;
    }
    fft_step1<R, TQ>(a, wk, tw, c, g);
    __syncthreads();
    fft_step2<R, TQ>(wk, a, tw, c, g);
#pragma unroll
    for (int k2 = 0; k2 < R; ++k2) ww[k2] = a[k2].x;
    if (p.cfl) {
        if (valid) {
#pragma unroll
            for (int k2 = 0; k2 < R; ++k2) {
                eig = fmax(eig, fabs(ww[k2]) * rdz);
                if (wall) slip = fmax(slip, ww[k2]);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            eig = fmax(eig, __shfl_xor_sync(0xffffffffu, eig, o));
            slip = fmax(slip, __shfl_xor_sync(0xffffffffu, slip, o));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMax(p.cfl, order_key(eig));
            atomicMax(p.cfl + 1, order_key(slip));
            atomicMax(p.cfl + 2, order_key(eig));
        }
    }

    const double sc = 1.0 / N;
    for (int pair = 0; pair < 3; ++pair) {
        // products at x = R k2 + c (forward input n = R n1 + n2, n2 = c, n1 = k2)
#pragma unroll
        for (int k2 = 0; k2 < R; ++k2) {
            const double x = uu[k2], y = vv[k2], z = ww[k2];
            a[k2] = (pair == 0) ? make_double2(x * x, y * y)
                  : (pair == 1) ? make_double2(z * z, x * y)
                                : make_double2(x * z, y * z);
        }
        __syncthreads();   // wk free (previous step 2 / separation done)
        fft_step1<R, TQ>(a, wk, tw, c, g);
        __syncthreads();
        fft_step2<R, TQ>(wk, a, tw, c, g);
        if (ALIAS) __syncthreads();
#pragma unroll
        for (int k2 = 0; k2 < R; ++k2) xs[(c + R * k2) * TQ + g] = a[k2];
        __syncthreads();
        for (int idx = threadIdx.x; idx < M * TQ; idx += NT) {
            const int i = idx / TQ, gg = idx - i * TQ;
            const long long qq = q0 + gg;
            if (qq >= P) continue;
            const double2 X = xs[i * TQ + gg], Y = xs[(i == 0 ? 0 : N - i) * TQ + gg];
            // A = (X + conj Y)/2, B = -i (X - conj Y)/2, both scaled by 1/N
            const double2 A = make_double2(0.5 * sc * (X.x + Y.x), 0.5 * sc * (X.y - Y.y));
            const double2 B = make_double2(0.5 * sc * (X.y + Y.y), -0.5 * sc * (X.x - Y.x));
            const double kx = p.xalp[i];
            const long long e = qq + (long long)i * P;
            const double2 iA = make_double2(-kx * A.y, kx * A.x);
            if (pair == 0) {            // A = uu, B = vv
                p.adv1[e] = iA;
                p.vv[e] = B;
            } else if (pair == 1) {     // A = ww, B = uv
                p.ww[e] = A;
                p.uv[e] = B;
                p.adv2[e] = make_double2(-kx * B.y, kx * B.x);
            } else {                    // A = uw, B = vw
                p.uw[e] = A;
                p.adv3[e] = iA;
                p.vw[e] = B;
            }
            if (p.stats2 && i == 0) {
                // statistics_fou2: x-means (mode 0, real part) in the order uu, vv, ww, uv, uw, vw
                const int sa = (pair == 0) ? 0 : (pair == 1) ? 2 : 4;
                const int sb = (pair == 0) ? 1 : (pair == 1) ? 3 : 5;
                p.stats2[sa * P + qq] += A.x;
                p.stats2[sb * P + qq] += B.x;
            }
        }
    }
}

template <int R, int TQ, int MINB = 1, bool ALIAS = false>
static int launch_advx(ductgpu_ctx ctx, const AdvParams &p)
{
    constexpr int N = R * R, NT = R * TQ;
    const double2 *tw = twiddle_table(ctx, N);
    if (!tw) return set_error(ctx, DUCTGPU_ESTATE, "advection3d: twiddle table for mgalx=%d unavailable", N);
    const size_t smem = ((size_t)N + (ALIAS ? 1 : 2) * (size_t)N * TQ) * sizeof(double2);
    DUCT_CUDA(ctx, cudaFuncSetAttribute(k_advx<R, TQ, MINB, ALIAS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const long long grid = (p.P + TQ - 1) / TQ;
    // algorithmic bytes: u, v, w read, eight product fields written
    if (ctx->prof_on && !ctx->capturing) ctx->prof_bytes[DUCTGPU_K_ADVECTION] += 11.0 * 16.0 * p.P * p.M;
    {
        LaunchScope ls(ctx, DUCTGPU_K_ADVECTION);
        k_advx<R, TQ, MINB, ALIAS><<<(unsigned)grid, NT, smem, ctx->stream>>>(p, tw);
    }
    return check_cuda(ctx, cudaGetLastError(), "k_advx");
}

static bool advx_supported(int mgalx) { return mgalx == 16 || mgalx == 64 || mgalx == 256 || mgalx == 144; }

static int advx_launch(ductgpu_ctx ctx, const AdvParams &p, int mgalx)
{
    switch (mgalx) {
    case 16: return launch_advx<4, 32>(ctx, p);
    case 64: return launch_advx<8, 16>(ctx, p);
    case 144: return launch_advx<12, 8>(ctx, p);
    // mgalx = 256: the pair spectrum aliased onto the step buffer (36 KB of
    // shared memory a CTA) and registers for four CTAs per SM (128, spilling):
    // 1.075 ms a config-4 step, against 1.096 for three CTAs aliased, 1.126
    // for three with separate buffers (168 registers), 1.21 for two (255)
    // and 1.21 for five (96); 64-thread CTAs (4 points) at 4 or 6 per SM
    // measured 1.27 / 1.19 ms
    case 256: return launch_advx<16, 8, 4, true>(ctx, p);
    default: return set_error(ctx, DUCTGPU_EARG, "advection3d: mgalx=%d (16, 64, 144 or 256)", mgalx);
    }
}

// ---------------------------------------------------------------------------
// Statistics.  One pass over u, v, w, p per recorded step: per point the
// energies of energy_fou (sum over modes i >= 1 of 2 |f_i|^2, and |f_0|^2,
// weighted by the mesh sizes dy dz), the mode-0 means and the x-mean of
// p^2 (statistics_fou), and the wall stress of wallstressx as a dot product
// of the mode-0 plane of u with four precomputed physical-space weight
// planes (the reference's 2D DCT of that plane followed by the weighted
// coefficient sums of cheb2_wallstress_circum is one linear functional per
// wall).  Per-CTA partial sums are combined in a fixed order by a finishing
// kernel, so the result does not depend on scheduling.
constexpr int kStatVals = 10;    // stress4[4], energy e (u, v, w) sums, energy e0 (mode 0) sums
constexpr int kStatThreads = 256;
constexpr int kStatBlocksMax = 296;

__device__ __forceinline__ double block_sum(double v, double *red)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x < 32) {
        s = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    }
    return s;   // valid in thread 0
}

struct StatParams {
    const double2 *f[4];     // u, v, w, p (p may be null: energies / stress only)
    const double *wcc;       // [P] dy dz
    const double *wst;       // [4][P] wall-stress weights, or null
    double *mean;            // [4][P] added, or null
    double *ppb;             // [P] added, or null
    double *partial;         // [gridDim][kStatVals]
    long long P;
    int M;
    int nf;                  // fields with energies (1..3)
};

__global__ void __launch_bounds__(kStatThreads) k_stats(const __grid_constant__ StatParams p)
{
    __shared__ double red[32];
    double acc[kStatVals];
#pragma unroll
    for (int k = 0; k < kStatVals; ++k) acc[k] = 0.0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < p.P; q += (long long)gridDim.x * blockDim.x) {
        const double wq = p.wcc[q];
        for (int c = 0; c < p.nf; ++c) {
            const double2 *f = p.f[c];
            double e = 0.0;
            for (int i = 1; i < p.M; ++i) {
                const double2 z = f[q + (long long)i * p.P];
                e = e + (z.x * z.x + z.y * z.y) * 2.0;
            }
            const double2 z0 = f[q];
            acc[4 + c] += e * wq;
            acc[7 + c] += (z0.x * z0.x + z0.y * z0.y) * wq;
            if (p.mean) p.mean[c * p.P + q] += z0.x;
        }
        if (p.wst) {
            const double u0 = p.f[0][q].x;
#pragma unroll
            for (int s = 0; s < 4; ++s) acc[s] += p.wst[s * p.P + q] * u0;
        }
        if (p.f[3]) {
            const double2 *f = p.f[3];
            double e = 0.0;
            for (int i = 1; i < p.M; ++i) {
                const double2 z = f[q + (long long)i * p.P];
                e = e + (z.x * z.x + z.y * z.y) * 2.0;
            }
            const double2 z0 = f[q];
            if (p.mean) p.mean[3 * p.P + q] += z0.x;
            if (p.ppb) p.ppb[q] += e + (z0.x * z0.x + z0.y * z0.y);
        }
    }
#pragma unroll
    for (int k = 0; k < kStatVals; ++k) {
        const double s = block_sum(acc[k], red);
        if (threadIdx.x == 0) p.partial[blockIdx.x * kStatVals + k] = s;
    }
}

// out[0..3] = stress4, out[4..6] = energy (u, v, w), out[7..9] = energy2
// (energy_fou: sqrt(e / area), sqrt((e + e0) / area)).  With a counter, the
// values go to out + 10 * (*counter) (a history row) and the counter
// advances; rows beyond cap are counted but not written.
__global__ void k_stats_finish(const double *partial, int nblocks, double area, double *out, int *counter, int cap)
{
    __shared__ double e[kStatVals];
    const int k = threadIdx.x;
    if (k < kStatVals) {
        double s = 0.0;
        for (int b = 0; b < nblocks; ++b) s += partial[b * kStatVals + k];
        e[k] = s;
    }
    __syncthreads();
    int row = 0;
    if (counter) {
        row = *counter;
        if (row >= cap) row = -1;
    }
    __syncthreads();
    if (row >= 0) {
        double *o = out + (size_t)kStatVals * row;
        if (k < 4) o[k] = e[k];
        else if (k < 7) {
            o[k] = sqrt(e[k] / area);
            o[k + 3] = sqrt((e[k] + e[k + 3]) / area);
        }
    }
    if (counter && k == 0) *counter += 1;
}

// statistics_fou's streamwise spectra at seven points: spec[c][s][i] +=
// |f_c(i, q_s)|^2 (times 2 for i >= 1).
__global__ void k_spectra(const double2 *u, const double2 *v, const double2 *w, const double2 *p, long long P, int M,
                          int my, int mz, double *spec)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 4 * 7 * M) return;
    const int i = t % M, s = (t / M) % 7, c = t / (7 * M);
    const int jin[7] = {my / 16, my / 8, my / 4, my / 2, my / 16, my / 8, my / 4};
    const int kin[7] = {mz / 2, mz / 2, mz / 2, mz / 2, mz / 16, mz / 8, mz / 4};
    if (jin[s] < 1 || kin[s] < 1) return;   // grids below 16 points: no such point
    const long long q = (long long)(jin[s] - 1) + (long long)my * (kin[s] - 1);
    const double2 *f = (c == 0) ? u : (c == 1) ? v : (c == 2) ? w : p;
    const double2 z = f[q + (long long)i * P];
    const double a = z.x * z.x + z.y * z.y;
    spec[((size_t)c * 7 + s) * M + i] += (i == 0) ? a : a * 2.0;
}

// Vorticity statistics of a recorded step (src/main1.f90:453-466): per
// component c of omega, statistics_omg2_fou (src/operators.F:1859-1955)
// om2[c] += |w_0|^2 + sum_{i>=1} 2 |w_i|^2 per point, and energy_fou's sums
// (907-973); for omega_x also energy_fou_zero_sector (1018-1099, |w_0|^2 dy
// dz per sector) and integral_abs_zero_sector (1462-1541, |Re w_0| dy dz).
// Sectors of point (j, k), 1-based: 1 j<k, j<mz+1-k; 2 j<k, j>mz+1-k;
// 3 j>k, j>mz+1-k; 4 j>k, j<mz+1-k; 5 on a diagonal.
constexpr int kOmgVals = 16;   // e (x, y, z), e0 (x, y, z), sector |w0|^2 [5], sector |Re w0| [5]

struct OmgParams {
    const double2 *f[3];     // omega_x, omega_y, omega_z
    const double *wcc;       // [P] dy dz
    double *om2;             // [3][P] added
    double *partial;         // [gridDim][kOmgVals]
    long long P;
    int M, my, mz;
};

__global__ void __launch_bounds__(kStatThreads) k_omg_stats(const __grid_constant__ OmgParams p)
{
    __shared__ double red[32];
    double acc[kOmgVals];
#pragma unroll
    for (int k = 0; k < kOmgVals; ++k) acc[k] = 0.0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < p.P; q += (long long)gridDim.x * blockDim.x) {
        const double wq = p.wcc[q];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double2 *f = p.f[c];
            double e = 0.0;
            for (int i = 1; i < p.M; ++i) {
                const double2 z = f[q + (long long)i * p.P];
                e = e + (z.x * z.x + z.y * z.y) * 2.0;
            }
            const double2 z0 = f[q];
            const double a0 = z0.x * z0.x + z0.y * z0.y;
            p.om2[c * p.P + q] += e + a0;
            acc[c] += e * wq;
            acc[3 + c] += a0 * wq;
        }
        const int j = (int)(q % p.my) + 1, k = (int)(q / p.my) + 1, kr = p.mz + 1 - k;
        const int s = (j < k && j < kr) ? 0 : (j < k && j > kr) ? 1 : (j > k && j > kr) ? 2 : (j > k && j < kr) ? 3 : 4;
        const double2 z0 = p.f[0][q];
#pragma unroll
        for (int t = 0; t < 5; ++t) {
            acc[6 + t] += (t == s) ? (z0.x * z0.x + z0.y * z0.y) * wq : 0.0;
            acc[11 + t] += (t == s) ? fabs(z0.x) * wq : 0.0;
        }
    }
#pragma unroll
    for (int k = 0; k < kOmgVals; ++k) {
        const double sum = block_sum(acc[k], red);
        if (threadIdx.x == 0) p.partial[blockIdx.x * kOmgVals + k] = sum;
    }
}

// The row of the step just recorded by k_stats_finish (*counter - 1):
// out[0..4] energomx4 (sector energies / area), out[5..9] energomxb4
// (sector |Re w0| integrals / area), out[10..12] energy_fou of omega_x,
// omega_y, omega_z (sqrt(e / area)), out[13..15] the same with mode 0.
__global__ void k_omg_finish(const double *partial, int nblocks, double area, double *out, const int *counter, int cap)
{
    __shared__ double e[kOmgVals];
    const int k = threadIdx.x;
    if (k < kOmgVals) {
        double sum = 0.0;
        for (int b = 0; b < nblocks; ++b) sum += partial[b * kOmgVals + k];
        e[k] = sum;
    }
    __syncthreads();
    const int row = *counter - 1;
    if (row < 0 || row >= cap) return;
    double *o = out + (size_t)kOmgVals * row;
    if (k < 3) {
        o[10 + k] = sqrt(e[k] / area);
        o[13 + k] = sqrt((e[k] + e[3 + k]) / area);
    } else if (k >= 6 && k < 16) {
        o[k - 6] = e[k] / area;
    }
}

// Host: the weights.  Nodes x_j = -s cos(pi j / (n - 1)); mesh sizes of
// src/ininewc.f90:102-112 (half the distance between the neighbours).
static void mesh_sizes(int n, double s, std::vector<double> &d)
{
    std::vector<double> x(n);
    for (int j = 0; j < n; ++j) x[j] = -s * cos(kPi * (double)j / (double)(n - 1));
    d.assign(n, 0.0);
    d[0] = (x[1] - x[0]) * 0.5;
    for (int j = 1; j < n - 1; ++j) d[j] = (x[j + 1] - x[j - 1]) * 0.5;
    d[n - 1] = (x[n - 1] - x[n - 2]) * 0.5;
}

// Forward transyz matrix C (n x n, c = C x): C[j][y] = sc_j w_y cos(pi j y / N)
// with N = n - 1, sc_j = 2/N (1/N at j = 0, N), w_y = 1/2 at y = 0, N.
static void dct_matrix(int n, std::vector<double> &C)
{
    const int N = n - 1;
    C.assign((size_t)n * n, 0.0);
    for (int j = 0; j < n; ++j) {
        const double sc = (j == 0 || j == N) ? 1.0 / N : 2.0 / N;
        for (int y = 0; y < n; ++y) {
            const double w = (y == 0 || y == N) ? 0.5 : 1.0;
            // cos(pi j y / N) with the argument reduced exactly (j y mod 2N)
            const long r = ((long)j * y) % (2L * N);
            C[(size_t)j * n + y] = sc * w * cos(kPi * (double)r / (double)N);
        }
    }
}

// Physical-space weight planes of wallstressx: stress_w = sum_q W_w[q] u0[q]
// with W_w = Cy^T Wc_w Cz and Wc_w the coefficient weights of
// cheb2_wallstress_circum (src/chebyshev.f90:642-690), divided by the
// circumference 4 + 4 aspect.
static void wallstress_weights(int my, int mz, double aspect, std::vector<double> &W)
{
    std::vector<double> Cy, Cz;
    dct_matrix(my, Cy);
    dct_matrix(mz, Cz);
    std::vector<double> Wc((size_t)4 * my * mz, 0.0);
    auto wc = [&](int s, int j, int k) -> double & { return Wc[((size_t)s * mz + k) * my + j]; };
    const double circ = 4.0 + 4.0 * aspect;
    for (int k = 0; k < mz; k += 2)
        for (int j = 0; j < my; ++j) {
            const double f = 2.0 * aspect * (double)j * j / (double)(k * k - 1);
            wc(0, j, k) = -f / circ;
            wc(1, j, k) = ((j & 1) ? 1.0 : -1.0) * f / circ;
        }
    for (int k = 0; k < mz; ++k)
        for (int j = 0; j < my; j += 2) {
            const double f = 2.0 / aspect * (double)k * k / (double)(j * j - 1);
            wc(2, j, k) = -f / circ;
            wc(3, j, k) = ((k & 1) ? 1.0 : -1.0) * f / circ;
        }
    W.assign((size_t)4 * my * mz, 0.0);
    std::vector<double> T((size_t)my * mz);
    for (int s = 0; s < 4; ++s) {
        // T[j][z] = sum_k Wc[j][k] Cz[k][z]
        for (int z = 0; z < mz; ++z)
            for (int j = 0; j < my; ++j) {
                double a = 0.0;
                for (int k = 0; k < mz; ++k) a += wc(s, j, k) * Cz[(size_t)k * mz + z];
                T[(size_t)z * my + j] = a;
            }
        // W[y][z] = sum_j Cy[j][y] T[j][z]
        for (int z = 0; z < mz; ++z)
            for (int y = 0; y < my; ++y) {
                double a = 0.0;
                for (int j = 0; j < my; ++j) a += Cy[(size_t)j * my + y] * T[(size_t)z * my + j];
                W[((size_t)s * mz + z) * my + y] = a;
            }
    }
}

// max |u| over the interior points of all modes (max_3din); the per-CTA
// maxima go through an atomic max on the bit pattern (|u| >= 0).
__global__ void k_maxabs(const double2 *u, int my, int mz, int M, double *out)
{
    const long long total = (long long)(my - 2) * (mz - 2) * M;
    double vmax = 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long j = 1 + t % (my - 2), r = t / (my - 2);
        const long long k = 1 + r % (mz - 2), i = r / (mz - 2);
        const double2 z = u[j + (long long)my * (k + (long long)mz * i)];
        vmax = fmax(vmax, hypot(z.x, z.y));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) vmax = fmax(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
    if ((threadIdx.x & 31) == 0 && vmax > 0.0)
        atomicMax(reinterpret_cast<unsigned long long *>(out), (unsigned long long)__double_as_longlong(vmax));
}

// ---------------------------------------------------------------------------
// Buffers of the operator entries, owned by the context.
struct DnsAux {
    double *xalp = nullptr;
    int xalp_cap = 0;
    int w_my = 0, w_mz = 0;
    double w_aspect = -1.0;
    double *wcc = nullptr, *wst = nullptr;   // [P] dy dz, [4][P] wall-stress weights
    double *partial = nullptr;               // [kStatBlocksMax][kStatVals]
    double *out = nullptr;                   // [kStatVals + 1]: statistics, then max |u|
};

void free_dns_aux(ductgpu_ctx ctx)
{
    DnsAux *a = ctx->dns_aux;
    if (!a) return;
    cudaFree(a->xalp);
    cudaFree(a->wcc);
    cudaFree(a->wst);
    cudaFree(a->partial);
    cudaFree(a->out);
    delete a;
    ctx->dns_aux = nullptr;
}

static int aux_get(ductgpu_ctx ctx, DnsAux **out)
{
    if (!ctx->dns_aux) {
        DnsAux *a = new (std::nothrow) DnsAux();
        if (!a) return set_error(ctx, DUCTGPU_EALLOC, "dns: out of host memory");
        if (cudaMalloc(&a->partial, sizeof(double) * kStatBlocksMax * kStatVals) != cudaSuccess ||
            cudaMalloc(&a->out, sizeof(double) * (kStatVals + 1)) != cudaSuccess) {
            cudaFree(a->partial);
            delete a;
            cudaGetLastError();
            return set_error(ctx, DUCTGPU_EALLOC, "dns: device buffers");
        }
        ctx->dns_aux = a;
    }
    *out = ctx->dns_aux;
    return DUCTGPU_OK;
}

// The wavenumbers to the device (stream-ordered after earlier launches).
static int upload_xalp(ductgpu_ctx ctx, const double *xalp, int nmodes, const double **dev)
{
    DnsAux *a = nullptr;
    int rc = aux_get(ctx, &a);
    if (rc) return rc;
    if (!xalp) return set_error(ctx, DUCTGPU_EARG, "xalp is null");
    if (nmodes > a->xalp_cap) {
        DUCT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        cudaFree(a->xalp);
        a->xalp = nullptr;
        a->xalp_cap = 0;
        DUCT_CUDA(ctx, cudaMalloc(&a->xalp, sizeof(double) * nmodes));
        a->xalp_cap = nmodes;
    }
    DUCT_CUDA(ctx, cudaMemcpyAsync(a->xalp, xalp, sizeof(double) * nmodes, cudaMemcpyHostToDevice, ctx->stream));
    *dev = a->xalp;
    return DUCTGPU_OK;
}

// Energy (mesh-size) and wall-stress weights on the device, for (my, mz, aspect).
static int make_weights(int my, int mz, double aspect, std::vector<double> &wcc, std::vector<double> &wst)
{
    std::vector<double> dy, dz;
    mesh_sizes(my, 1.0, dy);
    mesh_sizes(mz, aspect, dz);
    wcc.resize((size_t)my * mz);
    for (int k = 0; k < mz; ++k)
        for (int j = 0; j < my; ++j) wcc[(size_t)k * my + j] = dy[j] * dz[k];
    wallstress_weights(my, mz, aspect, wst);
    return 0;
}

static int aux_weights(ductgpu_ctx ctx, int my, int mz, double aspect, DnsAux **out)
{
    DnsAux *a = nullptr;
    int rc = aux_get(ctx, &a);
    if (rc) return rc;
    if (a->w_my != my || a->w_mz != mz || a->w_aspect != aspect) {
        std::vector<double> wcc, wst;
        make_weights(my, mz, aspect, wcc, wst);
        DUCT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        cudaFree(a->wcc);
        cudaFree(a->wst);
        a->wcc = a->wst = nullptr;
        a->w_my = 0;
        DUCT_CUDA(ctx, cudaMalloc(&a->wcc, sizeof(double) * wcc.size()));
        DUCT_CUDA(ctx, cudaMalloc(&a->wst, sizeof(double) * wst.size()));
        DUCT_CUDA(ctx, cudaMemcpy(a->wcc, wcc.data(), sizeof(double) * wcc.size(), cudaMemcpyHostToDevice));
        DUCT_CUDA(ctx, cudaMemcpy(a->wst, wst.data(), sizeof(double) * wst.size(), cudaMemcpyHostToDevice));
        a->w_my = my;
        a->w_mz = mz;
        a->w_aspect = aspect;
    }
    *out = a;
    return DUCTGPU_OK;
}

static int check_geom(ductgpu_ctx ctx, const char *who, int my, int mz, int nmodes, bool lines)
{
    if (my < 3 || mz < 3 || nmodes < 1)
        return set_error(ctx, DUCTGPU_EARG, "%s: my=%d mz=%d nmodes=%d", who, my, mz, nmodes);
    if (lines && (!lines_supported(my) || !lines_supported(mz)))
        return set_error(ctx, DUCTGPU_EARG, "%s: my-1=%d, mz-1=%d must be one of 16, 24, 32, 48, 64, 96, 128, 144, "
                         "192, 256", who, my - 1, mz - 1);
    return DUCTGPU_OK;
}

static int check_ptrs(ductgpu_ctx ctx, const char *who, std::initializer_list<const void *> ps)
{
    for (const void *p : ps)
        if (!p || ((uintptr_t)p & 15))
            return set_error(ctx, DUCTGPU_EARG, "%s: null or not 16-byte aligned field pointer", who);
    return DUCTGPU_OK;
}

static LineOut line_out(double *out, int order, double fac, double beta, double sigma = 1.0)
{
    LineOut o;
    o.out = out;
    o.order = order;
    o.fac = fac;
    o.beta = beta;
    o.sigma = sigma;
    return o;
}

// Adds the term (c0 + c1 i kx + c2 (i kx)^2) src to an output.
static void xterm(LineOut &o, const double *src, double c0, double c1, double c2)
{
    for (int t = 0; t < kLineXTerms; ++t)
        if (!o.xs[t]) {
            o.xs[t] = src;
            o.xc0[t] = c0;
            o.xc1[t] = c1;
            o.xc2[t] = c2;
            return;
        }
}

static LineParams line_params(char dir, int my, int mz, int nmodes, const double *xalp_dev, int real0 = 0)
{
    LineParams p;
    p.real0 = real0;
    p.dir = dir;
    p.my = my;
    p.mz = mz;
    p.nmodes = nmodes;
    p.xalp = xalp_dev;
    return p;
}

static void add_job(LineParams &p, const double *in, std::initializer_list<LineOut> outs)
{
    LineJob &J = p.job[p.njobs++];
    J.in = in;
    J.nout = 0;
    for (const LineOut &o : outs) J.o[J.nout++] = o;
}

// One more output of job `job` (from the same staged lines).
static void add_out(LineParams &p, int job, const LineOut &o)
{
    LineJob &J = p.job[job];
    if (J.nout < kMaxLineOut) J.o[J.nout++] = o;
}

}  // namespace duct

using namespace duct;

// ---- the reference's operators on device fields -------------------------
extern "C" int ductgpu_derivx_dev(ductgpu_ctx ctx, const double *u, double *du, int my, int mz, int nmodes,
                                  const double *xalp, int ider, double scal, char what)
{
    if (!ctx) return DUCTGPU_EARG;
    int rc = check_geom(ctx, "derivx", my, mz, nmodes, false);
    if (!rc) rc = check_ptrs(ctx, "derivx", {u, du});
    if (rc) return rc;
    if (ider != 1 && ider != 2) return set_error(ctx, DUCTGPU_EARG, "derivx: ider=%d", ider);
    cudaSetDevice(ctx->device);
    const double *xd;
    if ((rc = upload_xalp(ctx, xalp, nmodes, &xd))) return rc;
    // a line launch with an order-0 output only: du = [du +] scal (i kx)^ider u
    LineParams p = line_params('y', my, mz, nmodes, xd);
    LineOut o = line_out(du, 0, 0.0, what == 'n' ? 0.0 : 1.0);
    xterm(o, u, 0.0, ider == 1 ? scal : 0.0, ider == 2 ? scal : 0.0);
    add_job(p, u, {o});
    if (lines_supported(my)) return lines_launch(ctx, p);
    return set_error(ctx, DUCTGPU_EARG, "derivx: my-1=%d not a supported line length", my - 1);
}

extern "C" int ductgpu_laplacian3d_dev(ductgpu_ctx ctx, const double *u, double *flap, int my, int mz, int nmodes,
                                       const double *xalp, double aspect, double scal, char what)
{
    if (!ctx) return DUCTGPU_EARG;
    int rc = check_geom(ctx, "laplacian3d", my, mz, nmodes, true);
    if (!rc) rc = check_ptrs(ctx, "laplacian3d", {u, flap});
    if (rc) return rc;
    if (u == flap) return set_error(ctx, DUCTGPU_EARG, "laplacian3d: u and flap must differ");
    cudaSetDevice(ctx->device);
    const double *xd;
    if ((rc = upload_xalp(ctx, xalp, nmodes, &xd))) return rc;
    LineParams py = line_params('y', my, mz, nmodes, xd);
    LineOut oy = line_out(flap, 2, scal, what == 'n' ? 0.0 : 1.0);
    xterm(oy, u, 0.0, 0.0, scal);
    add_job(py, u, {oy});
    if ((rc = lines_launch(ctx, py))) return rc;
    LineParams pz = line_params('z', my, mz, nmodes, xd);
    add_job(pz, u, {line_out(flap, 2, scal / (aspect * aspect), 1.0)});
    return lines_launch(ctx, pz);
}

extern "C" int ductgpu_vorticity_dev(ductgpu_ctx ctx, const double *u, const double *v, const double *w, double *vort,
                                     int my, int mz, int nmodes, const double *xalp, double aspect, int iflag)
{
    if (!ctx) return DUCTGPU_EARG;
    int rc = check_geom(ctx, "vorticity", my, mz, nmodes, true);
    if (!rc) rc = check_ptrs(ctx, "vorticity", {u, v, w, vort});
    if (rc) return rc;
    if (iflag < 1 || iflag > 3) return set_error(ctx, DUCTGPU_EARG, "vorticity: component %d (1, 2, 3)", iflag);
    if (vort == u || vort == v || vort == w) return set_error(ctx, DUCTGPU_EARG, "vorticity: vort must differ from u, v, w");
    cudaSetDevice(ctx->device);
    const double *xd;
    if ((rc = upload_xalp(ctx, xalp, nmodes, &xd))) return rc;
    if (iflag == 1) {                       // om_x = w,y - v,z
        LineParams py = line_params('y', my, mz, nmodes, xd);
        add_job(py, w, {line_out(vort, 1, 1.0, 0.0)});
        if ((rc = lines_launch(ctx, py))) return rc;
        LineParams pz = line_params('z', my, mz, nmodes, xd);
        add_job(pz, v, {line_out(vort, 1, -1.0 / aspect, 1.0)});
        return lines_launch(ctx, pz);
    }
    if (iflag == 2) {                       // om_y = u,z - w,x
        LineParams pz = line_params('z', my, mz, nmodes, xd);
        LineOut o = line_out(vort, 1, 1.0 / aspect, 0.0);
        xterm(o, w, 0.0, -1.0, 0.0);
        add_job(pz, u, {o});
        return lines_launch(ctx, pz);
    }
    LineParams py = line_params('y', my, mz, nmodes, xd);   // om_z = v,x - u,y
    LineOut o = line_out(vort, 1, -1.0, 0.0);
    xterm(o, v, 0.0, 1.0, 0.0);
    add_job(py, u, {o});
    return lines_launch(ctx, py);
}

extern "C" int ductgpu_grad3d_dev(ductgpu_ctx ctx, const double *u, double *dxu, double *dyu, double *dzu, int my,
                                  int mz, int nmodes, const double *xalp, double aspect, double scal, char what)
{
    if (!ctx) return DUCTGPU_EARG;
    int rc = check_geom(ctx, "grad3d", my, mz, nmodes, true);
    if (!rc) rc = check_ptrs(ctx, "grad3d", {u, dxu, dyu, dzu});
    if (rc) return rc;
    cudaSetDevice(ctx->device);
    const double *xd;
    if ((rc = upload_xalp(ctx, xalp, nmodes, &xd))) return rc;
    const double beta = what == 'n' ? 0.0 : 1.0;
    LineParams py = line_params('y', my, mz, nmodes, xd);
    LineOut ox = line_out(dxu, 0, 0.0, beta);
    xterm(ox, u, 0.0, scal, 0.0);
    add_job(py, u, {line_out(dyu, 1, scal, beta), ox});
    if ((rc = lines_launch(ctx, py))) return rc;
    LineParams pz = line_params('z', my, mz, nmodes, xd);
    add_job(pz, u, {line_out(dzu, 1, scal / aspect, beta)});
    return lines_launch(ctx, pz);
}

extern "C" int ductgpu_div3d_dev(ductgpu_ctx ctx, const double *u, const double *v, const double *w, double *div,
                                 int my, int mz, int nmodes, const double *xalp, double aspect, double scal)
{
    if (!ctx) return DUCTGPU_EARG;
    int rc = check_geom(ctx, "div3d", my, mz, nmodes, true);
    if (!rc) rc = check_ptrs(ctx, "div3d", {u, v, w, div});
    if (rc) return rc;
    cudaSetDevice(ctx->device);
    const double *xd;
    if ((rc = upload_xalp(ctx, xalp, nmodes, &xd))) return rc;
    LineParams py = line_params('y', my, mz, nmodes, xd);
    LineOut o = line_out(div, 1, scal, 0.0);
    xterm(o, u, 0.0, scal, 0.0);
    add_job(py, v, {o});
    if ((rc = lines_launch(ctx, py))) return rc;
    LineParams pz = line_params('z', my, mz, nmodes, xd);
    add_job(pz, w, {line_out(div, 1, scal / aspect, 1.0)});
    return lines_launch(ctx, pz);
}

namespace duct {
// update_uvwp (no FILTER): p += phi - f1 lap(phi), u += s2 i kx phi,
// v += s2 phi_y, w += s2 phi_z, with f1 = (akk + bkk) dt nu, s2 = -dt (akk + bkk).
static int update_lines(ductgpu_ctx ctx, double *u, double *v, double *w, double *p, const double *phi, int my, int mz,
                        int nmodes, const double *xd, double aspect, double akk, double bkk, double dt, double fnu,
                        int real0 = 0)
{
    const double f1 = (akk + bkk) * dt * fnu, s2 = -dt * (akk + bkk);
    LineParams py = line_params('y', my, mz, nmodes, xd, real0);
    LineOut op = line_out(p, 2, -f1, 1.0);
    xterm(op, phi, 1.0, 0.0, -f1);
    LineOut ou = line_out(u, 0, 0.0, 1.0);
    xterm(ou, phi, 0.0, s2, 0.0);
    add_job(py, phi, {op, line_out(v, 1, s2, 1.0), ou});
    int rc = lines_launch(ctx, py);
    if (rc) return rc;
    LineParams pz = line_params('z', my, mz, nmodes, xd, real0);
    add_job(pz, phi, {line_out(p, 2, -f1 / (aspect * aspect), 1.0), line_out(w, 1, s2 / aspect, 1.0)});
    return lines_launch(ctx, pz);
}
}  // namespace duct

extern "C" int ductgpu_update_uvwp_dev(ductgpu_ctx ctx, double *u, double *v, double *w, double *p, const double *phi,
                                       int my, int mz, int nmodes, const double *xalp, double aspect, double akk,
                                       double bkk, double dt, double fnu)
{
    if (!ctx) return DUCTGPU_EARG;
    int rc = check_geom(ctx, "update_uvwp", my, mz, nmodes, true);
    if (!rc) rc = check_ptrs(ctx, "update_uvwp", {u, v, w, p, phi});
    if (rc) return rc;
    cudaSetDevice(ctx->device);
    const double *xd;
    if ((rc = upload_xalp(ctx, xalp, nmodes, &xd))) return rc;
    return update_lines(ctx, u, v, w, p, phi, my, mz, nmodes, xd, aspect, akk, bkk, dt, fnu);
}

namespace duct {
// advection3d on x-cut fields: the x-FFT products (k_advx) and the y / z
// derivatives of the off-diagonal and diagonal products (two line launches).
static int advection_issue(ductgpu_ctx ctx, const double *u, const double *v, const double *w, double *a1, double *a2,
                           double *a3, double *const prod[5], int my, int mz, int M, int mgalx, const double *xd,
                           double aspect, double *stats2, int real0 = 0, unsigned long long *cfl = nullptr,
                           const double *rdyz = nullptr, double hx = 0.0)
{
    AdvParams ap{};
    ap.u = reinterpret_cast<const double2 *>(u);
    ap.v = reinterpret_cast<const double2 *>(v);
    ap.w = reinterpret_cast<const double2 *>(w);
    ap.adv1 = reinterpret_cast<double2 *>(a1);
    ap.adv2 = reinterpret_cast<double2 *>(a2);
    ap.adv3 = reinterpret_cast<double2 *>(a3);
    ap.uv = reinterpret_cast<double2 *>(prod[0]);
    ap.uw = reinterpret_cast<double2 *>(prod[1]);
    ap.vv = reinterpret_cast<double2 *>(prod[2]);
    ap.vw = reinterpret_cast<double2 *>(prod[3]);
    ap.ww = reinterpret_cast<double2 *>(prod[4]);
    ap.stats2 = stats2;
    ap.xalp = xd;
    ap.P = (long long)my * mz;
    ap.M = M;
    ap.cfl = cfl;
    ap.rdyz = rdyz;
    ap.hx = hx;
    ap.my = my;
    ap.mz = mz;
    int rc = advx_launch(ctx, ap, mgalx);
    if (rc) return rc;
    // adv1 += d(uv)/dy + d(uw)/dz; adv2 += d(vv)/dy + d(vw)/dz; adv3 += d(vw)/dy + d(ww)/dz
    LineParams py = line_params('y', my, mz, M, xd, real0);
    add_job(py, prod[0], {line_out(a1, 1, 1.0, 1.0)});
    add_job(py, prod[2], {line_out(a2, 1, 1.0, 1.0)});
    add_job(py, prod[3], {line_out(a3, 1, 1.0, 1.0)});
    if ((rc = lines_launch(ctx, py))) return rc;
    LineParams pz = line_params('z', my, mz, M, xd, real0);
    add_job(pz, prod[1], {line_out(a1, 1, 1.0 / aspect, 1.0)});
    add_job(pz, prod[3], {line_out(a2, 1, 1.0 / aspect, 1.0)});
    add_job(pz, prod[4], {line_out(a3, 1, 1.0 / aspect, 1.0)});
    return lines_launch(ctx, pz);
}

static int mgalx_modes(int mgalx) { return (2 * (mgalx / 3)) / 2; }
}  // namespace duct

extern "C" int ductgpu_advection3d_dev(ductgpu_ctx ctx, const double *u, const double *v, const double *w,
                                       double *adv1, double *adv2, double *adv3, double *work, int my, int mz,
                                       int nmodes, int mgalx, const double *xalp, double aspect, double *stats2)
{
    if (!ctx) return DUCTGPU_EARG;
    int rc = check_geom(ctx, "advection3d", my, mz, nmodes, true);
    if (!rc) rc = check_ptrs(ctx, "advection3d", {u, v, w, adv1, adv2, adv3, work});
    if (rc) return rc;
    if (!advx_supported(mgalx)) return set_error(ctx, DUCTGPU_EARG, "advection3d: mgalx=%d (16, 64, 144, 256)", mgalx);
    if (nmodes != mgalx_modes(mgalx))
        return set_error(ctx, DUCTGPU_EARG, "advection3d: nmodes=%d, mgalx=%d keeps %d modes (mx = 2 (mgalx/3))",
                         nmodes, mgalx, mgalx_modes(mgalx));
    cudaSetDevice(ctx->device);
    const double *xd;
    if ((rc = upload_xalp(ctx, xalp, nmodes, &xd))) return rc;
    const size_t fd = 2ull * my * mz * nmodes;
    double *prod[5] = {work, work + fd, work + 2 * fd, work + 3 * fd, work + 4 * fd};
    return advection_issue(ctx, u, v, w, adv1, adv2, adv3, prod, my, mz, nmodes, mgalx, xd, aspect, stats2);
}

extern "C" int ductgpu_max_3din_dev(ductgpu_ctx ctx, const double *u, int my, int mz, int nmodes, double *divmax)
{
    if (!ctx) return DUCTGPU_EARG;
    int rc = check_geom(ctx, "max_3din", my, mz, nmodes, false);
    if (!rc) rc = check_ptrs(ctx, "max_3din", {u});
    if (rc) return rc;
    if (!divmax) return set_error(ctx, DUCTGPU_EARG, "max_3din: null output");
    cudaSetDevice(ctx->device);
    DnsAux *a = nullptr;
    if ((rc = aux_get(ctx, &a))) return rc;
    DUCT_CUDA(ctx, cudaMemsetAsync(a->out + kStatVals, 0, sizeof(double), ctx->stream));
    {
        LaunchScope ls(ctx, DUCTGPU_K_STATS);
        k_maxabs<<<2 * ctx->num_sms, 256, 0, ctx->stream>>>(reinterpret_cast<const double2 *>(u), my, mz, nmodes,
                                                            a->out + kStatVals);
    }
    DUCT_CUDA(ctx, cudaGetLastError());
    DUCT_CUDA(ctx, cudaMemcpyAsync(divmax, a->out + kStatVals, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    return check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "max_3din");
}

namespace duct {
static int stats_issue(ductgpu_ctx ctx, const double *const f[4], int nf, const double *wcc, const double *wst,
                       double *mean, double *ppb, double *partial, double *out, int *counter, int cap, long long P,
                       int M, double aspect)
{
    StatParams sp{};
    for (int c = 0; c < 4; ++c) sp.f[c] = reinterpret_cast<const double2 *>(f[c]);
    sp.wcc = wcc;
    sp.wst = wst;
    sp.mean = mean;
    sp.ppb = ppb;
    sp.partial = partial;
    sp.P = P;
    sp.M = M;
    sp.nf = nf;
    int blocks = (int)((P + kStatThreads - 1) / kStatThreads);
    if (blocks > kStatBlocksMax) blocks = kStatBlocksMax;
    {
        LaunchScope ls(ctx, DUCTGPU_K_STATS);
        k_stats<<<blocks, kStatThreads, 0, ctx->stream>>>(sp);
    }
    DUCT_CUDA(ctx, cudaGetLastError());
    {
        LaunchScope ls(ctx, DUCTGPU_K_STATS);
        k_stats_finish<<<1, 32, 0, ctx->stream>>>(partial, blocks, 4.0 * aspect, out, counter, cap);
    }
    return check_cuda(ctx, cudaGetLastError(), "k_stats");
}

// The vorticity statistics of one recorded step from omega (om) into the
// accumulators om2 and the history row the step's k_stats_finish opened.
static int omg_issue(ductgpu_ctx ctx, double *const om[3], const double *wcc, double *om2, double *partial,
                     double *out, const int *counter, int cap, int my, int mz, int M, double aspect)
{
    OmgParams op{};
    for (int c = 0; c < 3; ++c) op.f[c] = reinterpret_cast<const double2 *>(om[c]);
    op.wcc = wcc;
    op.om2 = om2;
    op.partial = partial;
    op.P = (long long)my * mz;
    op.M = M;
    op.my = my;
    op.mz = mz;
    int blocks = (int)((op.P + kStatThreads - 1) / kStatThreads);
    if (blocks > kStatBlocksMax) blocks = kStatBlocksMax;
    {
        LaunchScope ls(ctx, DUCTGPU_K_STATS);
        k_omg_stats<<<blocks, kStatThreads, 0, ctx->stream>>>(op);
    }
    DUCT_CUDA(ctx, cudaGetLastError());
    {
        LaunchScope ls(ctx, DUCTGPU_K_STATS);
        k_omg_finish<<<1, 32, 0, ctx->stream>>>(partial, blocks, 4.0 * aspect, out, counter, cap);
    }
    return check_cuda(ctx, cudaGetLastError(), "k_omg_stats");
}
}  // namespace duct

extern "C" int ductgpu_wallstressx_dev(ductgpu_ctx ctx, const double *u, int my, int mz, double aspect,
                                       double *stress4)
{
    if (!ctx) return DUCTGPU_EARG;
    int rc = check_geom(ctx, "wallstressx", my, mz, 1, false);
    if (!rc) rc = check_ptrs(ctx, "wallstressx", {u});
    if (rc) return rc;
    if (!stress4) return set_error(ctx, DUCTGPU_EARG, "wallstressx: null output");
    cudaSetDevice(ctx->device);
    DnsAux *a = nullptr;
    if ((rc = aux_weights(ctx, my, mz, aspect, &a))) return rc;
    const double *f[4] = {u, nullptr, nullptr, nullptr};
    if ((rc = stats_issue(ctx, f, 1, a->wcc, a->wst, nullptr, nullptr, a->partial, a->out, nullptr, 0,
                          (long long)my * mz, 1, aspect)))
        return rc;
    DUCT_CUDA(ctx, cudaMemcpyAsync(stress4, a->out, 4 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    return check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "wallstressx");
}

extern "C" int ductgpu_energy_fou_dev(ductgpu_ctx ctx, const double *u, int my, int mz, int nmodes, double aspect,
                                      double *energy, double *energy2)
{
    if (!ctx) return DUCTGPU_EARG;
    int rc = check_geom(ctx, "energy_fou", my, mz, nmodes, false);
    if (!rc) rc = check_ptrs(ctx, "energy_fou", {u});
    if (rc) return rc;
    if (!energy || !energy2) return set_error(ctx, DUCTGPU_EARG, "energy_fou: null output");
    cudaSetDevice(ctx->device);
    DnsAux *a = nullptr;
    if ((rc = aux_weights(ctx, my, mz, aspect, &a))) return rc;
    const double *f[4] = {u, nullptr, nullptr, nullptr};
    if ((rc = stats_issue(ctx, f, 1, a->wcc, nullptr, nullptr, nullptr, a->partial, a->out, nullptr, 0,
                          (long long)my * mz, nmodes, aspect)))
        return rc;
    double o[kStatVals];
    DUCT_CUDA(ctx, cudaMemcpyAsync(o, a->out, sizeof(o), cudaMemcpyDeviceToHost, ctx->stream));
    DUCT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *energy = o[4];
    *energy2 = o[7];
    return DUCTGPU_OK;
}

extern "C" int ductgpu_statistics_fou_dev(ductgpu_ctx ctx, const double *u, const double *v, const double *w,
                                          const double *p, int my, int mz, int nmodes, double *mean, double *ppb,
                                          double *spec)
{
    if (!ctx) return DUCTGPU_EARG;
    int rc = check_geom(ctx, "statistics_fou", my, mz, nmodes, false);
    if (!rc) rc = check_ptrs(ctx, "statistics_fou", {u, v, w, p});
    if (rc) return rc;
    if (!mean || !ppb || !spec) return set_error(ctx, DUCTGPU_EARG, "statistics_fou: null accumulator");
    if (my < 16 || mz < 16)
        return set_error(ctx, DUCTGPU_EARG, "statistics_fou: my=%d mz=%d (the spectra points need 16 or more)", my, mz);
    cudaSetDevice(ctx->device);
    DnsAux *a = nullptr;
    if ((rc = aux_weights(ctx, my, mz, 1.0, &a))) return rc;
    const double *f[4] = {u, v, w, p};
    if ((rc = stats_issue(ctx, f, 3, a->wcc, nullptr, mean, ppb, a->partial, a->out, nullptr, 0, (long long)my * mz,
                          nmodes, 1.0)))
        return rc;
    {
        LaunchScope ls(ctx, DUCTGPU_K_STATS);
        k_spectra<<<(4 * 7 * nmodes + 127) / 128, 128, 0, ctx->stream>>>(
            reinterpret_cast<const double2 *>(u), reinterpret_cast<const double2 *>(v),
            reinterpret_cast<const double2 *>(w), reinterpret_cast<const double2 *>(p), (long long)my * mz, nmodes,
            my, mz, spec);
    }
    DUCT_CUDA(ctx, cudaGetLastError());
    return check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "statistics_fou");
}

// ---------------------------------------------------------------------------
// The RK3/CN stepper (src/main1.f90:384-723) on device-resident fields.
namespace duct {
// Runge-Kutta coefficients, src/mod.f90:52-55
static const double kAkk[3] = {29.0 / 96.0, -3.0 / 40.0, 1.0 / 6.0};
static const double kBkk[3] = {37.0 / 160.0, 5.0 / 24.0, 1.0 / 6.0};
static const double kGkk[3] = {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};
static const double kRkk[3] = {0.0, -17.0 / 60.0, -5.0 / 12.0};
}  // namespace duct

struct ductgpu_dns_s {
    ductgpu_ctx ctx = nullptr;
    int my = 0, M = 0, mgalx = 0, precision = DUCTGPU_PREC_FP64;
    double alp = 1.0, fnu = 0.0, dt = 0.0, aspect = 1.0, dpdx = 0.0;
    int cmassflow = 1;
    double csum = 0.0;
    long long P = 0;
    size_t fdoubles = 0;         // doubles of a field
    double *mem = nullptr;       // all fields in one allocation
    double *vel[3] = {}, *p = nullptr;
    double *adv[2][3] = {};      // advection terms: substep k writes adv[k % 2], reads adv[(k - 1) % 2]
    double *h[3] = {};
    double *prod[5] = {};        // uv, uw, vv, vw, ww
    double *xalp = nullptr;      // device [M]
    double *lam_d[3] = {}, *lam_n = nullptr;
    // host copies: the Neumann fill finds the singular (kx = 0) planes on the host
    std::vector<double> lamh_d[3], lamh_n;
    // statistics accumulators and per-step history
    double *st_mean = nullptr, *st_prod = nullptr, *st_ppb = nullptr, *st_spec = nullptr;
    double *st_om2 = nullptr;    // [3][P] omx2, omy2, omz2 (statistics_omg2_fou)
    double *hist_om = nullptr;   // per recorded step: kOmgVals vorticity diagnostics
    double *wcc = nullptr, *wst = nullptr, *partial = nullptr;
    double *hist = nullptr;
    int *hist_n = nullptr;
    int hist_cap = 0;
    int nstat = 0;
    double *divmax = nullptr;    // [3], one per substep
    // time-step and slip checks of every step's first substep (order keys):
    // [0] max(|u| hx, |v|/dy, |w|/dz) of the last step, [1] the largest wall
    // velocity of the last step, [2] [0]'s maximum since the last read
    unsigned long long *cfl = nullptr;
    double *rdyz = nullptr;      // [2 my]: 1/dy, 1/dz
    // body force (src/main1.f90 (vi-b): forcings enter h like -grad p, h += (a + b) f)
    double *force = nullptr;     // 3 fields, owned
    bool forced = false;
    // reverse sweep: transposed derivative matrices, checkpoints, cotangents
    double *dmat = nullptr;      // [2][my][my] D1, D2 (real, column-major)
    double *adj = nullptr;       // adjoint work fields
    bool use_graphs = true;
    bool warm[3] = {};
    cudaGraphExec_t graph[3][2] = {};
};

namespace duct {

// The solves read the per-plane lambda from ctx->lam (device) and, for the
// Neumann fill's singular planes, from ctx->lam_host: both point at the
// stepper's own copies for the call.
static int dns_solve(ductgpu_dns d, FieldTask *t, int n, const double *lam, std::vector<double> &lamh)
{
    ductgpu_ctx ctx = d->ctx;
    double *saved = ctx->lam, *saved_h = ctx->lam_host;
    ctx->lam = const_cast<double *>(lam);
    ctx->lam_host = lamh.data();
    int rc;
    if (d->precision == DUCTGPU_PREC_MIXED) rc = solve_mixed(ctx, t, n);
    else rc = solve_fp64_ex(ctx, t, n, d->precision == DUCTGPU_PREC_INT8);
    ctx->lam = saved;
    ctx->lam_host = saved_h;
    return rc;
}

// One substep krk (1..3); stats: gather the statistics of the step (the
// reference does so at krk = 1).
// Work issued between side_fork and side_join runs on the context's first
// side stream, after everything issued before on its stream and concurrent
// with what is issued on it meanwhile.  Without the side stream (first needed
// inside a capture), and while launches are profiled one by one (whose
// event times would overlap), everything stays on one stream.
static bool side_fork(ductgpu_ctx ctx, cudaStream_t *main)
{
    *main = ctx->stream;
    if (ctx->prof_on) return false;
    if (!ctx->side[0]) {
        if (ctx->capturing) return false;
        if (!ctx->side_fork && cudaEventCreateWithFlags(&ctx->side_fork, cudaEventDisableTiming) != cudaSuccess)
            return false;
        if (cudaStreamCreateWithFlags(&ctx->side[0], cudaStreamNonBlocking) != cudaSuccess) return false;
        if (cudaEventCreateWithFlags(&ctx->side_join[0], cudaEventDisableTiming) != cudaSuccess) {
            cudaStreamDestroy(ctx->side[0]);
            ctx->side[0] = nullptr;
            return false;
        }
    }
    if (cudaEventRecord(ctx->side_fork, *main) != cudaSuccess ||
        cudaStreamWaitEvent(ctx->side[0], ctx->side_fork, 0) != cudaSuccess)
        return false;
    return true;
}

static int side_join(ductgpu_ctx ctx, cudaStream_t main)
{
    int rc = check_cuda(ctx, cudaEventRecord(ctx->side_join[0], ctx->side[0]), "side stream join");
    int rc2 = check_cuda(ctx, cudaStreamWaitEvent(main, ctx->side_join[0], 0), "side stream join");
    return rc ? rc : rc2;
}

static int dns_issue(ductgpu_dns d, int krk, bool stats)
{
    ductgpu_ctx ctx = d->ctx;
    const int k = krk - 1, my = d->my, M = d->M;
    const double a = kAkk[k], b = kBkk[k], gm = kGkk[k], rho = kRkk[k];
    const double nu = d->fnu, dt = d->dt, asp = d->aspect;
    double **an = d->adv[krk % 2], **ao = d->adv[(krk - 1) % 2];
    double *u = d->vel[0], *v = d->vel[1], *w = d->vel[2], *p = d->p;
    const double *xd = d->xalp;
    int rc = DUCTGPU_OK;
    // (ii) adv(u^{k-1}); statistics_fou2 of the products with the statistics.
    // The statistics kernels only read u, v, w, p: on the side stream,
    // concurrent with the advection
    cudaStream_t mainst = ctx->stream;
    const bool fork_stats = stats && side_fork(ctx, &mainst);
    if (stats) {
        if (fork_stats) ctx->stream = ctx->side[0];
        // wallstressx, energy_fou (u, v, w), statistics_fou (u, v, w, p)
        const double *f[4] = {u, v, w, p};
        rc = stats_issue(ctx, f, 3, d->wcc, d->wst, d->st_mean, d->st_ppb, d->partial, d->hist, d->hist_n,
                         d->hist_cap, d->P, M, asp);
        if (!rc) {
            LaunchScope ls(ctx, DUCTGPU_K_STATS);
            k_spectra<<<(4 * 7 * M + 127) / 128, 128, 0, ctx->stream>>>(
                reinterpret_cast<const double2 *>(u), reinterpret_cast<const double2 *>(v),
                reinterpret_cast<const double2 *>(w), reinterpret_cast<const double2 *>(p), d->P, M, my, my,
                d->st_spec);
        }
        if (!rc) rc = check_cuda(ctx, cudaGetLastError(), "k_spectra");
        ctx->stream = mainst;
    }
    if (!rc && krk == 1) rc = check_cuda(ctx, cudaMemsetAsync(d->cfl, 0, 2 * sizeof(unsigned long long), mainst),
                                          "dns: cfl reset");
    if (!rc)
        rc = advection_issue(ctx, u, v, w, an[0], an[1], an[2], d->prod, my, my, M, d->mgalx, xd, asp,
                             stats ? d->st_prod : nullptr, 1, krk == 1 ? d->cfl : nullptr, d->rdyz,
                             d->alp * d->mgalx / (2.0 * kPi));
    if (fork_stats) {
        const int rj = side_join(ctx, mainst);
        if (!rc) rc = rj;
    }
    if (rc) return rc;
    // (i), (iii)-(v), the x-part of (vi), (vi-b): along y,
    //   h = -rho adv_old - gamma adv + u/dt + a nu lap_x,y(u) [- (a+b) (i kx p + dpdx)]
    {
        LineParams py = line_params('y', my, my, M, xd, 1);
        for (int c = 0; c < 3; ++c) {
            LineOut o = line_out(d->h[c], 2, nu * a, 0.0);
            xterm(o, d->vel[c], 1.0 / dt, 0.0, nu * a);
            xterm(o, an[c], -gm, 0.0, 0.0);
            if (krk > 1) xterm(o, ao[c], -rho, 0.0, 0.0);
            if (c == 0) {
                xterm(o, p, 0.0, -(a + b), 0.0);
                if (!d->cmassflow) o.m0 = -(a + b) * d->dpdx;
            }
            if (d->forced) xterm(o, d->force + c * d->fdoubles, a + b, 0.0, 0.0);
            add_job(py, d->vel[c], {o});
        }
        if (stats) {
            // the vorticity diagnostics of src/main1.f90:453-466 from the
            // same staged lines, into the product fields (free once the
            // advection is done): omega_z = i kx v - du/dy, omega_x = dw/dy
            LineOut oz = line_out(d->prod[2], 1, -1.0, 0.0);
            xterm(oz, v, 0.0, 1.0, 0.0);
            add_out(py, 0, oz);
            add_out(py, 2, line_out(d->prod[0], 1, 1.0, 0.0));
        }
        if ((rc = lines_launch(ctx, py))) return rc;
    }
    // (vi) y and z parts of -(a+b) grad p: different outputs, the z part on
    // the side stream concurrent with the y part
    {
        LineParams py = line_params('y', my, my, M, xd, 1);
        add_job(py, p, {line_out(d->h[1], 1, -(a + b), 1.0)});
        LineParams pz = line_params('z', my, my, M, xd, 1);
        add_job(pz, p, {line_out(d->h[2], 1, -(a + b) / asp, 1.0)});
        const bool fork = side_fork(ctx, &mainst);
        rc = lines_launch(ctx, py);
        if (!rc) {
            if (fork) ctx->stream = ctx->side[0];
            rc = lines_launch(ctx, pz);
            ctx->stream = mainst;
        }
        if (fork) {
            const int rj = side_join(ctx, mainst);
            if (!rc) rc = rj;
        }
        if (rc) return rc;
    }
    // (iv) z part of the laplacian, then (vii) h *= -1/(nu beta)
    {
        LineParams pz = line_params('z', my, my, M, xd, 1);
        for (int c = 0; c < 3; ++c)
            add_job(pz, d->vel[c], {line_out(d->h[c], 2, nu * a / (asp * asp), 1.0, -1.0 / (nu * b))});
        if (stats) {
            // omega_x -= dv/dz, omega_y = du/dz - i kx w
            add_out(pz, 1, line_out(d->prod[0], 1, -1.0 / asp, 1.0));
            LineOut oy = line_out(d->prod[1], 1, 1.0 / asp, 0.0);
            xterm(oy, w, 0.0, -1.0, 0.0);
            add_out(pz, 0, oy);
        }
        if ((rc = lines_launch(ctx, pz))) return rc;
    }
    // the vorticity statistics on the side stream, concurrent with the
    // predictor solves (they read only the product fields)
    const bool fork_omg = stats && side_fork(ctx, &mainst);
    if (stats) {
        if (fork_omg) ctx->stream = ctx->side[0];
        rc = omg_issue(ctx, d->prod, d->wcc, d->st_om2, d->partial, d->hist_om, d->hist_n, d->hist_cap, my, my, M,
                       asp);
        ctx->stream = mainst;
        if (rc) {
            if (fork_omg) side_join(ctx, mainst);
            return rc;
        }
    }
    // (viii) predictor: helm3d 'd', helco = 1/(beta nu dt)
    {
        FieldTask t[3];
        for (int c = 0; c < 3; ++c) {
            t[c].rhs = d->h[c];
            t[c].sol = d->vel[c];
            t[c].nmodes = M;
            t[c].mode0 = 1;
            t[c].bound = 'd';
            t[c].plane0 = c * M;
            t[c].refine = 1;
        }
        rc = dns_solve(d, t, 3, d->lam_d[k], d->lamh_d[k]);
        if (fork_omg) {
            const int rj = side_join(ctx, mainst);
            if (!rc) rc = rj;
        }
        if (rc) return rc;
    }
    // (ix) rhs of the pseudo-pressure: div(u) / ((a+b) dt) -> h1
    const double sdiv = 1.0 / ((a + b) * dt);
    {
        LineParams py = line_params('y', my, my, M, xd, 1);
        LineOut o = line_out(d->h[0], 1, sdiv, 0.0);
        xterm(o, u, 0.0, sdiv, 0.0);
        add_job(py, v, {o});
        if ((rc = lines_launch(ctx, py))) return rc;
        LineParams pz = line_params('z', my, my, M, xd, 1);
        add_job(pz, w, {line_out(d->h[0], 1, sdiv / asp, 1.0)});
        if ((rc = lines_launch(ctx, pz))) return rc;
    }
    // (x) Poisson 'n' -> phi in h2
    {
        FieldTask t;
        t.rhs = d->h[0];
        t.sol = d->h[1];
        t.nmodes = M;
        t.mode0 = 1;
        t.bound = 'n';
        t.plane0 = 0;
        t.refine = ctx->refine_steps;
        if ((rc = dns_solve(d, &t, 1, d->lam_n, d->lamh_n))) return rc;
    }
    // (xi) update u, v, w, p
    if ((rc = update_lines(ctx, u, v, w, p, d->h[1], my, my, M, xd, asp, a, b, dt, nu, 1))) return rc;
    if (d->cmassflow) {
        double cs = d->csum;
        if ((rc = ductgpu_impose_mass_flow_dev(ctx, &cs, krk, u, 1))) return rc;
    }
    // divergence check: max |div u| over the interior (max_3din) -> divmax[k]
    DUCT_CUDA(ctx, cudaMemsetAsync(d->divmax + k, 0, sizeof(double), ctx->stream));
    {
        LineParams py = line_params('y', my, my, M, xd, 1);
        LineOut o = line_out(d->h[2], 1, 1.0, 0.0);
        xterm(o, u, 0.0, 1.0, 0.0);
        add_job(py, v, {o});
        if ((rc = lines_launch(ctx, py))) return rc;
        LineParams pz = line_params('z', my, my, M, xd, 1);
        LineOut oz = line_out(d->h[2], 1, 1.0 / asp, 1.0);
        oz.maxabs = d->divmax + k;
        add_job(pz, w, {oz});
        if ((rc = lines_launch(ctx, pz))) return rc;
    }
    return DUCTGPU_OK;
}

static void dns_free(ductgpu_dns d)
{
    if (!d) return;
    if (d->ctx) {
        cudaSetDevice(d->ctx->device);
        cudaStreamSynchronize(d->ctx->stream);
    }
    for (int k = 0; k < 3; ++k)
        for (int s = 0; s < 2; ++s)
            if (d->graph[k][s]) cudaGraphExecDestroy(d->graph[k][s]);
    cudaFree(d->mem);
    cudaFree(d->xalp);
    for (int k = 0; k < 3; ++k) cudaFree(d->lam_d[k]);
    cudaFree(d->lam_n);
    cudaFree(d->st_mean);
    cudaFree(d->wcc);
    cudaFree(d->hist);
    cudaFree(d->hist_om);
    cudaFree(d->hist_n);
    cudaFree(d->divmax);
    cudaFree(d->cfl);
    cudaFree(d->rdyz);
    cudaFree(d->force);
    cudaFree(d->dmat);
    cudaFree(d->adj);
    delete d;
}

}  // namespace duct

extern "C" int ductgpu_dns_create(ductgpu_ctx ctx, int mgalx, double alp, double fnu, double dt, double aspect,
                                  int cmassflow, double dpdx, int precision, int hist_cap, ductgpu_dns *out)
{
    if (!ctx || !out) return DUCTGPU_EARG;
    *out = nullptr;
    if (!ctx->ready) return set_error(ctx, DUCTGPU_ESTATE, "dns: operators not set up (call ductgpu_pseudomat)");
    const int my = ctx->my;
    if (ctx->mz != my) return set_error(ctx, DUCTGPU_EARG, "dns: square duct only (my=%d mz=%d)", my, ctx->mz);
    int rc = check_geom(ctx, "dns", my, my, 1, true);
    if (rc) return rc;
    if (!advx_supported(mgalx)) return set_error(ctx, DUCTGPU_EARG, "dns: mgalx=%d (16, 64, 144, 256)", mgalx);
    if (!(fnu > 0.0) || !(dt > 0.0) || !(aspect > 0.0))
        return set_error(ctx, DUCTGPU_EARG, "dns: nu=%g dt=%g aspect=%g", fnu, dt, aspect);
    if (precision != DUCTGPU_PREC_FP64 && precision != DUCTGPU_PREC_INT8 && precision != DUCTGPU_PREC_MIXED)
        return set_error(ctx, DUCTGPU_EARG, "dns: precision %d", precision);
    if (precision == DUCTGPU_PREC_INT8 && my - 2 > 127)
        return set_error(ctx, DUCTGPU_EARG, "dns: int8-emulated solve needs my <= 129 (my=%d)", my);
    if (hist_cap < 0) hist_cap = 0;
    cudaSetDevice(ctx->device);
    ductgpu_dns d = new (std::nothrow) ductgpu_dns_s();
    if (!d) return set_error(ctx, DUCTGPU_EALLOC, "dns: out of host memory");
    d->ctx = ctx;
    d->my = my;
    d->mgalx = mgalx;
    d->M = mgalx_modes(mgalx);
    d->alp = alp;
    d->fnu = fnu;
    d->dt = dt;
    d->aspect = aspect;
    d->cmassflow = cmassflow ? 1 : 0;
    d->dpdx = dpdx;
    d->precision = precision;
    d->P = (long long)my * my;
    d->fdoubles = 2ull * d->P * d->M;
    const int M = d->M;
    auto fail = [&](int code) {
        dns_free(d);
        return code;
    };
    // fields: u v w p, adv 2x3, h 3, prod 5 = 18
    if (cudaMalloc(&d->mem, sizeof(double) * d->fdoubles * 18) != cudaSuccess) {
        cudaGetLastError();
        return fail(set_error(ctx, DUCTGPU_EALLOC, "dns: %.1f MB of fields", 18.0 * d->fdoubles * 8 / 1e6));
    }
    double *f = d->mem;
    for (int c = 0; c < 3; ++c) d->vel[c] = f, f += d->fdoubles;
    d->p = f, f += d->fdoubles;
    for (int s = 0; s < 2; ++s)
        for (int c = 0; c < 3; ++c) d->adv[s][c] = f, f += d->fdoubles;
    for (int c = 0; c < 3; ++c) d->h[c] = f, f += d->fdoubles;
    for (int c = 0; c < 5; ++c) d->prod[c] = f, f += d->fdoubles;
    if (cudaMemsetAsync(d->mem, 0, sizeof(double) * d->fdoubles * 18, ctx->stream) != cudaSuccess)
        return fail(check_cuda(ctx, cudaGetLastError(), "dns: memset"));
    // wavenumbers and the lambda of every solve (per RK index)
    std::vector<double> xa(M), lam(3 * M);
    for (int i = 0; i < M; ++i) xa[i] = alp * i;
    if (cudaMalloc(&d->xalp, sizeof(double) * M) != cudaSuccess ||
        cudaMemcpy(d->xalp, xa.data(), sizeof(double) * M, cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(check_cuda(ctx, cudaGetLastError(), "dns: xalp"));
    for (int k = 0; k < 3; ++k) {
        const double helco = 1.0 / (kBkk[k] * fnu * dt);
        for (int c = 0; c < 3; ++c)
            for (int i = 0; i < M; ++i) lam[c * M + i] = helco + xa[i] * xa[i];
        d->lamh_d[k] = lam;
        if (cudaMalloc(&d->lam_d[k], sizeof(double) * 3 * M) != cudaSuccess ||
            cudaMemcpy(d->lam_d[k], lam.data(), sizeof(double) * 3 * M, cudaMemcpyHostToDevice) != cudaSuccess)
            return fail(check_cuda(ctx, cudaGetLastError(), "dns: lambda"));
    }
    for (int i = 0; i < M; ++i) lam[i] = xa[i] * xa[i];
    d->lamh_n.assign(lam.begin(), lam.begin() + M);
    if (cudaMalloc(&d->lam_n, sizeof(double) * M) != cudaSuccess ||
        cudaMemcpy(d->lam_n, lam.data(), sizeof(double) * M, cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(check_cuda(ctx, cudaGetLastError(), "dns: lambda"));
    // statistics: mean [4][P], prod [6][P], ppb [P], spec [4][7][M], om2 [3][P] in one block; weights
    const size_t nst = 4 * d->P + 6 * d->P + d->P + 4 * 7 * (size_t)M + 3 * d->P;
    if (cudaMalloc(&d->st_mean, sizeof(double) * nst) != cudaSuccess)
        return fail(check_cuda(ctx, cudaGetLastError(), "dns: statistics"));
    d->st_prod = d->st_mean + 4 * d->P;
    d->st_ppb = d->st_prod + 6 * d->P;
    d->st_spec = d->st_ppb + d->P;
    d->st_om2 = d->st_spec + 4 * 7 * (size_t)M;
    cudaMemset(d->st_mean, 0, sizeof(double) * nst);
    {
        std::vector<double> wcc, wst;
        make_weights(my, my, aspect, wcc, wst);
        // the partial sums of the statistics kernel, and one row of scratch results after them
        const size_t nw = wcc.size() + wst.size() + (size_t)(kStatBlocksMax + 1) * (kOmgVals > kStatVals ? kOmgVals : kStatVals);
        if (cudaMalloc(&d->wcc, sizeof(double) * nw) != cudaSuccess)
            return fail(check_cuda(ctx, cudaGetLastError(), "dns: weights"));
        d->wst = d->wcc + wcc.size();
        d->partial = d->wst + wst.size();
        cudaMemcpy(d->wcc, wcc.data(), sizeof(double) * wcc.size(), cudaMemcpyHostToDevice);
        cudaMemcpy(d->wst, wst.data(), sizeof(double) * wst.size(), cudaMemcpyHostToDevice);
    }
    d->hist_cap = hist_cap;
    if (cudaMalloc(&d->hist, sizeof(double) * kStatVals * (hist_cap > 0 ? hist_cap : 1)) != cudaSuccess ||
        cudaMalloc(&d->hist_om, sizeof(double) * kOmgVals * (hist_cap > 0 ? hist_cap : 1)) != cudaSuccess ||
        cudaMalloc(&d->hist_n, sizeof(int)) != cudaSuccess || cudaMemset(d->hist_n, 0, sizeof(int)) != cudaSuccess ||
        cudaMalloc(&d->divmax, sizeof(double) * 3) != cudaSuccess ||
        cudaMalloc(&d->cfl, sizeof(unsigned long long) * 3) != cudaSuccess ||
        cudaMemset(d->cfl, 0, sizeof(unsigned long long) * 3) != cudaSuccess)
        return fail(check_cuda(ctx, cudaGetLastError(), "dns: history"));
    {
        // 1/dy, 1/dz of determine_step (the mesh sizes of src/ininewc.f90:102-112)
        std::vector<double> dy, dz, r(2 * (size_t)my);
        mesh_sizes(my, 1.0, dy);
        mesh_sizes(my, aspect, dz);
        for (int j = 0; j < my; ++j) {
            r[j] = 1.0 / dy[j];
            r[my + j] = 1.0 / dz[j];
        }
        if (cudaMalloc(&d->rdyz, sizeof(double) * r.size()) != cudaSuccess ||
            cudaMemcpy(d->rdyz, r.data(), sizeof(double) * r.size(), cudaMemcpyHostToDevice) != cudaSuccess)
            return fail(check_cuda(ctx, cudaGetLastError(), "dns: mesh sizes"));
    }
    // the flow-rate forcing of CMASSFLOW: premassfu / premassf with alphak = beta_k
    if (d->cmassflow && (rc = ductgpu_precomp_mass_flow(ctx, dt, kBkk, 3, fnu, aspect, nullptr, nullptr)))
        return fail(rc);
    if ((rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "dns_create"))) return fail(rc);
    *out = d;
    return DUCTGPU_OK;
}

extern "C" int ductgpu_dns_destroy(ductgpu_dns d)
{
    if (!d) return DUCTGPU_EARG;
    dns_free(d);
    return DUCTGPU_OK;
}

// which: 0 u, 1 v, 2 w, 3 p
extern "C" int ductgpu_dns_field(ductgpu_dns d, int which, double **dev)
{
    if (!d || !dev || which < 0 || which > 3) return DUCTGPU_EARG;
    *dev = which < 3 ? d->vel[which] : d->p;
    return DUCTGPU_OK;
}

// After the fields were replaced: with CMASSFLOW the flow rate to hold is
// `csum` when given (> 0), else that of the new u, and the captured
// substeps (which bake it in) are re-captured.  Synchronises.
static int dns_fields_changed(ductgpu_dns d, double csum = 0.0)
{
    ductgpu_ctx ctx = d->ctx;
    if (d->cmassflow) {
        if (csum > 0.0) {
            d->csum = csum;
        } else {
            int rc = ductgpu_impose_mass_flow_dev(ctx, &d->csum, 1, d->vel[0], 0);
            if (rc) return rc;
        }
        for (int k = 0; k < 3; ++k)
            for (int s = 0; s < 2; ++s)
                if (d->graph[k][s]) {
                    cudaGraphExecDestroy(d->graph[k][s]);
                    d->graph[k][s] = nullptr;
                }
    }
    return check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "dns_set_fields");
}

extern "C" int ductgpu_dns_set_fields(ductgpu_dns d, const double *u, const double *v, const double *w,
                                      const double *p)
{
    if (!d) return DUCTGPU_EARG;
    ductgpu_ctx ctx = d->ctx;
    if (!u || !v || !w || !p) return set_error(ctx, DUCTGPU_EARG, "dns_set_fields: null field");
    cudaSetDevice(ctx->device);
    const double *src[4] = {u, v, w, p};
    double *dst[4] = {d->vel[0], d->vel[1], d->vel[2], d->p};
    for (int c = 0; c < 4; ++c)
        DUCT_CUDA(ctx, cudaMemcpyAsync(dst[c], src[c], sizeof(double) * d->fdoubles, cudaMemcpyDefault, ctx->stream));
    return dns_fields_changed(d);
}

// The stepper's state as a uvwp_NNNN.h5 file (src/main1.f90:735-752 with
// save_4fields_fou_hdf5) and back (the irestart read).
extern "C" int ductgpu_dns_save_hdf5(ductgpu_dns d, const char *filename, double time, double cfl, double slip)
{
    if (!d) return DUCTGPU_EARG;
    ductgpu_ctx ctx = d->ctx;
    cudaSetDevice(ctx->device);
    ductgpu_h5_header h{};
    h.nparams = 7;
    h.numerop = 1;
    h.mgalx = d->mgalx;
    h.my = h.mz = d->my;
    h.mx1 = d->M - 1;
    h.alp = d->alp;
    h.aspect = d->aspect;
    h.time = time;
    h.fnu = d->fnu;
    h.cfl = cfl;
    h.dtfixed = d->dt;
    h.cmassflow = d->cmassflow ? d->csum : 0.0;
    h.slip = slip;
    double dv[3];
    unsigned long long key[2];
    DUCT_CUDA(ctx, cudaMemcpyAsync(dv, d->divmax, sizeof dv, cudaMemcpyDeviceToHost, ctx->stream));
    DUCT_CUDA(ctx, cudaMemcpyAsync(key, d->cfl, sizeof key, cudaMemcpyDeviceToHost, ctx->stream));
    DUCT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    h.divergence = dv[2];
    // slip NaN: the wall slip slip_velocity_3d measured at the last step
    if (slip != slip) h.slip = key[1] ? order_key_value(key[1]) : 0.0;
    return ductgpu_save_4fields_fou_hdf5_dev(ctx, filename, d->vel[0], d->vel[1], d->vel[2], d->p, &h);
}

extern "C" int ductgpu_dns_write_statistics_hdf5(ductgpu_dns d, const char *filename, double time, double timef)
{
    if (!d) return DUCTGPU_EARG;
    ductgpu_ctx ctx = d->ctx;
    if (!filename) return set_error(ctx, DUCTGPU_EARG, "write_statistics_hdf5: NULL file name");
    cudaSetDevice(ctx->device);
    DUCT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    const size_t P = d->P, M = d->M;
    // mean, prod, ppb, spec, om2 are one contiguous block on the device
    const size_t n = 4 * P + 6 * P + P + 4 * 7 * M + 3 * P;
    std::vector<double> h(n);
    DUCT_CUDA(ctx, cudaMemcpy(h.data(), d->st_mean, sizeof(double) * n, cudaMemcpyDeviceToHost));
    H5Stats st;
    st.mgalx = d->mgalx;
    st.my = st.mz = d->my;
    st.nmodes = d->M;
    st.nstat = d->nstat;
    st.timef = timef;
    st.time = time;
    st.fnu = d->fnu;
    st.alp = d->alp;
    st.aspect = d->aspect;
    st.mean = h.data();
    st.prod = st.mean + 4 * P;
    st.ppb = st.prod + 6 * P;
    st.spec = st.ppb + P;
    st.om2 = st.spec + 4 * 7 * M;
    return h5_write_statistics(ctx, filename, st);
}

extern "C" int ductgpu_dns_load_hdf5(ductgpu_dns d, const char *filename, double *time)
{
    if (!d) return DUCTGPU_EARG;
    ductgpu_ctx ctx = d->ctx;
    cudaSetDevice(ctx->device);
    ductgpu_h5_header h{};
    int rc = ductgpu_read_4fields_fou_hdf5_dev(ctx, filename, d->vel[0], d->vel[1], d->vel[2], d->p, d->my, d->my,
                                              d->M, &h);
    if (rc) return rc;
    if (time) *time = h.time;
    // the run's constant flow rate travels in the file (writeheader_hdf5's
    // cmassflow), so a restart holds exactly the saved run's
    return dns_fields_changed(d, h.cmassflow);
}

extern "C" int ductgpu_dns_get_fields(ductgpu_dns d, double *u, double *v, double *w, double *p)
{
    if (!d) return DUCTGPU_EARG;
    ductgpu_ctx ctx = d->ctx;
    cudaSetDevice(ctx->device);
    double *dst[4] = {u, v, w, p};
    const double *src[4] = {d->vel[0], d->vel[1], d->vel[2], d->p};
    for (int c = 0; c < 4; ++c)
        if (dst[c])
            DUCT_CUDA(ctx, cudaMemcpyAsync(dst[c], src[c], sizeof(double) * d->fdoubles, cudaMemcpyDefault, ctx->stream));
    return check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "dns_get_fields");
}

extern "C" int ductgpu_dns_set_graphs(ductgpu_dns d, int on)
{
    if (!d) return DUCTGPU_EARG;
    d->use_graphs = on != 0;
    return DUCTGPU_OK;
}

namespace duct {
static int dns_run_substep(ductgpu_dns d, int krk, bool stats)
{
    ductgpu_ctx ctx = d->ctx;
    const int k = krk - 1, s = stats ? 1 : 0;
    if (!d->use_graphs || ctx->prof_on) return dns_issue(d, krk, stats);
    if (!d->graph[k][s]) {
        // the first run of each RK index is uncaptured: it sizes the
        // workspaces and builds the twiddle tables; later runs capture
        // the substep once (without executing it) and replay the graph
        if (!d->warm[k]) {
            int rc = dns_issue(d, krk, stats);
            if (rc) return rc;
            DUCT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            d->warm[k] = true;
            return DUCTGPU_OK;
        }
        ctx->capturing = true;
        cudaGraph_t g = nullptr;
        int rc = DUCTGPU_OK;
        cudaError_t e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            rc = dns_issue(d, krk, stats);
            cudaError_t e2 = cudaStreamEndCapture(ctx->stream, &g);
            if (!rc && e2 != cudaSuccess) rc = check_cuda(ctx, e2, "cudaStreamEndCapture");
        } else {
            rc = check_cuda(ctx, e, "cudaStreamBeginCapture");
        }
        ctx->capturing = false;
        if (!rc) rc = check_cuda(ctx, cudaGraphInstantiate(&d->graph[k][s], g, 0), "cudaGraphInstantiate");
        if (g) cudaGraphDestroy(g);
        if (rc) return rc;
    }
    ctx->launches += 1;
    return check_cuda(ctx, cudaGraphLaunch(d->graph[k][s], ctx->stream), "cudaGraphLaunch");
}
}  // namespace duct

extern "C" int ductgpu_dns_substep(ductgpu_dns d, int krk, int stats)
{
    if (!d) return DUCTGPU_EARG;
    if (krk < 1 || krk > 3) return set_error(d->ctx, DUCTGPU_EARG, "dns_substep: krk=%d (1..3)", krk);
    cudaSetDevice(d->ctx->device);
    const bool st = stats && krk == 1;
    int rc = dns_run_substep(d, krk, st);
    if (!rc && st) d->nstat += 1;
    return rc;
}

// nsteps full RK3 steps; statistics gathered at every stats_every-th step
// (0: none), counting from the first step of this call.  Asynchronous.
extern "C" int ductgpu_dns_steps(ductgpu_dns d, int nsteps, int stats_every)
{
    if (!d) return DUCTGPU_EARG;
    if (nsteps < 0) return set_error(d->ctx, DUCTGPU_EARG, "dns_steps: nsteps=%d", nsteps);
    cudaSetDevice(d->ctx->device);
    for (int s = 0; s < nsteps; ++s) {
        const int st = (stats_every > 0 && s % stats_every == 0) ? 1 : 0;
        for (int krk = 1; krk <= 3; ++krk) {
            int rc = ductgpu_dns_substep(d, krk, st);
            if (rc) return rc;
        }
    }
    return DUCTGPU_OK;
}

// Accumulated statistics (device -> host; null outputs skipped): mean
// [4][my][my] (u, v, w, p mode-0 real parts, summed over the recorded
// steps), prod [6][my][my] (uu, vv, ww, uv, uw, vw), ppb [my][my], spec
// [4][7][M]; hist [nrows][10] rows of stress4[4], energy[3], energy2[3];
// nstat recorded steps, nhist rows written (at most the capacity given to
// ductgpu_dns_create).  divmax3: max |div u| after each substep of the last
// step.  Synchronises.
extern "C" int ductgpu_dns_statistics(ductgpu_dns d, double *mean, double *prod, double *ppb, double *spec,
                                      double *hist, int *nstat, int *nhist, double *divmax3)
{
    if (!d) return DUCTGPU_EARG;
    ductgpu_ctx ctx = d->ctx;
    cudaSetDevice(ctx->device);
    DUCT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    const size_t P = d->P;
    if (mean) DUCT_CUDA(ctx, cudaMemcpy(mean, d->st_mean, sizeof(double) * 4 * P, cudaMemcpyDeviceToHost));
    if (prod) DUCT_CUDA(ctx, cudaMemcpy(prod, d->st_prod, sizeof(double) * 6 * P, cudaMemcpyDeviceToHost));
    if (ppb) DUCT_CUDA(ctx, cudaMemcpy(ppb, d->st_ppb, sizeof(double) * P, cudaMemcpyDeviceToHost));
    if (spec) DUCT_CUDA(ctx, cudaMemcpy(spec, d->st_spec, sizeof(double) * 4 * 7 * d->M, cudaMemcpyDeviceToHost));
    int nh = 0;
    DUCT_CUDA(ctx, cudaMemcpy(&nh, d->hist_n, sizeof(int), cudaMemcpyDeviceToHost));
    if (nh > d->hist_cap) nh = d->hist_cap;
    if (hist && nh > 0) DUCT_CUDA(ctx, cudaMemcpy(hist, d->hist, sizeof(double) * kStatVals * nh, cudaMemcpyDeviceToHost));
    if (nstat) *nstat = d->nstat;
    if (nhist) *nhist = nh;
    if (divmax3) DUCT_CUDA(ctx, cudaMemcpy(divmax3, d->divmax, sizeof(double) * 3, cudaMemcpyDeviceToHost));
    return DUCTGPU_OK;
}

extern "C" int ductgpu_dns_cfl(ductgpu_dns d, double *cfl, double *slip, double *cfl_max)
{
    if (!d) return DUCTGPU_EARG;
    ductgpu_ctx ctx = d->ctx;
    cudaSetDevice(ctx->device);
    DUCT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    unsigned long long k[3];
    DUCT_CUDA(ctx, cudaMemcpy(k, d->cfl, sizeof k, cudaMemcpyDeviceToHost));
    DUCT_CUDA(ctx, cudaMemset(d->cfl + 2, 0, sizeof(unsigned long long)));
    // before any step the keys are 0: nothing measured
    if (cfl) *cfl = k[0] ? d->dt * order_key_value(k[0]) : 0.0;
    if (slip) *slip = k[1] ? order_key_value(k[1]) : 0.0;
    if (cfl_max) *cfl_max = k[2] ? d->dt * order_key_value(k[2]) : 0.0;
    return DUCTGPU_OK;
}

extern "C" int ductgpu_dns_statistics_omg(ductgpu_dns d, double *om2, double *hist, int *nhist)
{
    if (!d) return DUCTGPU_EARG;
    ductgpu_ctx ctx = d->ctx;
    cudaSetDevice(ctx->device);
    DUCT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (om2) DUCT_CUDA(ctx, cudaMemcpy(om2, d->st_om2, sizeof(double) * 3 * d->P, cudaMemcpyDeviceToHost));
    int nh = 0;
    DUCT_CUDA(ctx, cudaMemcpy(&nh, d->hist_n, sizeof(int), cudaMemcpyDeviceToHost));
    if (nh > d->hist_cap) nh = d->hist_cap;
    if (hist && nh > 0)
        DUCT_CUDA(ctx, cudaMemcpy(hist, d->hist_om, sizeof(double) * kOmgVals * nh, cudaMemcpyDeviceToHost));
    if (nhist) *nhist = nh;
    return DUCTGPU_OK;
}

// ---------------------------------------------------------------------------
// Body force and the gradient of the four-wall shear functional through one
// RK3/CN step by reverse mode (the discrete adjoint of the step above).
//
// Forward step: three substeps S_k mapping (u, v, w, p, A_{k-1}) to
// (u', v', w', p', A_k), linear in everything but the advection A_k =
// adv(u, v, w).  J = sum over the four walls of wallstressx(u) after the
// step, a linear functional of the mode-0 real part of u.  The reverse
// sweep applies, substep by substep from the last, the transpose of every
// linear map in the coefficient inner product <a, b> = Re sum conj(a) b:
//   mass flow   u += pu (csum - Q u)/pf         ->  u_ -= Q^T <pu, u_> / pf
//   update      p' = p + phi - f1 Lap phi, u' = u* + s2 grad phi
//   pressure    phi = S_n(div u* / ((a+b) dt))  ->  the adjoint Neumann solve
//   predictor   u* = S_d(sigma h)               ->  the adjoint Dirichlet solve
//   rhs         h = a nu Lap u + u/dt - gamma A_k - rho A_{k-1} - (a+b) grad p + (a+b) f
//   advection   A_i = sum_j d_j P(u_i u_j)      ->  linearised at the substep's
//               entry velocities (kept as in-memory checkpoints):
//               u_m += sum_j W Spec(u_j Phys(W^-1 (Q_mj + Q_jm))), Q_ij = d_j^T A_i,
//               W = diag(1, 2, 2, ...) the weights of the Hermitian modes.
// Derivative transposes: i kx -> -i kx along x; along y and z the real
// collocation matrices D1, D2 of the line kernel (built by applying it to
// the unit vectors) transposed.
namespace duct {

static void dns_drop_graphs(ductgpu_dns d)
{
    for (int k = 0; k < 3; ++k)
        for (int s = 0; s < 2; ++s)
            if (d->graph[k][s]) {
                cudaGraphExecDestroy(d->graph[k][s]);
                d->graph[k][s] = nullptr;
            }
}

// out = beta out + fac A^T in along lines (A nn x nn column-major real);
// mode 0 keeps a zero imaginary part with real0 (the forward derivative
// terms of a real mode-0 line are real).
__global__ void k_lines_mat_t(const double *A, int nn, const double2 *in, double2 *out, int my, int mz, int M,
                              int ydir, double fac, double beta, int real0)
{
    const long long P = (long long)my * mz, total = P * M;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long mode = t / P, q = t - mode * P;
        const int y = (int)(q % my), z = (int)(q / my);
        const int j = ydir ? y : z;
        const double2 *line = in + mode * P + (ydir ? (long long)my * z : (long long)y);
        const long long es = ydir ? 1 : my;
        const double *col = A + (long long)nn * j;
        double ax = 0.0, ay = 0.0;
        for (int k = 0; k < nn; ++k) {
            const double2 v = line[k * es];
            ax += col[k] * v.x;
            ay += col[k] * v.y;
        }
        if (real0 && mode == 0) ay = 0.0;
        double2 o = make_double2(fac * ax, fac * ay);
        if (beta != 0.0) {
            const double2 w = out[t];
            o.x += beta * w.x;
            o.y += beta * w.y;
        }
        out[t] = o;
    }
}

__global__ void k_real_part(const double2 *in, double *out, long long n)
{
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        out[t] = in[t].x;
}

__global__ void k_unit_plane(double2 *e, int nn)
{
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)nn * nn;
         t += (long long)gridDim.x * blockDim.x)
        e[t] = make_double2((t % nn) == (t / nn) ? 1.0 : 0.0, 0.0);
}

// dJ/du: the mode-0 real part gets the sum of the four wall-stress weights.
__global__ void k_seed_wall(double2 *ub, const double *wst, long long P)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < P; q += (long long)gridDim.x * blockDim.x)
        ub[q].x += wst[q] + wst[P + q] + wst[2 * P + q] + wst[3 * P + q];
}

// Transpose of impose_mass_flow's correction u0 += pu (csum - Q u0) / pf,
// Q u0 = aspect sum w_j w_k Re u0: u0_ -= aspect w_j w_k <pu, Re u0_> / pf.
__global__ void __launch_bounds__(1024) k_mf_adj(double2 *u, const double *w, int m, double aspect, const double *pu,
                                                 const double *pf)
{
    __shared__ double red[33];
    const long long plane = (long long)m * m;
    double acc = 0.0;
    for (long long i = threadIdx.x; i < plane; i += blockDim.x) acc += pu[i] * u[i].x;
    const double s = block_sum(acc, red);
    __shared__ double sh;
    if (threadIdx.x == 0) sh = s;
    __syncthreads();
    const double f = aspect * sh / *pf;
    for (long long i = threadIdx.x; i < plane; i += blockDim.x) u[i].x -= f * w[i % m] * w[i / m];
}

struct AdjAdvParams {
    const double2 *u, *v, *w;    // entry velocities of the substep
    const double2 *S[6];         // Q_mj + Q_jm for (m, j) = 11, 22, 33, 12, 13, 23
    double2 *ub[3];              // cotangents of u, v, w (added)
    long long P;
    int M;
};

// Transposed advection products per (y, z) point (see the block comment):
// r_m = sum_j u_j Phys(W^-1 S_mj), u_m += W Spec(r_m).
template <int R, int TQ>
__global__ void __launch_bounds__(R * TQ) k_advx_adj(const __grid_constant__ AdjAdvParams p,
                                                     const double2 *__restrict__ twg)
{
    constexpr int N = R * R, NT = R * TQ;
    extern __shared__ __align__(16) double2 sm[];
    double2 *tw = sm, *wk = tw + N, *xs = wk + N * TQ;
    const int c = threadIdx.x / TQ, g = threadIdx.x - c * TQ;
    const long long q0 = (long long)blockIdx.x * TQ, q = q0 + g;
    const bool valid = q < p.P;
    const int M = p.M;
    const long long P = p.P;
    for (int t = threadIdx.x; t < N; t += NT) cp_async16(tw + t, twg + t);
    cp_async_wait_all();
    __syncthreads();
    double2 a[R];
    // physical values of X + i Y along x (each a Hermitian spectrum, modes
    // >= 1 scaled by sc): re into xr, im into yr
    auto ifft_pair = [&](const double2 *X, const double2 *Y, double sc, double (&xr)[R], double (&yr)[R]) {
#pragma unroll
        for (int n1 = 0; n1 < R; ++n1) {
            const int k = R * n1 + c;
            double2 z = make_double2(0.0, 0.0);
            if (valid && k < M) {
                const double2 x = X[q + (long long)k * P], y = Y ? Y[q + (long long)k * P] : make_double2(0.0, 0.0);
                z = (k == 0) ? make_double2(x.x, -y.x) : make_double2(sc * (x.x - y.y), -sc * (x.y + y.x));
            } else if (valid && k > N - M) {
                const long long kk = N - k;
                const double2 x = X[q + kk * P], y = Y ? Y[q + kk * P] : make_double2(0.0, 0.0);
                z = make_double2(sc * (x.x + y.y), -sc * (y.x - x.y));
            }
            a[n1] = z;
        }
        __syncthreads();
        fft_step1<R, TQ>(a, wk, tw, c, g);
        __syncthreads();
        fft_step2<R, TQ>(wk, a, tw, c, g);
#pragma unroll
        for (int k2 = 0; k2 < R; ++k2) {
            xr[k2] = a[k2].x;
            yr[k2] = -a[k2].y;
        }
    };
    double uu[R], vv[R], ww[R], r1[R], r2[R], r3[R], s1[R], s2[R];
    ifft_pair(p.u, p.v, 1.0, uu, vv);
    ifft_pair(p.w, nullptr, 1.0, ww, s1);
    ifft_pair(p.S[0], p.S[1], 0.5, s1, s2);          // S11, S22
#pragma unroll
    for (int k = 0; k < R; ++k) {
        r1[k] = uu[k] * s1[k];
        r2[k] = vv[k] * s2[k];
    }
    ifft_pair(p.S[2], p.S[3], 0.5, s1, s2);          // S33, S12
#pragma unroll
    for (int k = 0; k < R; ++k) {
        r3[k] = ww[k] * s1[k];
        r1[k] += vv[k] * s2[k];
        r2[k] += uu[k] * s2[k];
    }
    ifft_pair(p.S[4], p.S[5], 0.5, s1, s2);          // S13, S23
#pragma unroll
    for (int k = 0; k < R; ++k) {
        r1[k] += ww[k] * s1[k];
        r3[k] += uu[k] * s1[k] + vv[k] * s2[k];
        r2[k] += ww[k] * s2[k];
    }
    const double sc = 1.0 / N;
    for (int pair = 0; pair < 2; ++pair) {
#pragma unroll
        for (int k2 = 0; k2 < R; ++k2) a[k2] = pair == 0 ? make_double2(r1[k2], r2[k2]) : make_double2(r3[k2], 0.0);
        __syncthreads();
        fft_step1<R, TQ>(a, wk, tw, c, g);
        __syncthreads();
        fft_step2<R, TQ>(wk, a, tw, c, g);
#pragma unroll
        for (int k2 = 0; k2 < R; ++k2) xs[(c + R * k2) * TQ + g] = a[k2];
        __syncthreads();
        for (int idx = threadIdx.x; idx < M * TQ; idx += NT) {
            const int i = idx / TQ, gg = idx - i * TQ;
            const long long qq = q0 + gg;
            if (qq >= P) continue;
            const double2 X = xs[i * TQ + gg], Y = xs[(i == 0 ? 0 : N - i) * TQ + gg];
            const double wgt = (i == 0) ? sc : 2.0 * sc;   // W Spec
            const double2 A = make_double2(0.5 * wgt * (X.x + Y.x), 0.5 * wgt * (X.y - Y.y));
            const double2 B = make_double2(0.5 * wgt * (X.y + Y.y), -0.5 * wgt * (X.x - Y.x));
            const long long e = qq + (long long)i * P;
            double2 *o0 = p.ub[pair == 0 ? 0 : 2];
            double2 t0 = o0[e];
            o0[e] = make_double2(t0.x + A.x, t0.y + A.y);
            if (pair == 0) {
                double2 t1 = p.ub[1][e];
                p.ub[1][e] = make_double2(t1.x + B.x, t1.y + B.y);
            }
        }
    }
}

template <int R, int TQ>
static int launch_advx_adj(ductgpu_ctx ctx, const AdjAdvParams &p)
{
    constexpr int N = R * R, NT = R * TQ;
    const double2 *tw = twiddle_table(ctx, N);
    if (!tw) return set_error(ctx, DUCTGPU_ESTATE, "adjoint advection: twiddle table unavailable");
    const size_t smem = ((size_t)N + 2 * (size_t)N * TQ) * sizeof(double2);
    DUCT_CUDA(ctx, cudaFuncSetAttribute(k_advx_adj<R, TQ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    {
        LaunchScope ls(ctx, DUCTGPU_K_ADVECTION);
        k_advx_adj<R, TQ><<<(unsigned)((p.P + TQ - 1) / TQ), NT, smem, ctx->stream>>>(p, tw);
    }
    return check_cuda(ctx, cudaGetLastError(), "k_advx_adj");
}

static int advx_adj_launch(ductgpu_ctx ctx, const AdjAdvParams &p, int mgalx)
{
    switch (mgalx) {
    case 16: return launch_advx_adj<4, 32>(ctx, p);
    case 64: return launch_advx_adj<8, 16>(ctx, p);
    case 144: return launch_advx_adj<12, 8>(ctx, p);
    case 256: return launch_advx_adj<16, 8>(ctx, p);
    default: return set_error(ctx, DUCTGPU_EARG, "adjoint advection: mgalx=%d", mgalx);
    }
}

// Work fields of the reverse sweep (offsets in fields of fdoubles).
enum AdjSlot {
    kSave = 0,          // u, v, w, p at the start (restored after the sweep)
    kCk = 4,            // 3 substeps x (u, v, w) entry velocities
    kUb = 13,           // u_, v_, w_, p_
    kAnext = 17,        // 3: cotangent of A_{k} from substep k + 1
    kAcur = 20,         // 3: total cotangent of this substep's A_k
    kHb = 23,           // 3: cotangents of the solves' right-hand sides
    kPhib = 26, kRb = 27,
    kS = 28,            // 6: Q_mj + Q_jm
    kFb = 34,           // 3: dJ/df
    kE = 37,            // 2 planes: unit vectors, operator (set-up of D1, D2)
    kAdjFields = 38
};

static int dns_adj_ensure(ductgpu_dns d)
{
    ductgpu_ctx ctx = d->ctx;
    if (d->adj) return DUCTGPU_OK;
    if (cudaMalloc(&d->adj, sizeof(double) * d->fdoubles * kAdjFields) != cudaSuccess ||
        cudaMalloc(&d->dmat, sizeof(double) * 2 * d->my * d->my) != cudaSuccess) {
        cudaGetLastError();
        return set_error(ctx, DUCTGPU_EALLOC, "dns gradient: work fields");
    }
    // D1, D2: the line kernel applied to the unit vectors of one plane
    const int m = d->my;
    double *E = d->adj + kE * d->fdoubles, *O = E + 2ull * m * m;
    k_unit_plane<<<(m * m + 255) / 256, 256, 0, ctx->stream>>>(reinterpret_cast<double2 *>(E), m);
    for (int ord = 1; ord <= 2; ++ord) {
        LineParams py = line_params('y', m, m, 1, d->xalp);
        add_job(py, E, {line_out(O, ord, 1.0, 0.0)});
        int rc = lines_launch(ctx, py);
        if (rc) return rc;
        k_real_part<<<(m * m + 255) / 256, 256, 0, ctx->stream>>>(reinterpret_cast<const double2 *>(O),
                                                                  d->dmat + (size_t)(ord - 1) * m * m, (long long)m * m);
    }
    ctx->launches += 3;
    return check_cuda(ctx, cudaGetLastError(), "dns gradient set-up");
}

// out = beta out + fac D_ord^T in along dir
static int mat_t(ductgpu_dns d, int ord, char dir, const double *in, double *out, double fac, double beta)
{
    ductgpu_ctx ctx = d->ctx;
    const long long total = d->P * d->M;
    int blocks = (int)((total + 255) / 256);
    if (blocks > 8 * ctx->num_sms) blocks = 8 * ctx->num_sms;
    {
        LaunchScope ls(ctx, DUCTGPU_K_LINES);
        k_lines_mat_t<<<blocks, 256, 0, ctx->stream>>>(d->dmat + (size_t)(ord - 1) * d->my * d->my, d->my,
                                                       reinterpret_cast<const double2 *>(in),
                                                       reinterpret_cast<double2 *>(out), d->my, d->my, d->M,
                                                       dir == 'y', fac, beta, 1);
    }
    return check_cuda(ctx, cudaGetLastError(), "k_lines_mat_t");
}

// out = sigma (beta out + sum_t (c0 + c1 i kx + c2 (i kx)^2) src_t) (pointwise)
struct PTerm {
    const double *src;
    double c0, c1, c2;
};
static int pointwise(ductgpu_dns d, double *out, double beta, std::initializer_list<PTerm> terms)
{
    LineParams p = line_params('y', d->my, d->my, d->M, d->xalp, 1);
    LineOut o = line_out(out, 0, 0.0, beta);
    for (const PTerm &t : terms) xterm(o, t.src, t.c0, t.c1, t.c2);
    add_job(p, nullptr, {o});
    return lines_launch(d->ctx, p);
}

static int dns_adj_solve(ductgpu_dns d, char bound, const double *const *g, double *const *out, int n, int k)
{
    ductgpu_ctx ctx = d->ctx;
    FieldTask t[3];
    for (int c = 0; c < n; ++c) {
        t[c].rhs = const_cast<double *>(g[c]);
        t[c].sol = out[c];
        t[c].nmodes = d->M;
        t[c].mode0 = 1;
        t[c].bound = bound;
        t[c].plane0 = c * d->M;
        t[c].refine = 1;
    }
    double *saved = ctx->lam, *saved_h = ctx->lam_host;
    ctx->lam = bound == 'n' ? d->lam_n : d->lam_d[k];
    ctx->lam_host = bound == 'n' ? d->lamh_n.data() : d->lamh_d[k].data();
    const int rc = solve_adjoint(ctx, t, n);
    ctx->lam = saved;
    ctx->lam_host = saved_h;
    return rc;
}

static int dns_gradient(ductgpu_dns d, double *J)
{
    ductgpu_ctx ctx = d->ctx;
    int rc = dns_adj_ensure(d);
    if (rc) return rc;
    const size_t F = d->fdoubles, fb = sizeof(double) * F;
    const int m = d->my, M = d->M;
    const double nu = d->fnu, dt = d->dt, asp = d->aspect;
    double *W = d->adj;
    auto slot = [&](int s) { return W + (size_t)s * F; };
    double *vel[4] = {d->vel[0], d->vel[1], d->vel[2], d->p};
    for (int c = 0; c < 4; ++c) DUCT_CUDA(ctx, cudaMemcpyAsync(slot(kSave + c), vel[c], fb, cudaMemcpyDeviceToDevice, ctx->stream));
    // forward step with the substeps' entry velocities kept
    for (int krk = 1; krk <= 3; ++krk) {
        for (int c = 0; c < 3; ++c)
            DUCT_CUDA(ctx, cudaMemcpyAsync(slot(kCk + 3 * (krk - 1) + c), d->vel[c], fb, cudaMemcpyDeviceToDevice,
                                           ctx->stream));
        if ((rc = dns_issue(d, krk, false))) return rc;
    }
    // J = sum of the four wall stresses of the final u
    {
        const double *f[4] = {d->vel[0], nullptr, nullptr, nullptr};
        double *out = d->partial + (size_t)kStatBlocksMax * kStatVals;   // the scratch row
        if ((rc = stats_issue(ctx, f, 1, d->wcc, d->wst, nullptr, nullptr, d->partial, out, nullptr, 0, d->P, 1,
                              asp)))
            return rc;
        double s4[4];
        DUCT_CUDA(ctx, cudaMemcpyAsync(s4, out, sizeof(s4), cudaMemcpyDeviceToHost, ctx->stream));
        DUCT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        *J = s4[0] + s4[1] + s4[2] + s4[3];
    }
    // reverse sweep
    DUCT_CUDA(ctx, cudaMemsetAsync(slot(kUb), 0, 4 * fb, ctx->stream));
    DUCT_CUDA(ctx, cudaMemsetAsync(slot(kAnext), 0, 3 * fb, ctx->stream));
    DUCT_CUDA(ctx, cudaMemsetAsync(slot(kFb), 0, 3 * fb, ctx->stream));
    k_seed_wall<<<(unsigned)((d->P + 255) / 256), 256, 0, ctx->stream>>>(reinterpret_cast<double2 *>(slot(kUb)), d->wst,
                                                                         d->P);
    ctx->launches += 1;
    double *ub[3] = {slot(kUb), slot(kUb + 1), slot(kUb + 2)}, *pb = slot(kUb + 3);
    double *an[3] = {slot(kAnext), slot(kAnext + 1), slot(kAnext + 2)};
    double *ac[3] = {slot(kAcur), slot(kAcur + 1), slot(kAcur + 2)};
    double *hb[3] = {slot(kHb), slot(kHb + 1), slot(kHb + 2)};
    double *phib = slot(kPhib), *rb = slot(kRb), *fbar[3] = {slot(kFb), slot(kFb + 1), slot(kFb + 2)};
    double *S[6];
    for (int i = 0; i < 6; ++i) S[i] = slot(kS + i);
    for (int krk = 3; krk >= 1; --krk) {
        const int k = krk - 1;
        const double a = kAkk[k], b = kBkk[k], gm = kGkk[k], rho = kRkk[k];
        const double f1 = (a + b) * dt * nu, s2 = -dt * (a + b), sdiv = 1.0 / ((a + b) * dt), sig = -1.0 / (nu * b);
        // (mass flow)
        if (d->cmassflow) {
            LaunchScope ls(ctx, DUCTGPU_K_OTHER);
            k_mf_adj<<<1, 1024, 0, ctx->stream>>>(reinterpret_cast<double2 *>(ub[0]), ctx->ccw, m, ctx->mf_aspect,
                                                   ctx->mf_u + (size_t)m * m * k, ctx->mf_f + k);
        }
        // (update) phi_ = (I - f1 Lap)^T p_ + s2 grad^T u_
        if ((rc = pointwise(d, phib, 0.0, {{pb, 1.0, 0.0, -f1}, {ub[0], 0.0, -s2, 0.0}}))) return rc;
        if ((rc = mat_t(d, 2, 'y', pb, phib, -f1, 1.0))) return rc;
        if ((rc = mat_t(d, 2, 'z', pb, phib, -f1 / (asp * asp), 1.0))) return rc;
        if ((rc = mat_t(d, 1, 'y', ub[1], phib, s2, 1.0))) return rc;
        if ((rc = mat_t(d, 1, 'z', ub[2], phib, s2 / asp, 1.0))) return rc;
        // (pressure) r_ = S_n^T phi_ ; u*_ += sdiv grad^T r_
        {
            const double *g[1] = {phib};
            double *o[1] = {rb};
            if ((rc = dns_adj_solve(d, 'n', g, o, 1, k))) return rc;
        }
        if ((rc = pointwise(d, ub[0], 1.0, {{rb, 0.0, -sdiv, 0.0}}))) return rc;
        if ((rc = mat_t(d, 1, 'y', rb, ub[1], sdiv, 1.0))) return rc;
        if ((rc = mat_t(d, 1, 'z', rb, ub[2], sdiv / asp, 1.0))) return rc;
        // (predictor) h_ = S_d^T u*_ ; the right-hand side's cotangent is sig h_
        {
            const double *g[3] = {ub[0], ub[1], ub[2]};
            if ((rc = dns_adj_solve(d, 'd', g, hb, 3, k))) return rc;
        }
        // p_ -= (a+b) sig grad^T h_
        if ((rc = pointwise(d, pb, 1.0, {{hb[0], 0.0, (a + b) * sig, 0.0}}))) return rc;
        if ((rc = mat_t(d, 1, 'y', hb[1], pb, -(a + b) * sig, 1.0))) return rc;
        if ((rc = mat_t(d, 1, 'z', hb[2], pb, -(a + b) * sig / asp, 1.0))) return rc;
        for (int c = 0; c < 3; ++c) {
            // A_k's cotangent; the previous substep's; f_; u_ entering the substep
            if ((rc = pointwise(d, ac[c], 0.0, {{an[c], 1.0, 0.0, 0.0}, {hb[c], -gm * sig, 0.0, 0.0}}))) return rc;
            if ((rc = pointwise(d, an[c], 0.0, {{hb[c], -rho * sig, 0.0, 0.0}}))) return rc;
            if ((rc = pointwise(d, fbar[c], 1.0, {{hb[c], (a + b) * sig, 0.0, 0.0}}))) return rc;
            if ((rc = pointwise(d, ub[c], 0.0, {{hb[c], sig / dt, 0.0, sig * a * nu}}))) return rc;
            if ((rc = mat_t(d, 2, 'y', hb[c], ub[c], sig * a * nu, 1.0))) return rc;
            if ((rc = mat_t(d, 2, 'z', hb[c], ub[c], sig * a * nu / (asp * asp), 1.0))) return rc;
        }
        // (advection) S_mj = Q_mj + Q_jm, Q_ij = d_j^T A_i
        if ((rc = pointwise(d, S[0], 0.0, {{ac[0], 0.0, -2.0, 0.0}}))) return rc;          // 2 Q11
        if ((rc = mat_t(d, 1, 'y', ac[1], S[1], 2.0, 0.0))) return rc;                       // 2 Q22
        if ((rc = mat_t(d, 1, 'z', ac[2], S[2], 2.0 / asp, 0.0))) return rc;                 // 2 Q33
        if ((rc = pointwise(d, S[3], 0.0, {{ac[1], 0.0, -1.0, 0.0}}))) return rc;          // Q21
        if ((rc = mat_t(d, 1, 'y', ac[0], S[3], 1.0, 1.0))) return rc;                       // + Q12
        if ((rc = pointwise(d, S[4], 0.0, {{ac[2], 0.0, -1.0, 0.0}}))) return rc;          // Q31
        if ((rc = mat_t(d, 1, 'z', ac[0], S[4], 1.0 / asp, 1.0))) return rc;                 // + Q13
        if ((rc = mat_t(d, 1, 'y', ac[2], S[5], 1.0, 0.0))) return rc;                       // Q32
        if ((rc = mat_t(d, 1, 'z', ac[1], S[5], 1.0 / asp, 1.0))) return rc;                 // + Q23
        AdjAdvParams ap{};
        ap.u = reinterpret_cast<const double2 *>(slot(kCk + 3 * k));
        ap.v = reinterpret_cast<const double2 *>(slot(kCk + 3 * k + 1));
        ap.w = reinterpret_cast<const double2 *>(slot(kCk + 3 * k + 2));
        for (int i = 0; i < 6; ++i) ap.S[i] = reinterpret_cast<const double2 *>(S[i]);
        for (int c = 0; c < 3; ++c) ap.ub[c] = reinterpret_cast<double2 *>(ub[c]);
        ap.P = d->P;
        ap.M = M;
        if ((rc = advx_adj_launch(ctx, ap, d->mgalx))) return rc;
    }
    // the state as it was
    for (int c = 0; c < 4; ++c) DUCT_CUDA(ctx, cudaMemcpyAsync(vel[c], slot(kSave + c), fb, cudaMemcpyDeviceToDevice, ctx->stream));
    return check_cuda(ctx, cudaGetLastError(), "dns gradient");
}

}  // namespace duct

extern "C" int ductgpu_dns_set_forcing(ductgpu_dns d, const double *f1, const double *f2, const double *f3)
{
    if (!d) return DUCTGPU_EARG;
    ductgpu_ctx ctx = d->ctx;
    cudaSetDevice(ctx->device);
    const bool on = f1 || f2 || f3;
    if (on && !d->force && cudaMalloc(&d->force, sizeof(double) * 3 * d->fdoubles) != cudaSuccess) {
        cudaGetLastError();
        return set_error(ctx, DUCTGPU_EALLOC, "dns_set_forcing: 3 fields");
    }
    const double *src[3] = {f1, f2, f3};
    for (int c = 0; c < 3 && on; ++c) {
        double *dst = d->force + c * d->fdoubles;
        if (src[c]) DUCT_CUDA(ctx, cudaMemcpyAsync(dst, src[c], sizeof(double) * d->fdoubles, cudaMemcpyDefault, ctx->stream));
        else DUCT_CUDA(ctx, cudaMemsetAsync(dst, 0, sizeof(double) * d->fdoubles, ctx->stream));
    }
    if (on != d->forced) dns_drop_graphs(d);   // the substep graphs were captured with the other choice
    d->forced = on;
    return check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "dns_set_forcing");
}

extern "C" int ductgpu_dns_grad_wallstress(ductgpu_dns d, double *J, double *fbar)
{
    if (!d || !J) return DUCTGPU_EARG;
    ductgpu_ctx ctx = d->ctx;
    cudaSetDevice(ctx->device);
    int rc = dns_gradient(d, J);
    if (rc) return rc;
    if (fbar)
        DUCT_CUDA(ctx, cudaMemcpyAsync(fbar, d->adj + (size_t)kFb * d->fdoubles, sizeof(double) * 3 * d->fdoubles,
                                       cudaMemcpyDefault, ctx->stream));
    return check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "dns_grad_wallstress");
}

// J = the four-wall stress of u after nsteps RK3 steps from the current
// state (left unchanged): the functional the gradient differentiates.
extern "C" int ductgpu_dns_wallstress_after(ductgpu_dns d, int nsteps, double *J)
{
    if (!d || !J || nsteps < 0) return DUCTGPU_EARG;
    ductgpu_ctx ctx = d->ctx;
    cudaSetDevice(ctx->device);
    int rc = dns_adj_ensure(d);
    if (rc) return rc;
    const size_t fb = sizeof(double) * d->fdoubles;
    double *vel[4] = {d->vel[0], d->vel[1], d->vel[2], d->p};
    for (int c = 0; c < 4; ++c)
        DUCT_CUDA(ctx, cudaMemcpyAsync(d->adj + (size_t)(kSave + c) * d->fdoubles, vel[c], fb, cudaMemcpyDeviceToDevice,
                                       ctx->stream));
    for (int s = 0; s < nsteps; ++s)
        for (int krk = 1; krk <= 3; ++krk)
            if ((rc = dns_issue(d, krk, false))) return rc;
    const double *f[4] = {d->vel[0], nullptr, nullptr, nullptr};
    double *out = d->partial + (size_t)kStatBlocksMax * kStatVals;
    if ((rc = stats_issue(ctx, f, 1, d->wcc, d->wst, nullptr, nullptr, d->partial, out, nullptr, 0, d->P, 1,
                          d->aspect)))
        return rc;
    double s4[4];
    DUCT_CUDA(ctx, cudaMemcpyAsync(s4, out, sizeof(s4), cudaMemcpyDeviceToHost, ctx->stream));
    for (int c = 0; c < 4; ++c)
        DUCT_CUDA(ctx, cudaMemcpyAsync(vel[c], d->adj + (size_t)(kSave + c) * d->fdoubles, fb, cudaMemcpyDeviceToDevice,
                                       ctx->stream));
    DUCT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *J = s4[0] + s4[1] + s4[2] + s4[3];
    return DUCTGPU_OK;
}
