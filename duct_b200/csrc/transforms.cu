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
// complex line on tiles of lines staged in shared memory with cp.async.
//
// Pencil transposes (src/parallel.F:476-529): 32x32 tiles of complex
// elements through padded shared memory.
#include <math.h>

#include "internal.h"
#include "fft.cuh"

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


// One radix-R Stockham stage over all lines of the CTA; twiddles from the
// table tw[t] = exp(-2 pi i t / L).
template <int R>
__device__ __forceinline__ void stockham_stage(const double2 *x, double2 *y, const double2 *tw, int L, int LS, int Ns,
                                               int lpb)
{
    const int nb = L / R;
    const int tstep = L / (Ns * R);
    for (int idx = threadIdx.x; idx < nb * lpb; idx += blockDim.x) {
        const int l = idx / nb, j = idx - l * nb;
        const double2 *xl = x + l * LS;
        double2 *yl = y + l * LS;
        const int k = j % Ns;
        double2 v[4];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = xl[j + r * nb];
        if (Ns > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) v[r] = cmul(v[r], tw[r * k * tstep]);
        }
        dft<R>(v);
        const int d = (j / Ns) * Ns * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) yl[d + r * Ns] = v[r];
    }
}

// Lines of a CTA: lpb consecutive lines of one plane (the launch keeps a
// CTA inside one Fourier mode), staged with cp.async; y-lines are
// contiguous, z-lines are read as rows of lpb consecutive y (128 B for 8).
__global__ void __launch_bounds__(256) k_dct(const __grid_constant__ DctParams p)
{
    extern __shared__ __align__(16) double2 buf[];
    const int L = p.L, LS = p.L + 1, N = p.nn - 1, nn = p.nn;   // LS: padded line stride
    double2 *tw = buf;
    double2 *x = buf + L, *y = x + p.lpb * LS;
    const int cpm = (p.lines_per_mode + p.lpb - 1) / p.lpb;   // CTAs per mode
    const int mode = blockIdx.x / cpm;
    const int q0 = (blockIdx.x - mode * cpm) * p.lpb;
    const int nl = min(p.lpb, p.lines_per_mode - q0);
    double2 *g = reinterpret_cast<double2 *>(p.f) + mode * p.mode_stride + (long long)q0 * p.line_stride;
    const bool contiguous = (p.elem_stride == 1);
    for (int idx = threadIdx.x; idx < nl * nn; idx += blockDim.x) {
        int l, j;
        if (contiguous) { l = idx / nn; j = idx - l * nn; }
        else { j = idx / nl; l = idx - j * nl; }
        cp_async16(x + l * LS + j, g + l * p.line_stride + (long long)j * p.elem_stride);
    }
    for (int t = threadIdx.x; t < L; t += blockDim.x) {
        double sn, cs;
        sincospi(-2.0 * (double)t / (double)L, &sn, &cs);
        tw[t] = make_double2(cs, sn);
    }
    cp_async_wait_all();
    __syncthreads();
    // even extension; the inverse weights the interior points by 1/2
    const double si = (p.iopt >= 0) ? 0.5 : 1.0;
    for (int idx = threadIdx.x; idx < p.lpb * (N - 1); idx += blockDim.x) {
        const int l = idx / (N - 1), j = 1 + idx - l * (N - 1);
        double2 v = make_double2(0.0, 0.0);
        if (l < nl) {
            v = x[l * LS + j];
            v = make_double2(si * v.x, si * v.y);
        }
        x[l * LS + j] = v;
        x[l * LS + (L - j)] = v;
    }
    for (int l = nl + threadIdx.x; l < p.lpb; l += blockDim.x) {   // unused lines: zero ends
        x[l * LS] = make_double2(0.0, 0.0);
        x[l * LS + N] = make_double2(0.0, 0.0);
    }
    __syncthreads();
    int Ns = 1;
    for (int s = 0; s < p.nstages; ++s) {
        const int R = p.radix[s];
        if (R == 4) stockham_stage<4>(x, y, tw, L, LS, Ns, p.lpb);
        else if (R == 2) stockham_stage<2>(x, y, tw, L, LS, Ns, p.lpb);
        else stockham_stage<3>(x, y, tw, L, LS, Ns, p.lpb);
        Ns *= R;
        __syncthreads();
        double2 *t = x; x = y; y = t;
    }
    const double dn1 = 1.0 / (double)N, dn2 = 0.5 * dn1;
    for (int idx = threadIdx.x; idx < nl * nn; idx += blockDim.x) {
        int l, j;
        if (contiguous) { l = idx / nn; j = idx - l * nn; }
        else { j = idx / nl; l = idx - j * nl; }
        double2 v = x[l * LS + j];
        if (p.iopt < 0) {
            const double sc = (j == 0 || j == N) ? dn2 : dn1;
            v = make_double2(sc * v.x, sc * v.y);
        }
        g[l * p.line_stride + (long long)j * p.elem_stride] = v;
    }
}

// ---------------------------------------------------------------------------
// Two-pass register FFT of the even extension, L = R1 * R2 (four-step):
//   X[k1 + R1 k2] = sum_n2 W_R2^(n2 k2) W_L^(n2 k1) sum_n1 x[R2 n1 + n2] W_R1^(n1 k1)
// Step 1: one thread per (line, n2) runs the R1-point DFT in registers and
// applies W_L^(n2 k1); step 2: one thread per (line, k1) runs the R2-point
// DFT.  Shared memory is touched once per step (reads and writes) instead
// of once per radix stage.  The register DFTs are compile-time Stockham
// sequences of radix 4, 3, 2 stages; their twiddles W_(Ns P)^(r k) come from
// the W_L table (broadcast reads).
// One padded line buffer per line: point j lives at j + j / R2 (a pad word
// after every R2 points), so the step-1 columns (stride R2) and the step-2
// rows (R2 consecutive points) are both conflict-free, and both steps work
// in place (step 1: each thread reads and writes its own column; step 2:
// rows are read into registers before a barrier, then results written).
template <int R1, int R2>
__global__ void __launch_bounds__(256) k_dct2(const __grid_constant__ DctParams p, const double2 *__restrict__ twg)
{
    extern __shared__ __align__(16) double2 buf[];
    constexpr int L = R1 * R2, LS = R1 * (R2 + 1);
    constexpr int LPB = 256 / (R1 > R2 ? R1 : R2);   // lines per CTA (compile time: cheap index math)
    const int N = p.nn - 1, nn = p.nn;
    double2 *tw = buf;
    double2 *x = buf + L;                       // [LPB][LS]
    auto at = [](int j) { return j + j / R2; };
    const int cpm = (p.lines_per_mode + LPB - 1) / LPB;
    const int mode = blockIdx.x / cpm;
    const int q0 = (blockIdx.x - mode * cpm) * LPB;
    const int nl = min(LPB, p.lines_per_mode - q0);
    double2 *g = reinterpret_cast<double2 *>(p.f) + mode * p.mode_stride + (long long)q0 * p.line_stride;
    const bool contiguous = (p.elem_stride == 1);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // y-lines: a warp per line, lanes along the line; z-lines: consecutive
    // threads on consecutive lines (l fastest), LPB a compile-time divisor
    if (contiguous) {
        for (int l = warp; l < nl; l += 8)
            for (int j = lane; j < nn; j += 32) cp_async16(x + l * LS + at(j), g + l * p.line_stride + j);
    } else {
        for (int idx = threadIdx.x; idx < LPB * nn; idx += 256) {
            const int j = idx / LPB, l = idx - j * LPB;
            if (l < nl) cp_async16(x + l * LS + at(j), g + l + (long long)j * p.elem_stride);
        }
    }
    for (int t = threadIdx.x; t < L; t += 256) cp_async16(tw + t, twg + t);
    cp_async_wait_all();
    __syncthreads();
    const double si = (p.iopt >= 0) ? 0.5 : 1.0;
    for (int l = warp; l < LPB; l += 8) {
        double2 *xl = x + l * LS;
        if (l < nl) {
            for (int j = 1 + lane; j < N; j += 32) {
                double2 v = xl[at(j)];
                v = make_double2(si * v.x, si * v.y);
                xl[at(j)] = v;
                xl[at(L - j)] = v;
            }
        } else {
            for (int j = lane; j < L; j += 32) xl[at(j)] = make_double2(0.0, 0.0);
        }
    }
    __syncthreads();
    // step 1: R1-point DFTs along n1 (column n2), twiddle W_L^(n2 k1), in place
    {
        const int l = threadIdx.x / R2, n2 = threadIdx.x - l * R2;
        if (l < LPB) {
            double2 *xl = x + l * LS;
            double2 v[R1];
#pragma unroll
            for (int n1 = 0; n1 < R1; ++n1) v[n1] = xl[n1 * (R2 + 1) + n2];
            reg_fft<R1, 0, 1>(v, tw, L);
#pragma unroll
            for (int k1 = 0; k1 < R1; ++k1) xl[k1 * (R2 + 1) + n2] = (k1 == 0) ? v[0] : cmul(v[k1], tw[n2 * k1]);
        }
    }
    __syncthreads();
    // step 2: R2-point DFTs along row k1; results X[k1 + R1 k2] after a barrier
    {
        const int l = threadIdx.x / R1, k1 = threadIdx.x - l * R1;
        const bool act = l < LPB;
        double2 w[R2];
        if (act) {
            const double2 *xr = x + l * LS + k1 * (R2 + 1);
#pragma unroll
            for (int n2 = 0; n2 < R2; ++n2) w[n2] = xr[n2];
            reg_fft<R2, 0, 1>(w, tw, L);
        }
        __syncthreads();
        if (act) {
#pragma unroll
            for (int k2 = 0; k2 < R2; ++k2) {
                const int j = k1 + R1 * k2;
                if (j <= N) x[l * LS + at(j)] = w[k2];
            }
        }
    }
    __syncthreads();
    const double dn1 = 1.0 / (double)N, dn2 = 0.5 * dn1;
    const bool fwd = p.iopt < 0;
    if (contiguous) {
        for (int l = warp; l < nl; l += 8)
            for (int j = lane; j < nn; j += 32) {
                double2 v = x[l * LS + at(j)];
                if (fwd) {
                    const double sc = (j == 0 || j == N) ? dn2 : dn1;
                    v = make_double2(sc * v.x, sc * v.y);
                }
                g[l * p.line_stride + j] = v;
            }
    } else {
        for (int idx = threadIdx.x; idx < LPB * nn; idx += 256) {
            const int j = idx / LPB, l = idx - j * LPB;
            if (l >= nl) continue;
            double2 v = x[l * LS + at(j)];
            if (fwd) {
                const double sc = (j == 0 || j == N) ? dn2 : dn1;
                v = make_double2(sc * v.x, sc * v.y);
            }
            g[l + (long long)j * p.elem_stride] = v;
        }
    }
}

__global__ void k_twiddles(int L, double2 *tw)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < L; t += gridDim.x * blockDim.x) {
        double sn, cs;
        sincospi(-2.0 * (double)t / (double)L, &sn, &cs);
        tw[t] = make_double2(cs, sn);
    }
}

// W_L table in device memory, one per length, kept in the context
const double2 *twiddle_table(ductgpu_ctx ctx, int L)
{
    for (int i = 0; i < ductgpu_ctx_s::kTwTables; ++i)
        if (ctx->tw_len[i] == L) return reinterpret_cast<const double2 *>(ctx->tw_tab[i]);
    for (int i = 0; i < ductgpu_ctx_s::kTwTables; ++i)
        if (!ctx->tw_len[i]) {
            if (ctx->capturing) return nullptr;     // no allocation inside a capture
            if (cudaMalloc(&ctx->tw_tab[i], (size_t)L * sizeof(double2)) != cudaSuccess) return nullptr;
            k_twiddles<<<(L + 255) / 256, 256, 0, ctx->stream>>>(L, reinterpret_cast<double2 *>(ctx->tw_tab[i]));
            ctx->launches += 1;
            ctx->tw_len[i] = L;
            return reinterpret_cast<const double2 *>(ctx->tw_tab[i]);
        }
    return nullptr;
}

template <int R1, int R2>
static int launch_dct2(ductgpu_ctx ctx, DctParams &p, int nmodes)
{
    constexpr int L = R1 * R2;
    constexpr int RM = R1 > R2 ? R1 : R2;
    const double2 *tw = twiddle_table(ctx, L);
    if (!tw) return -1;                             // no table: the radix-stage kernel
    p.lpb = 256 / RM;                               // the kernel's LPB
    const size_t smem = ((size_t)L + (size_t)p.lpb * R1 * (R2 + 1)) * sizeof(double2);
    DUCT_CUDA(ctx, cudaFuncSetAttribute(k_dct2<R1, R2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int grid = nmodes * ((p.lines_per_mode + p.lpb - 1) / p.lpb);
    {
        LaunchScope ls(ctx, DUCTGPU_K_TRANSFORM);
        k_dct2<R1, R2><<<grid, 256, smem, ctx->stream>>>(p, tw);
    }
    return check_cuda(ctx, cudaGetLastError(), "k_dct2");
}

// Threads per CTA of k_dcth: a CTA holds 64 / max(R1, R2) lines (4 at
// N = 192) and runs its steps (staging, pre-step, two FFT steps, post-step,
// store) between CTA barriers, so many small CTAs on an SM overlap the steps
// of one another; measured at my = 193 (fraction of the HBM copy rate,
// y / z): 256 threads 0.315 / 0.289, 128 threads 0.343 / 0.321, 64 threads
// 0.351 / 0.324.
constexpr int kDcthThreads = 64;

// Half-length DCT-I (N = R1 R2 even, N + 1 points a line).  With F the
// DCT-I of a line, F_k = (x_0 + (-1)^k x_N) / 2 + sum_{j=1}^{N-1} x_j cos(pi j k / N)
// (the 2N even-extension FFT of k_dct2 gives 2 F_k), the sequence
//   g_0 = (x_0 + x_N) / 2,  g_{N/2} = x_{N/2},
//   g_j = (x_j + x_{N-j}) / 2 - sin(pi j / N) (x_j - x_{N-j})   (0 < j < N, j != N/2)
// has the length-N DFT G_k with (by the symmetric / antisymmetric split of
// each term under j -> N - j, and 2 sin a sin b = cos(a - b) - cos(a + b))
//   F_{2k} = (G_k + G_{N-k}) / 2,   F_{2k+1} = F_{2k-1} + i (G_k - G_{N-k}) / 2,
//   F_1 = (x_0 - x_N) / 2 + sum_{j=1}^{N/2-1} cos(pi j / N) (x_j - x_{N-j}).
// g is real-linear in x, so the complex line (re + i im) goes through one
// complex FFT of length N and these formulas directly -- the half-length
// real-data DCT of Press et al. (Numerical Recipes, sec. 12.3), here for a
// pair of real lines at once.  Half the FFT of the even extension and half
// its shared memory.
// Shared line layout: point j at j + j / R2 (as k_dct2), x_N at R1 (R2 + 1).
// Results: F_{2k} in slot k, F_{2k+1} in slot N - k (slot N for F_1).
template <int R1, int R2, int NT>
__global__ void __launch_bounds__(NT) k_dcth(const __grid_constant__ DctParams p, const double2 *__restrict__ twg,
                                             const double2 *__restrict__ tw2)
{
    extern __shared__ __align__(16) double2 buf[];
    constexpr int N = R1 * R2, LS = R1 * (R2 + 1) + 1;
    constexpr int LPB = NT / (R1 > R2 ? R1 : R2), NW = NT / 32;
    double2 *tw = buf;                          // W_N^t, N entries
    double2 *ha = tw + N;                       // W_2N^j, j <= N/2: (cos, -sin)(pi j / N)
    double2 *x = ha + (N / 2 + 1);              // [LPB][LS]
    double2 *f1 = x + LPB * LS;                 // [LPB] F_1 of each line
    auto at = [](int j) { return j + j / R2; };
    const int cpm = (p.lines_per_mode + LPB - 1) / LPB;
    const int mode = blockIdx.x / cpm;
    const int q0 = (blockIdx.x - mode * cpm) * LPB;
    const int nl = min(LPB, p.lines_per_mode - q0);
    double2 *g = reinterpret_cast<double2 *>(p.f) + mode * p.mode_stride + (long long)q0 * p.line_stride;
    const bool contiguous = (p.elem_stride == 1);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (contiguous) {
        for (int l = warp; l < nl; l += NW)
            for (int j = lane; j <= N; j += 32) cp_async16(x + l * LS + at(j), g + l * p.line_stride + j);
    } else {
        for (int idx = threadIdx.x; idx < LPB * (N + 1); idx += NT) {
            const int j = idx / LPB, l = idx - j * LPB;
            if (l < nl) cp_async16(x + l * LS + at(j), g + l + (long long)j * p.elem_stride);
        }
    }
    for (int t = threadIdx.x; t < N; t += NT) cp_async16(tw + t, twg + t);
    for (int t = threadIdx.x; t <= N / 2; t += NT) cp_async16(ha + t, tw2 + t);
    cp_async_wait_all();
    __syncthreads();
    // g in place (a warp per line); the inverse halves the interior points first
    const double si = (p.iopt >= 0) ? 0.5 : 1.0;
    for (int l = warp; l < LPB; l += NW) {
        double2 *xl = x + l * LS;
        if (l >= nl) {
            for (int j = lane; j < LS; j += 32) xl[j] = make_double2(0.0, 0.0);
            continue;
        }
        double sx = 0.0, sy = 0.0;
        for (int j = 1 + lane; j < N / 2; j += 32) {
            const double2 a = xl[at(j)], b = xl[at(N - j)];
            const double2 u = make_double2(0.5 * si * (a.x + b.x), 0.5 * si * (a.y + b.y));
            const double2 v = make_double2(si * (a.x - b.x), si * (a.y - b.y));
            const double2 w = ha[j];   // (cos(pi j/N), -sin(pi j/N))
            xl[at(j)] = make_double2(u.x + w.y * v.x, u.y + w.y * v.y);
            xl[at(N - j)] = make_double2(u.x - w.y * v.x, u.y - w.y * v.y);
            sx += w.x * v.x;
            sy += w.x * v.y;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            sx += __shfl_xor_sync(0xffffffffu, sx, o);
            sy += __shfl_xor_sync(0xffffffffu, sy, o);
        }
        if (lane == 0) {
            const double2 x0 = xl[at(0)], xn = xl[at(N)], xm = xl[at(N / 2)];
            f1[l] = make_double2(0.5 * (x0.x - xn.x) + sx, 0.5 * (x0.y - xn.y) + sy);
            xl[at(0)] = make_double2(0.5 * (x0.x + xn.x), 0.5 * (x0.y + xn.y));
            xl[at(N / 2)] = make_double2(si * xm.x, si * xm.y);
        }
    }
    __syncthreads();
    // FFT of length N in place: R1-point DFTs along n1 (column n2) with the
    // twiddle W_N^(n2 k1), then R2-point DFTs along each row k1
    {
        const int l = threadIdx.x / R2, n2 = threadIdx.x - l * R2;
        if (l < LPB) {
            double2 *xl = x + l * LS;
            double2 v[R1];
#pragma unroll
            for (int n1 = 0; n1 < R1; ++n1) v[n1] = xl[n1 * (R2 + 1) + n2];
            reg_fft<R1, 0, 1>(v, tw, N);
#pragma unroll
            for (int k1 = 0; k1 < R1; ++k1) xl[k1 * (R2 + 1) + n2] = (k1 == 0) ? v[0] : cmul(v[k1], tw[n2 * k1]);
        }
    }
    __syncthreads();
    {
        const int l = threadIdx.x / R1, k1 = threadIdx.x - l * R1;
        const bool act = l < LPB;
        double2 w[R2];
        if (act) {
            const double2 *xr = x + l * LS + k1 * (R2 + 1);
#pragma unroll
            for (int n2 = 0; n2 < R2; ++n2) w[n2] = xr[n2];
            reg_fft<R2, 0, 1>(w, tw, N);
        }
        __syncthreads();
        if (act) {
#pragma unroll
            for (int k2 = 0; k2 < R2; ++k2) x[l * LS + at(k1 + R1 * k2)] = w[k2];
        }
    }
    __syncthreads();
    // From G to F, a warp per line: lane q owns the pairs (k, N - k) of a run
    // of consecutive k <= N/2; F_{2k} = (G_k + G_{N-k}) / 2 goes to slot k and
    // F_{2k+1} = F_1 + sum_{i=1}^{k} i (G_i - G_{N-i}) / 2 to slot N - k
    // (the increments scanned across the warp with shuffles), F_1 to slot N.
    for (int l = warp; l < nl; l += NW) {
        double2 *xl = x + l * LS;
        constexpr int CH = (N / 2 + 1 + 31) / 32;
        const int k0 = lane * CH, k1 = min(N / 2 + 1, k0 + CH);
        double sx = 0.0, sy = 0.0;
        for (int k = k0; k < k1; ++k) {
            if (k == 0 || k == N / 2) continue;
            const double2 gk = xl[at(k)], gm = xl[at(N - k)];
            sx -= 0.5 * (gk.y - gm.y);
            sy += 0.5 * (gk.x - gm.x);
        }
        double ix = sx, iy = sy;   // inclusive prefix over lanes 0..lane
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double tx = __shfl_up_sync(0xffffffffu, ix, o), ty = __shfl_up_sync(0xffffffffu, iy, o);
            if (lane >= o) {
                ix += tx;
                iy += ty;
            }
        }
        const double2 b1 = f1[l];
        double rx = b1.x + ix - sx, ry = b1.y + iy - sy;
        for (int k = k0; k < k1; ++k) {
            const double2 gk = xl[at(k)], gm = xl[at(k == 0 ? 0 : N - k)];
            xl[at(k)] = make_double2(0.5 * (gk.x + gm.x), 0.5 * (gk.y + gm.y));
            if (k > 0 && k < N / 2) {
                rx -= 0.5 * (gk.y - gm.y);
                ry += 0.5 * (gk.x - gm.x);
                xl[at(N - k)] = make_double2(rx, ry);
            }
        }
        if (lane == 0) xl[at(N)] = b1;
    }
    __syncthreads();
    // out_j = 2 F_j, scaled by 1/(2N) at the ends and 1/N inside (forward)
    const bool fwd = p.iopt < 0;
    auto value = [&](int l, int j) {
        const int slot = (j & 1) ? N - (j >> 1) : (j >> 1);
        const double2 v = x[l * LS + at(slot)];
        const double sc = fwd ? ((j == 0 || j == N) ? 1.0 / N : 2.0 / N) : 2.0;
        return make_double2(sc * v.x, sc * v.y);
    };
    if (contiguous) {
        for (int l = warp; l < nl; l += NW)
            for (int j = lane; j <= N; j += 32) g[l * p.line_stride + j] = value(l, j);
    } else {
        for (int idx = threadIdx.x; idx < LPB * (N + 1); idx += NT) {
            const int j = idx / LPB, l = idx - j * LPB;
            if (l < nl) g[l + (long long)j * p.elem_stride] = value(l, j);
        }
    }
}

template <int R1, int R2, int NT = kDcthThreads>
static int launch_dcth(ductgpu_ctx ctx, DctParams &p, int nmodes)
{
    constexpr int N = R1 * R2, LS = R1 * (R2 + 1) + 1;
    constexpr int LPB = NT / (R1 > R2 ? R1 : R2);
    const double2 *tw = twiddle_table(ctx, N);
    const double2 *tw2 = twiddle_table(ctx, 2 * N);
    if (!tw || !tw2) return -1;
    p.lpb = LPB;
    const size_t smem = ((size_t)N + (N / 2 + 1) + (size_t)LPB * LS + LPB) * sizeof(double2);
    DUCT_CUDA(ctx, cudaFuncSetAttribute(k_dcth<R1, R2, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int grid = nmodes * ((p.lines_per_mode + LPB - 1) / LPB);
    {
        LaunchScope ls(ctx, DUCTGPU_K_TRANSFORM);
        k_dcth<R1, R2, NT><<<grid, NT, smem, ctx->stream>>>(p, tw, tw2);
    }
    return check_cuda(ctx, cudaGetLastError(), "k_dcth");
}

// Half-length plans (R1 x R2 = N = nn - 1); -1 if none.
static int dcth_dispatch(ductgpu_ctx ctx, DctParams &p, int nmodes)
{
    switch (p.nn - 1) {
    case 16: return launch_dcth<4, 4>(ctx, p, nmodes);
    case 24: return launch_dcth<4, 6>(ctx, p, nmodes);
    case 32: return launch_dcth<4, 8>(ctx, p, nmodes);
    case 48: return launch_dcth<6, 8>(ctx, p, nmodes);
    case 64: return launch_dcth<8, 8>(ctx, p, nmodes);
    case 96: return launch_dcth<8, 12>(ctx, p, nmodes);
    case 128: return launch_dcth<8, 16>(ctx, p, nmodes);
    case 144: return launch_dcth<12, 12>(ctx, p, nmodes);
    case 192: return launch_dcth<12, 16>(ctx, p, nmodes);
    case 256: return launch_dcth<16, 16>(ctx, p, nmodes);
    default: return -1;
    }
}

// Register-FFT plans (R1 x R2 = L) for the line lengths in use; -1 if none.
static int dct2_dispatch(ductgpu_ctx ctx, DctParams &p, int nmodes)
{
    switch (p.L) {
    case 16: return launch_dct2<4, 4>(ctx, p, nmodes);
    case 24: return launch_dct2<4, 6>(ctx, p, nmodes);
    case 32: return launch_dct2<4, 8>(ctx, p, nmodes);
    case 48: return launch_dct2<6, 8>(ctx, p, nmodes);
    case 64: return launch_dct2<8, 8>(ctx, p, nmodes);
    case 96: return launch_dct2<8, 12>(ctx, p, nmodes);
    case 128: return launch_dct2<8, 16>(ctx, p, nmodes);
    case 144: return launch_dct2<12, 12>(ctx, p, nmodes);
    case 192: return launch_dct2<12, 16>(ctx, p, nmodes);
    case 256: return launch_dct2<16, 16>(ctx, p, nmodes);
    case 288: return launch_dct2<12, 24>(ctx, p, nmodes);
    case 384: return launch_dct2<16, 24>(ctx, p, nmodes);
    case 512: return launch_dct2<16, 32>(ctx, p, nmodes);
    default: return -1;
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
    int lpb;              // lines per CTA
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

// lines per CTA of k_deriv: y lines (contiguous) / z lines (a point of
// consecutive lines contiguous); 16 keeps 4 CTAs on an SM at my = 193
constexpr int kDerivLinesY = 16, kDerivLinesZ = 16;

// A tile of p.lpb lines of one mode staged with cp.async (padded odd
// row length, conflict-free for both the y and the z access pattern), the
// recurrence run in place by one thread per line (it reads c_k before it
// writes out_k and then only lower indices), coalesced stores.
__global__ void __launch_bounds__(256) k_deriv(const __grid_constant__ DerivParams p)
{
    extern __shared__ __align__(16) double2 sm[];
    const int nn = p.nn, ld = nn | 1;
    const int cpm = (p.lines_per_mode + p.lpb - 1) / p.lpb;
    const int mode = blockIdx.x / cpm;
    const int q0 = (blockIdx.x - mode * cpm) * p.lpb;
    const int nl = min(p.lpb, p.lines_per_mode - q0);
    const long long base = mode * p.mode_stride + (long long)q0 * p.line_stride;
    const double2 *U = reinterpret_cast<const double2 *>(p.u) + base;
    double2 *DU = reinterpret_cast<double2 *>(p.du) + base;
    const bool contiguous = (p.elem_stride == 1);
    for (int idx = threadIdx.x; idx < nl * nn; idx += blockDim.x) {
        int l, k;
        if (contiguous) { l = idx / nn; k = idx - l * nn; }
        else { k = idx / nl; l = idx - k * nl; }
        cp_async16(sm + l * ld + k, U + l * p.line_stride + (long long)k * p.elem_stride);
    }
    cp_async_wait_all();
    __syncthreads();
    if (threadIdx.x < nl) {
        double2 *c = sm + threadIdx.x * ld;
        if (p.ider == 1) {
            deriv_rec(c, 1, c, 1, nn, p.fac, false);
        } else {
            deriv_rec(c, 1, c, 1, nn, 1.0, false);
            deriv_rec(c, 1, c, 1, nn, p.fac, false);
        }
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < nl * nn; idx += blockDim.x) {
        int l, k;
        if (contiguous) { l = idx / nn; k = idx - l * nn; }
        else { k = idx / nl; l = idx - k * nl; }
        const long long g = l * p.line_stride + (long long)k * p.elem_stride;
        const double2 v = sm[l * ld + k];
        DU[g] = p.accumulate ? make_double2(DU[g].x + v.x, DU[g].y + v.y) : v;
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
    p.iopt = iopt;
    // the half-length DCT where a plan exists, then the two-pass register
    // FFT of the even extension, else the radix stages
    {
        const int rc = dcth_dispatch(ctx, p, nmodes);
        if (rc >= 0) return rc;
    }
    {
        const int rc = dct2_dispatch(ctx, p, nmodes);
        if (rc >= 0) return rc;
    }
    // lines per CTA: two line buffers + the twiddle table in ~100 KB, so
    // two CTAs share an SM
    p.lpb = (int)((100 * 1024 / sizeof(double2) - p.L) / (2 * (p.L + 1)));
    if (p.lpb < 1) p.lpb = 1;
    if (p.lpb > 32) p.lpb = 32;
    if (p.lpb > p.lines_per_mode) p.lpb = p.lines_per_mode;
    p.iopt = iopt;
    const size_t smem = (2 * (size_t)p.lpb * (p.L + 1) + p.L) * sizeof(double2);
    DUCT_CUDA(ctx, cudaFuncSetAttribute(k_dct, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int grid = nmodes * ((p.lines_per_mode + p.lpb - 1) / p.lpb);
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
    p.lpb = (cdir == 'y') ? kDerivLinesY : kDerivLinesZ;
    const size_t smem = (size_t)p.lpb * (p.nn | 1) * sizeof(double2);
    DUCT_CUDA(ctx, cudaFuncSetAttribute(k_deriv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int grid = nmodes * ((p.lines_per_mode + p.lpb - 1) / p.lpb);
    {
        LaunchScope ls(ctx, DUCTGPU_K_TRANSFORM);
        k_deriv<<<grid, 256, smem, ctx->stream>>>(p);
    }
    return check_cuda(ctx, cudaGetLastError(), "k_deriv");
}

int transpose_dev(ductgpu_ctx ctx, const double *in, double *out, long long A, long long Q)
{
    // the TMA form where a tensor map describes the arrays, else 32 x 32
    // tiles through shared memory
    const int rt = transpose_tma(ctx, in, out, A, Q);
    if (rt >= 0) return rt;
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
