// cheb_lines.cu -- fused Chebyshev derivative lines with a pointwise
// epilogue (FP64), the workhorse of the operators around the solve.
//
// The reference differentiates along y or z in three full passes over a
// field: transyz(f,cdir,-1) to Chebyshev coefficients, derivyz (the
// backward recurrence once or twice), transyz(out,cdir,+1) back to the
// nodes, and then a daxpy into the target (e.g. laplacian3d / grad3d /
// div3d / update_uvwp, src/operators.F:278-605, and the y / z terms of
// advection3d, src/operators.F:9-276).  Here one kernel does all of it per
// line in shared memory: a field is read once, every output is written
// once, and the x-derivative terms (derivx, src/fourier.F:120-188: i kx f
// and -kx^2 f) and the daxpy / dscal combinations of the RK3/CN substep
// (src/main1.f90:384-723) are folded into the store:
//
//   out = sigma * (beta * out + fac * D^order(in) + sum_t (c0_t + c1_t i kx
//                  + c2_t (i kx)^2) src_t + [mode 0] m0)
//
// D^order is the reference's derivative: transyz -1 (DCT-I, ends 1/N,
// interior 2/N), the recurrence d_{k-1} = d_{k+1} + 2k c_k with the sign of
// the solver grid x = -cos (out_k = -d_k, out_0 = -d_0/2), applied `order`
// times, then transyz +1.  The DCT-I is the half-length form (one complex
// FFT of N points for the real and imaginary lines at once, Press et al.,
// Numerical Recipes sec. 12.3; the same transform as transforms.cu's k_dcth),
// and both scans of the recurrence (one per parity class) run across a warp
// with shuffles.  A job may produce two outputs from one input line (e.g.
// phi_y and phi_yy of update_uvwp): one forward transform, both recurrences,
// one inverse per output.
#include "fft.cuh"
#include "internal.h"

namespace duct {

// Scans of the forward / inverse post-step and of the recurrence, and the
// forward / inverse pre-step, one warp per line.  Layout of a line in the
// FFT buffer: point j at j + j / R2 (a pad word every R2 points), point N
// last.

// Forward pre-step on the staged line in x (in place):
//   g_0 = (x_0 + x_N)/2, g_{N/2} = x_{N/2},
//   g_j = (x_j + x_{N-j})/2 - sin(pi j/N)(x_j - x_{N-j}),
//   F_1 = (x_0 - x_N)/2 + sum_{j=1}^{N/2-1} cos(pi j/N)(x_j - x_{N-j}).
// src (natural order, or null for x itself) gives the inverse's input,
// whose two ends count twice (y_0 = 2 c_0, y_N = 2 c_N).
template <int R2, int N>
__device__ __forceinline__ void pre_step(double2 *xl, const double2 *src, const double2 *ha, double2 &f1, int lane)
{
    auto at = [](int j) { return j + j / R2; };
    double sx = 0.0, sy = 0.0;
    for (int j = 1 + lane; j < N / 2; j += 32) {
        const double2 a = src ? src[j] : xl[at(j)], b = src ? src[N - j] : xl[at(N - j)];
        const double2 u = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y + b.y));
        const double2 v = make_double2(a.x - b.x, a.y - b.y);
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
        double2 x0, xn, xm;
        if (src) {
            x0 = make_double2(2.0 * src[0].x, 2.0 * src[0].y);
            xn = make_double2(2.0 * src[N].x, 2.0 * src[N].y);
            xm = src[N / 2];
        } else {
            x0 = xl[at(0)];
            xn = xl[at(N)];
            xm = xl[at(N / 2)];
        }
        f1 = make_double2(0.5 * (x0.x - xn.x) + sx, 0.5 * (x0.y - xn.y) + sy);
        xl[at(0)] = make_double2(0.5 * (x0.x + xn.x), 0.5 * (x0.y + xn.y));
        xl[at(N / 2)] = xm;
    }
}

// Length-N FFT of every line in place: R1-point DFTs along n1 (column n2)
// with the twiddle W_N^(n2 k1), then R2-point DFTs along each row k1.
template <int R1, int R2, int NT, int LPB, int LS>
__device__ __forceinline__ void fft_lines(double2 *x, const double2 *tw)
{
    constexpr int N = R1 * R2;
    auto at = [](int j) { return j + j / R2; };
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
}

// Post-step: F_{2k} = (G_k + G_{N-k})/2, F_{2k+1} = F_1 + sum_{m=1}^{k}
// i (G_m - G_{N-m})/2 (a warp scan of the increments).  nat != null: the
// coefficients c = scale F (ends 1/N, interior 2/N: transyz -1) in natural
// order into nat; else F in place in slot order (F_{2k} in slot k,
// F_{2k+1} in slot N - k, F_1 in slot N).
template <int R2, int N>
__device__ __forceinline__ void post_step(double2 *xl, double2 *nat, double2 f1, int lane)
{
    auto at = [](int j) { return j + j / R2; };
    constexpr int CH = (N / 2 + 1 + 31) / 32;
    const int k0 = lane * CH, k1 = min(N / 2 + 1, k0 + CH);
    double sx = 0.0, sy = 0.0;
    for (int k = k0; k < k1; ++k) {
        if (k == 0 || k == N / 2) continue;
        const double2 gk = xl[at(k)], gm = xl[at(N - k)];
        sx -= 0.5 * (gk.y - gm.y);
        sy += 0.5 * (gk.x - gm.x);
    }
    double ix = sx, iy = sy;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double tx = __shfl_up_sync(0xffffffffu, ix, o), ty = __shfl_up_sync(0xffffffffu, iy, o);
        if (lane >= o) {
            ix += tx;
            iy += ty;
        }
    }
    double rx = f1.x + ix - sx, ry = f1.y + iy - sy;
    constexpr double s_in = 2.0 / N, s_end = 1.0 / N;
    for (int k = k0; k < k1; ++k) {
        const double2 gk = xl[at(k)], gm = xl[at(k == 0 ? 0 : N - k)];
        const double2 fe = make_double2(0.5 * (gk.x + gm.x), 0.5 * (gk.y + gm.y));
        if (k > 0 && k < N / 2) {
            rx -= 0.5 * (gk.y - gm.y);
            ry += 0.5 * (gk.x - gm.x);
        }
        if (nat) {
            const double se = (k == 0 || k == N / 2) ? s_end : s_in;
            nat[2 * k] = make_double2(se * fe.x, se * fe.y);
            if (k < N / 2) nat[2 * k + 1] = make_double2(s_in * rx, s_in * ry);
        } else {
            xl[at(k)] = fe;
            if (k > 0 && k < N / 2) xl[at(N - k)] = make_double2(rx, ry);
        }
    }
    if (!nat && lane == 0) xl[at(N)] = f1;
}

// Derivative recurrence on a natural-order coefficient line s -> t:
//   e_k = sum_{j >= k, j = k mod 2} 2 j s_j,  t_m = -e_{m+1} (m >= 1),
//   t_0 = -e_1 / 2, t_N = 0
// (src/chebyshev.f90:44-58; e_k is the reference's running value cri).
// Lane q owns k in [1 + q CH, 1 + (q + 1) CH); the two parity classes are
// suffix-scanned across the warp.
template <int N>
__device__ __forceinline__ void recurrence(const double2 *s, double2 *t, int lane)
{
    constexpr int CH = (N + 31) / 32;
    const int k0 = 1 + lane * CH, k1 = min(N + 1, k0 + CH);
    double2 se = make_double2(0.0, 0.0), so = se;
    for (int k = k0; k < k1; ++k) {
        const double2 v = s[k];
        const double f = 2.0 * k;
        if (k & 1) { so.x += f * v.x; so.y += f * v.y; }
        else { se.x += f * v.x; se.y += f * v.y; }
    }
    double2 ie = se, io = so;   // inclusive suffix sums over lanes >= lane
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double ax = __shfl_down_sync(0xffffffffu, ie.x, o), ay = __shfl_down_sync(0xffffffffu, ie.y, o);
        const double bx = __shfl_down_sync(0xffffffffu, io.x, o), by = __shfl_down_sync(0xffffffffu, io.y, o);
        if (lane + o < 32) {
            ie.x += ax; ie.y += ay;
            io.x += bx; io.y += by;
        }
    }
    double2 re = make_double2(ie.x - se.x, ie.y - se.y), ro = make_double2(io.x - so.x, io.y - so.y);
    for (int k = k1 - 1; k >= k0; --k) {
        const double2 v = s[k];
        const double f = 2.0 * k;
        double2 e;
        if (k & 1) { ro.x += f * v.x; ro.y += f * v.y; e = ro; }
        else { re.x += f * v.x; re.y += f * v.y; e = re; }
        const double h = (k == 1) ? -0.5 : -1.0;
        t[k - 1] = make_double2(h * e.x, h * e.y);
    }
    if (lane == 0) t[N] = make_double2(0.0, 0.0);
}

struct LineGeom {
    long long ls, es, ms;   // complex strides: line, element, mode
    int lpm;                // lines per mode
};

__device__ __forceinline__ double2 xterm_coef(const LineOut &o, int t, double kx)
{
    // (c0 + c1 i kx + c2 (i kx)^2)
    return make_double2(o.xc0[t] - o.xc2[t] * kx * kx, o.xc1[t] * kx);
}

__device__ __forceinline__ void atomic_max_nonneg(double *a, double v)
{
    atomicMax(reinterpret_cast<unsigned long long *>(a), (unsigned long long)__double_as_longlong(v));
}

// Stores one output of a CTA's lines.  slotted: the transform's result in
// slot order in x (null for an order-0 output).
template <int R2, int N, int NT, int LPB, int LS>
__device__ __forceinline__ void store_output(const LineOut &o, const double2 *x, bool contiguous, const LineGeom &g,
                                             long long base, int nl, int q0, int mode, double kx, bool real0)
{
    auto at = [](int j) { return j + j / R2; };
    double2 *out = reinterpret_cast<double2 *>(o.out) + base;
    double2 cf[kLineXTerms];
    const double2 *xs[kLineXTerms];
#pragma unroll
    for (int t = 0; t < kLineXTerms; ++t) {
        cf[t] = xterm_coef(o, t, kx);
        xs[t] = o.xs[t] ? reinterpret_cast<const double2 *>(o.xs[t]) + base : nullptr;
    }
    const double m0 = (mode == 0) ? o.m0 : 0.0;
    const bool deriv = o.order > 0;
    double vmax = 0.0;
    auto one = [&](int l, int j) {
        const long long gi = l * g.ls + (long long)j * g.es;
        double2 v = make_double2(m0, 0.0);
        if (deriv) {
            const int slot = (j & 1) ? N - (j >> 1) : (j >> 1);
            const double2 f = x[l * LS + at(slot)];
            v.x += o.fac * f.x;
            // the real and imaginary lines share one FFT; a real mode-0
            // line keeps an exactly real derivative, as with real DCTs
            if (!real0) v.y += o.fac * f.y;
        }
#pragma unroll
        for (int t = 0; t < kLineXTerms; ++t)
            if (xs[t]) {
                const double2 s = xs[t][gi];
                v.x += cf[t].x * s.x - cf[t].y * s.y;
                v.y += cf[t].x * s.y + cf[t].y * s.x;
            }
        if (o.beta != 0.0) {
            const double2 w = out[gi];
            v.x += o.beta * w.x;
            v.y += o.beta * w.y;
        }
        v.x *= o.sigma;
        v.y *= o.sigma;
        out[gi] = v;
        if (o.maxabs && j > 0 && j < N && q0 + l > 0 && q0 + l < g.lpm - 1) vmax = fmax(vmax, hypot(v.x, v.y));
    };
    if (contiguous) {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        for (int l = warp; l < nl; l += NT / 32)
            for (int j = lane; j <= N; j += 32) one(l, j);
    } else {
        for (int idx = threadIdx.x; idx < LPB * (N + 1); idx += NT) {
            const int j = idx / LPB, l = idx - j * LPB;
            if (l < nl) one(l, j);
        }
    }
    if (o.maxabs) {
#pragma unroll
        for (int s = 16; s > 0; s >>= 1) vmax = fmax(vmax, __shfl_xor_sync(0xffffffffu, vmax, s));
        if ((threadIdx.x & 31) == 0 && vmax > 0.0) atomic_max_nonneg(o.maxabs, vmax);
    }
}

template <int R1, int R2, int NT>
__global__ void __launch_bounds__(NT) k_lines(const __grid_constant__ LineParams p, const double2 *__restrict__ twg,
                                              const double2 *__restrict__ tw2g)
{
    constexpr int N = R1 * R2, NN = N + 1, LS = R1 * (R2 + 1) + 1;
    constexpr int LPB = NT / (R1 > R2 ? R1 : R2), NW = NT / 32;
    extern __shared__ __align__(16) double2 sm[];
    double2 *tw = sm;                   // W_N^t, N entries
    double2 *ha = tw + N;               // (cos, -sin)(pi j / N), j <= N/2
    double2 *x = ha + (N / 2 + 1);      // [LPB][LS] FFT buffer
    double2 *c = x + LPB * LS;          // [LPB][NN] coefficients, then order-2 coefficients
    double2 *d = c + LPB * NN;          // [LPB][NN] order-1 coefficients
    double2 *f1 = d + LPB * NN;         // [LPB]
    auto at = [](int j) { return j + j / R2; };

    const int job = blockIdx.x / p.ctas_per_job;
    const int r = blockIdx.x - job * p.ctas_per_job;
    const LineJob &J = p.job[job];
    LineGeom g;
    const bool contiguous = (p.dir == 'y');
    g.ms = (long long)p.my * p.mz;
    if (contiguous) { g.ls = p.my; g.es = 1; g.lpm = p.mz; }
    else { g.ls = 1; g.es = p.my; g.lpm = p.my; }
    const int cpm = (g.lpm + LPB - 1) / LPB;
    const int mode = r / cpm;
    const int q0 = (r - mode * cpm) * LPB;
    const int nl = min(LPB, g.lpm - q0);
    const long long base = mode * g.ms + (long long)q0 * g.ls;
    const double kx = p.xalp[mode];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

    bool any_deriv = false, need2 = false;
    for (int k = 0; k < J.nout; ++k) {
        any_deriv |= J.o[k].order > 0;
        need2 |= J.o[k].order == 2;
    }
    if (any_deriv) {
        const double2 *in = reinterpret_cast<const double2 *>(J.in) + base;
        if (contiguous) {
            for (int l = warp; l < nl; l += NW)
                for (int j = lane; j <= N; j += 32) cp_async16(x + l * LS + at(j), in + l * g.ls + j);
        } else {
            for (int idx = threadIdx.x; idx < LPB * NN; idx += NT) {
                const int j = idx / LPB, l = idx - j * LPB;
                if (l < nl) cp_async16(x + l * LS + at(j), in + l + (long long)j * g.es);
            }
        }
        for (int t = threadIdx.x; t < N; t += NT) cp_async16(tw + t, twg + t);
        for (int t = threadIdx.x; t <= N / 2; t += NT) cp_async16(ha + t, tw2g + t);
        cp_async_wait_all();
        __syncthreads();
        // forward transform -> c (natural order, transyz -1 scaling)
        for (int l = warp; l < LPB; l += NW) {
            double2 *xl = x + l * LS;
            if (l >= nl) {
                for (int j = lane; j < LS; j += 32) xl[j] = make_double2(0.0, 0.0);
                continue;
            }
            pre_step<R2, N>(xl, nullptr, ha, f1[l], lane);
        }
        __syncthreads();
        fft_lines<R1, R2, NT, LPB, LS>(x, tw);
        for (int l = warp; l < nl; l += NW) post_step<R2, N>(x + l * LS, c + l * NN, f1[l], lane);
        __syncthreads();
        // order 1 -> d; order 2 -> c (over the coefficients, no longer needed)
        for (int l = warp; l < nl; l += NW) {
            recurrence<N>(c + l * NN, d + l * NN, lane);
            __syncwarp();
            if (need2) recurrence<N>(d + l * NN, c + l * NN, lane);
        }
        __syncthreads();
    }
    for (int oi = 0; oi < J.nout; ++oi) {
        const LineOut &o = J.o[oi];
        if (o.order > 0) {
            const double2 *y = (o.order == 1) ? d : c;
            for (int l = warp; l < LPB; l += NW) {
                if (l >= nl) continue;   // zeroed above; the FFT of zeros stays zero
                pre_step<R2, N>(x + l * LS, y + l * NN, ha, f1[l], lane);
            }
            __syncthreads();
            fft_lines<R1, R2, NT, LPB, LS>(x, tw);
            for (int l = warp; l < nl; l += NW) post_step<R2, N>(x + l * LS, nullptr, f1[l], lane);
            __syncthreads();
        }
        store_output<R2, N, NT, LPB, LS>(o, x, contiguous, g, base, nl, q0, mode, kx, p.real0 && mode == 0);
        __syncthreads();
    }
}

const double2 *twiddle_table(ductgpu_ctx ctx, int L);

template <int R1, int R2, int NT>
static int launch_lines(ductgpu_ctx ctx, const LineParams &p0)
{
    constexpr int N = R1 * R2, NN = N + 1, LS = R1 * (R2 + 1) + 1;
    constexpr int LPB = NT / (R1 > R2 ? R1 : R2);
    const double2 *tw = twiddle_table(ctx, N);
    const double2 *tw2 = twiddle_table(ctx, 2 * N);
    if (!tw || !tw2)
        return set_error(ctx, DUCTGPU_ESTATE, "lines: twiddle tables for N=%d unavailable%s", N,
                         ctx->capturing ? " (first use inside a capture)" : "");
    LineParams p = p0;
    const int lpm = (p.dir == 'y') ? p.mz : p.my;
    p.ctas_per_job = p.nmodes * ((lpm + LPB - 1) / LPB);
    const size_t smem = ((size_t)N + (N / 2 + 1) + (size_t)LPB * LS + 2 * (size_t)LPB * NN + LPB) * sizeof(double2);
    DUCT_CUDA(ctx, cudaFuncSetAttribute(k_lines<R1, R2, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const long long grid = (long long)p.ctas_per_job * p.njobs;
    if (grid > 0x7fffffffLL) return set_error(ctx, DUCTGPU_EARG, "lines: grid too large");
    {
        LaunchScope ls(ctx, DUCTGPU_K_LINES);
        k_lines<R1, R2, NT><<<(unsigned)grid, NT, smem, ctx->stream>>>(p, tw, tw2);
    }
    return check_cuda(ctx, cudaGetLastError(), "k_lines");
}

bool lines_supported(int nn)
{
    switch (nn - 1) {
    case 16: case 24: case 32: case 48: case 64: case 96: case 128: case 144: case 192: case 256: return true;
    default: return false;
    }
}

int lines_launch(ductgpu_ctx ctx, const LineParams &p)
{
    if (p.njobs < 1 || p.njobs > kMaxLineJobs) return set_error(ctx, DUCTGPU_EARG, "lines: %d jobs", p.njobs);
    if (p.dir != 'y' && p.dir != 'z') return set_error(ctx, DUCTGPU_EARG, "lines: direction '%c'", p.dir);
    if (!p.xalp || p.nmodes < 1) return set_error(ctx, DUCTGPU_EARG, "lines: modes");
    for (int i = 0; i < p.njobs; ++i) {
        const LineJob &J = p.job[i];
        if (J.nout < 1 || J.nout > kMaxLineOut) return set_error(ctx, DUCTGPU_EARG, "lines: job %d has %d outputs", i, J.nout);
        for (int k = 0; k < J.nout; ++k) {
            if (!J.o[k].out || J.o[k].order < 0 || J.o[k].order > 2)
                return set_error(ctx, DUCTGPU_EARG, "lines: job %d output %d", i, k);
            if (J.o[k].order > 0 && !J.in) return set_error(ctx, DUCTGPU_EARG, "lines: job %d has no input", i);
        }
    }
    const int nn = (p.dir == 'y') ? p.my : p.mz;
    switch (nn - 1) {
    case 16: return launch_lines<4, 4, 64>(ctx, p);
    case 24: return launch_lines<4, 6, 64>(ctx, p);
    case 32: return launch_lines<4, 8, 64>(ctx, p);
    case 48: return launch_lines<6, 8, 64>(ctx, p);
    case 64: return launch_lines<8, 8, 64>(ctx, p);
    case 96: return launch_lines<8, 12, 64>(ctx, p);
    case 128: return launch_lines<8, 16, 64>(ctx, p);
    case 144: return launch_lines<12, 12, 64>(ctx, p);
    case 192: return launch_lines<12, 16, 64>(ctx, p);
    case 256: return launch_lines<16, 16, 64>(ctx, p);
    default:
        return set_error(ctx, DUCTGPU_EARG, "lines: line length %d - 1 is not one of 16, 24, 32, 48, 64, 96, 128, "
                         "144, 192, 256", nn);
    }
}

}  // namespace duct
