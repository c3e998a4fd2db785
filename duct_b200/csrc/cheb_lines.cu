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
// and both scans of the recurrence (one per parity class) run across the
// lanes that own the line with shuffles.  A job may produce up to three
// outputs from one input line (e.g. p, v and u of update_uvwp): one forward
// transform, the recurrences, one inverse per derivative output.
//
// Work split: a line belongs to a segment of LPL consecutive lanes (16 for
// N = 96..256, 8 or 4 below), so a warp carries 32 / LPL lines through the
// whole chain on its own -- warp-synchronous, with no CTA barrier after the
// twiddle tables are loaded -- and many independent warps per SM hide the
// FP64 and shared-memory latencies of the short dependent phases (pre-step,
// two FFT steps, scans).  The two lines of a warp are neighbours (z and
// z + 1 for y lines, y and y + 1 for z lines), so the strided accesses of
// z lines still move whole 32-byte sectors.
#include "fft.cuh"
#include "internal.h"

namespace duct {

// Shuffles within a segment of W lanes.
template <int W>
__device__ __forceinline__ double seg_sum(double v)
{
#pragma unroll
    for (int o = W / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, W);
    return v;
}

// Chunk of a scan over n values on W lanes, rounded up to an odd count:
// lanes then start their chunks on distinct 16-byte banks of a quarter warp.
__host__ __device__ constexpr int odd_chunk(int n, int w) { return ((n + w - 1) / w) | 1; }

// Layout of a line in its FFT buffer: point j at j + j / R2 (a pad word every
// R2 points), point N last.
template <int R2>
__device__ __forceinline__ int at(int j) { return j + j / R2; }

// Pre-step, in place on the staged line (src null) or from a natural-order
// line src -- the staged physical line, or (DOUBLE_ENDS) a coefficient line
// whose two ends count twice (y_0 = 2 c_0, y_N = 2 c_N):
//   g_0 = (x_0 + x_N)/2, g_{N/2} = x_{N/2},
//   g_j = (x_j + x_{N-j})/2 - sin(pi j/N)(x_j - x_{N-j}),
//   F_1 = (x_0 - x_N)/2 + sum_{j=1}^{N/2-1} cos(pi j/N)(x_j - x_{N-j}) -> *f1.
template <int R2, int N, int W, bool DOUBLE_ENDS>
__device__ __forceinline__ void pre_seg(double2 *xl, const double2 *src, const double2 *ha, double2 *f1, int s)
{
    double sx = 0.0, sy = 0.0;
    constexpr int IT = (N / 2 - 1 + W - 1) / W;
#pragma unroll
    for (int it = 0; it < IT; ++it) {
        const int j = 1 + s + it * W;
        if (j >= N / 2) break;
        const double2 a = src ? src[j] : xl[at<R2>(j)], b = src ? src[N - j] : xl[at<R2>(N - j)];
        const double2 u = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y + b.y));
        const double2 v = make_double2(a.x - b.x, a.y - b.y);
        const double2 w = ha[j];   // (cos(pi j/N), -sin(pi j/N))
        xl[at<R2>(j)] = make_double2(u.x + w.y * v.x, u.y + w.y * v.y);
        xl[at<R2>(N - j)] = make_double2(u.x - w.y * v.x, u.y - w.y * v.y);
        sx += w.x * v.x;
        sy += w.x * v.y;
    }
    sx = seg_sum<W>(sx);
    sy = seg_sum<W>(sy);
    if (s == 0) {
        double2 x0, xn, xm;
        if (src) {
            const double e = DOUBLE_ENDS ? 2.0 : 1.0;
            x0 = make_double2(e * src[0].x, e * src[0].y);
            xn = make_double2(e * src[N].x, e * src[N].y);
            xm = src[N / 2];
        } else {
            x0 = xl[at<R2>(0)];
            xn = xl[at<R2>(N)];
            xm = xl[at<R2>(N / 2)];
        }
        *f1 = make_double2(0.5 * (x0.x - xn.x) + sx, 0.5 * (x0.y - xn.y) + sy);
        xl[at<R2>(0)] = make_double2(0.5 * (x0.x + xn.x), 0.5 * (x0.y + xn.y));
        xl[at<R2>(N / 2)] = xm;
    }
    __syncwarp();
}

// Length-N FFT of a line in place (N = R1 R2, R1, R2 <= W): lane n2 runs the
// R1-point DFT of column n2 and applies W_N^(n2 k1), then lane k1 the
// R2-point DFT of row k1.
// twT[k1 R2 + n2] = W_N^(n2 k1): the inter-step twiddles laid out so that
// the lanes of a segment (n2) read consecutive words.
template <int R1, int R2, int W>
__device__ __forceinline__ void fft_seg(double2 *xl, const double2 *tw, const double2 *twT, int s)
{
    constexpr int N = R1 * R2;
    if (s < R2) {
        double2 v[R1];
#pragma unroll
        for (int n1 = 0; n1 < R1; ++n1) v[n1] = xl[n1 * (R2 + 1) + s];
        reg_fft<R1, 0, 1>(v, tw, N);
#pragma unroll
        for (int k1 = 0; k1 < R1; ++k1) xl[k1 * (R2 + 1) + s] = (k1 == 0) ? v[0] : cmul(v[k1], twT[k1 * R2 + s]);
    }
    __syncwarp();
    double2 w[R2];
    if (s < R1) {
#pragma unroll
        for (int n2 = 0; n2 < R2; ++n2) w[n2] = xl[s * (R2 + 1) + n2];
        reg_fft<R2, 0, 1>(w, tw, N);
    }
    __syncwarp();
    if (s < R1) {
#pragma unroll
        for (int k2 = 0; k2 < R2; ++k2) xl[at<R2>(s + R1 * k2)] = w[k2];
    }
    __syncwarp();
}

// Post-step: F_{2k} = (G_k + G_{N-k})/2, F_{2k+1} = F_1 + sum_{m=1}^{k}
// i (G_m - G_{N-m})/2 (a scan of the increments over the segment).  nat !=
// null: the coefficients c = scale F (ends 1/N, interior 2/N: transyz -1)
// in natural order into nat; else F in place in slot order (F_{2k} in slot
// k, F_{2k+1} in slot N - k, F_1 in slot N).
template <int R2, int N, int W>
__device__ __forceinline__ void post_seg(double2 *xl, double2 *nat, double2 f1, int s)
{
    constexpr int CH = odd_chunk(N / 2 + 1, W);
    const int k0 = s * CH, k1 = min(N / 2 + 1, k0 + CH);
    double sx = 0.0, sy = 0.0;
#pragma unroll
    for (int i = 0; i < CH; ++i) {
        const int k = k0 + i;
        if (k >= k1) break;
        if (k == 0 || k == N / 2) continue;
        const double2 gk = xl[at<R2>(k)], gm = xl[at<R2>(N - k)];
        sx -= 0.5 * (gk.y - gm.y);
        sy += 0.5 * (gk.x - gm.x);
    }
    double ix = sx, iy = sy;
#pragma unroll
    for (int o = 1; o < W; o <<= 1) {
        const double tx = __shfl_up_sync(0xffffffffu, ix, o, W), ty = __shfl_up_sync(0xffffffffu, iy, o, W);
        if (s >= o) {
            ix += tx;
            iy += ty;
        }
    }
    double rx = f1.x + ix - sx, ry = f1.y + iy - sy;
    constexpr double s_in = 2.0 / N, s_end = 1.0 / N;
#pragma unroll
    for (int i = 0; i < CH; ++i) {
        const int k = k0 + i;
        if (k >= k1) break;
        const double2 gk = xl[at<R2>(k)], gm = xl[at<R2>(k == 0 ? 0 : N - k)];
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
            xl[at<R2>(k)] = fe;
            if (k > 0 && k < N / 2) xl[at<R2>(N - k)] = make_double2(rx, ry);
        }
    }
    if (!nat && s == 0) xl[at<R2>(N)] = f1;
    __syncwarp();
}

// Derivative recurrence in place on a natural-order coefficient line:
//   e_k = sum_{j >= k, j = k mod 2} 2 j c_j,  c_m <- -e_{m+1} (m >= 1),
//   c_0 <- -e_1 / 2, c_N <- 0
// (src/chebyshev.f90:44-58; e_k is the reference's running value cri).
// Lane s owns k in [1 + s CH, 1 + (s + 1) CH): a first pass sums its chunk
// per parity class, the sums are suffix-scanned over the segment, and a
// backward pass writes c[k-1], reading c[k-1] just before.  The only
// element a lane overwrites in another lane's chunk is that lane's top one,
// which every lane keeps in a register before the warp barrier.
template <int N, int W>
__device__ __forceinline__ void rec_seg(double2 *c, int s)
{
    constexpr int CH = odd_chunk(N, W);
    const int k0 = 1 + s * CH, k1 = min(N + 1, k0 + CH);
    double2 se = make_double2(0.0, 0.0), so = se, top = se;
#pragma unroll
    for (int i = 0; i < CH; ++i) {
        const int k = k0 + i;
        if (k >= k1) break;
        const double2 v = c[k];
        const double f = 2.0 * k;
        if (k & 1) { so.x += f * v.x; so.y += f * v.y; }
        else { se.x += f * v.x; se.y += f * v.y; }
        top = v;
    }
    double2 ie = se, io = so;   // inclusive suffix sums over lanes >= s
#pragma unroll
    for (int o = 1; o < W; o <<= 1) {
        const double ax = __shfl_down_sync(0xffffffffu, ie.x, o, W), ay = __shfl_down_sync(0xffffffffu, ie.y, o, W);
        const double bx = __shfl_down_sync(0xffffffffu, io.x, o, W), by = __shfl_down_sync(0xffffffffu, io.y, o, W);
        if (s + o < W) {
            ie.x += ax; ie.y += ay;
            io.x += bx; io.y += by;
        }
    }
    double2 re = make_double2(ie.x - se.x, ie.y - se.y), ro = make_double2(io.x - so.x, io.y - so.y);
    __syncwarp();
    double2 cur = top;
#pragma unroll
    for (int i = CH - 1; i >= 0; --i) {
        const int k = k0 + i;
        if (k >= k1) continue;
        const double2 v = cur;
        if (k > k0) cur = c[k - 1];   // read before this iteration overwrites it
        const double f = 2.0 * k;
        double2 e;
        if (k & 1) { ro.x += f * v.x; ro.y += f * v.y; e = ro; }
        else { re.x += f * v.x; re.y += f * v.y; e = re; }
        const double h = (k == 1) ? -0.5 : -1.0;
        c[k - 1] = make_double2(h * e.x, h * e.y);
    }
    if (s == 0) c[N] = make_double2(0.0, 0.0);
    __syncwarp();
}

__device__ __forceinline__ double2 xterm_coef(const LineOut &o, int t, double kx)
{
    // (c0 + c1 i kx + c2 (i kx)^2)
    return make_double2(o.xc0[t] - o.xc2[t] * kx * kx, o.xc1[t] * kx);
}

// Stores one output of a line.  deriv: the transform's result in slot order
// in xl.  maxabs: the interior points' max |out|, reduced over the warp.
template <int R2, int N, int W>
__device__ __forceinline__ void store_seg(const LineOut &o, const double2 *xl, bool deriv, long long lbase,
                                          long long es, bool act, bool interior_line, int mode, double kx, bool real0,
                                          int s)
{
    double vmax = 0.0;
    if (act) {
        double2 *out = reinterpret_cast<double2 *>(o.out) + lbase;
        double2 cf[kLineXTerms];
        const double2 *xs[kLineXTerms];
#pragma unroll
        for (int t = 0; t < kLineXTerms; ++t) {
            cf[t] = xterm_coef(o, t, kx);
            xs[t] = o.xs[t] ? reinterpret_cast<const double2 *>(o.xs[t]) + lbase : nullptr;
        }
        const double m0 = (mode == 0) ? o.m0 : 0.0;
#pragma unroll 4
        for (int j = s; j <= N; j += W) {
            const long long gi = (long long)j * es;
            double2 v = make_double2(m0, 0.0);
            if (deriv) {
                const int slot = (j & 1) ? N - (j >> 1) : (j >> 1);
                const double2 f = xl[at<R2>(slot)];
                v.x += o.fac * f.x;
                // the real and imaginary lines share one FFT; a real mode-0
                // line keeps an exactly real derivative, as with real DCTs
                if (!real0) v.y += o.fac * f.y;
            }
#pragma unroll
            for (int t = 0; t < kLineXTerms; ++t)
                if (xs[t]) {
                    const double2 sv = xs[t][gi];
                    v.x += cf[t].x * sv.x - cf[t].y * sv.y;
                    v.y += cf[t].x * sv.y + cf[t].y * sv.x;
                }
            if (o.beta != 0.0) {
                const double2 w = out[gi];
                v.x += o.beta * w.x;
                v.y += o.beta * w.y;
            }
            v.x *= o.sigma;
            v.y *= o.sigma;
            out[gi] = v;
            if (interior_line && j > 0 && j < N) vmax = fmax(vmax, hypot(v.x, v.y));
        }
    }
    if (o.maxabs) {
#pragma unroll
        for (int t = 16; t > 0; t >>= 1) vmax = fmax(vmax, __shfl_xor_sync(0xffffffffu, vmax, t));
        if ((threadIdx.x & 31) == 0 && vmax > 0.0)
            atomicMax(reinterpret_cast<unsigned long long *>(o.maxabs), (unsigned long long)__double_as_longlong(vmax));
    }
}

// Shared memory per line: the FFT buffer (LS), the coefficients (N + 1; also
// the landing place of the next line's prefetch) and F_1.
template <int R1, int R2>
struct LineShape {
    static constexpr int N = R1 * R2, NN = N + 1, LS = R1 * (R2 + 1) + 1, PL = LS + NN + 1;
};

template <int R1, int R2, int W, int WPB>
__global__ void __launch_bounds__(32 * WPB, 16 / WPB) k_lines(const __grid_constant__ LineParams p,
                                                              const double2 *__restrict__ twg,
                                                              const double2 *__restrict__ tw2g)
{
    using S = LineShape<R1, R2>;
    constexpr int N = S::N, LS = S::LS, PL = S::PL, LPW = 32 / W, NT = 32 * WPB;
    extern __shared__ __align__(16) double2 sm[];
    double2 *tw = sm;                   // W_N^t, N entries
    double2 *twT = tw + N;              // W_N^(n2 k1) at k1 R2 + n2, N entries
    double2 *ha = twT + N;              // (cos, -sin)(pi j / N), j <= N/2
    double2 *lines = ha + (N / 2 + 1);  // [WPB * LPW][PL]
    for (int t = threadIdx.x; t < N; t += NT) {
        tw[t] = twg[t];
        const int k1 = t / R2, n2 = t - k1 * R2;
        twT[t] = twg[(n2 * k1) % N];
    }
    for (int t = threadIdx.x; t <= N / 2; t += NT) ha[t] = tw2g[t];
    __syncthreads();

    // persistent warps over work items = (job, mode, pair of neighbouring lines)
    const bool ydir = (p.dir == 'y');
    const long long ms = (long long)p.my * p.mz;
    const long long ls = ydir ? p.my : 1, es = ydir ? 1 : p.my;
    const int lpm = ydir ? p.mz : p.my;
    const int gpm = (lpm + LPW - 1) / LPW;              // line groups per mode
    const long long per_job = (long long)gpm * p.nmodes;
    const long long items = per_job * p.njobs;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int s = lane % W, seg = lane / W;
    const long long wstep = (long long)gridDim.x * WPB;
    double2 *xl = lines + (warp * LPW + seg) * PL, *cl = xl + LS, *f1 = cl + S::NN;

    struct Item {
        int job, mode, q;
        bool act;
        long long lbase;
    };
    auto item_of = [&](long long it) {
        Item I;
        I.job = (int)(it / per_job);
        const long long r = it - (long long)I.job * per_job;
        I.mode = (int)(r / gpm);
        I.q = (int)(r - (long long)I.mode * gpm) * LPW + seg;
        I.act = I.q < lpm;
        I.lbase = I.mode * ms + (long long)(I.act ? I.q : 0) * ls;
        return I;
    };
    auto needs_input = [&](int job) {
        const LineJob &J = p.job[job];
        for (int k = 0; k < J.nout; ++k)
            if (J.o[k].order > 0) return true;
        return false;
    };
    // the physical line of an item into cl (natural order), asynchronously
    auto prefetch = [&](const Item &I) {
        if (I.act && needs_input(I.job)) {
            const double2 *in = reinterpret_cast<const double2 *>(p.job[I.job].in) + I.lbase;
#pragma unroll
            for (int j = s; j <= N; j += W) cp_async16(cl + j, in + (long long)j * es);
        }
        asm volatile("cp.async.commit_group;\n" ::);
    };

    long long it = (long long)blockIdx.x * WPB + warp;
    Item I = item_of(it);
    if (it < items) prefetch(I);
    for (; it < items; it += wstep) {
        const LineJob &J = p.job[I.job];
        const double kx = p.xalp[I.mode];
        const bool real0 = p.real0 && I.mode == 0;
        const bool interior_line = I.q > 0 && I.q < lpm - 1;
        const Item next = item_of(it + wstep);
        const bool has_next = it + wstep < items;
        int maxord = 0, last = -1;
        for (int k = 0; k < J.nout; ++k) {
            maxord = max(maxord, J.o[k].order);
            if (J.o[k].order > 0) last = k;
        }
        asm volatile("cp.async.wait_group 0;\n" ::);
        __syncwarp();
        if (maxord > 0) {
            if (!I.act)
                for (int j = s; j <= N; j += W) cl[j] = make_double2(0.0, 0.0);
            __syncwarp();
            pre_seg<R2, N, W, false>(xl, cl, ha, f1, s);
            fft_seg<R1, R2, W>(xl, tw, twT, s);
            post_seg<R2, N, W>(xl, cl, *f1, s);
            // order 1 outputs, then (one more recurrence) order 2 outputs;
            // the next item's line is fetched into cl once its last read is done
            bool fetched = false;
            for (int ord = 1; ord <= maxord; ++ord) {
                rec_seg<N, W>(cl, s);
                for (int k = 0; k < J.nout; ++k) {
                    const LineOut &o = J.o[k];
                    if (o.order != ord) continue;
                    pre_seg<R2, N, W, true>(xl, cl, ha, f1, s);
                    if (k == last && ord == maxord && has_next) {
                        prefetch(next);
                        fetched = true;
                    }
                    fft_seg<R1, R2, W>(xl, tw, twT, s);
                    post_seg<R2, N, W>(xl, nullptr, *f1, s);
                    store_seg<R2, N, W>(o, xl, true, I.lbase, es, I.act, interior_line, I.mode, kx, real0, s);
                    __syncwarp();
                }
            }
            if (!fetched && has_next) prefetch(next);
        } else if (has_next) {
            prefetch(next);
        }
        for (int k = 0; k < J.nout; ++k)
            if (J.o[k].order == 0)
                store_seg<R2, N, W>(J.o[k], xl, false, I.lbase, es, I.act, interior_line, I.mode, kx, real0, s);
        I = next;
    }
    asm volatile("cp.async.wait_group 0;\n" ::);
}

template <int R1, int R2, int W, int WPB>
static int launch_lines(ductgpu_ctx ctx, const LineParams &p0)
{
    using S = LineShape<R1, R2>;
    constexpr int N = S::N, LPB = (32 / W) * WPB;
    static_assert(R1 <= W && R2 <= W && 32 % W == 0, "a line's FFT columns and rows fit its lane segment");
    const double2 *tw = twiddle_table(ctx, N);
    const double2 *tw2 = twiddle_table(ctx, 2 * N);
    if (!tw || !tw2)
        return set_error(ctx, DUCTGPU_ESTATE, "lines: twiddle tables for N=%d unavailable%s", N,
                         ctx->capturing ? " (first use inside a capture)" : "");
    LineParams p = p0;
    const int lpm = (p.dir == 'y') ? p.mz : p.my;
    // one work item (job, mode, line pair) per warp: measured at my = 193
    // (a cfg4 DNS step) this beats persistent warps that prefetch their next
    // item (16 / WPB CTAs per SM; 10.4 against 9.6 ms of line kernels a step)
    const long long items = (long long)p.njobs * p.nmodes * ((lpm + 32 / W - 1) / (32 / W));
    const long long grid = (items + WPB - 1) / WPB;
    if (grid > 0x7fffffffLL) return set_error(ctx, DUCTGPU_EARG, "lines: grid too large");
    p.ctas_per_job = 0;
    const size_t smem = (2 * (size_t)N + (N / 2 + 1) + (size_t)LPB * S::PL) * sizeof(double2);
    DUCT_CUDA(ctx, cudaFuncSetAttribute(k_lines<R1, R2, W, WPB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)smem));
    if (ctx->prof_on && !ctx->capturing) {
        // algorithmic bytes: the input once (if transformed), every output
        // written once and read once more if accumulated, every x-term source
        double fields = 0.0;
        for (int i = 0; i < p.njobs; ++i) {
            const LineJob &J = p.job[i];
            bool in = false;
            for (int k = 0; k < J.nout; ++k) {
                const LineOut &o = J.o[k];
                in |= o.order > 0;
                fields += 1.0 + (o.beta != 0.0 ? 1.0 : 0.0);
                for (int t = 0; t < kLineXTerms; ++t) fields += o.xs[t] ? 1.0 : 0.0;
            }
            fields += in ? 1.0 : 0.0;
        }
        ctx->prof_bytes[DUCTGPU_K_LINES] += fields * 16.0 * p.my * p.mz * p.nmodes;
    }
    {
        LaunchScope ls(ctx, DUCTGPU_K_LINES);
        k_lines<R1, R2, W, WPB><<<(unsigned)grid, 32 * WPB, smem, ctx->stream>>>(p, tw, tw2);
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
    // an output's destination and sources against the other outputs' destinations
    for (int i = 0; i < p.njobs; ++i)
        for (int k = 0; k < p.job[i].nout; ++k) {
            const LineOut &o = p.job[i].o[k];
            for (int i2 = 0; i2 < p.njobs; ++i2)
                for (int k2 = 0; k2 < p.job[i2].nout; ++k2) {
                    if (i2 == i && k2 == k) continue;
                    const double *w = p.job[i2].o[k2].out;
                    bool hit = (o.out == w);       // two writers of one field, or beta reading the other's

                    for (int t = 0; t < kLineXTerms; ++t) hit |= (o.xs[t] == w);
                    if (hit)
                        return set_error(ctx, DUCTGPU_EARG, "lines: job %d output %d reads or writes what job %d output %d writes",
                                         i, k, i2, k2);
                }
        }
    // a job's input against the other jobs' destinations (its own may be in place)
    for (int i = 0; i < p.njobs; ++i)
        for (int i2 = 0; i2 < p.njobs; ++i2)
            for (int k2 = 0; k2 < p.job[i2].nout && i2 != i; ++k2)
                if (p.job[i].in && p.job[i].in == p.job[i2].o[k2].out)
                    return set_error(ctx, DUCTGPU_EARG, "lines: job %d reads what job %d output %d writes", i, i2, k2);
    const int nn = (p.dir == 'y') ? p.my : p.mz;
    if (ctx->dlines && dlines_supported(nn)) return dlines_launch(ctx, p);
    switch (nn - 1) {
    case 16: return launch_lines<4, 4, 4, 4>(ctx, p);
    case 24: return launch_lines<4, 6, 8, 4>(ctx, p);
    case 32: return launch_lines<4, 8, 8, 4>(ctx, p);
    case 48: return launch_lines<6, 8, 8, 4>(ctx, p);
    case 64: return launch_lines<8, 8, 8, 4>(ctx, p);
    case 96: return launch_lines<8, 12, 16, 8>(ctx, p);
    case 128: return launch_lines<8, 16, 16, 8>(ctx, p);
    case 144: return launch_lines<12, 12, 16, 8>(ctx, p);
    case 192: return launch_lines<12, 16, 16, 8>(ctx, p);
    case 256: return launch_lines<16, 16, 16, 8>(ctx, p);
    default:
        return set_error(ctx, DUCTGPU_EARG, "lines: line length %d - 1 is not one of 16, 24, 32, 48, 64, 96, 128, "
                         "144, 192, 256", nn);
    }
}

}  // namespace duct
