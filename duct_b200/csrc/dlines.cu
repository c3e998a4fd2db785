// dlines.cu -- the Chebyshev derivative lines of cheb_lines.cu on the FP64
// tensor cores (mma.sync m16n8k16 f64, "DMMA").
//
// For one line length nn = 2 ho + 1 the reference's derivative (transyz -1,
// the recurrence once or twice, transyz +1) is a fixed real nn x nn matrix
// D (D1 or D2), built on the host in long double from that same chain.  On
// the symmetric Gauss-Lobatto nodes D1 anticommutes with the reflection J
// (point k <-> nn-1-k) and D2 commutes with it, so with the line split into
// u_c = x_c + x_{nn-1-c} and v_c = x_c - x_{nn-1-c} (c < ho) and the middle
// point x_ho the derivative is, for the rows r < ho,
//   P_r = sum_{c<ho} Ap(r,c) u_c + D(r,ho) x_ho,  Ap(r,c) = (D(r,c) + D(r,nn-1-c)) / 2
//   M_r = sum_{c<ho} Am(r,c) v_c,                Am(r,c) = (D(r,c) - D(r,nn-1-c)) / 2
//   y_r = P_r + M_r,  y_{nn-1-r} = s (P_r - M_r)   (s = -1 for D1, +1 for D2)
// and for the middle row y_ho = sum_{c<ho} (Ap(ho,c) u_c + Am(ho,c) v_c) +
// D(ho,ho) x_ho: two ho x ho GEMMs on the tensor cores (half the flops of
// the full matrix), the middle column a rank-1 update of P and the middle
// row a dot product in FP64 FMAs, so that ho = 16 MT (nn = 2^k + 1) pads
// nothing.  The store is k_lines' epilogue (out = sigma (beta out + fac y +
// x-terms + [mode 0] m0), the max |out| reduction), so lines_launch hands a
// launch either to k_lines (the FFT form) or to this kernel.
//
// A CTA takes 16 complex lines (32 real columns) of one mode of one job,
// staged once with cp.async and folded in place (u_k to row k, v_k to row
// nn-1-k, x_ho stays); a warp per 16 rows r < ho (MT = ceil(ho / 16) warps)
// runs the two GEMMs of every derivative output of the job over them,
// reading its A fragments straight from L2 (the operators are at most
// 0.5 MB), with no CTA barrier inside the K loop.
#include <math.h>

#include <type_traits>
#include <vector>

#include "internal.h"

namespace duct {

// A CTA of NT n-tiles takes 4 NT complex lines (8 NT real columns); the
// staged rows are 8 NT + 4 doubles apart, a stride of 4 mod 16 doubles, so
// that the B-fragment loads of a half-warp (rows t, columns g < 4) meet 16
// distinct bank pairs.
template <int NT> struct DlShape {
    static constexpr int lines = 4 * NT, cols = 8 * NT, nld = 8 * NT + 4;
};
constexpr int kDlMaxMT = 8;                  // ho <= 128: line lengths up to 257

// Operators of one order, HR = 16 MT: Ap and Am (HR x HR each, rows and
// columns >= ho zero, DMMA A-fragment order), then the vectors D(r, ho)
// (r < ho), Ap(ho, c), Am(ho, c) (c < ho) and D(ho, ho), HR doubles each.
inline size_t dl_chunk(int HR) { return 2 * (size_t)HR * HR + 4 * (size_t)HR; }

struct DLineParams {
    LineParams lp;
    const double *op[2];     // [order - 1]
    int nn, ho;
    int ctas_per_job;
};

__device__ __forceinline__ void dl_cp16(void *smem, const void *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}

// D += A(16x16) B(16x8), m16n8k16 f64 fragments (PTX ISA):
// a[v] = A[g + 8(v&1)][t + 4(v>>1)], b[v] = B[t + 4v][g],
// d = {D[g][2t], D[g][2t+1], D[g+8][2t], D[g+8][2t+1]}.
__device__ __forceinline__ void dl_mma(double (&d)[4], const double (&a)[8], const double (&b)[4])
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 "
        "{%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, {%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]),
          "d"(b[0]), "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

__device__ __forceinline__ double2 dl_xcoef(const LineOut &o, int t, double kx)
{
    return make_double2(o.xc0[t] - o.xc2[t] * kx * kx, o.xc1[t] * kx);
}

// One output element: out[gi] = sigma (beta out + fac y + x-terms + m0).
// Returns |out| for the interior max (0 where it does not count).
template <int NXM>
__device__ __forceinline__ double dl_store(const LineOut &o, long long gi, double2 y, bool deriv, double kx,
                                           double m0, bool real0, bool interior)
{
    double2 *out = reinterpret_cast<double2 *>(o.out);
    double2 v = make_double2(m0, 0.0);
    if (deriv) {
        v.x += o.fac * y.x;
        if (!real0) v.y += o.fac * y.y;
    }
#pragma unroll
    for (int t = 0; t < NXM; ++t)
        if (o.xs[t]) {
            const double2 c = dl_xcoef(o, t, kx);
            const double2 s = reinterpret_cast<const double2 *>(o.xs[t])[gi];
            v.x += c.x * s.x - c.y * s.y;
            v.y += c.x * s.y + c.y * s.x;
        }
    if (o.beta != 0.0) {
        const double2 w = out[gi];
        v.x += o.beta * w.x;
        v.y += o.beta * w.y;
    }
    v.x *= o.sigma;
    v.y *= o.sigma;
    out[gi] = v;
    return interior ? hypot(v.x, v.y) : 0.0;
}

// Registers for about WARPS resident warps per SM, two CTAs at least (a
// latency-bound kernel: the staging, the L2 operator loads and the
// epilogue's loads are hidden by other warps rather than by prefetching).
// NXM: the x-terms an output of the launch may have (1, or all
// kLineXTerms): fewer registers where the launch's outputs have at most one
template <int MT, int NT, int WARPS, int NXM>
__global__ void __launch_bounds__(32 * MT, WARPS / MT > 2 ? WARPS / MT : 2)
    k_dlines(const __grid_constant__ DLineParams q)
{
    constexpr int kDlLines = DlShape<NT>::lines, kDlCols = DlShape<NT>::cols, kDlNld = DlShape<NT>::nld;
    constexpr int HR = 16 * MT;
    constexpr size_t blk = (size_t)HR * HR;
    extern __shared__ __align__(16) double Xs[];   // [nn][kDlNld] lines ((re, im) column pairs), then red

    const LineParams &p = q.lp;
    const int job = blockIdx.x / q.ctas_per_job;
    const int rr = blockIdx.x - job * q.ctas_per_job;
    const LineJob &J = p.job[job];
    const bool ydir = (p.dir == 'y');
    const long long ms = (long long)p.my * p.mz;
    const long long ls = ydir ? p.my : 1, es = ydir ? 1 : p.my;
    const int lpm = ydir ? p.mz : p.my;
    const int cpm = (lpm + kDlLines - 1) / kDlLines;
    const int mode = rr / cpm;
    const int q0 = (rr - mode * cpm) * kDlLines;
    const int L = min(kDlLines, lpm - q0);
    const long long base = mode * ms + (long long)q0 * ls;
    const int lsi = (int)ls, esi = (int)es;  // strides within a mode (a plane holds < 2^31 points)
    const double kx = p.xalp[mode];
    const bool real0 = p.real0 && mode == 0;
    const int nn = q.nn, ho = q.ho;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const double m0 = (mode == 0) ? 1.0 : 0.0;
    double *red = Xs + (size_t)nn * kDlNld;  // [2][MT][32]: the middle row's partial sums

    // element idx of the CTA's lines: line idx % 16, point idx / 16 (a warp
    // touches two points of 16 lines: whole 32-byte sectors along y, 512
    // contiguous bytes along z; 16-byte shared stores without conflicts)
    int maxord = 0;
    for (int k = 0; k < J.nout; ++k) maxord = max(maxord, J.o[k].order);
    if (maxord > 0) {
        const double2 *in = reinterpret_cast<const double2 *>(J.in) + base;
        for (int idx = tid; idx < nn * kDlLines; idx += 32 * MT) {
            const int l = idx % kDlLines, j = idx / kDlLines;
            double *dst = Xs + j * kDlNld + 2 * l;
            if (l < L) dl_cp16(dst, in + (l * lsi + j * esi));
            else { dst[0] = 0.0; dst[1] = 0.0; }
        }
        asm volatile("cp.async.commit_group;\n" ::);
        asm volatile("cp.async.wait_group 0;\n" ::);
        __syncthreads();
        // fold in place: u_k = x_k + x_{nn-1-k} to row k, v_k = x_k - x_{nn-1-k}
        // to row nn-1-k (k < ho); row ho keeps x_ho
        for (int idx = tid; idx < ho * kDlCols; idx += 32 * MT) {
            const int k = idx / kDlCols, c = idx - k * kDlCols;
            const double a = Xs[k * kDlNld + c], b = Xs[(nn - 1 - k) * kDlNld + c];
            Xs[k * kDlNld + c] = a + b;
            Xs[(nn - 1 - k) * kDlNld + c] = a - b;
        }
        __syncthreads();
    }
    double vmax = 0.0;
    const double *maxabs_out = nullptr;
    const int mt = warp;                     // this warp's 16 rows and 16-column slice of the middle row
    for (int oi = 0; oi < J.nout; ++oi) {
        const LineOut &o = J.o[oi];
        if (o.maxabs) maxabs_out = o.maxabs;
        if (o.order == 0) {
            // four elements at a time, their loads before their stores
            constexpr int B = 4;
            for (int i0 = tid; i0 < nn * kDlLines; i0 += B * 32 * MT) {
                double2 v[B];
                int gi[B];
                bool ok[B];
#pragma unroll
                for (int e = 0; e < B; ++e) {
                    const int idx = i0 + e * 32 * MT, l = idx % kDlLines, j = idx / kDlLines;
                    ok[e] = idx < nn * kDlLines && l < L;
                    gi[e] = l * lsi + j * esi;
                    v[e] = make_double2(m0 * o.m0, 0.0);
                }
#pragma unroll
                for (int tt = 0; tt < NXM; ++tt)
                    if (o.xs[tt]) {
                        const double2 c = dl_xcoef(o, tt, kx);
#pragma unroll
                        for (int e = 0; e < B; ++e)
                            if (ok[e]) {
                                const double2 x = (reinterpret_cast<const double2 *>(o.xs[tt]) + base)[gi[e]];
                                v[e].x += c.x * x.x - c.y * x.y;
                                v[e].y += c.x * x.y + c.y * x.x;
                            }
                    }
                double2 *out = reinterpret_cast<double2 *>(o.out) + base;
                if (o.beta != 0.0) {
#pragma unroll
                    for (int e = 0; e < B; ++e)
                        if (ok[e]) {
                            const double2 w = out[gi[e]];
                            v[e].x += o.beta * w.x;
                            v[e].y += o.beta * w.y;
                        }
                }
#pragma unroll
                for (int e = 0; e < B; ++e)
                    if (ok[e]) {
                        const int idx = i0 + e * 32 * MT, l = idx % kDlLines, j = idx / kDlLines;
                        const double2 w = make_double2(o.sigma * v[e].x, o.sigma * v[e].y);
                        out[gi[e]] = w;
                        if (o.maxabs && j > 0 && j < nn - 1 && q0 + l > 0 && q0 + l < lpm - 1)
                            vmax = fmax(vmax, hypot(w.x, w.y));
                    }
            }
            continue;
        }
        const double *opb = q.op[o.order - 1];
        // the middle row: this warp's 16 columns of it for real column `lane`
        {
            const double *rowP = opb + 2 * blk + HR, *rowM = opb + 2 * blk + 2 * HR;
            const int cl = lane < kDlCols ? lane : 0;     // lanes beyond the columns repeat column 0
            double part = (mt == 0) ? __ldg(opb + 2 * blk + 3 * HR) * Xs[ho * kDlNld + cl] : 0.0;
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const int c = mt * 16 + i;
                if (c < ho)
                    part = fma(__ldg(rowP + c), Xs[c * kDlNld + cl],
                               fma(__ldg(rowM + c), Xs[(nn - 1 - c) * kDlNld + cl], part));
            }
            red[((oi & 1) * MT + mt) * 32 + lane] = part;
        }
        // the middle column's coefficients D(r, ho) of this thread's rows
        const double d0 = __ldg(opb + 2 * blk + mt * 16 + g), d1 = __ldg(opb + 2 * blk + mt * 16 + g + 8);
        double acc[2][NT][4];
#pragma unroll
        for (int pm = 0; pm < 2; ++pm)
#pragma unroll
            for (int nt = 0; nt < NT; ++nt)
#pragma unroll
                for (int v = 0; v < 4; ++v) acc[pm][nt][v] = 0.0;
        // P = Ap u, then M = Am v (one GEMM at a time: fewer live registers).
        // B fragments of K step ks: u_k from row k, v_k from row nn-1-k; only
        // the last step can reach k >= ho (zero there)
#pragma unroll
        for (int pm = 0; pm < 2; ++pm) {
            const double2 *Asrc = reinterpret_cast<const double2 *>(opb + pm * blk + (size_t)mt * 256) + lane;
            auto step = [&](int ks, const double (&a)[8], auto last) {
#pragma unroll
                for (int nt = 0; nt < NT; ++nt) {
                    const int col = nt * 8 + g;
                    double b[4];
#pragma unroll
                    for (int v = 0; v < 4; ++v) {
                        const int k = ks * 16 + t + 4 * v;
                        const int row = pm ? nn - 1 - k : k;
                        if (decltype(last)::value) b[v] = (k < ho) ? Xs[row * kDlNld + col] : 0.0;
                        else b[v] = Xs[row * kDlNld + col];
                    }
                    dl_mma(acc[pm][nt], a, b);
                }
            };
#pragma unroll 1
            for (int ks = 0; ks < MT; ++ks) {
                double a[8];
#pragma unroll
                for (int h = 0; h < 4; ++h) {
                    const double2 v = __ldg(Asrc + (size_t)ks * MT * 128 + 32 * h);
                    a[2 * h] = v.x;
                    a[2 * h + 1] = v.y;
                }
                if (ks + 1 < MT) step(ks, a, std::false_type());
                else step(ks, a, std::true_type());
            }
            if (pm == 0) {
                // the middle column: P_r += D(r, ho) x_ho
#pragma unroll
                for (int nt = 0; nt < NT; ++nt) {
                    const double xr = Xs[ho * kDlNld + nt * 8 + 2 * t], xi = Xs[ho * kDlNld + nt * 8 + 2 * t + 1];
                    acc[0][nt][0] = fma(d0, xr, acc[0][nt][0]);
                    acc[0][nt][1] = fma(d0, xi, acc[0][nt][1]);
                    acc[0][nt][2] = fma(d1, xr, acc[0][nt][2]);
                    acc[0][nt][3] = fma(d1, xi, acc[0][nt][3]);
                }
            }
        }
        // y_r = P_r + M_r, y_{nn-1-r} = s (P_r - M_r); columns (2t, 2t+1) of
        // n-tile nt are (re, im) of line 4 nt + t.  Every load of the
        // epilogue comes before its first store, so the loads of the 16
        // elements need not wait for stores the compiler cannot prove
        // disjoint from them.
        {
            const double s = (o.order == 1) ? -1.0 : 1.0;
            double2 v[NT][2][2];
#pragma unroll
            for (int nt = 0; nt < NT; ++nt)
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const double pr = acc[0][nt][2 * h], pi = acc[0][nt][2 * h + 1];
                    const double mr = acc[1][nt][2 * h], mi = acc[1][nt][2 * h + 1];
                    v[nt][h][0] = make_double2(m0 * o.m0 + o.fac * (pr + mr), real0 ? 0.0 : o.fac * (pi + mi));
                    v[nt][h][1] = make_double2(m0 * o.m0 + o.fac * s * (pr - mr), real0 ? 0.0 : o.fac * s * (pi - mi));
                }
            auto valid = [&](int nt, int h) { return nt * 4 + t < L && mt * 16 + g + 8 * h < ho; };
            // offsets from the CTA's first element: within one mode, 32 bits
            auto gidx = [&](int nt, int h, int m) {
                const int r = mt * 16 + g + 8 * h;
                return (nt * 4 + t) * lsi + (m ? nn - 1 - r : r) * esi;
            };
#pragma unroll
            for (int tt = 0; tt < NXM; ++tt)
                if (o.xs[tt]) {
                    const double2 c = dl_xcoef(o, tt, kx);
                    const double2 *src = reinterpret_cast<const double2 *>(o.xs[tt]) + base;
#pragma unroll
                    for (int nt = 0; nt < NT; ++nt)
#pragma unroll
                        for (int h = 0; h < 2; ++h)
#pragma unroll
                            for (int m = 0; m < 2; ++m)
                                if (valid(nt, h)) {
                                    const double2 x = src[gidx(nt, h, m)];
                                    v[nt][h][m].x += c.x * x.x - c.y * x.y;
                                    v[nt][h][m].y += c.x * x.y + c.y * x.x;
                                }
                }
            double2 *out = reinterpret_cast<double2 *>(o.out) + base;
            if (o.beta != 0.0) {
#pragma unroll
                for (int nt = 0; nt < NT; ++nt)
#pragma unroll
                    for (int h = 0; h < 2; ++h)
#pragma unroll
                        for (int m = 0; m < 2; ++m)
                            if (valid(nt, h)) {
                                const double2 w = out[gidx(nt, h, m)];
                                v[nt][h][m].x += o.beta * w.x;
                                v[nt][h][m].y += o.beta * w.y;
                            }
            }
#pragma unroll
            for (int nt = 0; nt < NT; ++nt) {
                const int l = nt * 4 + t;
                const bool chk = o.maxabs && q0 + l > 0 && q0 + l < lpm - 1;
#pragma unroll
                for (int h = 0; h < 2; ++h)
#pragma unroll
                    for (int m = 0; m < 2; ++m)
                        if (valid(nt, h)) {
                            const double2 w = make_double2(o.sigma * v[nt][h][m].x, o.sigma * v[nt][h][m].y);
                            out[gidx(nt, h, m)] = w;
                            if (chk && mt * 16 + g + 8 * h > 0) vmax = fmax(vmax, hypot(w.x, w.y));
                        }
            }
        }
        __syncthreads();                     // the partial sums of the middle row
        if (warp == 0) {
            double y = 0.0;
#pragma unroll
            for (int w = 0; w < MT; ++w) y += red[((oi & 1) * MT + w) * 32 + lane];
            const double yi = __shfl_down_sync(0xffffffffu, y, 1);
            const int l = lane >> 1;
            if (!(lane & 1) && l < L) {
                const bool chk = o.maxabs && q0 + l > 0 && q0 + l < lpm - 1;
                vmax = fmax(vmax, dl_store<NXM>(o, base + (long long)l * ls + (long long)ho * es, make_double2(y, yi), true,
                                           kx, m0 * o.m0, real0, chk));
            }
        }
    }
    if (maxabs_out) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) vmax = fmax(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
        if (lane == 0 && vmax > 0.0)
            atomicMax(reinterpret_cast<unsigned long long *>(const_cast<double *>(maxabs_out)),
                      (unsigned long long)__double_as_longlong(vmax));
    }
}

// odd line lengths of the FFT kernel with ho <= 128 (17 .. 257)
bool dlines_supported(int nn) { return (nn & 1) && nn >= 17 && lines_supported(nn) && nn / 2 <= 16 * kDlMaxMT; }

void free_dlines(ductgpu_ctx ctx)
{
    for (int i = 0; i < ductgpu_ctx_s::kDlineSlots; ++i) {
        cudaFree(ctx->dl_ops[i]);
        ctx->dl_ops[i] = nullptr;
        ctx->dl_nn[i] = 0;
    }
}

// The derivative matrix D = B R^ord F of one line of nn = N + 1 points,
// column-major, in long double: F the forward tcheb (src/tchebw.f:62-192:
// c_k = w_k (x_0 + (-1)^k x_N + 2 sum_{0<j<N} x_j cos(pi j k / N)), w_k =
// 1/N inside, 1/(2N) at k = 0, N), R the derivative recurrence of derivyz
// (src/chebyshev.f90:44-58: d_N = 0, d_{k-1} = d_{k+1} + 2 k c_k, out_k =
// -d_k for k >= 1, out_0 = -d_0 / 2), B the inverse tcheb (x_j = sum_k c_k
// cos(pi j k / N)).  The 64-bit significand keeps the entries' own error
// (~ 2^-64 N^4 at the corners of D2) below their FP64 rounding; the same
// chain run in FP64 on unit vectors leaves errors ~ 2^-53 N^3 on entries
// of size N^2 that a whole line then sums.
static void cheb_deriv_matrix(int nn, int ord, std::vector<long double> &D)
{
    const int N = nn - 1;
    const long double pi = 3.141592653589793238462643383279502884L;
    std::vector<long double> ct(2 * (size_t)N), c(nn), d(nn);
    for (int q = 0; q < 2 * N; ++q) ct[q] = cosl(pi * (long double)q / (long double)N);
    D.assign((size_t)nn * nn, 0.0L);
    for (int col = 0; col < nn; ++col) {
        const long double sc = (col == 0 || col == N) ? 1.0L : 2.0L;
        for (int k = 0; k < nn; ++k) {
            const long double w = (k == 0 || k == N) ? 0.5L / N : 1.0L / N;
            c[k] = w * sc * ct[(size_t)((long)col * k % (2 * N))];
        }
        for (int o = 0; o < ord; ++o) {
            long double dk1 = 0.0L, dk = 0.0L;     // d_{k+1}, d_k, walking k down from N
            d[N] = 0.0L;
            for (int k = N; k >= 1; --k) {
                const long double dm = dk1 + 2.0L * k * c[k];   // d_{k-1}
                d[k] = -dk;
                dk1 = dk;
                dk = dm;
            }
            d[0] = -0.5L * dk;
            c.swap(d);
        }
        for (int j = 0; j < nn; ++j) {
            long double x = 0.0L;
            for (int k = 0; k < nn; ++k) x += c[k] * ct[(size_t)((long)j * k % (2 * N))];
            D[(size_t)j + (size_t)nn * col] = x;
        }
    }
}

// The folded, packed operators of line length nn (built on first use:
// not inside a stream capture): [order 1 chunk][order 2 chunk].
static int dlines_ops(ductgpu_ctx ctx, int nn, const double **ops, int *hr)
{
    const int ho = nn / 2, MT = (ho + 15) / 16, HR = 16 * MT;
    const size_t blk = (size_t)HR * HR, chunk = dl_chunk(HR);
    *hr = HR;
    int slot = -1;
    for (int i = 0; i < ductgpu_ctx_s::kDlineSlots; ++i)
        if (ctx->dl_nn[i] == nn) { *ops = ctx->dl_ops[i]; return DUCTGPU_OK; }
    for (int i = 0; i < ductgpu_ctx_s::kDlineSlots && slot < 0; ++i)
        if (!ctx->dl_nn[i]) slot = i;
    if (slot < 0) return set_error(ctx, DUCTGPU_ESTATE, "derivative lines: more than %d line lengths",
                                   ductgpu_ctx_s::kDlineSlots);
    if (ctx->capturing)
        return set_error(ctx, DUCTGPU_ESTATE, "derivative lines: operators for nn=%d first built inside a capture", nn);
    std::vector<double> packed(2 * chunk, 0.0);
    std::vector<long double> M;
    for (int ord = 0; ord < 2; ++ord) {
        cheb_deriv_matrix(nn, ord + 1, M);
        auto d = [&](int r, int c) { return M[(size_t)r + (size_t)nn * c]; };
        double *dst = packed.data() + ord * chunk;
        for (size_t idx = 0; idx < blk; ++idx) {
            int row, col;
            pack_slot((int)idx, MT, row, col);
            if (row < ho && col < ho) {
                dst[idx] = (double)(0.5L * (d(row, col) + d(row, nn - 1 - col)));
                dst[blk + idx] = (double)(0.5L * (d(row, col) - d(row, nn - 1 - col)));
            }
        }
        for (int r = 0; r < ho; ++r) {
            dst[2 * blk + r] = (double)d(r, ho);
            dst[2 * blk + HR + r] = (double)(0.5L * (d(ho, r) + d(ho, nn - 1 - r)));
            dst[2 * blk + 2 * HR + r] = (double)(0.5L * (d(ho, r) - d(ho, nn - 1 - r)));
        }
        dst[2 * blk + 3 * HR] = (double)d(ho, ho);
    }
    double *dev = nullptr;
    DUCT_CUDA(ctx, cudaMalloc(&dev, packed.size() * sizeof(double)));
    DUCT_CUDA(ctx, cudaMemcpy(dev, packed.data(), packed.size() * sizeof(double), cudaMemcpyHostToDevice));
    ctx->dl_ops[slot] = dev;
    ctx->dl_nn[slot] = nn;
    *ops = dev;
    return DUCTGPU_OK;
}

template <int MT, int NT, int WARPS, int NXM>
static int launch_dlines(ductgpu_ctx ctx, DLineParams &q)
{
    const size_t smem = ((size_t)q.nn * DlShape<NT>::nld + 2 * (size_t)MT * 32) * sizeof(double);
    DUCT_CUDA(ctx, cudaFuncSetAttribute(k_dlines<MT, NT, WARPS, NXM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const long long grid = (long long)q.ctas_per_job * q.lp.njobs;
    if (grid > 0x7fffffffLL) return set_error(ctx, DUCTGPU_EARG, "derivative lines: grid too large");
    if (ctx->prof_on && !ctx->capturing) {
        double fields = 0.0;
        for (int i = 0; i < q.lp.njobs; ++i) {
            const LineJob &J = q.lp.job[i];
            bool in = false;
            for (int k = 0; k < J.nout; ++k) {
                const LineOut &o = J.o[k];
                in |= o.order > 0;
                fields += 1.0 + (o.beta != 0.0 ? 1.0 : 0.0);
                for (int t = 0; t < kLineXTerms; ++t) fields += o.xs[t] ? 1.0 : 0.0;
            }
            fields += in ? 1.0 : 0.0;
        }
        ctx->prof_bytes[DUCTGPU_K_LINES] += fields * 16.0 * q.lp.my * q.lp.mz * q.lp.nmodes;
        // per CTA and derivative output: 2 GEMMs x MT warps x MT K steps x NT
        // m16n8k16 MMAs of 2 x 16 x 8 x 16 flops
        int nderiv = 0;
        for (int i = 0; i < q.lp.njobs; ++i)
            for (int k = 0; k < q.lp.job[i].nout; ++k) nderiv += q.lp.job[i].o[k].order > 0;
        ctx->prof_flops[DUCTGPU_K_LINES] += (double)q.ctas_per_job * nderiv * 2.0 * MT * MT * NT * 4096.0;
    }
    {
        LaunchScope ls(ctx, DUCTGPU_K_LINES);
        k_dlines<MT, NT, WARPS, NXM><<<(unsigned)grid, 32 * MT, smem, ctx->stream>>>(q);
    }
    return check_cuda(ctx, cudaGetLastError(), "k_dlines");
}

int dlines_launch(ductgpu_ctx ctx, const LineParams &p)
{
    const int nn = (p.dir == 'y') ? p.my : p.mz;
    DLineParams q;
    q.lp = p;
    q.nn = nn;
    q.ho = nn / 2;
    const double *ops = nullptr;
    int HR = 0;
    int rc = dlines_ops(ctx, nn, &ops, &HR);
    if (rc) return rc;
    q.op[0] = ops;
    q.op[1] = ops + dl_chunk(HR);
    const int lpm = (p.dir == 'y') ? p.mz : p.my;
    // dlines 1: 8 lines per CTA with registers for 32 resident warps per SM
    // (the fastest measured on the 193 x 193, 85-mode DNS step: 9.56 ms a
    // step, against 9.97 ms with 24 warps, 10.8 ms with 16 and 10.9 ms for
    // 16 lines per CTA with 16 warps; 4 lines per CTA: 10.1 ms); 2: 16
    // lines per CTA, 16 warps (each operator fragment feeds twice the MMAs)
    const bool wide = ctx->dlines == 2;
    // at most one x-term per output (xterm() fills the slots in order)
    bool one_x = true;
    for (int i = 0; i < p.njobs; ++i)
        for (int k = 0; k < p.job[i].nout; ++k)
            for (int t = 1; t < kLineXTerms; ++t) one_x = one_x && !p.job[i].o[k].xs[t];
    const int lines = wide ? DlShape<4>::lines : DlShape<2>::lines;
    q.ctas_per_job = p.nmodes * ((lpm + lines - 1) / lines);
#define DL_CASE(mt) \
    case mt:                                                                                      \
        return wide ? (one_x ? launch_dlines<mt, 4, 16, 1>(ctx, q) : launch_dlines<mt, 4, 16, kLineXTerms>(ctx, q)) \
                    : (one_x ? launch_dlines<mt, 2, 32, 1>(ctx, q) : launch_dlines<mt, 2, 32, kLineXTerms>(ctx, q));
    switch (HR / 16) {
        DL_CASE(1) DL_CASE(2) DL_CASE(3) DL_CASE(4) DL_CASE(5) DL_CASE(6) DL_CASE(7) DL_CASE(8)
    default: return set_error(ctx, DUCTGPU_EARG, "derivative lines: line length %d", nn);
    }
#undef DL_CASE
}

}  // namespace duct

// The derivative matrix of one Chebyshev line, for callers and tests on the
// host: no context, no GPU.
extern "C" int ductgpu_cheb_deriv_matrix(int n, int order, double *D)
{
    if (n < 3 || n > 1025 || order < 1 || order > 2 || !D) return DUCTGPU_EARG;
    std::vector<long double> M;
    duct::cheb_deriv_matrix(n, order, M);
    for (size_t i = 0; i < M.size(); ++i) D[i] = (double)M[i];
    return DUCTGPU_OK;
}
