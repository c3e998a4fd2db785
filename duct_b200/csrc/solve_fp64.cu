// solve_fp64.cu -- plain FP64 diagonalisation solve on the B200 FP64 tensor
// cores (mma.sync m16n8k8 f64, "DMMA"; tcgen05 has no f64 kind).
//
// The reference solves one real plane at a time with four dgemm calls, two
// explicit transposes and a divide (src/solvediag.f90:47-80, GPU variant
// :82-128 with cublasDgemm, transpose_gpu and mat_invdiag):
//     U = P [ (P^-1 F P^-T) / (E_i + E_j - lambda) ] P^T .
// Here every plane of every field goes through four batched passes, each a
// GEMM of a fixed n x n operator against many short "lines" of the field:
//     y-pass  out(o, z) = sum_y A(o,y) in(y, z)      (A = P^-1, then P)
//     z-pass  out(y, o) = sum_z A(o,z) in(y, z)      (A = P^-1 with the
//                          eigenvalue divide fused in the epilogue, then P)
// The complex field is never de-interleaved in memory: a CTA stages 32
// complex lines (64 real columns: re and im side by side) of one plane in
// shared memory and multiplies the whole padded operator against them, so
// the transposes of the reference disappear into the addressing.  The
// operator streams through shared memory in K chunks of 32 with cp.async,
// pre-packed in the DMMA A-fragment order (16-byte loads, no bank
// conflicts); with 16-wide K chunks a CTA stays under 113 KB of shared
// memory for n <= 127, so two CTAs share an SM and hide each other's
// staging latency.
#include <math.h>

#include "internal.h"

namespace duct {

constexpr int kLines = kPassLines;   // complex lines per CTA
constexpr int kNld = 68;     // leading dim of the staged tile (64 + 4 pad)
constexpr int kKC = 16;      // K chunk of the streamed operator (one k16 step)
constexpr int kThreads = 256;
constexpr int kParityLines = 16;   // lines per CTA of the flip-symmetric passes (3 CTAs per SM)

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
// 16-byte copy, or 16 zero bytes when !valid (gmem is then not read)
__device__ __forceinline__ void cp_async16_zfill(void *smem, const void *gmem, bool valid)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const int n = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// D += A(16x16) * B(16x8), fragments as in the PTX ISA for m16n8k16 f64:
// a[v] = A[g + 8(v&1)][t + 4(v>>1)], b[v] = B[t + 4v][g],
// d = {D[g][2t], D[g][2t+1], D[g+8][2t], D[g+8][2t+1]}.
__device__ __forceinline__ void dmma16(double (&d)[4], const double (&a)[8], const double (&b)[4])
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 "
        "{%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, {%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]),
          "d"(b[0]), "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

// MTW: 16-row tiles per warp along M of the launch (fields with smaller
// operators skip the tiles they do not have).
template <int MTW, int LINES>
__global__ void __launch_bounds__(kThreads, LINES == 16 ? 3 : (MTW == 3 ? 1 : 2)) k_pass_fp64(const __grid_constant__ PassParams p)
{
    extern __shared__ __align__(16) double smem[];
    constexpr int NLD = 2 * LINES + 4, NTW = LINES / 8;
    constexpr int a_chunk_max = (kKC / 16) * (4 * MTW) * 256;
    double *As = smem;
    double *Bs = smem + 2 * a_chunk_max;

    int fi = 0;
    while (fi + 1 < p.nf && (int)blockIdx.x >= p.cta_start[fi + 1]) ++fi;
    const PassField &F = p.f[fi];
    const int local = blockIdx.x - p.cta_start[fi];
    const int plane = local / F.nchunks;
    const int chunk = local - plane * F.nchunks;
    const int l0 = chunk * LINES;
    const int L = min(LINES, F.nlines - l0);
    const double *src = F.src + (long long)plane * F.plane_stride;
    double *dst = F.dst + (long long)plane * F.plane_stride;
    const int tid = threadIdx.x;
    const int kpad = F.kpad, mtiles = F.mtiles;
    const int nkc = kpad / kKC;
    const int a_chunk = (kKC / 16) * mtiles * 256;

    auto load_a = [&](int c, int buf) {
        const double *g = F.A + (size_t)c * a_chunk;
        double *s = As + buf * a_chunk_max;
        for (int i = tid * 2; i < a_chunk; i += kThreads * 2) cp_async16(s + i, g + i);
        cp_async_commit();
    };
    load_a(0, 0);

    // Stage the lines: Bs[k][2l + c] = in(k, l0 + l) component c, zero
    // padded; cp.async keeps all of a thread's copies in flight at once (the
    // first K step's wait covers them)
    const int n = F.n, sk = F.sk, sl = F.sl, o1 = F.off;
    auto stage = [&](int k, int l) {
        const bool ok = k < n && l < L;
        const double *gp = ok ? src + 2 * ((long long)(k + o1) * sk + (long long)(l0 + l + o1) * sl) : src;
        cp_async16_zfill(Bs + k * NLD + 2 * l, gp, ok);
    };
    if (sk == 1) {
        for (int idx = tid; idx < kpad * LINES; idx += kThreads) stage(idx % kpad, idx / kpad);
    } else {
        for (int idx = tid; idx < kpad * LINES; idx += kThreads) stage(idx / LINES, idx % LINES);
    }
    cp_async_commit();

    const int lane = tid & 31, warp = tid >> 5;
    const int wm = warp & 3, wn = warp >> 2;
    const int g = lane >> 2, t = lane & 3;
    double acc[MTW][NTW][4];
#pragma unroll
    for (int i = 0; i < MTW; ++i)
#pragma unroll
        for (int j = 0; j < NTW; ++j)
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[i][j][v] = 0.0;

    for (int c = 0; c < nkc; ++c) {
        if (c + 1 < nkc) {
            load_a(c + 1, (c + 1) & 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const double *Ab = As + (c & 1) * a_chunk_max;
#pragma unroll
        for (int ks = 0; ks < kKC / 16; ++ks) {
            const int kg = c * kKC + ks * 16 + t;
            double b[NTW][4];
#pragma unroll
            for (int nt = 0; nt < NTW; ++nt) {
                const int col = wn * LINES + nt * 8 + g;
#pragma unroll
                for (int v = 0; v < 4; ++v) b[nt][v] = Bs[(kg + 4 * v) * NLD + col];
            }
#pragma unroll
            for (int mt = 0; mt < MTW; ++mt) {
                const int mtg = wm * MTW + mt;
                if (mtg >= mtiles) continue;
                double a[8];
                const double2 *q = reinterpret_cast<const double2 *>(Ab + (ks * mtiles + mtg) * 256) + lane;
#pragma unroll
                for (int h = 0; h < 4; ++h) {
                    const double2 v = q[32 * h];
                    a[2 * h] = v.x;
                    a[2 * h + 1] = v.y;
                }
#pragma unroll
                for (int nt = 0; nt < NTW; ++nt) dmma16(acc[mt][nt], a, b[nt]);
            }
        }
        __syncthreads();
    }

    // Epilogue: rows of the accumulator are the output index o, column pairs
    // (2t, 2t+1) are (re, im) of line l.
    const double lam = p.lam[F.plane0 + plane];
    const bool singular = (F.sing_io >= 0) && fabs(lam) <= 1.0e-10;
    const bool im0 = p.zero_im_mode0 && F.mode0 && plane == 0;
#pragma unroll
    for (int mt = 0; mt < MTW; ++mt)
#pragma unroll
        for (int nt = 0; nt < NTW; ++nt) {
            const int l = wn * (LINES / 2) + nt * 4 + t;
            if (l >= L) continue;
            const int lg = l0 + l;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int o = (wm * MTW + mt) * 16 + g + 8 * h;
                if (o >= n) continue;
                double re = acc[mt][nt][2 * h], im = acc[mt][nt][2 * h + 1];
                if (p.divide) {
                    if (singular && o == F.sing_io && lg == F.sing_l) {
                        re = 0.0;
                        im = 0.0;
                    } else {
                        const double rden = 1.0 / ((F.E[o] + F.El[lg]) - lam);
                        re *= rden;
                        im *= rden;
                    }
                }
                const long long off = 2 * ((long long)(o + o1) * sk + (long long)(lg + o1) * sl);
                if (p.residual) {
                    const long long po = (long long)plane * F.plane_stride + off;
                    const double2 f = *reinterpret_cast<const double2 *>(F.resF + po);
                    const double2 tt = *reinterpret_cast<const double2 *>(F.resT + po);
                    const double2 uu = *reinterpret_cast<const double2 *>(F.resU + po);
                    re = (f.x - tt.x) - re + lam * uu.x;
                    im = (f.y - tt.y) - im + lam * uu.y;
                }
                if (im0) im = 0.0;
                *reinterpret_cast<double2 *>(dst + off) = make_double2(re, im);
            }
        }
}

// ---------------------------------------------------------------------------
// Flip-symmetric variant (fold_operators in setup.cu): the operator is the
// two half blocks stacked, 2 H x H (H = kpad = 32 MTW), so warps 0-1 along M
// own the even block and warps 2-3 the odd one, each over its own H rows of
// the staged data -- half the K loop of k_pass_fp64 at the same tile shape.
// par 1 (P^-1 passes): the physical input is folded while it is staged
//   (rows 0..H-1: in_k + in_{n-1-k}, in_k alone at the middle point when n
//   is odd; rows H..2H-1: in_k - in_{n-1-k}); the output is in mode order
//   (he even modes, then ho odd ones), the eigenvalue divide as usual.
// par 2 (P passes): the mode-ordered input is staged as the two halves; the
//   accumulators go through shared memory, and out_o = even_o + odd_o,
//   out_{n-1-o} = even_o - odd_o.
// One tile (field fi, the field's tile `local` = plane * nchunks + chunk)
// of a flip-symmetric pass, by every thread of the CTA; smem as sized by
// pass_smem_bytes for this MTW (with the eigenvalue staging).
template <int MTW, int LINES, bool SINGLE = false>
__device__ __forceinline__ void pass_s_tile(const PassParams &p, int fi, int local, double *smem)
{
    constexpr int NLD = 2 * LINES + 4, NTW = LINES / 8;
    constexpr int a_chunk_max = (kKC / 16) * (4 * MTW) * 256;
    double *As = smem;
    double *Bs = smem + (SINGLE ? 1 : 2) * a_chunk_max;

    const PassField &F = p.f[fi];
    const int plane = local / F.nchunks;
    const int chunk = local - plane * F.nchunks;
    const int l0 = chunk * LINES;
    const int L = min(LINES, F.nlines - l0);
    const double *src = F.src + (long long)plane * F.plane_stride;
    double *dst = F.dst + (long long)plane * F.plane_stride;
    const int tid = threadIdx.x;
    const int H = F.kpad, mtiles = F.mtiles, rows = 2 * H;
    const int nkc = H / kKC;
    const int a_chunk = (kKC / 16) * mtiles * 256;
    const int n = F.n, he = F.he, ho = F.ho, sk = F.sk, sl = F.sl, o1 = F.off;

    auto load_a = [&](int c, int buf) {
        const double *g = F.A + (size_t)c * a_chunk;
        double *sa = As + buf * a_chunk_max;
        for (int i = tid * 2; i < a_chunk; i += kThreads * 2) cp_async16(sa + i, g + i);
        cp_async_commit();
    };
    load_a(0, 0);

    // Raw rows by cp.async (all of a thread's copies in flight), placed so
    // that the fold is in place: row r < H holds point / mode r (r < he),
    // row H + j the partner of row j -- point n-1-j for par 1, odd mode
    // he + j for par 2 (j < ho); the other rows are zero.
    auto stage = [&](int r, int l) {
        const int j = r - H;
        const int k = (r < H) ? (r < he ? r : -1) : (j < ho ? (F.par == 1 ? n - 1 - j : he + j) : -1);
        const bool ok = k >= 0 && l < L;
        const double *gp = ok ? src + 2 * ((long long)(k + o1) * sk + (long long)(l0 + l + o1) * sl) : src;
        cp_async16_zfill(Bs + r * NLD + 2 * l, gp, ok);
    };
    if (sk == 1) {
        // groups of 8 threads take 4 consecutive points of 2 lines: 64-byte
        // runs in global memory, 8 distinct bank groups in shared memory
        const int rq = rows / 4;
        for (int idx = tid; idx < rows * LINES; idx += kThreads) {
            const int rest = idx >> 3;
            stage((rest % rq) * 4 + (idx & 3), (rest / rq) * 2 + ((idx >> 2) & 1));
        }
    } else {
        for (int idx = tid; idx < rows * LINES; idx += kThreads) stage(idx / LINES, idx % LINES);
    }
    cp_async_commit();
    if (F.par == 1) {
        // fold the pairs: row j <- in_j + in_{n-1-j}, row H + j <- in_j - in_{n-1-j}
        // (the middle point of an odd n stays in row ho of the even half)
        cp_async_wait<0>();
        __syncthreads();
        for (int idx = tid; idx < ho * LINES; idx += kThreads) {
            const int j = idx / LINES, l = idx % LINES;
            double2 *pa = reinterpret_cast<double2 *>(Bs + j * NLD + 2 * l);
            double2 *pb = reinterpret_cast<double2 *>(Bs + (H + j) * NLD + 2 * l);
            const double2 a = *pa, b = *pb;
            *pa = make_double2(a.x + b.x, a.y + b.y);
            *pb = make_double2(a.x - b.x, a.y - b.y);
        }
    }

    const int lane = tid & 31, warp = tid >> 5;
    const int wm = warp & 3, wn = warp >> 2;
    const int g = lane >> 2, t = lane & 3;
    const int kb0 = (wm * MTW * 16 >= H) ? H : 0;   // this warp's half of the staged rows
    // eigenvalues of the divide epilogue in shared memory (E of every row,
    // El of the CTA's lines), staged while the operator and lines arrive
    double *Es = Bs + rows * NLD;
    if (F.par == 1 && p.divide) {
        for (int i = tid; i < n; i += kThreads) Es[i] = F.E[i];
        for (int i = tid; i < L; i += kThreads) Es[rows + i] = F.El[l0 + i];
    }
    double acc[MTW][NTW][4];
#pragma unroll
    for (int i = 0; i < MTW; ++i)
#pragma unroll
        for (int j = 0; j < NTW; ++j)
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[i][j][v] = 0.0;

    for (int c = 0; c < nkc; ++c) {
        if (SINGLE) {
            // one operator buffer: chunk c is loaded once every warp is done
            // with chunk c - 1 (the barrier closing the previous iteration)
            if (c > 0) load_a(c, 0);
            cp_async_wait<0>();
        } else if (c + 1 < nkc) {
            load_a(c + 1, (c + 1) & 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const double *Ab = As + (SINGLE ? 0 : (c & 1) * a_chunk_max);
#pragma unroll
        for (int ks = 0; ks < kKC / 16; ++ks) {
            const int kg = kb0 + c * kKC + ks * 16 + t;
            double b[NTW][4];
#pragma unroll
            for (int nt = 0; nt < NTW; ++nt) {
                const int col = wn * LINES + nt * 8 + g;
#pragma unroll
                for (int v = 0; v < 4; ++v) b[nt][v] = Bs[(kg + 4 * v) * NLD + col];
            }
#pragma unroll
            for (int mt = 0; mt < MTW; ++mt) {
                const int mtg = wm * MTW + mt;
                double a[8];
                const double2 *q = reinterpret_cast<const double2 *>(Ab + (ks * mtiles + mtg) * 256) + lane;
#pragma unroll
                for (int h = 0; h < 4; ++h) {
                    const double2 v = q[32 * h];
                    a[2 * h] = v.x;
                    a[2 * h + 1] = v.y;
                }
#pragma unroll
                for (int nt = 0; nt < NTW; ++nt) dmma16(acc[mt][nt], a, b[nt]);
            }
        }
        __syncthreads();
    }

    const double lam = p.lam[F.plane0 + plane];
    const bool im0 = p.zero_im_mode0 && F.mode0 && plane == 0;
    if (F.par == 1) {
        const bool singular = (F.sing_io >= 0) && fabs(lam) <= 1.0e-10;
#pragma unroll
        for (int mt = 0; mt < MTW; ++mt)
#pragma unroll
            for (int nt = 0; nt < NTW; ++nt) {
                const int l = wn * (LINES / 2) + nt * 4 + t;
                if (l >= L) continue;
                const int lg = l0 + l;
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int orow = (wm * MTW + mt) * 16 + g + 8 * h;
                    const int o = orow < H ? (orow < he ? orow : -1) : (orow - H < ho ? he + orow - H : -1);
                    if (o < 0) continue;
                    double re = acc[mt][nt][2 * h], im = acc[mt][nt][2 * h + 1];
                    if (p.divide) {
                        if (singular && o == F.sing_io && lg == F.sing_l) {
                            re = 0.0;
                            im = 0.0;
                        } else {
                            const double rden = 1.0 / ((Es[o] + Es[rows + l]) - lam);
                            re *= rden;
                            im *= rden;
                        }
                    }
                    if (im0) im = 0.0;
                    const long long off = 2 * ((long long)(o + o1) * sk + (long long)(lg + o1) * sl);
                    *reinterpret_cast<double2 *>(dst + off) = make_double2(re, im);
                }
            }
        return;
    }
    // par 2: both halves through shared memory (the staged data is consumed).
    // With the output points contiguous in memory (sk == 1) the halves are
    // laid out line-major, 2H + 2 complex per line (conflict-free for the
    // accumulator writes), so consecutive threads read consecutive 16-byte
    // words and write consecutive points; otherwise row-major as staged.
    auto emit = [&](const double2 *ev, const double2 *od, int rs, int o, int l) {
        const int oh = o < he ? o : n - 1 - o;   // row of the halves (stride rs)
        double2 v = ev[oh * rs];
        if (oh < ho) {
            const double2 d = od[oh * rs];
            v = (o < he) ? make_double2(v.x + d.x, v.y + d.y) : make_double2(v.x - d.x, v.y - d.y);
        }
        if (im0) v.y = 0.0;
        *reinterpret_cast<double2 *>(dst + 2 * ((long long)(o + o1) * sk + (long long)(l0 + l + o1) * sl)) = v;
    };
    if (sk == 1) {
        double2 *Cs = reinterpret_cast<double2 *>(Bs);
        const int cld = 2 * H + 2;
#pragma unroll
        for (int mt = 0; mt < MTW; ++mt)
#pragma unroll
            for (int nt = 0; nt < NTW; ++nt)
#pragma unroll
                for (int h = 0; h < 2; ++h)
                    Cs[(wn * (LINES / 2) + nt * 4 + t) * cld + (wm * MTW + mt) * 16 + g + 8 * h] =
                        make_double2(acc[mt][nt][2 * h], acc[mt][nt][2 * h + 1]);
        __syncthreads();
        for (int idx = tid; idx < n * LINES; idx += kThreads) {
            const int o = idx % n, l = idx / n;
            if (l < L) emit(Cs + l * cld, Cs + l * cld + H, 1, o, l);
        }
    } else {
#pragma unroll
        for (int mt = 0; mt < MTW; ++mt)
#pragma unroll
            for (int nt = 0; nt < NTW; ++nt)
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int orow = (wm * MTW + mt) * 16 + g + 8 * h;
                    *reinterpret_cast<double2 *>(Bs + orow * NLD + wn * LINES + nt * 8 + 2 * t) =
                        make_double2(acc[mt][nt][2 * h], acc[mt][nt][2 * h + 1]);
                }
        __syncthreads();
        const double2 *Rs = reinterpret_cast<const double2 *>(Bs);
        for (int idx = tid; idx < n * LINES; idx += kThreads) {
            const int o = idx / LINES, l = idx % LINES;
            if (l < L) emit(Rs + l, Rs + H * (NLD / 2) + l, NLD / 2, o, l);
        }
    }
}

template <int MTW, int LINES, bool SINGLE = false>
__global__ void __launch_bounds__(kThreads, SINGLE ? 4 : (LINES == 16 ? 3 : (MTW == 3 ? 1 : 2)))
    k_pass_fp64s(const __grid_constant__ PassParams p)
{
    extern __shared__ __align__(16) double smem[];
    int fi = 0;
    while (fi + 1 < p.nf && (int)blockIdx.x >= p.cta_start[fi + 1]) ++fi;
    pass_s_tile<MTW, LINES, SINGLE>(p, fi, (int)blockIdx.x - p.cta_start[fi], smem);
}

// ---------------------------------------------------------------------------
// The four flip-symmetric passes of a batched solve in ONE persistent launch.
// CTAs take tiles from a global counter in pass order -- (pass, field,
// plane, chunk) -- and a tile of pass k > 0 first waits until every tile of
// the earlier passes of its plane is done (per-plane completion counters,
// released with a fence and an atomic add), so passes of different planes
// overlap and no launch boundary separates them.  Tiles are dequeued in
// dependency order by CTAs that are running, so every wait ends; each is
// still bounded: a wait that runs out raises the error word (code 1) and
// an abort flag that ends the other CTAs' waits and their dequeue loops.
struct PassQueue {
    PassParams pass[4];
    int items[5];                  // first tile of each pass; items[4]: all tiles
    int need[4][kMaxFields];       // tiles per plane of field i in the passes before k
    int plane_base[kMaxFields];    // field i's first per-plane counter
};
constexpr unsigned kQueueSpin = 1u << 22;

// ctr[0]: dequeue counter, ctr[1]: abort flag, ctr[2 + plane_base[i] + plane]:
// tiles done of that plane (all zero at launch)
__device__ __forceinline__ void queue_release(int *cnt)
{
    asm volatile("red.release.gpu.global.add.s32 [%0], 1;\n" ::"l"(cnt) : "memory");
}

// Thread 0 takes the next tile while the current one runs (the atomic's
// result is used only after it) and polls the new tile's dependency; warp 1
// releases the finished tile's count (one release after the CTA barrier
// that follows the tile's stores) in parallel with that poll.
template <int MTWMAX>
__global__ void __launch_bounds__(kThreads, MTWMAX == 3 ? 2 : 3)
    k_pass_fp64q(const __grid_constant__ PassQueue q, int *ctr, int *err)
{
    extern __shared__ __align__(16) double smem[];
    __shared__ int s_cur, s_stop;
    volatile int *abort = ctr + 1;
    const int tid = threadIdx.x, total = q.items[4];
    if (tid == 0) s_cur = atomicAdd(ctr, 1);
    __syncthreads();
    int *pending = nullptr;     // warp 1's lane 0: the count of the tile to release
    for (;;) {
        const int item = s_cur;
        if (item >= total) {
            if (tid == 32 && pending) queue_release(pending);
            return;
        }
        int k = 0;
        while (item >= q.items[k + 1]) ++k;
        const PassParams &p = q.pass[k];
        const int idx = item - q.items[k];
        int fi = 0;
        while (fi + 1 < p.nf && idx >= p.cta_start[fi + 1]) ++fi;
        const int local = idx - p.cta_start[fi];
        int *cnt = ctr + 2 + q.plane_base[fi] + local / p.f[fi].nchunks;
        int next = total;
        if (tid == 0) {
            next = *abort ? total : atomicAdd(ctr, 1);
            int stop = 0;
            if (k > 0) {
                const int need = q.need[k][fi];
                for (unsigned it = 0;; ++it) {
                    int v;
                    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];\n" : "=r"(v) : "l"(cnt) : "memory");
                    if (v >= need) break;
                    if ((it & 63) == 63 && *abort) {
                        stop = 1;
                        break;
                    }
                    if (it >= kQueueSpin) {
                        stop = 1;
                        atomicExch(err, 1);
                        atomicExch(ctr + 1, 1);
                        break;
                    }
                    __nanosleep(it < 64 ? 32 : 256);
                }
            }
            s_stop = stop;
        }
        if (tid == 32 && pending) {
            queue_release(pending);
            pending = nullptr;
        }
        __syncthreads();    // s_stop; every thread has read s_cur
        if (s_stop) return;
        const int mtw = p.f[fi].kpad / 32;
        if (mtw == 1) pass_s_tile<1, kParityLines>(p, fi, local, smem);
        else if (mtw == 2 && MTWMAX >= 2) pass_s_tile<MTWMAX >= 2 ? 2 : 1, kParityLines>(p, fi, local, smem);
        else if (MTWMAX >= 3) pass_s_tile<MTWMAX >= 3 ? 3 : 1, kParityLines>(p, fi, local, smem);
        if (tid == 32) pending = cnt;
        __syncthreads();    // the tile's stores issued, its shared memory consumed
        if (tid == 0) s_cur = next;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Register-streamed variant: the CTA stages its 32 complex lines once, in
// B-fragment order (so a lane's four k values are two contiguous 16-byte
// words), and each warp then runs its whole K loop without a CTA barrier:
// the operator fragments come straight from L2 (the packed operator is
// 128 KB at n = 127 and stays resident) with a one-k-step register
// prefetch.  WM warps along M own MT consecutive 16-row tiles each; the
// 8 / WM warps along N own 8 / (8 / WM) of the 8 column tiles.
// Packed B: index (((ks * 8 + nt) * 2 + half) * 32 + lane) * 2 + vv holds
// B[ks*16 + t + 4 (2 half + vv)][nt*8 + g], lane = 4 g + t.
template <int WM, int MT>
__global__ void __launch_bounds__(kThreads, (MT == 1) ? 2 : 1) k_pass_fp64r(const __grid_constant__ PassParams p)
{
    extern __shared__ __align__(16) double smem[];
    constexpr int WN = 8 / WM, NTW = 8 / WN;
    double *Bp = smem;

    int fi = 0;
    while (fi + 1 < p.nf && (int)blockIdx.x >= p.cta_start[fi + 1]) ++fi;
    const PassField &F = p.f[fi];
    const int local = blockIdx.x - p.cta_start[fi];
    const int plane = local / F.nchunks;
    const int chunk = local - plane * F.nchunks;
    const int l0 = chunk * kLines;
    const int L = min(kLines, F.nlines - l0);
    const double *src = F.src + (long long)plane * F.plane_stride;
    double *dst = F.dst + (long long)plane * F.plane_stride;
    const int tid = threadIdx.x;
    const int kpad = F.kpad, mtiles = F.mtiles;
    const int n = F.n, sk = F.sk, sl = F.sl, o1 = F.off;

    // stage: element (k, line l) -> real columns 2l (re), 2l+1 (im)
    for (int idx = tid; idx < kpad * kLines; idx += kThreads) {
        int k, l;
        if (sk == 1) { k = idx % kpad; l = idx / kpad; }
        else { l = idx % kLines; k = idx / kLines; }
        double2 v = make_double2(0.0, 0.0);
        if (k < n && l < L)
            v = *reinterpret_cast<const double2 *>(src + 2 * ((long long)(k + o1) * sk + (long long)(l0 + l + o1) * sl));
        const int ks = k >> 4, kk = k & 15, t = kk & 3, vq = kk >> 2;
        const int half = vq >> 1, vv = vq & 1;
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            const int col = 2 * l + c, nt = col >> 3, g = col & 7;
            Bp[((((ks * 8 + nt) * 2 + half) * 32 + (g * 4 + t)) * 2) + vv] = c ? v.y : v.x;
        }
    }
    __syncthreads();

    const int lane = tid & 31, warp = tid >> 5;
    const int wm = warp % WM, wn = warp / WM;
    const int g = lane >> 2, t = lane & 3;
    double acc[MT][NTW][4];
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < NTW; ++j)
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[i][j][v] = 0.0;

    const int nks = kpad >> 4;
    auto load_a = [&](int ks, int mt, double (&a)[8]) {
        const int mtg = wm * MT + mt;
        if (mtg >= mtiles) return;
        const double2 *q = reinterpret_cast<const double2 *>(F.A + (size_t)(ks * mtiles + mtg) * 256) + lane;
#pragma unroll
        for (int h = 0; h < 4; ++h) {
            const double2 v = __ldg(q + 32 * h);
            a[2 * h] = v.x;
            a[2 * h + 1] = v.y;
        }
    };
    double a_cur[MT][8], a_nxt[MT][8];
#pragma unroll
    for (int mt = 0; mt < MT; ++mt) load_a(0, mt, a_cur[mt]);
    for (int ks = 0; ks < nks; ++ks) {
        if (ks + 1 < nks) {
#pragma unroll
            for (int mt = 0; mt < MT; ++mt) load_a(ks + 1, mt, a_nxt[mt]);
        }
#pragma unroll
        for (int q = 0; q < NTW; ++q) {
            const int nt = wn * NTW + q;
            const double2 *bq = reinterpret_cast<const double2 *>(Bp + ((ks * 8 + nt) * 2) * 64) + lane;
            const double2 b01 = bq[0], b23 = bq[32];
            const double b[4] = {b01.x, b01.y, b23.x, b23.y};
#pragma unroll
            for (int mt = 0; mt < MT; ++mt) {
                if (wm * MT + mt >= mtiles) continue;
                dmma16(acc[mt][q], a_cur[mt], b);
            }
        }
#pragma unroll
        for (int mt = 0; mt < MT; ++mt)
#pragma unroll
            for (int v = 0; v < 8; ++v) a_cur[mt][v] = a_nxt[mt][v];
    }

    // epilogue as in k_pass_fp64: rows o of the accumulator, column pairs
    // (2t, 2t+1) of tile nt = (re, im) of line 4 nt + t
    const double lam = p.lam[F.plane0 + plane];
    const bool singular = (F.sing_io >= 0) && fabs(lam) <= 1.0e-10;
    const bool im0 = p.zero_im_mode0 && F.mode0 && plane == 0;
#pragma unroll
    for (int mt = 0; mt < MT; ++mt)
#pragma unroll
        for (int q = 0; q < NTW; ++q) {
            const int l = (wn * NTW + q) * 4 + t;
            if (l >= L) continue;
            const int lg = l0 + l;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int o = (wm * MT + mt) * 16 + g + 8 * h;
                if (o >= n) continue;
                double re = acc[mt][q][2 * h], im = acc[mt][q][2 * h + 1];
                if (p.divide) {
                    if (singular && o == F.sing_io && lg == F.sing_l) {
                        re = 0.0;
                        im = 0.0;
                    } else {
                        const double rden = 1.0 / ((F.E[o] + F.El[lg]) - lam);
                        re *= rden;
                        im *= rden;
                    }
                }
                const long long off = 2 * ((long long)(o + o1) * sk + (long long)(lg + o1) * sl);
                if (p.residual) {
                    const long long po = (long long)plane * F.plane_stride + off;
                    const double2 f = *reinterpret_cast<const double2 *>(F.resF + po);
                    const double2 tt = *reinterpret_cast<const double2 *>(F.resT + po);
                    const double2 uu = *reinterpret_cast<const double2 *>(F.resU + po);
                    re = (f.x - tt.x) - re + lam * uu.x;
                    im = (f.y - tt.y) - im + lam * uu.y;
                }
                if (im0) im = 0.0;
                *reinterpret_cast<double2 *>(dst + off) = make_double2(re, im);
            }
        }
}

template <int WM, int MT>
static cudaError_t launch_pass_r(ductgpu_ctx ctx, const PassParams &pp, int grid, int kpad_max)
{
    const size_t smem = (size_t)kpad_max * 64 * sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(k_pass_fp64r<WM, MT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    LaunchScope ls(ctx, DUCTGPU_K_PASS_FP64);
    k_pass_fp64r<WM, MT><<<grid, kThreads, smem, ctx->stream>>>(pp);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Persistent variant for operators up to 128 rows (n <= 127): one CTA per
// SM, 8 warps, each warp holding the A fragments of its 16-row tile for the
// whole K extent in registers (KS x 8 doubles per lane, loaded once per
// operator), looping over a contiguous range of 32-line tiles.  The next
// tile's lines are copied into the other half of a double-buffered shared
// memory tile with cp.async (zero-filled outside the field) while the
// current one is multiplied, so the DMMA pipe only idles for the epilogue
// and one barrier per tile.  MTILES 8: warp w owns rows 16w..16w+15 and all
// 64 columns; MTILES 4: warps w and w+4 share rows 16(w&3).. and split the
// columns.
template <int KS, int MTILES>
__global__ void __launch_bounds__(kThreads, 1) k_pass_fp64p(const __grid_constant__ PassParams p, int ntiles)
{
    extern __shared__ __align__(16) double smem[];
    constexpr int KPAD = 16 * KS, NTW = (MTILES == 8) ? 8 : 4;
    constexpr int TILE = KPAD * kNld;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int mtg = (MTILES == 8) ? warp : (warp & 3);
    const int ntb = (MTILES == 8) ? 0 : (warp >> 2) * 4;
    // this CTA's contiguous tile range
    const int per = ntiles / gridDim.x, extra = ntiles % gridDim.x;
    const int t0 = blockIdx.x * per + min((int)blockIdx.x, extra);
    const int t1 = t0 + per + ((int)blockIdx.x < extra ? 1 : 0);
    if (t0 >= t1) return;

    auto locate = [&](int tile, int &fi, int &plane, int &l0) {
        fi = 0;
        while (fi + 1 < p.nf && tile >= p.cta_start[fi + 1]) ++fi;
        const int local = tile - p.cta_start[fi];
        plane = local / p.f[fi].nchunks;
        l0 = (local - plane * p.f[fi].nchunks) * kLines;
    };
    auto stage = [&](int tile, int buf) {
        int fi, plane, l0;
        locate(tile, fi, plane, l0);
        const PassField &F = p.f[fi];
        const int L = min(kLines, F.nlines - l0);
        const double *src = F.src + (long long)plane * F.plane_stride;
        double *Bs = smem + buf * TILE;
        for (int idx = tid; idx < KPAD * kLines; idx += kThreads) {
            int k, l;
            if (F.sk == 1) { k = idx % KPAD; l = idx / KPAD; }
            else { l = idx % kLines; k = idx / kLines; }
            const bool ok = k < F.n && l < L;
            const double *gp = ok ? src + 2 * ((long long)(k + F.off) * F.sk + (long long)(l0 + l + F.off) * F.sl) : src;
            cp_async16_zfill(Bs + k * kNld + 2 * l, gp, ok);
        }
        cp_async_commit();
    };

    double a[KS][8];
    const double *a_src = nullptr;
    stage(t0, 0);
    for (int tile = t0; tile < t1; ++tile) {
        const int buf = (tile - t0) & 1;
        if (tile + 1 < t1) {
            stage(tile + 1, buf ^ 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        int fi, plane, l0;
        locate(tile, fi, plane, l0);
        const PassField &F = p.f[fi];
        if (F.A != a_src) {   // operator of this field: fragments into registers
            a_src = F.A;
#pragma unroll
            for (int ks = 0; ks < KS; ++ks) {
                const double2 *q = reinterpret_cast<const double2 *>(F.A + (size_t)(ks * MTILES + mtg) * 256) + lane;
#pragma unroll
                for (int h = 0; h < 4; ++h) {
                    const double2 v = __ldg(q + 32 * h);
                    a[ks][2 * h] = v.x;
                    a[ks][2 * h + 1] = v.y;
                }
            }
        }
        const double *Bs = smem + buf * TILE;
        double acc[NTW][4];
#pragma unroll
        for (int q = 0; q < NTW; ++q)
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[q][v] = 0.0;
#pragma unroll
        for (int ks = 0; ks < KS; ++ks) {
            const int kg = ks * 16 + t;
#pragma unroll
            for (int q = 0; q < NTW; ++q) {
                const int col = (ntb + q) * 8 + g;
                double b[4];
#pragma unroll
                for (int v = 0; v < 4; ++v) b[v] = Bs[(kg + 4 * v) * kNld + col];
                dmma16(acc[q], a[ks], b);
            }
        }
        // epilogue (as k_pass_fp64)
        const int L = min(kLines, F.nlines - l0);
        double *dst = F.dst + (long long)plane * F.plane_stride;
        const double lam = p.lam[F.plane0 + plane];
        const bool singular = (F.sing_io >= 0) && fabs(lam) <= 1.0e-10;
        const bool im0 = p.zero_im_mode0 && F.mode0 && plane == 0;
        const int n = F.n, sk = F.sk, sl = F.sl, o1 = F.off;
#pragma unroll
        for (int q = 0; q < NTW; ++q) {
            const int l = (ntb + q) * 4 + t;
            if (l >= L) continue;
            const int lg = l0 + l;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int o = mtg * 16 + g + 8 * h;
                if (o >= n) continue;
                double re = acc[q][2 * h], im = acc[q][2 * h + 1];
                if (p.divide) {
                    if (singular && o == F.sing_io && lg == F.sing_l) {
                        re = 0.0;
                        im = 0.0;
                    } else {
                        const double rden = 1.0 / ((F.E[o] + F.El[lg]) - lam);
                        re *= rden;
                        im *= rden;
                    }
                }
                const long long off = 2 * ((long long)(o + o1) * sk + (long long)(lg + o1) * sl);
                if (p.residual) {
                    const long long po = (long long)plane * F.plane_stride + off;
                    const double2 f = *reinterpret_cast<const double2 *>(F.resF + po);
                    const double2 tt = *reinterpret_cast<const double2 *>(F.resT + po);
                    const double2 uu = *reinterpret_cast<const double2 *>(F.resU + po);
                    re = (f.x - tt.x) - re + lam * uu.x;
                    im = (f.y - tt.y) - im + lam * uu.y;
                }
                if (im0) im = 0.0;
                *reinterpret_cast<double2 *>(dst + off) = make_double2(re, im);
            }
        }
        __syncthreads();   // the buffer is refilled by the next iteration's stage
    }
}

template <int KS, int MTILES>
static cudaError_t launch_pass_p(ductgpu_ctx ctx, const PassParams &pp, int ntiles)
{
    const size_t smem = 2 * (size_t)16 * KS * kNld * sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(k_pass_fp64p<KS, MTILES>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int grid = ntiles < ctx->num_sms ? ntiles : ctx->num_sms;
    LaunchScope ls(ctx, DUCTGPU_K_PASS_FP64);
    k_pass_fp64p<KS, MTILES><<<grid, kThreads, smem, ctx->stream>>>(pp, ntiles);
    return cudaGetLastError();
}

static size_t pass_smem_bytes(int mtw, int kpad, int lines, int abuf = 2)
{
    const size_t a_chunk = (size_t)(kKC / 16) * (4 * mtw) * 256;
    return (abuf * a_chunk + (size_t)kpad * (2 * lines + 4)) * sizeof(double);
}

template <int MTW, int LINES, bool SINGLE = false>
static cudaError_t launch_pass_s(ductgpu_ctx ctx, const PassParams &pp, int hpad_max)
{
    // LINES-line tiles: re-cut the callers' 32-line grid
    PassParams q = pp;
    int grid = 0;
    for (int i = 0; i < q.nf; ++i) {
        q.f[i].nchunks = (q.f[i].nlines + LINES - 1) / LINES;
        q.cta_start[i] = grid;
        grid += q.f[i].nmodes * q.f[i].nchunks;
    }
    q.cta_start[q.nf] = grid;
    // + the eigenvalue staging of the divide epilogue (n <= 2 hpad rows, LINES lines)
    const size_t smem = pass_smem_bytes(MTW, 2 * hpad_max, LINES, SINGLE ? 1 : 2) +
                        (size_t)(2 * hpad_max + LINES) * sizeof(double);
    cudaError_t e =
        cudaFuncSetAttribute(k_pass_fp64s<MTW, LINES, SINGLE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    LaunchScope ls(ctx, DUCTGPU_K_PASS_FP64);
    k_pass_fp64s<MTW, LINES, SINGLE><<<grid, kThreads, smem, ctx->stream>>>(q);
    return cudaGetLastError();
}

template <int MTWMAX>
static int launch_pass_q(ductgpu_ctx ctx, const PassQueue &q, int *ctr, int tiles)
{
    const int hmax = 32 * MTWMAX;
    const size_t smem = pass_smem_bytes(MTWMAX, 2 * hmax, kParityLines) + (size_t)(2 * hmax + kParityLines) * sizeof(double);
    DUCT_CUDA(ctx, cudaFuncSetAttribute(k_pass_fp64q<MTWMAX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    DUCT_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pass_fp64q<MTWMAX>, kThreads, smem));
    if (per_sm < 1) return set_error(ctx, DUCTGPU_ECUDA, "queued passes: no CTA fits an SM");
    const int grid = tiles < per_sm * ctx->num_sms ? tiles : per_sm * ctx->num_sms;
    {
        LaunchScope ls(ctx, DUCTGPU_K_PASS_FP64);
        k_pass_fp64q<MTWMAX><<<grid, kThreads, smem, ctx->stream>>>(q, ctr, ctx->dev_err);
    }
    return check_cuda(ctx, cudaGetLastError(), "k_pass_fp64q");
}

// The four flip-symmetric passes pp[0..3] of a batched solve (every field
// folded, the same fields in each pass) as one persistent launch.
int fp64_pass_queue(ductgpu_ctx ctx, const PassParams *pp)
{
    PassQueue q{};
    const int nf = pp[0].nf;
    int tiles = 0, mtw = 1, planes = 0;
    for (int k = 0; k < 4; ++k) {
        PassParams &p = q.pass[k];
        p = pp[k];
        if (p.nf != nf || p.residual) return set_error(ctx, DUCTGPU_EARG, "queued passes: pass %d", k);
        int grid = 0;
        for (int i = 0; i < nf; ++i) {
            PassField &f = p.f[i];
            if (!f.par || (f.kpad != 32 && f.kpad != 64 && f.kpad != 96) || f.nmodes != pp[0].f[i].nmodes)
                return set_error(ctx, DUCTGPU_EARG, "queued passes: pass %d field %d", k, i);
            f.nchunks = (f.nlines + kParityLines - 1) / kParityLines;
            p.cta_start[i] = grid;
            grid += f.nmodes * f.nchunks;
            mtw = f.kpad / 32 > mtw ? f.kpad / 32 : mtw;
        }
        p.cta_start[nf] = grid;
        q.items[k] = tiles;
        tiles += grid;
    }
    q.items[4] = tiles;
    for (int i = 0; i < nf; ++i) {
        q.plane_base[i] = planes;
        planes += q.pass[0].f[i].nmodes;
        int acc = 0;
        for (int k = 0; k < 4; ++k) {
            q.need[k][i] = acc;
            acc += q.pass[k].f[i].nchunks;
        }
    }
    if (tiles <= 0) return DUCTGPU_OK;
    const size_t cbytes = (size_t)(2 + planes) * sizeof(int);
    // sized once for 16 fields x 256 modes: a captured graph keeps the pointer
    const size_t cap = cbytes > (2 + 16 * 256) * sizeof(int) ? cbytes : (2 + 16 * 256) * sizeof(int);
    if (ctx->pq_cap < cbytes) {
        if (ctx->capturing)
            return set_error(ctx, DUCTGPU_ESTATE, "queued passes: counters first sized inside a capture");
        cudaFree(ctx->pq_ctr);
        ctx->pq_ctr = nullptr;
        ctx->pq_cap = 0;
        DUCT_CUDA(ctx, cudaMalloc(&ctx->pq_ctr, cap));
        ctx->pq_cap = cap;
    }
    DUCT_CUDA(ctx, cudaMemsetAsync(ctx->pq_ctr, 0, cbytes, ctx->stream));
    switch (mtw) {
    case 1: return launch_pass_q<1>(ctx, q, ctx->pq_ctr, tiles);
    case 2: return launch_pass_q<2>(ctx, q, ctx->pq_ctr, tiles);
    default: return launch_pass_q<3>(ctx, q, ctx->pq_ctr, tiles);
    }
}

template <int MTW, int LINES>
static cudaError_t launch_pass(ductgpu_ctx ctx, const PassParams &pp, int grid, int kpad_max)
{
    const size_t smem = pass_smem_bytes(MTW, kpad_max, LINES);
    cudaError_t e = cudaFuncSetAttribute(k_pass_fp64<MTW, LINES>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    LaunchScope ls(ctx, DUCTGPU_K_PASS_FP64);
    k_pass_fp64<MTW, LINES><<<grid, kThreads, smem, ctx->stream>>>(pp);
    return cudaGetLastError();
}

void pass_geometry(PassField &f, const BoundOps &b, const double *El, int nlines, int sk, int sl,
                   long long plane_stride)
{
    f.n = b.n;
    f.kpad = b.kpad;
    f.mtiles = b.mtiles;
    f.E = b.E;
    f.El = El;
    f.nlines = nlines;
    f.nchunks = (nlines + kLines - 1) / kLines;
    f.sk = sk;
    f.sl = sl;
    f.off = 1;
    f.plane_stride = plane_stride;
}

// ---------------------------------------------------------------------------
// Walls of Dirichlet fields: helm3d zeroes the four wall lines of rhs in
// place (src/helm3d.f90:48-60) and the solution keeps them
// (src/solvediag.f90:131-135 writes only the interior); mode 0 has a zero
// imaginary part everywhere (src/int2d3d.f90:91-96).
struct WallParams {
    double *rhs[kMaxFields];
    double *sol[kMaxFields];
    int cta_start[kMaxFields + 1];
    int nf;
    int m;
    long long plane_stride;
};

__global__ void k_zero_walls(const __grid_constant__ WallParams p)
{
    int fi = 0;
    while (fi + 1 < p.nf && (int)blockIdx.x >= p.cta_start[fi + 1]) ++fi;
    const int plane = blockIdx.x - p.cta_start[fi];
    const int m = p.m;
    double *r = p.rhs[fi] + (long long)plane * p.plane_stride;
    double *s = p.sol[fi] + (long long)plane * p.plane_stride;
    for (int i = threadIdx.x; i < 4 * m; i += blockDim.x) {
        const int side = i / m, q = i % m;
        long long off;
        if (side == 0) off = q;                           // U(q,1)
        else if (side == 1) off = q + (long long)m * (m - 1);  // U(q,m)
        else if (side == 2) off = (long long)m * q;       // U(1,q)
        else off = (m - 1) + (long long)m * q;            // U(m,q)
        const double2 z = make_double2(0.0, 0.0);
        *reinterpret_cast<double2 *>(r + 2 * off) = z;
        *reinterpret_cast<double2 *>(s + 2 * off) = z;
    }
}

// ---------------------------------------------------------------------------
// Neumann walls, corners and the singular kx=0 mode: src/solvediag.f90:
// 161-206 (pin), 250-276 (wall lines from DC), 278-322 (corners via AM1).
// One CTA per complex plane; the interior is already solved.
constexpr int kMaxSing = 64;   // singular planes per pin launch
struct FillParams {
    double *sol[kMaxFields];
    int mode0[kMaxFields];
    int plane0[kMaxFields];
    int cta_start[kMaxFields + 1];
    int nf;
    const double *DC, *AM1, *ccw, *pcol, *lam;
    const double *dcr;          // rows 1 and m of DC, contiguous
    double *pin_cc;             // [2 * kMaxSing] point-gauge coefficients
    int sing_fi[kMaxSing], sing_plane[kMaxSing], nsing;
    double wanted;
    int m, io, gauge;
    long long plane_stride;
};

__device__ __forceinline__ double2 operator+(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 operator*(double s, double2 a) { return make_double2(s * a.x, s * a.y); }

template <int NV>
__device__ void block_sum(double (&v)[NV], double *red)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int i = 0; i < NV; ++i)
        for (int o = 16; o > 0; o >>= 1) v[i] += __shfl_xor_sync(0xffffffffu, v[i], o);
    __syncthreads();
    if (lane == 0)
        for (int i = 0; i < NV; ++i) red[warp * NV + i] = v[i];
    __syncthreads();
    for (int i = 0; i < NV; ++i) {
        double s = 0.0;
        for (int w = 0; w < nw; ++w) s += red[w * NV + i];
        v[i] = s;
    }
    __syncthreads();
}

__device__ __forceinline__ int fill_field(const FillParams &p)
{
    int fi = 0;
    while (fi + 1 < p.nf && (int)blockIdx.x >= p.cta_start[fi + 1]) ++fi;
    return fi;
}

// Point gauge of the singular planes (|lambda| <= 1e-10, the kx = 0
// pressure mode): the field plus c P(:,io) P(:,io)^T, with c chosen so that
// the point (iofzero+1, iofzero+1) takes the value wanted
// (src/solvediag.f90:195-206, the reference's choice of FT(iofzero,iofzero)).
// Two steps, so that the update can be spread over many CTAs: k_pin_coef
// reads the point of every listed plane and stores c; k_neumann_partials
// applies it block by block and never reads the point it may be changing.
__global__ void k_pin_coef(const __grid_constant__ FillParams p)
{
    const int s = threadIdx.x;
    if (s >= p.nsing) return;
    const int m = p.m, io = p.io;
    const double2 *U = reinterpret_cast<const double2 *>(p.sol[p.sing_fi[s]] + (long long)p.sing_plane[s] * p.plane_stride);
    const double2 u0 = U[(io + 1) + (long long)m * (io + 1)];
    const double pio = p.pcol[io];
    p.pin_cc[2 * s] = (p.wanted - u0.x) / (pio * pio);
    p.pin_cc[2 * s + 1] = (p.wanted - u0.y) / (pio * pio);
}

// Neumann walls, corners and (for the zero-mean gauge) the constant shift,
// in two kernels that read each interior plane once.
// k_neumann_partials: one CTA per 32 x 32 interior block (blockIdx.y =
// T tz + ty, T = ceil(n / 32) blocks a direction) applies the point gauge to its block (singular planes, c from
// k_pin_coef) and writes, for each of its columns, the sums over its rows
// of DC(1,i) U(i,j) and DC(m,i) U(i,j) (the y walls' dot products,
// src/solvediag.f90:253-264), and for each of its rows the sums over its
// columns of DC(1,j) U(i,j) and DC(m,j) U(i,j) (the z walls, :265-276).
// k_neumann_finish: one CTA per plane adds the T blocks' partial sums in
// a fixed order, writes the wall lines, then the corners through AM1
// (:278-322) and, for the zero-mean gauge, the constant shift.
__global__ void __launch_bounds__(256) k_neumann_partials(const __grid_constant__ FillParams p, double *part)
{
    __shared__ double zs[8][32][4];
    const int fi = fill_field(p);
    const int plane = blockIdx.x - p.cta_start[fi], gp = blockIdx.x;
    const int m = p.m, n = m - 2, np = gridDim.x, T = (n + 31) / 32;
    const int ty = blockIdx.y % T, tz = blockIdx.y / T;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double2 *U = reinterpret_cast<double2 *>(p.sol[fi] + (long long)plane * p.plane_stride);
    int sg = -1;
    for (int q = 0; q < p.nsing; ++q)
        if (p.sing_fi[q] == fi && p.sing_plane[q] == plane) sg = q;
    const double2 cc = (sg >= 0) ? make_double2(p.pin_cc[2 * sg], p.pin_cc[2 * sg + 1]) : make_double2(0.0, 0.0);
    const int i = 1 + ty * 32 + lane;
    const bool iok = i <= n;
    const double ai = iok ? p.dcr[i] : 0.0, bi = iok ? p.dcr[m + i] : 0.0;
    const double pin_i = (sg >= 0 && iok) ? p.pcol[i - 1] : 0.0;
    double z[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const int j = 1 + tz * 32 + warp * 4 + c;
        const bool jok = j <= n;
        double2 v = make_double2(0.0, 0.0);
        if (iok && jok) {
            v = U[i + (long long)m * j];
            if (sg >= 0) {
                const double w = pin_i * p.pcol[j - 1];
                v = make_double2(v.x + w * cc.x, v.y + w * cc.y);
                U[i + (long long)m * j] = v;
            }
        }
        double y[4] = {ai * v.x, ai * v.y, bi * v.x, bi * v.y};
#pragma unroll
        for (int q = 0; q < 4; ++q)
            for (int o = 16; o > 0; o >>= 1) y[q] += __shfl_xor_sync(0xffffffffu, y[q], o);
        if (lane == 0 && jok) {
            double *py = part + ((long long)(gp * T + ty) * m + j) * 4;
#pragma unroll
            for (int q = 0; q < 4; ++q) py[q] = y[q];
        }
        const double aj = jok ? p.dcr[j] : 0.0, bj = jok ? p.dcr[m + j] : 0.0;
        z[0] += aj * v.x; z[1] += aj * v.y; z[2] += bj * v.x; z[3] += bj * v.y;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) zs[warp][lane][q] = z[q];
    __syncthreads();
    if (warp == 0 && iok) {
        double *pz = part + (long long)np * T * m * 4 + ((long long)(gp * T + tz) * m + i) * 4;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            double t = zs[0][lane][q];
            for (int w = 1; w < 8; ++w) t += zs[w][lane][q];
            pz[q] = t;
        }
    }
}

__global__ void __launch_bounds__(256) k_neumann_finish(const __grid_constant__ FillParams p, const double *part)
{
    __shared__ double red[8 * 8];
    const int fi = fill_field(p);
    const int plane = blockIdx.x - p.cta_start[fi], gp = blockIdx.x;
    const int m = p.m, n = m - 2, np = gridDim.x, T = (n + 31) / 32;
    double2 *U = reinterpret_cast<double2 *>(p.sol[fi] + (long long)plane * p.plane_stride);
    auto u = [&](int i, int j) -> double2 & { return U[i + (long long)m * j]; };
    const double *DC = p.DC;
    const double d11 = DC[0], d1m = DC[(long long)m * (m - 1)];
    const double dm1 = DC[m - 1], dmm = DC[(m - 1) + (long long)m * (m - 1)];
    const double idet = 1.0 / (d11 * dmm - d1m * dm1);
    for (int k = 1 + threadIdx.x; k <= n; k += blockDim.x) {
        double sy[4] = {0.0, 0.0, 0.0, 0.0}, sz[4] = {0.0, 0.0, 0.0, 0.0};
        for (int t = 0; t < T; ++t) {
            const double *py = part + ((long long)(gp * T + t) * m + k) * 4;
            const double *pz = part + (long long)np * T * m * 4 + ((long long)(gp * T + t) * m + k) * 4;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                sy[q] += py[q];
                sz[q] += pz[q];
            }
        }
        // y walls of column k, z walls of row k
        u(0, k) = make_double2((-dmm * sy[0] + d1m * sy[2]) * idet, (-dmm * sy[1] + d1m * sy[3]) * idet);
        u(m - 1, k) = make_double2((dm1 * sy[0] - d11 * sy[2]) * idet, (dm1 * sy[1] - d11 * sy[3]) * idet);
        u(k, 0) = make_double2((-dmm * sz[0] + d1m * sz[2]) * idet, (-dmm * sz[1] + d1m * sz[3]) * idet);
        u(k, m - 1) = make_double2((dm1 * sz[0] - d11 * sz[2]) * idet, (dm1 * sz[1] - d11 * sz[3]) * idet);
    }
    __syncthreads();   // the wall lines of this plane, written above, feed the corners
    double f[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int i = 1 + threadIdx.x; i < m - 1; i += blockDim.x) {
        const double a = p.dcr[i], b = p.dcr[m + i];
        const double2 ui0 = u(i, 0), u0i = u(0, i), umi = u(m - 1, i), uim = u(i, m - 1);
        f[0] += -a * (ui0.x + u0i.x);            f[1] += -a * (ui0.y + u0i.y);
        f[2] += -a * umi.x + b * ui0.x;          f[3] += -a * umi.y + b * ui0.y;
        f[4] += -b * (uim.x + umi.x);            f[5] += -b * (uim.y + umi.y);
        f[6] += -a * uim.x + b * u0i.x;          f[7] += -a * uim.y + b * u0i.y;
    }
    block_sum<8>(f, red);
    if (threadIdx.x == 0) {
        const double *A = p.AM1;
        double c[8];
        for (int r = 0; r < 4; ++r) {
            c[2 * r] = c[2 * r + 1] = 0.0;
            for (int i = 0; i < 4; ++i) {
                c[2 * r] += A[r + 4 * i] * f[2 * i];
                c[2 * r + 1] += A[r + 4 * i] * f[2 * i + 1];
            }
        }
        u(0, 0) = make_double2(c[0], c[1]);
        u(m - 1, 0) = make_double2(c[2], c[3]);
        u(m - 1, m - 1) = make_double2(c[4], c[5]);
        u(0, m - 1) = make_double2(c[6], c[7]);
    }
    const double lam = p.lam[p.plane0[fi] + plane];
    if (p.gauge == DUCTGPU_GAUGE_MEAN && fabs(lam) <= 1.0e-10) {
        __syncthreads();
        // Zero mean over [-1,1]^2 with the Clenshaw-Curtis weights of the
        // nodes: subtract integral/4 (a constant keeps the Neumann walls).
        double s[2] = {0.0, 0.0};
        for (int idx = threadIdx.x; idx < m * m; idx += blockDim.x) {
            const int i = idx % m, j = idx / m;
            const double w = p.ccw[i] * p.ccw[j];
            const double2 v = u(i, j);
            s[0] += w * v.x;
            s[1] += w * v.y;
        }
        block_sum<2>(s, red);
        for (int idx = threadIdx.x; idx < m * m; idx += blockDim.x) {
            const int i = idx % m, j = idx / m;
            u(i, j) = make_double2(u(i, j).x - 0.25 * s[0], u(i, j).y - 0.25 * s[1]);
        }
    }
}

// ---------------------------------------------------------------------------

static int plane_count(const FieldTask *t, int nt)
{
    int s = 0;
    for (int i = 0; i < nt; ++i) s += t[i].nmodes;
    return s;
}

int fp64_pass(ductgpu_ctx ctx, const PassParams &pp, int grid)
{
    int mt_max = 4, kpad_max = 32;
    for (int i = 0; i < pp.nf; ++i) {
        mt_max = pp.f[i].mtiles > mt_max ? pp.f[i].mtiles : mt_max;
        kpad_max = pp.f[i].kpad > kpad_max ? pp.f[i].kpad : kpad_max;
    }
    const int mtw = mt_max / 4;
    if (mtw < 1 || mtw > 3) return set_error(ctx, DUCTGPU_EARG, "operator larger than %d", kMaxN);
    const int variant = ctx->pass_variant[mtw - 1];
    cudaError_t e;
    if (pp.f[0].par) {
        // flip-symmetric half operators: solve_fp64_ex sets every field or
        // none, kpad = hpad = 32 mtw, and uses no residual epilogue
        for (int i = 0; i < pp.nf; ++i)
            if (!pp.f[i].par || pp.f[i].kpad != 32 * mtw || pp.residual)
                return set_error(ctx, DUCTGPU_EARG, "flip-symmetric pass: inconsistent field %d", i);
        // the persistent warp-specialised form pays one operator load per
        // CTA: used when every SM gets several 16-line tiles
        long long tiles = 0;
        bool lines_fit = true;   // the persistent form stages the line eigenvalues in 2 hpad slots
        for (int i = 0; i < pp.nf; ++i) {
            tiles += (long long)pp.f[i].nmodes * ((pp.f[i].nlines + 15) / 16);
            lines_fit = lines_fit && pp.f[i].nlines <= 2 * pp.f[i].kpad;
        }
        if (ctx->parity_ws && mtw <= 2 && lines_fit && tiles >= 6LL * ctx->num_sms) {
            e = fp64_pass_ws(ctx, pp, 32 * mtw);
            return e == cudaSuccess ? DUCTGPU_OK : check_cuda(ctx, e, "k_pass_fp64w");
        }
        switch (mtw) {
        case 1: e = launch_pass_s<1, kParityLines>(ctx, pp, kpad_max); break;
        case 2: e = launch_pass_s<2, kParityLines>(ctx, pp, kpad_max); break;
        // 96-row half blocks: 8 lines and one operator buffer, 57 KB, four
        // CTAs per SM (the double-buffered 16-line tile takes 106 KB and
        // fits twice): config-4 solves 2.99 -> 2.74 ms a step.  The same
        // form at 32 rows was slower (config 2: 0.410 -> 0.473 ms), at 64
        // rows no faster (0.412 ms either way).
        default: e = launch_pass_s<3, 8, true>(ctx, pp, kpad_max); break;
        }
        return e == cudaSuccess ? DUCTGPU_OK : check_cuda(ctx, e, "k_pass_fp64s");
    }
    bool uniform = true;
    for (int i = 1; i < pp.nf; ++i)
        uniform = uniform && pp.f[i].kpad == pp.f[0].kpad && pp.f[i].mtiles == pp.f[0].mtiles;
    if (variant == DUCTGPU_PASS_PERSIST && uniform && (pp.f[0].mtiles == 4 || pp.f[0].mtiles == 8)) {
        const int ks = pp.f[0].kpad / 16;
        if (pp.f[0].mtiles == 8) {
            switch (ks) {
            case 6: e = launch_pass_p<6, 8>(ctx, pp, grid); break;
            default: e = launch_pass_p<8, 8>(ctx, pp, grid); break;
            }
        } else {
            switch (ks) {
            case 2: e = launch_pass_p<2, 4>(ctx, pp, grid); break;
            default: e = launch_pass_p<4, 4>(ctx, pp, grid); break;
            }
        }
    } else if (variant == DUCTGPU_PASS_REGISTER) {
        switch (mtw) {
        case 1: e = launch_pass_r<4, 1>(ctx, pp, grid, kpad_max); break;
        case 2: e = launch_pass_r<8, 1>(ctx, pp, grid, kpad_max); break;
        default: e = launch_pass_r<4, 3>(ctx, pp, grid, kpad_max); break;
        }
    } else if (variant == DUCTGPU_PASS_STAGED16) {
        // 16 lines per CTA: the callers' grid is for 32; re-cut it
        PassParams q = pp;
        int cta = 0;
        for (int i = 0; i < q.nf; ++i) {
            q.f[i].nchunks = (q.f[i].nlines + 15) / 16;
            q.cta_start[i] = cta;
            cta += q.f[i].nmodes * q.f[i].nchunks;
        }
        q.cta_start[q.nf] = cta;
        switch (mtw) {
        case 1: e = launch_pass<1, 16>(ctx, q, cta, kpad_max); break;
        case 2: e = launch_pass<2, 16>(ctx, q, cta, kpad_max); break;
        default: e = launch_pass<3, 16>(ctx, q, cta, kpad_max); break;
        }
    } else {
        switch (mtw) {
        case 1: e = launch_pass<1, 32>(ctx, pp, grid, kpad_max); break;
        case 2: e = launch_pass<2, 32>(ctx, pp, grid, kpad_max); break;
        default: e = launch_pass<3, 32>(ctx, pp, grid, kpad_max); break;
        }
    }
    return e == cudaSuccess ? DUCTGPU_OK : check_cuda(ctx, e, "k_pass_fp64");
}

// Grid of a pass: CTA ranges per field (planes x line chunks).
static int pass_grid(PassParams &pp, const FieldTask *tasks, int ntasks)
{
    int cta = 0;
    for (int i = 0; i < ntasks; ++i) {
        pp.cta_start[i] = cta;
        cta += tasks[i].nmodes * pp.f[i].nchunks;
    }
    pp.cta_start[ntasks] = cta;
    pp.nf = ntasks;
    return cta;
}

int solve_fp64(ductgpu_ctx ctx, const FieldTask *tasks, int ntasks) { return solve_fp64_ex(ctx, tasks, ntasks, false); }

bool use_fold(ductgpu_ctx ctx, const FieldTask *tasks, int ntasks)
{
    const int v = ctx->pass_variant[(ctx->dir.mtiles / 4) - 1];
    if (v != DUCTGPU_PASS_PARITY && v != DUCTGPU_PASS_PARITY_QUEUE) return false;
    for (int i = 0; i < ntasks; ++i)
        if (!((tasks[i].bound == 'n') ? ctx->neu : ctx->dir).fold_ok) return false;
    return true;
}

void fold_field(PassField &f, const BoundOps &b, int par, const double *A, bool neumann)
{
    f.par = par;
    f.A = A;
    f.kpad = b.hpad;
    f.mtiles = 2 * b.hpad / 16;
    f.he = b.he;
    f.ho = b.ho;
    f.E = f.El = b.Eperm;
    f.sing_io = f.sing_l = neumann ? b.sing_perm : -1;
}

int solve_fp64_ex(ductgpu_ctx ctx, const FieldTask *tasks, int ntasks, bool emulate)
{
    if (ntasks < 1 || ntasks > kMaxFields)
        return set_error(ctx, DUCTGPU_EARG, "solve: %d fields (1..%d)", ntasks, kMaxFields);
    const int m = ctx->my, n = m - 2;
    const long long ps = 2LL * m * m;
    const int planes = plane_count(tasks, ntasks);
    int rc = ensure(ctx, ctx->work, (size_t)2 * planes * ps * sizeof(double));
    if (rc) return rc;
    double *w1 = ctx->work.buf;
    double *w2 = w1 + (size_t)planes * ps;

    PassParams pp{};
    pp.lam = ctx->lam;
    // flip-symmetric half operators for all four passes (the intermediate
    // mode order differs), when selected and every field's operators have them
    const bool fold = !emulate && use_fold(ctx, tasks, ntasks);
    for (int i = 0; i < ntasks; ++i) {
        pp.f[i].nmodes = tasks[i].nmodes;
        pp.f[i].mode0 = tasks[i].mode0;
        pp.f[i].plane0 = tasks[i].plane0;
        pp.f[i].sing_io = (tasks[i].bound == 'n') ? ctx->neu.iofzero - 1 : -1;
        pp.f[i].sing_l = pp.f[i].sing_io;
    }
    // the four folded passes as one persistent launch
    const bool queue = fold && ctx->pass_variant[(ctx->dir.mtiles / 4) - 1] == DUCTGPU_PASS_PARITY_QUEUE;
    PassParams qp[4];
    // pass 1 (y, P^-1): rhs -> w1 ; pass 2 (z, P^-1, divide): w1 -> w2 ;
    // pass 3 (z, P): w2 -> w1 ; pass 4 (y, P): w1 -> sol
    for (int pass = 0; pass < 4; ++pass) {
        long long off = 0;
        const bool ypass = (pass == 0 || pass == 3);
        for (int i = 0; i < ntasks; ++i) {
            const BoundOps &b = (tasks[i].bound == 'n') ? ctx->neu : ctx->dir;
            double *a1 = w1 + off * ps, *a2 = w2 + off * ps;
            off += tasks[i].nmodes;
            switch (pass) {
            case 0: pp.f[i].src = tasks[i].rhs; pp.f[i].dst = a1; pp.f[i].A = b.Qpack; break;
            case 1: pp.f[i].src = a1; pp.f[i].dst = a2; pp.f[i].A = b.Qpack; break;
            case 2: pp.f[i].src = a2; pp.f[i].dst = a1; pp.f[i].A = b.Ppack; break;
            default: pp.f[i].src = a1; pp.f[i].dst = tasks[i].sol; pp.f[i].A = b.Ppack; break;
            }
            pp.f[i].Ai8 = (pass < 2) ? b.Qi8 : b.Pi8;
            pp.f[i].Aexp = (pass < 2) ? b.Qexp8 : b.Pexp8;
            pass_geometry(pp.f[i], b, b.E, n, ypass ? 1 : m, ypass ? m : 1, ps);
            if (fold)
                fold_field(pp.f[i], b, (pass < 2) ? 1 : 2, (pass < 2) ? b.Qfold : b.Pfold, tasks[i].bound == 'n');
        }
        const int cta = pass_grid(pp, tasks, ntasks);
        pp.divide = (pass == 1);
        pp.zero_im_mode0 = (pass == 3);
        pp.residual = 0;
        if (queue) qp[pass] = pp;
        else if ((rc = emulate ? i8_pass(ctx, pp, cta) : fp64_pass(ctx, pp, cta))) return rc;
    }
    if (queue && (rc = fp64_pass_queue(ctx, qp))) return rc;
    if ((rc = zero_walls(ctx, tasks, ntasks))) return rc;
    return neumann_fill(ctx, tasks, ntasks);
}

int zero_walls(ductgpu_ctx ctx, const FieldTask *tasks, int ntasks)
{
    WallParams wp{};
    int cta = 0;
    for (int i = 0; i < ntasks; ++i) {
        if (tasks[i].bound != 'd') continue;
        wp.rhs[wp.nf] = tasks[i].rhs;
        wp.sol[wp.nf] = tasks[i].sol;
        wp.cta_start[wp.nf] = cta;
        cta += tasks[i].nmodes;
        wp.nf++;
    }
    if (!wp.nf) return DUCTGPU_OK;
    wp.cta_start[wp.nf] = cta;
    wp.m = ctx->my;
    wp.plane_stride = 2LL * ctx->my * ctx->my;
    {
        LaunchScope ls(ctx, DUCTGPU_K_WALLS);
        k_zero_walls<<<cta, 128, 0, ctx->stream>>>(wp);
    }
    return check_cuda(ctx, cudaGetLastError(), "k_zero_walls");
}

int neumann_fill(ductgpu_ctx ctx, const FieldTask *tasks, int ntasks)
{
    FillParams fp{};
    int cta = 0;
    for (int i = 0; i < ntasks; ++i) {
        if (tasks[i].bound != 'n') continue;
        fp.sol[fp.nf] = tasks[i].sol;
        fp.mode0[fp.nf] = tasks[i].mode0;
        fp.plane0[fp.nf] = tasks[i].plane0;
        fp.cta_start[fp.nf] = cta;
        cta += tasks[i].nmodes;
        fp.nf++;
    }
    if (!fp.nf) return DUCTGPU_OK;
    fp.cta_start[fp.nf] = cta;
    fp.DC = ctx->DC;
    fp.dcr = ctx->dcr;
    fp.pin_cc = ctx->pin_cc;
    fp.AM1 = ctx->AM1;
    fp.ccw = ctx->ccw;
    fp.pcol = ctx->neu.pcol;
    fp.lam = ctx->lam;
    fp.wanted = ctx->wanted;
    fp.m = ctx->my;
    fp.io = ctx->neu.iofzero > 0 ? pin_index(ctx) : -1;
    fp.gauge = ctx->gauge;
    fp.plane_stride = 2LL * ctx->my * ctx->my;
    // the pin only acts on singular planes (|lambda| <= 1e-10, the kx=0
    // pressure mode), listed on the host; the coefficient kernel is launched
    // only when there are any
    for (int i = 0, f = 0; i < ntasks && fp.io >= 0; ++i) {
        if (tasks[i].bound != 'n') continue;
        for (int k = 0; k < tasks[i].nmodes; ++k)
            if (fabs(ctx->lam_host[tasks[i].plane0 + k]) <= 1.0e-10) {
                if (fp.nsing == kMaxSing)
                    return set_error(ctx, DUCTGPU_EARG, "more than %d singular (lambda = 0) Neumann planes in one call", kMaxSing);
                fp.sing_fi[fp.nsing] = f;
                fp.sing_plane[fp.nsing] = k;
                ++fp.nsing;
            }
        ++f;
    }
    if (fp.nsing) {
        LaunchScope ls(ctx, DUCTGPU_K_NEUMANN);
        k_pin_coef<<<1, kMaxSing, 0, ctx->stream>>>(fp);
    }
    // partial sums in the pass workspace (free once the passes are done:
    // (T = ceil(n/32)) x m x 4 doubles per plane and direction)
    const int n = ctx->my - 2, T = (n + 31) / 32;
    if (ctx->work.bytes < (size_t)2 * cta * T * ctx->my * 4 * sizeof(double))
        return set_error(ctx, DUCTGPU_EARG, "Neumann fill: workspace smaller than its partial sums");
    {
        LaunchScope ls(ctx, DUCTGPU_K_NEUMANN);
        k_neumann_partials<<<dim3(cta, T * T), 256, 0, ctx->stream>>>(fp, ctx->work.buf);
    }
    {
        LaunchScope ls(ctx, DUCTGPU_K_NEUMANN);
        k_neumann_finish<<<cta, 256, 0, ctx->stream>>>(fp, ctx->work.buf);
    }
    return check_cuda(ctx, cudaGetLastError(), "k_neumann");
}

}  // namespace duct
