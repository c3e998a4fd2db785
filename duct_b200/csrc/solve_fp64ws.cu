// solve_fp64ws.cu -- warp-specialised persistent form of the flip-symmetric
// FP64 pass (k_pass_fp64s in solve_fp64.cu; the operator algebra is
// described at fold_operators in setup.cu).
//
// One CTA per SM walks a contiguous range of 16-line tiles of one field, so
// the field's folded operator (2H x H, fragment order of k_pack_a) is loaded
// once and stays in shared memory.  Roles:
//   warps 0-3   producers: stage tile j into stage j % 4 of a ring with
//               cp.async (each thread copies both rows of its point pairs,
//               so a P^-1 pass folds them in place after its own copies
//               land), one tile ahead of the one they finish (two
//               ahead was measured slower: the deeper stage wait couples
//               the producers to the group two tiles back);
//   warps 4-19  two consumer groups of 8 warps take alternate tiles: DMMA
//               over the stage (warps 4 x 2 along M x N, as k_pass_fp64s),
//               then the epilogue -- direct stores with the eigenvalue
//               divide, or the unfold through the stage.
// Hand-offs: mbarriers full[s] (128 producer arrivals) and empty[s] (one
// arrival by the consumer group that released the stage).  Every wait is
// bounded; a role that times out raises the error word and the abort flag,
// and each consumer group takes its go / stop decision as a whole (bar.red)
// so that no thread is left at a group barrier.
#include <math.h>

#include "internal.h"

namespace duct {

namespace {

constexpr int kWsLinesF = 16;                 // complex lines per tile
constexpr int kWsNld = 2 * kWsLinesF + 4;     // staged row length (doubles)
constexpr int kWsStages = 4;
constexpr int kWsProd = 128;                  // producer threads
constexpr int kWsGroup = 256;                 // threads per consumer group
constexpr int kWsThreads = kWsProd + 2 * kWsGroup;
constexpr unsigned kWsSpin = 1u << 24;

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void cp16z(void *dst, const void *src, bool valid)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
                 "r"(valid ? 16 : 0));
}

__device__ __forceinline__ void mma_f64(double (&d)[4], const double (&a)[8], const double (&b)[4])
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 "
        "{%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, {%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]),
          "d"(b[0]), "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

__device__ __forceinline__ bool bar_try(uint64_t *bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return ok != 0;
}

// bounded wait; false after the limit or once another role has failed
__device__ __forceinline__ bool bar_wait(uint64_t *bar, unsigned parity, volatile int *abort,
                                         unsigned limit = kWsSpin)
{
    for (unsigned it = 0; it < limit; ++it) {
        if (bar_try(bar, parity)) return true;
        if ((it & 255) == 255 && *abort) return false;
        if (it > 64) __nanosleep(64);
    }
    return false;
}

__device__ __forceinline__ void bar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}

// barrier of one consumer group (named barrier 1 + g, 256 threads) that
// also returns whether any of its threads reported a failure
__device__ __forceinline__ bool group_any(int g, bool fail)
{
    unsigned any;
    asm volatile("{\n\t.reg .pred p, q;\n\t"
                 "setp.ne.u32 p, %1, 0;\n\t"
                 "bar.red.or.pred q, %2, 256, p;\n\t"
                 "selp.u32 %0, 1, 0, q;\n\t}\n"
                 : "=r"(any) : "r"(fail ? 1u : 0u), "r"(1 + g) : "memory");
    return any != 0;
}

__device__ __forceinline__ void group_sync(int g)
{
    asm volatile("bar.sync %0, 256;\n" ::"r"(1 + g) : "memory");
}

}  // namespace

// cstart[i] .. cstart[i+1]-1: the CTAs of field i (the launcher splits the
// grid over the fields in proportion to their tiles)
struct WsSplit {
    int cstart[kMaxFields + 1];
};

template <int H>
__global__ void __launch_bounds__(kWsThreads, 1)
k_pass_fp64w(const __grid_constant__ PassParams p, const __grid_constant__ WsSplit sp, int *err)
{
    constexpr int MTILES = 2 * H / 16, MTW = MTILES / 4, NTW = kWsLinesF / 8, KS = H / 16;
    constexpr int ROWS = 2 * H, STAGE = ROWS * kWsNld, AOP = KS * MTILES * 256;
    extern __shared__ __align__(16) double smem[];
    double *As = smem;                          // folded operator, resident
    double *St = As + AOP;                      // kWsStages staged tiles
    double *Es = St + kWsStages * STAGE;        // E (pass direction), 2H
    double *Els = Es + ROWS;                    // El (line direction), 2H
    uint64_t *full = reinterpret_cast<uint64_t *>(Els + ROWS);
    uint64_t *empty = full + kWsStages;
    volatile int *abort = reinterpret_cast<volatile int *>(empty + kWsStages);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    int fi = 0;
    while (fi + 1 < p.nf && (int)blockIdx.x >= sp.cstart[fi + 1]) ++fi;
    const PassField &F = p.f[fi];
    const int nctas = sp.cstart[fi + 1] - sp.cstart[fi], cl = blockIdx.x - sp.cstart[fi];
    const int ntiles_f = F.nmodes * F.nchunks;
    const int per = ntiles_f / nctas, extra = ntiles_f % nctas;
    const int t0 = cl * per + min(cl, extra);
    const int ntile = per + (cl < extra ? 1 : 0);
    const int n = F.n, he = F.he, ho = F.ho, sk = F.sk, sl = F.sl, o1 = F.off;

    if (tid == 0) {
        for (int s = 0; s < kWsStages; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(full + s)), "r"(kWsProd));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(empty + s)), "r"(1));
        }
        *abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    auto tile_at = [&](int j, int &plane, int &l0) {
        const int t = t0 + j;
        plane = t / F.nchunks;
        l0 = (t - plane * F.nchunks) * kWsLinesF;
    };
    // point pair (r, H + r) of line l per item: row r holds point / mode
    // r (r < he), row H + r point n-1-r (P^-1 passes) or odd mode he + r
    // (P passes), r < ho; the other rows are zero
    auto item = [&](int idx, int &r, int &l) {
        if (sk == 1) {   // 4 points x 2 lines per 8 threads
            const int rest = idx >> 3;
            r = (rest % (H / 4)) * 4 + (idx & 3);
            l = (rest / (H / 4)) * 2 + ((idx >> 2) & 1);
        } else {
            r = idx / kWsLinesF;
            l = idx % kWsLinesF;
        }
    };
    auto issue = [&](int j) {
        int plane, l0;
        tile_at(j, plane, l0);
        const int L = min(kWsLinesF, F.nlines - l0);
        const double *src = F.src + (long long)plane * F.plane_stride;
        double *S = St + (j % kWsStages) * STAGE;
        for (int idx = tid; idx < H * kWsLinesF; idx += kWsProd) {
            int r, l;
            item(idx, r, l);
            const bool lok = l < L;
            const int kb = (F.par == 1) ? n - 1 - r : he + r;
            const bool oka = lok && r < he, okb = lok && r < ho;
            const long long col = (long long)(l0 + l + o1) * sl;
            cp16z(S + r * kWsNld + 2 * l, oka ? src + 2 * ((long long)(r + o1) * sk + col) : src, oka);
            cp16z(S + (H + r) * kWsNld + 2 * l, okb ? src + 2 * ((long long)(kb + o1) * sk + col) : src, okb);
        }
        asm volatile("cp.async.commit_group;\n" ::);
    };
    // operator and eigenvalues of the field, by every thread; the producers
    // queue the first tile with them (its stage is fresh), so the two loads
    // overlap
    for (int i = tid * 2; i < AOP; i += kWsThreads * 2) {
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(As + i)), "l"(F.A + i));
    }
    asm volatile("cp.async.commit_group;\n" ::);
    if (warp < 4 && ntile > 0) issue(0);
    if (p.divide) {
        for (int i = tid; i < n; i += kWsThreads) Es[i] = F.E[i];
        for (int i = tid; i < F.nlines; i += kWsThreads) Els[i] = F.El[i];
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();
    if (ntile <= 0) return;

    auto fail = [&]() {
        *abort = 1;
        atomicExch(err, 1);     // a wait ran out (code 2 is the tcgen05 kernels' misaligned base)
    };

    if (warp < 4) {
        // ---- producers -------------------------------------------------
        bool ok = true;   // tile 0 was queued with the operator
        for (int j = 0; j < ntile && ok; ++j) {
            if (j + 1 < ntile) {
                const int s1 = (j + 1) % kWsStages, u1 = (j + 1) / kWsStages;
                if (!bar_wait(empty + s1, (u1 & 1) ^ 1, abort)) { ok = false; break; }
                issue(j + 1);
                asm volatile("cp.async.wait_group 1;\n" ::: "memory");
            } else {
                asm volatile("cp.async.wait_group 0;\n" ::: "memory");
            }
            if (F.par == 1) {   // fold this thread's own pairs
                double *S = St + (j % kWsStages) * STAGE;
                for (int idx = tid; idx < H * kWsLinesF; idx += kWsProd) {
                    int r, l;
                    item(idx, r, l);
                    if (r >= ho) continue;
                    double2 *pa = reinterpret_cast<double2 *>(S + r * kWsNld + 2 * l);
                    double2 *pb = reinterpret_cast<double2 *>(S + (H + r) * kWsNld + 2 * l);
                    const double2 x = *pa, y = *pb;
                    *pa = make_double2(x.x + y.x, x.y + y.y);
                    *pb = make_double2(x.x - y.x, x.y - y.y);
                }
            }
            bar_arrive(full + (j % kWsStages));
        }
        if (!ok) fail();
        asm volatile("cp.async.wait_all;\n" ::: "memory");
        return;
    }

    // ---- consumers -------------------------------------------------------
    const int g = (warp - 4) >> 3, cw = (warp - 4) & 7, gt = tid - kWsProd - g * kWsGroup;
    const int wm = cw & 3, wn = cw >> 2, gg = lane >> 2, t = lane & 3;
    const int kb0 = (wm * MTW * 16 >= H) ? H : 0;
    for (int j = g; j < ntile; j += 2) {
        const int s = j % kWsStages, u = j / kWsStages;
        const bool waited = bar_wait(full + s, u & 1, abort);
        if (group_any(g, !waited)) {
            if (gt == 0) fail();
            break;
        }
        double *S = St + s * STAGE;
        double acc[MTW][NTW][4];
#pragma unroll
        for (int i = 0; i < MTW; ++i)
#pragma unroll
            for (int q = 0; q < NTW; ++q)
#pragma unroll
                for (int v = 0; v < 4; ++v) acc[i][q][v] = 0.0;
#pragma unroll
        for (int ks = 0; ks < KS; ++ks) {
            const int kg = kb0 + ks * 16 + t;
            double b[NTW][4];
#pragma unroll
            for (int nt = 0; nt < NTW; ++nt) {
                const int col = wn * kWsLinesF + nt * 8 + gg;
#pragma unroll
                for (int v = 0; v < 4; ++v) b[nt][v] = S[(kg + 4 * v) * kWsNld + col];
            }
#pragma unroll
            for (int mt = 0; mt < MTW; ++mt) {
                const double2 *q = reinterpret_cast<const double2 *>(As + (ks * MTILES + wm * MTW + mt) * 256) + lane;
                double a[8];
#pragma unroll
                for (int h = 0; h < 4; ++h) {
                    const double2 v = q[32 * h];
                    a[2 * h] = v.x;
                    a[2 * h + 1] = v.y;
                }
#pragma unroll
                for (int nt = 0; nt < NTW; ++nt) mma_f64(acc[mt][nt], a, b[nt]);
            }
        }
        int plane, l0;
        tile_at(j, plane, l0);
        const int L = min(kWsLinesF, F.nlines - l0);
        double *dst = F.dst + (long long)plane * F.plane_stride;
        const double lam = p.lam[F.plane0 + plane];
        const bool im0 = p.zero_im_mode0 && F.mode0 && plane == 0;
        group_sync(g);   // the group is done reading the stage
        if (F.par == 1) {
            if (gt == 0) bar_arrive(empty + s);
            const bool singular = (F.sing_io >= 0) && fabs(lam) <= 1.0e-10;
#pragma unroll
            for (int mt = 0; mt < MTW; ++mt)
#pragma unroll
                for (int nt = 0; nt < NTW; ++nt) {
                    const int l = wn * (kWsLinesF / 2) + nt * 4 + t;
                    if (l >= L) continue;
                    const int lg = l0 + l;
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int orow = (wm * MTW + mt) * 16 + gg + 8 * h;
                        const int o = orow < H ? (orow < he ? orow : -1) : (orow - H < ho ? he + orow - H : -1);
                        if (o < 0) continue;
                        double re = acc[mt][nt][2 * h], im = acc[mt][nt][2 * h + 1];
                        if (p.divide) {
                            if (singular && o == F.sing_io && lg == F.sing_l) {
                                re = 0.0;
                                im = 0.0;
                            } else {
                                const double rden = 1.0 / ((Es[o] + Els[lg]) - lam);
                                re *= rden;
                                im *= rden;
                            }
                        }
                        if (im0) im = 0.0;
                        const long long off = 2 * ((long long)(o + o1) * sk + (long long)(lg + o1) * sl);
                        *reinterpret_cast<double2 *>(dst + off) = make_double2(re, im);
                    }
                }
            continue;
        }
        // unfold through the stage (layouts as k_pass_fp64s)
        auto emit = [&](const double2 *ev, const double2 *od, int rs, int o, int l) {
            const int oh = o < he ? o : n - 1 - o;
            double2 v = ev[oh * rs];
            if (oh < ho) {
                const double2 d = od[oh * rs];
                v = (o < he) ? make_double2(v.x + d.x, v.y + d.y) : make_double2(v.x - d.x, v.y - d.y);
            }
            if (im0) v.y = 0.0;
            *reinterpret_cast<double2 *>(dst + 2 * ((long long)(o + o1) * sk + (long long)(l0 + l + o1) * sl)) = v;
        };
        if (sk == 1) {
            double2 *Cs = reinterpret_cast<double2 *>(S);
            const int cld = 2 * H + 2;
#pragma unroll
            for (int mt = 0; mt < MTW; ++mt)
#pragma unroll
                for (int nt = 0; nt < NTW; ++nt)
#pragma unroll
                    for (int h = 0; h < 2; ++h)
                        Cs[(wn * (kWsLinesF / 2) + nt * 4 + t) * cld + (wm * MTW + mt) * 16 + gg + 8 * h] =
                            make_double2(acc[mt][nt][2 * h], acc[mt][nt][2 * h + 1]);
            group_sync(g);
            for (int idx = gt; idx < n * kWsLinesF; idx += kWsGroup) {
                const int o = idx % n, l = idx / n;
                if (l < L) emit(Cs + l * cld, Cs + l * cld + H, 1, o, l);
            }
        } else {
#pragma unroll
            for (int mt = 0; mt < MTW; ++mt)
#pragma unroll
                for (int nt = 0; nt < NTW; ++nt)
#pragma unroll
                    for (int h = 0; h < 2; ++h)
                        *reinterpret_cast<double2 *>(S + ((wm * MTW + mt) * 16 + gg + 8 * h) * kWsNld + wn * kWsLinesF +
                                                     nt * 8 + 2 * t) =
                            make_double2(acc[mt][nt][2 * h], acc[mt][nt][2 * h + 1]);
            group_sync(g);
            const double2 *Rs = reinterpret_cast<const double2 *>(S);
            for (int idx = gt; idx < n * kWsLinesF; idx += kWsGroup) {
                const int o = idx / kWsLinesF, l = idx % kWsLinesF;
                if (l < L) emit(Rs + l, Rs + H * (kWsNld / 2) + l, kWsNld / 2, o, l);
            }
        }
        group_sync(g);   // the stage is free again
        if (gt == 0) bar_arrive(empty + s);
    }
}

// Self-test of the failure path: one CTA waits, with the pass kernel's
// bounded wait, on an mbarrier that nothing arrives at.  The wait gives up
// after `limit` polls and raises the error word, as a role of the pass
// kernel does when its partner never hands over; nothing faults or hangs.
__global__ void k_wait_selftest(unsigned limit, int *err)
{
    __shared__ uint64_t bar;
    __shared__ int abort_flag;
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(&bar)), "r"(1));
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    const bool ok = bar_wait(&bar, 0, &abort_flag, limit);   // phase 0 never completes
    if (!__all_sync(0xffffffffu, ok) && threadIdx.x == 0) atomicExch(err, 3);
}

cudaError_t wait_selftest(ductgpu_ctx ctx, unsigned polls)
{
    LaunchScope ls(ctx, DUCTGPU_K_OTHER);
    k_wait_selftest<<<1, 32, 0, ctx->stream>>>(polls, ctx->dev_err);
    return cudaGetLastError();
}

template <int H>
static cudaError_t launch_ws(ductgpu_ctx ctx, const PassParams &pp)
{
    // 16-line tiles; the grid split over the fields in proportion to their
    // tiles, at least one CTA each
    PassParams q = pp;
    int tiles[kMaxFields], total = 0;
    for (int i = 0; i < q.nf; ++i) {
        q.f[i].nchunks = (q.f[i].nlines + kWsLinesF - 1) / kWsLinesF;
        tiles[i] = q.f[i].nmodes * q.f[i].nchunks;
        total += tiles[i];
    }
    const int G = ctx->num_sms > q.nf ? ctx->num_sms : q.nf;
    WsSplit sp{};
    int c = 0;
    for (int i = 0; i < q.nf; ++i) {
        sp.cstart[i] = c;
        int k = (int)((long long)G * tiles[i] / total);
        if (k < 1) k = 1;
        if (k > tiles[i]) k = tiles[i];
        c += k;
    }
    sp.cstart[q.nf] = c;
    constexpr int ROWS = 2 * H, STAGE = ROWS * kWsNld, AOP = (H / 16) * (2 * H / 16) * 256;
    const size_t smem = (size_t)(AOP + kWsStages * STAGE + 2 * ROWS) * sizeof(double) + 2 * kWsStages * 8 + 16;
    cudaError_t e = cudaFuncSetAttribute(k_pass_fp64w<H>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    LaunchScope ls(ctx, DUCTGPU_K_PASS_FP64);
    k_pass_fp64w<H><<<c, kWsThreads, smem, ctx->stream>>>(q, sp, ctx->dev_err);
    return cudaGetLastError();
}

cudaError_t fp64_pass_ws(ductgpu_ctx ctx, const PassParams &pp, int hpad)
{
    return (hpad == 32) ? launch_ws<32>(ctx, pp) : launch_ws<64>(ctx, pp);
}

}  // namespace duct
