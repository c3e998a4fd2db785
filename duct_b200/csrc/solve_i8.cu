// solve_i8.cu -- FP64-accurate GEMM passes emulated with int8 slices on the
// tcgen05 tensor cores (kind::i8, exact int32 accumulation): the Ozaki
// scheme with enough slices that no refinement is needed.
//
//   A (operator row o)   = 2^(e_o + 1) sum_{s=1..7} 2^-7s SA_s
//   B (data column c)    = 2^(e_c + 1) sum_{t=1..7} 2^-7t SB_t
// with integer slices |S| <= 64 (the value is pre-scaled below 1/2, each
// rounding remainder is at most 1/2 and is scaled by 2^7 again).  A slice
// product is below 2^12, a K = 128 sum below 2^19 and the at most seven
// products of one level L = s + t below 2^22: every level is exact in an
// int32 TMEM accumulator.  Keeping the levels L = 2..8 (28 products) drops
// only terms below 2^-56 of the row and column scales, so the pass matches
// an FP64 GEMM to about 1e-15 relative to those scales -- no FP64 residual
// and no refinement, unlike the BF16 path of solve_mixed.cu.
//
// Kernel (same tile and addressing as the FP64 pass: 32 complex lines of
// one plane, 64 real columns): operator slices (7 x 16 KB) resident in
// shared memory per field; data loaded in FP64 and split into 7 slices in
// the 128-byte-swizzled K-major layout; one thread issues 28 x 4 MMAs (M=128, N=64, K=32)
// into 7 TMEM accumulators (448 columns) and commits to an mbarrier (bounded
// wait); 8 warps read the levels back and recombine them in FP64.
#include <math.h>

#include "internal.h"

namespace duct {

constexpr int kI8Lines = 32;          // complex lines per tile (64 real columns)
constexpr int kI8N = 64;              // MMA N
constexpr int kI8M = 128;             // MMA M (padded operator rows)
constexpr int kI8K = 128;             // padded K
constexpr int kI8Slices = 7;
constexpr int kI8Levels = 7;          // L = 2..8
constexpr int kI8Bits = 7;
constexpr int kI8OpSlice = kI8M * kI8K;     // 16 KB
constexpr int kI8DataSlice = kI8N * kI8K;   // 8 KB
constexpr int kI8TmemCols = 512;            // 7 x 64 = 448 used
constexpr unsigned kI8Spin = 1u << 24;

// kind::i8 instruction descriptor: D S32 (c_format 2 at bit 4), A and B
// signed 8-bit (format 1 at bits 7 and 10), both K-major, N = 64, M = 128.
constexpr uint32_t kI8Idesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kI8N >> 3) << 17) |
                              ((uint32_t)(kI8M >> 4) << 24);

__device__ __forceinline__ unsigned i8_smem(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t i8_desc(unsigned saddr, unsigned lbo, unsigned sbo)
{
    // shared-memory matrix descriptor, K-major with the 128-byte swizzle
    // (layout type 2 at bits 61-63), version 1 (bit 46), base offset 0 (the
    // 8-row x 128-byte swizzle atoms are 1024-byte aligned)
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n"
        :: "r"(tmem_d), "l"(da), "l"(db), "r"(kI8Idesc), "r"(accumulate));
}

__device__ __forceinline__ bool i8_try_wait(uint64_t *bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok) : "r"(i8_smem(bar)), "r"(parity) : "memory");
    return ok != 0;
}

__device__ __forceinline__ void i8_tmem_ld16(uint32_t taddr, int (&v)[16])
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = (int)r[i];
}

// K-major layout of a rows x 128 int8 tile with the 128-byte swizzle: a row
// is one 128-byte line, 8 rows form a 1024-byte atom, and the 16-byte chunk
// c of row r sits at chunk position c ^ (r % 8).  Byte offset of (row, k).
__device__ __forceinline__ int i8_off(int row, int k)
{
    return ((row >> 3) << 10) + ((row & 7) << 7) + ((((k >> 4) ^ (row & 7))) << 4) + (k & 15);
}

__device__ __forceinline__ double i8_pow2(int e)
{
    e = max(-1022, min(1023, e));
    return __longlong_as_double((long long)(e + 1023) << 52);
}

// x = 2^(e+1) sum_s 2^-7s S_s with |x| < 2^e; slices in [-64, 64].
__device__ __forceinline__ void split7(double x, int e, int (&s)[kI8Slices])
{
    double r = (e > -1000) ? x * i8_pow2(-(e + 1)) : 0.0;
#pragma unroll
    for (int i = 0; i < kI8Slices; ++i) {
        r *= (double)(1 << kI8Bits);
        const double q = rint(r);
        s[i] = (int)q;
        r -= q;
    }
}

// ---- operator slicing (set-up) --------------------------------------------
__global__ void k_split_operator_i8(int n, const double *A, int8_t *slices, int *rexp)
{
    const int o = blockIdx.x;          // 128 rows
    __shared__ int e_s;
    if (threadIdx.x == 0) e_s = -1074;
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const double x = (o < n) ? A[o + (size_t)n * k] : 0.0;
        if (x != 0.0) {
            int e;
            frexp(x, &e);
            atomicMax(&e_s, e);
        }
    }
    __syncthreads();
    const int e = e_s;
    if (threadIdx.x == 0) rexp[o] = e;
    for (int k = threadIdx.x; k < kI8K; k += blockDim.x) {
        const double x = (o < n && k < n) ? A[o + (size_t)n * k] : 0.0;
        int s[kI8Slices];
        split7(x, e, s);
        for (int i = 0; i < kI8Slices; ++i) slices[i * kI8OpSlice + i8_off(o, k)] = (int8_t)s[i];
    }
}

int split_operator_i8(ductgpu_ctx ctx, int n, const double *A, int8_t **slices, int **rexp)
{
    if (n > kI8K) return set_error(ctx, DUCTGPU_EARG, "int8 operator slices: n=%d > %d", n, kI8K);
    if (!*slices) DUCT_CUDA(ctx, cudaMalloc(slices, kI8Slices * kI8OpSlice));
    if (!*rexp) DUCT_CUDA(ctx, cudaMalloc(rexp, kI8M * sizeof(int)));
    {
        LaunchScope ls(ctx, DUCTGPU_K_OTHER);
        k_split_operator_i8<<<kI8M, 128, 0, ctx->stream>>>(n, A, *slices, *rexp);
    }
    return check_cuda(ctx, cudaGetLastError(), "k_split_operator_i8");
}


// ---- the pass --------------------------------------------------------------
__global__ void __launch_bounds__(256, 1) k_pass_i8(const __grid_constant__ PassParams p, int ntiles, int *err)
{
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t *As = smem;                                   // 7 x 16 KB
    uint8_t *Bs = smem + kI8Slices * kI8OpSlice;          // 7 x 8 KB
    int *ecol = reinterpret_cast<int *>(Bs + kI8Slices * kI8DataSlice);   // 64
    uint64_t *bar = reinterpret_cast<uint64_t *>(ecol + kI8N);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // 1024-byte aligned base for the swizzled buffers (see k_pass_i8ws)
    if (i8_smem(smem) & 1023u) {
        if (tid == 0) atomicExch(err, 2);
        return;
    }

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n"
                     :: "r"(i8_smem(tslot)), "r"(kI8TmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" :: "r"(i8_smem(bar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tbase = *tslot;
    const int8_t *loaded = nullptr;
    unsigned phase = 0;
    bool failed = false;

    // contiguous tile range per CTA (the operator slices change at most at
    // the field boundaries inside it)
    const int per = ntiles / gridDim.x, extra = ntiles % gridDim.x;
    const int t0 = blockIdx.x * per + min((int)blockIdx.x, extra);
    const int t1 = t0 + per + ((int)blockIdx.x < extra ? 1 : 0);

    // data: thread owns (line l, 16 consecutive k); the next tile's values
    // are loaded into the same registers while the current tile's MMAs and
    // epilogue run
    auto tile_geom = [&](int tile, int &fi, int &plane, int &l0) {
        fi = 0;
        while (fi + 1 < p.nf && tile >= p.cta_start[fi + 1]) ++fi;
        const int local = tile - p.cta_start[fi];
        plane = local / p.f[fi].nchunks;
        l0 = (local - plane * p.f[fi].nchunks) * kI8Lines;
    };
    double2 v[16];
    auto load_tile = [&](int tile) {
        int fi, plane, l0;
        tile_geom(tile, fi, plane, l0);
        const PassField &G = p.f[fi];
        const int Lg = min(kI8Lines, G.nlines - l0);
        const double *gsrc = G.src + (long long)plane * G.plane_stride;
        int l, kb;
        if (G.sk == 1) { l = tid >> 3; kb = tid & 7; }
        else { l = tid & 31; kb = tid >> 5; }
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const int k = kb * 16 + q;
            v[q] = make_double2(0.0, 0.0);
            if (k < G.n && l < Lg)
                v[q] = __ldg(reinterpret_cast<const double2 *>(gsrc + 2 * ((long long)(k + G.off) * G.sk +
                                                                          (long long)(l0 + l + G.off) * G.sl)));
        }
    };
    if (t0 < t1) load_tile(t0);

    for (int tile = t0; tile < t1; ++tile) {
        int fi, plane, l0;
        tile_geom(tile, fi, plane, l0);
        const PassField &F = p.f[fi];
        const int L = min(kI8Lines, F.nlines - l0);
        const int n = F.n, sk = F.sk, sl = F.sl, o1 = F.off;
        double *dst = F.dst + (long long)plane * F.plane_stride;

        if (F.Ai8 != loaded) {   // operator slices of this field
            for (int i = tid * 16; i < kI8Slices * kI8OpSlice; i += 256 * 16)
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(i8_smem(As + i)), "l"(F.Ai8 + i));
            asm volatile("cp.async.commit_group;\n" ::);
            loaded = F.Ai8;
        }
        if (tid < kI8N) ecol[tid] = -1074;

        int l, kb;
        if (sk == 1) { l = tid >> 3; kb = tid & 7; }
        else { l = tid & 31; kb = tid >> 5; }
        int emax_re = -1074, emax_im = -1074;
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            int e;
            if (v[q].x != 0.0) { frexp(v[q].x, &e); emax_re = max(emax_re, e); }
            if (v[q].y != 0.0) { frexp(v[q].y, &e); emax_im = max(emax_im, e); }
        }
        __syncthreads();   // ecol initialised
        atomicMax(&ecol[2 * l], emax_re);
        atomicMax(&ecol[2 * l + 1], emax_im);
        __syncthreads();
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            const int col = 2 * l + c;
            const int e = ecol[col];
            uint32_t w[kI8Slices][4];
#pragma unroll
            for (int i = 0; i < kI8Slices; ++i)
#pragma unroll
                for (int h = 0; h < 4; ++h) w[i][h] = 0u;
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                int s[kI8Slices];
                split7(c ? v[q].y : v[q].x, e, s);
#pragma unroll
                for (int i = 0; i < kI8Slices; ++i) w[i][q >> 2] |= ((uint32_t)s[i] & 0xFFu) << (8 * (q & 3));
            }
#pragma unroll
            for (int i = 0; i < kI8Slices; ++i)
                *reinterpret_cast<uint4 *>(Bs + i * kI8DataSlice + i8_off(col, kb * 16)) =
                    make_uint4(w[i][0], w[i][1], w[i][2], w[i][3]);
        }
        if (tile + 1 < t1) load_tile(tile + 1);   // in flight during the MMAs and the epilogue
        asm volatile("cp.async.wait_all;\n" ::);
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");

        if (tid == 0) {
            const unsigned a0 = i8_smem(As), b0 = i8_smem(Bs);
            const unsigned sbo = 1024;                 // next 8-row atom
#pragma unroll 1
            for (int lv = 0; lv < kI8Levels; ++lv) {
                const int Ls = lv + 2;
                bool first = true;
#pragma unroll 1
                for (int si = 1; si <= kI8Slices; ++si) {
                    const int ti = Ls - si;
                    if (ti < 1 || ti > kI8Slices) continue;
#pragma unroll
                    for (int ks = 0; ks < kI8K / 32; ++ks) {
                        // K step of 32 bytes: advance the start address inside the atom
                        const uint64_t da = i8_desc(a0 + (si - 1) * kI8OpSlice + ks * 32, 16, sbo);
                        const uint64_t db = i8_desc(b0 + (ti - 1) * kI8DataSlice + ks * 32, 16, sbo);
                        mma_i8(tbase + lv * kI8N, da, db, first ? 0u : 1u);
                        first = false;
                    }
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n"
                         :: "r"(i8_smem(bar)) : "memory");
        }
        bool ok = false;
        for (unsigned it = 0; it < kI8Spin; ++it) {
            if (i8_try_wait(bar, phase)) { ok = true; break; }
            if (it > 64) __nanosleep(32);
        }
        ok = __all_sync(0xffffffffu, ok);   // tcgen05.ld below is warp-collective
        phase ^= 1u;
        if (!ok) {
            atomicExch(err, 1);
            failed = true;
        } else {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            // epilogue: warp w -> TMEM lanes 32 (w % 4).. (rows o), columns 32 (w / 4)..
            const int qd = warp & 3, half = warp >> 2;
            const int o = qd * 32 + lane;
            const double lam = p.lam[F.plane0 + plane];
            const bool singular = (F.sing_io >= 0) && fabs(lam) <= 1.0e-10;
            const bool im0 = p.zero_im_mode0 && F.mode0 && plane == 0;
            const int eo = (o < kI8M) ? F.Aexp[o] : 0;
#pragma unroll 1
            for (int ch = 0; ch < 2; ++ch) {
                int acc[kI8Levels][16];
#pragma unroll
                for (int lv = 0; lv < kI8Levels; ++lv)
                    i8_tmem_ld16(tbase + ((uint32_t)(qd * 32) << 16) + lv * kI8N + half * 32 + ch * 16, acc[lv]);
                asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
                if (o >= n) continue;
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const int lq = half * 16 + ch * 8 + q;
                    if (lq >= L) continue;
                    const int lg = l0 + lq;
                    double val[2];
#pragma unroll
                    for (int c = 0; c < 2; ++c) {
                        double sacc = 0.0;
#pragma unroll
                        for (int lv = kI8Levels - 1; lv >= 0; --lv)
                            sacc += (double)acc[lv][2 * q + c] * i8_pow2(-kI8Bits * (lv + 2));
                        val[c] = sacc * i8_pow2(eo + ecol[2 * lq + c] + 2);
                    }
                    if (p.divide) {
                        if (singular && o == F.sing_io && lg == F.sing_l) {
                            val[0] = val[1] = 0.0;
                        } else {
                            const double den = (F.E[o] + F.El[lg]) - lam;
                            val[0] /= den;
                            val[1] /= den;
                        }
                    }
                    const long long off = 2 * ((long long)(o + o1) * sk + (long long)(lg + o1) * sl);
                    if (p.residual) {
                        const long long po = (long long)plane * F.plane_stride + off;
                        const double2 f = *reinterpret_cast<const double2 *>(F.resF + po);
                        const double2 tt = *reinterpret_cast<const double2 *>(F.resT + po);
                        const double2 uu = *reinterpret_cast<const double2 *>(F.resU + po);
                        val[0] = (f.x - tt.x) - val[0] + lam * uu.x;
                        val[1] = (f.y - tt.y) - val[1] + lam * uu.y;
                    }
                    if (im0) val[1] = 0.0;
                    *reinterpret_cast<double2 *>(dst + off) = make_double2(val[0], val[1]);
                }
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
        __syncthreads();   // TMEM read and Bs consumed before the next tile
        if (failed) break;
    }
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" :: "r"(tbase), "r"(kI8TmemCols));
}

// ---- warp-specialised, double-buffered pass --------------------------------
// 9 warps: 0-3 split tiles of 16 complex lines (32 real columns) into a
// two-stage B buffer, warp 8 issues the MMAs (one elected lane) into one of
// two TMEM accumulator sets, 4-7 read finished accumulators back and store.
// Hand-offs through mbarriers (full/empty per B stage, tfull/tempty per TMEM
// set); every wait is bounded and a timeout stops the role and raises the
// error word.  A (operator slices) is reloaded by warp 8 when the field
// changes, after the MMAs in flight have completed.
constexpr int kWsLines = 16;                        // complex lines per tile
constexpr int kWsN = 32;                            // real columns per tile
constexpr int kWsBSlice = kWsN * kI8K;              // 4 KB
constexpr int kWsBStage = kI8Slices * kWsBSlice;    // 28 KB
constexpr int kWsAcc = kI8Levels * kWsN;            // 224 TMEM columns per set
static_assert(kI8OpSlice % 1024 == 0 && kI8DataSlice % 1024 == 0 && kWsBStage % 1024 == 0,
              "swizzle atoms of the operand buffers must stay 1024-byte aligned");
constexpr uint32_t kWsIdesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kWsN >> 3) << 17) |
                              ((uint32_t)(kI8M >> 4) << 24);

__device__ __forceinline__ void ws_mma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n"
        :: "r"(tmem_d), "l"(da), "l"(db), "r"(kWsIdesc), "r"(accumulate));
}
__device__ __forceinline__ void ws_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" :: "r"(i8_smem(bar)) : "memory");
}
__device__ __forceinline__ void ws_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n"
                 :: "r"(i8_smem(bar)) : "memory");
}
// bounded wait; false after the limit (or when another role already failed)
__device__ __forceinline__ bool ws_wait(uint64_t *bar, unsigned parity, volatile int *abort)
{
    for (unsigned it = 0; it < kI8Spin; ++it) {
        if (i8_try_wait(bar, parity)) return true;
        if ((it & 255) == 255 && *abort) return false;
        if (it > 64) __nanosleep(64);
    }
    return false;
}

__device__ __forceinline__ void i8_tmem_ld8(uint32_t taddr, int (&v)[8])
{
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = (int)r[i];
}

// Biased exponent field of x (0 for zero and subnormals, treated as zero).
__device__ __forceinline__ int i8_bexp(double x) { return (int)((__double_as_longlong(x) >> 52) & 0x7FF); }

// Data slices by bit extraction: with the column exponent ec (|x| < 2^ec),
// M = trunc(|x| 2^(49 - ec)) < 2^49 and the slices are its seven base-128
// digits, most significant first, with the sign of x: x = 2^ec sum_t
// SB_t 2^-7t up to 2^(ec - 49).  Integer operations only.
__device__ __forceinline__ void split7_bits(double x, int ec, int (&d)[kI8Slices])
{
    const unsigned long long b = (unsigned long long)__double_as_longlong(x);
    const int E = (int)((b >> 52) & 0x7FF);
    const int sh = 1026 + ec - E;
    unsigned long long M = 0;
    if (E != 0 && sh < 64) M = ((b & 0x000FFFFFFFFFFFFFull) | 0x0010000000000000ull) >> sh;
    const int neg = (int)(b >> 63);
#pragma unroll
    for (int i = 0; i < kI8Slices; ++i) {
        const int v = (int)((M >> (7 * (kI8Slices - 1 - i))) & 127u);
        d[i] = neg ? -v : v;
    }
}

// 17 warps: 0-7 producers, 8-15 epilogue, 16 MMA issuer (see above).
__global__ void __launch_bounds__(544, 1) k_pass_i8ws(const __grid_constant__ PassParams p, int ntiles, int *err)
{
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t *As = smem;                                          // 7 x 16 KB
    uint8_t *Bs = smem + kI8Slices * kI8OpSlice;                 // 2 x 28 KB
    int *ecol = reinterpret_cast<int *>(Bs + 2 * kWsBStage);     // [4][32] exponent ring
    double *elr = reinterpret_cast<double *>(ecol + 4 * kWsN);   // [4][16] line eigenvalues (divide)
    uint64_t *bars = reinterpret_cast<uint64_t *>(elr + 4 * kWsLines);
    uint64_t *full = bars, *empty = bars + 2, *tfull = bars + 4, *tempty = bars + 6, *abar = bars + 8;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 9);
    volatile int *abort = reinterpret_cast<volatile int *>(tslot + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    constexpr int kProd = 256, kEpi = 256, kMmaWarp = 16;
    // The carve-up above keeps every 128-byte-swizzled buffer on a 1024-byte
    // boundary relative to the base (7 x 16 KB, then 2 x 28 KB), the
    // mbarriers on 8 bytes and the TMEM slot on 4, provided the base itself
    // is 1024-byte aligned.  Dynamic shared memory starts on such a boundary
    // when the kernel declares no static shared memory; a variant that adds
    // some (e.g. timing arrays) moves the base to a 16-byte boundary only,
    // which misaligns the descriptors and mbarriers.  Checked before any
    // barrier or TMEM allocation: the whole CTA returns and the host reads
    // code 2 from the error word.
    if (i8_smem(smem) & 1023u) {
        if (tid == 0) atomicExch(err, 2);
        return;
    }

    if (warp == kMmaWarp) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n"
                     :: "r"(i8_smem(tslot)), "r"(kI8TmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    if (tid == 0) {
        for (int s = 0; s < 2; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" :: "r"(i8_smem(full + s)), "r"(kProd));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" :: "r"(i8_smem(empty + s)), "r"(1));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" :: "r"(i8_smem(tfull + s)), "r"(1));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" :: "r"(i8_smem(tempty + s)), "r"(kEpi));
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" :: "r"(i8_smem(abar)), "r"(1));
        *abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tbase = *tslot;

    const int per = ntiles / gridDim.x, extra = ntiles % gridDim.x;
    const int t0 = blockIdx.x * per + min((int)blockIdx.x, extra);
    const int t1 = t0 + per + ((int)blockIdx.x < extra ? 1 : 0);
    auto tile_geom = [&](int tile, int &fi, int &plane, int &l0) {
        fi = 0;
        while (fi + 1 < p.nf && tile >= p.cta_start[fi + 1]) ++fi;
        const int local = tile - p.cta_start[fi];
        plane = local / p.f[fi].nchunks;
        l0 = (local - plane * p.f[fi].nchunks) * kWsLines;
    };
    auto fail = [&]() {
        *abort = 1;
        atomicExch(err, 1);
    };

    if (warp < 8) {
        // ---- producers: load, exponents, split into the B stage ----------
        double2 v[8];
        auto mapping = [&](int sk, int &l, int &kb) {
            if (sk == 1) { l = tid >> 4; kb = tid & 15; }   // 8 consecutive k of one line
            else { l = tid & 15; kb = tid >> 4; }          // 16 consecutive lines at one k
        };
        auto load_tile = [&](int tile) {
            int fi, plane, l0;
            tile_geom(tile, fi, plane, l0);
            const PassField &G = p.f[fi];
            const int Lg = min(kWsLines, G.nlines - l0);
            const double *gsrc = G.src + (long long)plane * G.plane_stride;
            int l, kb;
            mapping(G.sk, l, kb);
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int k = kb * 8 + q;
                v[q] = make_double2(0.0, 0.0);
                if (k < G.n && l < Lg)
                    v[q] = __ldg(reinterpret_cast<const double2 *>(gsrc + 2 * ((long long)(k + G.off) * G.sk +
                                                                              (long long)(l0 + l + G.off) * G.sl)));
            }
        };
        if (t0 < t1) load_tile(t0);
        for (int tile = t0; tile < t1; ++tile) {
            const int j = tile - t0, s = j & 1, use = j >> 1;
            int fi, plane, l0;
            tile_geom(tile, fi, plane, l0);
            int l, kb;
            mapping(p.f[fi].sk, l, kb);
            int emax_re = 0, emax_im = 0;
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                emax_re = max(emax_re, i8_bexp(v[q].x));
                emax_im = max(emax_im, i8_bexp(v[q].y));
            }
            // stage (and exponent slot j % 4) free once the MMAs of tile j - 2
            // completed (so the epilogue of tile j - 4 is done too); all
            // producers take the go / stop decision together
            const bool waited = ws_wait(empty + s, (use & 1) ^ 1, abort);
            int anyfail;
            asm volatile("{\n\t.reg .pred p, q;\n\t"
                         "setp.eq.u32 p, %1, 0;\n\t"
                         "bar.red.or.pred q, 1, 256, p;\n\t"
                         "selp.u32 %0, 1, 0, q;\n\t}\n"
                         : "=r"(anyfail) : "r"(waited ? 1u : 0u) : "memory");
            if (anyfail) { fail(); break; }
            int *ec = ecol + (j & 3) * kWsN;
            if (tid < kWsN) ec[tid] = 0;
            if (p.divide && tid < kWsLines) {   // the tile's line eigenvalues, for the epilogue
                const PassField &G = p.f[fi];
                elr[(j & 3) * kWsLines + tid] = (l0 + tid < G.nlines) ? G.El[l0 + tid] : 0.0;
            }
            asm volatile("bar.sync 1, 256;\n" ::: "memory");
            atomicMax(&ec[2 * l], emax_re);
            atomicMax(&ec[2 * l + 1], emax_im);
            asm volatile("bar.sync 1, 256;\n" ::: "memory");
            uint8_t *B = Bs + s * kWsBStage;
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const int col = 2 * l + c;
                const int e = ec[col] - 1022;   // column exponent: |x| < 2^e
                uint32_t w[kI8Slices][2];
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    // four consecutive k: digit magnitudes packed byte-wise,
                    // then the signs applied to the four bytes at once
                    uint32_t wd[kI8Slices], sgn = 0u;
#pragma unroll
                    for (int i = 0; i < kI8Slices; ++i) wd[i] = 0u;
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const double x = c ? v[4 * h + u].y : v[4 * h + u].x;
                        const unsigned long long b = (unsigned long long)__double_as_longlong(x);
                        const int E = (int)((b >> 52) & 0x7FF);
                        const int sh = 1026 + e - E;
                        unsigned long long M = 0;
                        if (E != 0 && sh < 64) M = ((b & 0x000FFFFFFFFFFFFFull) | 0x0010000000000000ull) >> sh;
                        sgn |= (uint32_t)(b >> 63) * (0xFFu << (8 * u));
#pragma unroll
                        for (int i = 0; i < kI8Slices; ++i)
                            wd[i] |= ((uint32_t)(M >> (7 * (kI8Slices - 1 - i))) & 0x7Fu) << (8 * u);
                    }
#pragma unroll
                    for (int i = 0; i < kI8Slices; ++i) {
                        // -d mod 256 = (0x80 - d) ^ 0x80 for 0 <= d <= 127, byte-parallel
                        const uint32_t neg = (0x80808080u - wd[i]) ^ 0x80808080u;
                        w[i][h] = (neg & sgn) | (wd[i] & ~sgn);
                    }
                }
#pragma unroll
                for (int i = 0; i < kI8Slices; ++i)
                    *reinterpret_cast<uint2 *>(B + i * kWsBSlice + i8_off(col, kb * 8)) = make_uint2(w[i][0], w[i][1]);
            }
            if (tile + 1 < t1) load_tile(tile + 1);   // next tile's values in flight
            asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
            ws_arrive(full + s);
        }
    } else if (warp == kMmaWarp) {
        // ---- MMA issuer ---------------------------------------------------
        const int8_t *loaded = nullptr;
        unsigned aphase = 0;
        bool pending = false;
        for (int tile = t0; tile < t1; ++tile) {
            const int j = tile - t0, s = j & 1, use = j >> 1;
            int fi, plane, l0;
            tile_geom(tile, fi, plane, l0);
            const int8_t *Ai = p.f[fi].Ai8;
            if (Ai != loaded) {
                if (pending) {   // the MMAs reading the old slices must be done
                    if (lane == 0) ws_commit(abar);
                    __syncwarp();
                    if (!__all_sync(0xffffffffu, ws_wait(abar, aphase, abort))) { fail(); break; }
                    aphase ^= 1u;
                }
                for (int i = lane * 16; i < kI8Slices * kI8OpSlice; i += 32 * 16)
                    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(i8_smem(As + i)), "l"(Ai + i));
                asm volatile("cp.async.commit_group;\n" ::);
                asm volatile("cp.async.wait_all;\n" ::);
                asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
                __syncwarp();
                loaded = Ai;
            }
            if (!__all_sync(0xffffffffu, ws_wait(full + s, use & 1, abort))) { fail(); break; }
            if (!__all_sync(0xffffffffu, ws_wait(tempty + s, (use & 1) ^ 1, abort))) { fail(); break; }
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            if (lane == 0) {
                // descriptors differ from the base ones only in the start
                // address (16-byte units, no carry out of the 14-bit field):
                // every offset below is a compile-time constant
                const uint64_t da0 = i8_desc(i8_smem(As), 16, 1024);
                const uint64_t db0 = i8_desc(i8_smem(Bs + s * kWsBStage), 16, 1024);
                const uint32_t dacc = tbase + s * kWsAcc;
#pragma unroll
                for (int lv = 0; lv < kI8Levels; ++lv) {
#pragma unroll
                    for (int si = 1; si <= kI8Slices; ++si) {
                        const int ti = lv + 2 - si;
                        if (ti < 1 || ti > kI8Slices) continue;
                        const bool first_pair = (si == (lv + 2 - kI8Slices > 1 ? lv + 2 - kI8Slices : 1));
#pragma unroll
                        for (int ks = 0; ks < kI8K / 32; ++ks)
                            ws_mma(dacc + lv * kWsN, da0 + (uint64_t)(((si - 1) * kI8OpSlice + ks * 32) >> 4),
                                   db0 + (uint64_t)(((ti - 1) * kWsBSlice + ks * 32) >> 4),
                                   (first_pair && ks == 0) ? 0u : 1u);
                    }
                }
                ws_commit(empty + s);
                ws_commit(tfull + s);
            }
            __syncwarp();
            pending = true;
        }
    } else {
        // ---- epilogue: TMEM -> FP64 -> global -----------------------------
        const int ew = warp - 8, qd = ew & 3, chh = ew >> 2;   // lane quarter, column half
        const int o = qd * 32 + lane;
        for (int tile = t0; tile < t1; ++tile) {
            const int j = tile - t0, s = j & 1, use = j >> 1;
            int fi, plane, l0;
            tile_geom(tile, fi, plane, l0);
            const PassField &F = p.f[fi];
            // E of this row, read before the wait (the line eigenvalues come
            // staged with the tile's exponents)
            const double Eo = (p.divide && o < F.n) ? __ldg(F.E + o) : 0.0;
            if (!__all_sync(0xffffffffu, ws_wait(tfull + s, use & 1, abort))) { fail(); break; }
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const int L = min(kWsLines, F.nlines - l0);
            const double *el = elr + (j & 3) * kWsLines;
            const int n = F.n, sk = F.sk, sl = F.sl, o1 = F.off;
            double *dst = F.dst + (long long)plane * F.plane_stride;
            const double lam = p.lam[F.plane0 + plane];
            const bool singular = (F.sing_io >= 0) && fabs(lam) <= 1.0e-10;
            const bool im0 = p.zero_im_mode0 && F.mode0 && plane == 0;
            const int eo = F.Aexp[o];
            const int *ec = ecol + (j & 3) * kWsN;
#pragma unroll 1
            for (int ch = 0; ch < 2; ++ch) {
                const int c0 = chh * 16 + ch * 8;   // first real column of this chunk
                int acc[kI8Levels][8];
#pragma unroll
                for (int lv = 0; lv < kI8Levels; ++lv)
                    i8_tmem_ld8(tbase + ((uint32_t)(qd * 32) << 16) + s * kWsAcc + lv * kWsN + c0, acc[lv]);
                asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
                if (o >= n) continue;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int lq = (c0 >> 1) + q;
                    if (lq >= L) continue;
                    const int lg = l0 + lq;
                    double val[2];
#pragma unroll
                    for (int c = 0; c < 2; ++c) {
                        const int cc = 2 * q + c;
                        // levels 2..4 and 5..8 combined exactly in 64-bit integers
                        const long long hi = ((long long)acc[0][cc] << 14) + ((long long)acc[1][cc] << 7) + acc[2][cc];
                        const long long lo = ((long long)acc[3][cc] << 21) + ((long long)acc[4][cc] << 14) +
                                             ((long long)acc[5][cc] << 7) + acc[6][cc];
                        const double sacc = fma((double)hi, 0x1p-28, (double)lo * 0x1p-56);
                        val[c] = sacc * i8_pow2(eo + 1 + ec[2 * lq + c] - 1022);
                    }
                    if (p.divide) {
                        if (singular && o == F.sing_io && lg == F.sing_l) {
                            val[0] = val[1] = 0.0;
                        } else {
                            const double rden = 1.0 / ((Eo + el[lq]) - lam);
                            val[0] *= rden;
                            val[1] *= rden;
                        }
                    }
                    const long long off = 2 * ((long long)(o + o1) * sk + (long long)(lg + o1) * sl);
                    if (p.residual) {
                        const long long po = (long long)plane * F.plane_stride + off;
                        const double2 f = *reinterpret_cast<const double2 *>(F.resF + po);
                        const double2 tt = *reinterpret_cast<const double2 *>(F.resT + po);
                        const double2 uu = *reinterpret_cast<const double2 *>(F.resU + po);
                        val[0] = (f.x - tt.x) - val[0] + lam * uu.x;
                        val[1] = (f.y - tt.y) - val[1] + lam * uu.y;
                    }
                    if (im0) val[1] = 0.0;
                    *reinterpret_cast<double2 *>(dst + off) = make_double2(val[0], val[1]);
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
            ws_arrive(tempty + s);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (warp == kMmaWarp)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" :: "r"(tbase), "r"(kI8TmemCols));
}

int i8_pass(ductgpu_ctx ctx, const PassParams &pp, int grid)
{
    if (ctx->i8_kernel == 1) {
        for (int i = 0; i < pp.nf; ++i)
            if (!pp.f[i].Ai8 || pp.f[i].n > kI8K)
                return set_error(ctx, DUCTGPU_EARG, "int8 pass: operator of field %d not sliced (n <= 127 only)", i);
        // 16 lines per tile: re-cut the callers' 32-line grid
        PassParams q = pp;
        int tiles = 0;
        for (int i = 0; i < q.nf; ++i) {
            q.f[i].nchunks = (q.f[i].nlines + kWsLines - 1) / kWsLines;
            q.cta_start[i] = tiles;
            tiles += q.f[i].nmodes * q.f[i].nchunks;
        }
        q.cta_start[q.nf] = tiles;
        const size_t smem = (size_t)kI8Slices * kI8OpSlice + 2 * (size_t)kWsBStage + 4 * kWsN * sizeof(int) +
                            4 * kWsLines * sizeof(double) + 128;
        DUCT_CUDA(ctx, cudaFuncSetAttribute(k_pass_i8ws, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        const int ctas = tiles < ctx->num_sms ? tiles : ctx->num_sms;
        {
            LaunchScope ls(ctx, DUCTGPU_K_MIXED_GEMM);
            k_pass_i8ws<<<ctas, 544, smem, ctx->stream>>>(q, tiles, ctx->dev_err);
        }
        return check_cuda(ctx, cudaGetLastError(), "k_pass_i8ws");
    }
    for (int i = 0; i < pp.nf; ++i)
        if (!pp.f[i].Ai8 || pp.f[i].n > kI8K || pp.f[i].nchunks * kI8Lines < pp.f[i].nlines)
            return set_error(ctx, DUCTGPU_EARG, "int8 pass: operator of field %d not sliced (n <= 127 only)", i);
    const size_t smem = (size_t)kI8Slices * (kI8OpSlice + kI8DataSlice) + kI8N * sizeof(int) + 64;
    DUCT_CUDA(ctx, cudaFuncSetAttribute(k_pass_i8, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int ctas = grid < ctx->num_sms ? grid : ctx->num_sms;   // one CTA per SM (shared memory, TMEM)
    {
        LaunchScope ls(ctx, DUCTGPU_K_MIXED_GEMM);
        k_pass_i8<<<ctas, 256, smem, ctx->stream>>>(pp, grid, ctx->dev_err);
    }
    return check_cuda(ctx, cudaGetLastError(), "k_pass_i8");
}

}  // namespace duct
