// solve_mixed.cu -- split-precision diagonalisation solve on the tcgen05
// tensor cores with FP64 iterative refinement.
//
// Each GEMM pass of the solve (same four passes and addressing as the FP64
// path in solve_fp64.cu) runs as an Ozaki-style product of BF16 slices:
//   A (fixed operator, per-row exponent e_o) = 2^e_o sum_i 2^-7i SA_i
//   B (data lines,    per-column exponent e_c) = 2^e_c sum_j 2^-7j SB_j
// with integer slices |S| <= 128, which BF16 holds exactly.  Products of
// slices are integers below 2^14, a K <= 128 sum stays below 2^21, and the
// (up to four) slice pairs of one level L = i + j add below 2^23: every
// level is accumulated EXACTLY in an FP32 TMEM accumulator.  Four slices
// and the levels L = 2..5 (ten slice products) give a product accurate to
// ~2^-28 relative; FP64 iterative refinement on the residual of the
// reference's own FP64 operator (D2 interior blocks, on the DMMA pass)
// brings the solution to FP64 accuracy.
//
// Kernel shape (one CTA per 32 complex lines of a plane, as the FP64 pass):
//   * operator slices (4 x 128 x 128 BF16, pre-split at setup) copied to
//     shared memory in the UMMA no-swizzle K-major core-matrix layout;
//   * the 64 real columns of data loaded in FP64, split into 4 slices
//     with per-column exponents by all threads;
//   * one elected thread issues the 10 x (K/16) tcgen05.mma (M=128, N=64,
//     K=16, kind::f16 BF16 -> FP32) into 4 TMEM accumulators and commits
//     to an mbarrier (bounded wait: a timeout sets an error flag);
//   * 8 warps read TMEM back (tcgen05.ld 32x32b), recombine the levels in
//     FP64 with the exponents, divide by the eigenvalue sum when asked, and
//     store FP64.
#include <cuda_bf16.h>
#include <math.h>

#include "internal.h"

namespace duct {

constexpr int kMxLines = 32;        // complex lines per CTA (64 real columns)
constexpr int kMxN = 64;            // MMA N
constexpr int kMxM = 128;           // MMA M (padded operator rows)
constexpr int kMxK = 128;           // padded K
constexpr int kSlices = 4;
constexpr int kLevels = 4;          // L = 2..5
constexpr int kSliceBits = 7;
constexpr int kOpSliceBytes = kMxM * kMxK * 2;   // 32 KB
constexpr int kDataSliceBytes = kMxN * kMxK * 2; // 16 KB
static_assert(kOpSliceBytes % 1024 == 0 && kDataSliceBytes % 1024 == 0,
              "swizzle atoms of the operand buffers must stay 1024-byte aligned");
constexpr int kTmemCols = kLevels * kMxN;        // 256
constexpr unsigned kSpinLimit = 1u << 24;

struct MixedField {
    const double *src;
    double *dst;
    const double *add;       // optional addend (same layout as dst), or null
    const uint8_t *Aslices;  // operator slices, kSlices x 32 KB
    const int *Aexp;         // per-row exponents (128)
    const double *E;
    int nmodes, mode0, plane0, sing_io;
};

struct MixedParams {
    MixedField f[kMaxFields];
    int cta_start[kMaxFields + 1];
    int nf;
    const double *lam;
    long long plane_stride;
    int n, nchunks, sk, sl;
    int divide, zero_im_mode0;
    int *err;                // set to 1 when a bounded wait gives up
};

// ---- small PTX wrappers ---------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t umma_desc(unsigned saddr, unsigned lbo, unsigned sbo)
{
    // SM100 shared-memory matrix descriptor, no swizzle (layout type 0),
    // version 1 (bits 46-47), base offset 0, addresses in 16-byte units.
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// kind::f16 instruction descriptor: D FP32, A and B BF16, both K-major,
// N = 64 (n_dim = N >> 3 at bit 17), M = 128 (m_dim = M >> 4 at bit 24).
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kMxN >> 3) << 17) |
                            ((uint32_t)(kMxM >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        :: "r"(tmem_d), "l"(da), "l"(db), "r"(kIdesc), "r"(accumulate));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" :: "r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return ok != 0;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16])
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void cp_async16_m(void *smem, const void *gmem)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(smem)), "l"(gmem));
}

// Core-matrix (8 rows x 16 bytes) K-major layout of a rows x 128 BF16 tile:
// byte offset of element (row, k).
__device__ __forceinline__ int core_off(int row, int k)
{
    return (((row >> 3) * (kMxK / 8) + (k >> 3)) << 7) + ((row & 7) << 4) + ((k & 7) << 1);
}

// 2^e for -1022 <= e <= 1023 (clamped), built from the exponent bits.
__device__ __forceinline__ double pow2(int e)
{
    e = max(-1022, min(1023, e));
    return __longlong_as_double((long long)(e + 1023) << 52);
}

// Split x (|x| < 2^e) into kSlices integer slices of kSliceBits each; a
// column whose largest magnitude is below 2^-1000 is treated as zero.
__device__ __forceinline__ void split4(double x, int e, float (&s)[kSlices])
{
    double r = (e > -1000) ? x * pow2(-e) : 0.0;
#pragma unroll
    for (int i = 0; i < kSlices; ++i) {
        r *= (double)(1 << kSliceBits);
        const double q = rint(r);
        s[i] = (float)q;
        r -= q;
    }
}

__global__ void __launch_bounds__(256, 1) k_pass_mixed(const __grid_constant__ MixedParams p)
{
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t *As = smem;                                  // kSlices x 32 KB
    uint8_t *Bs = smem + kSlices * kOpSliceBytes;        // kSlices x 16 KB
    int *ecol = reinterpret_cast<int *>(Bs + kSlices * kDataSliceBytes);   // 64
    uint64_t *bar = reinterpret_cast<uint64_t *>(ecol + kMxN);             // 8-byte aligned
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int n = p.n, sk = p.sk, sl = p.sl;
    // the 128-byte-swizzled operand buffers need a 1024-byte aligned base
    // (dynamic shared memory starts there only when the kernel has no static
    // shared memory); checked before any barrier or TMEM allocation, the
    // whole CTA returns together and the host reads code 2
    if (smem_u32(smem) & 1023u) {
        if (tid == 0) atomicExch(p.err, 2);
        return;
    }

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n"
                     :: "r"(smem_u32(tslot)), "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    if (tid == 0) {
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tbase = *tslot;
    const uint8_t *loaded = nullptr;
    unsigned phase = 0;
    bool failed = false;

    // persistent loop over tiles (32 complex lines of one plane each); the
    // operator slices stay in shared memory while consecutive tiles use them
    for (int tile = blockIdx.x; tile < p.cta_start[p.nf]; tile += gridDim.x) {
        int fi = 0;
        while (fi + 1 < p.nf && tile >= p.cta_start[fi + 1]) ++fi;
        const MixedField &F = p.f[fi];
        const int local = tile - p.cta_start[fi];
        const int plane = local / p.nchunks;
        const int chunk = local - plane * p.nchunks;
        const int l0 = chunk * kMxLines;
        const int L = min(kMxLines, p.n - l0);
        const double *src = F.src + (long long)plane * p.plane_stride;
        double *dst = F.dst + (long long)plane * p.plane_stride;

        if (F.Aslices != loaded) {
            for (int i = tid * 16; i < kSlices * kOpSliceBytes; i += 256 * 16) cp_async16_m(As + i, F.Aslices + i);
            asm volatile("cp.async.commit_group;\n" ::);
            loaded = F.Aslices;
        }
        if (tid < kMxN) ecol[tid] = -1074;

        // data: thread owns (line l, 16 consecutive k); coalesced for both passes
        int l, kb;
        if (sk == 1) { l = tid >> 3; kb = tid & 7; }
        else { l = tid & 31; kb = tid >> 5; }
        double2 v[16];
        int emax_re = -1074, emax_im = -1074;
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const int k = kb * 16 + q;
            v[q] = make_double2(0.0, 0.0);
            if (k < n && l < L)
                v[q] = *reinterpret_cast<const double2 *>(src + 2 * ((long long)(k + 1) * sk + (long long)(l0 + l + 1) * sl));
            int e;
            if (v[q].x != 0.0) { frexp(v[q].x, &e); emax_re = max(emax_re, e); }
            if (v[q].y != 0.0) { frexp(v[q].y, &e); emax_im = max(emax_im, e); }
        }
        __syncthreads();   // ecol initialised
        atomicMax(&ecol[2 * l], emax_re);
        atomicMax(&ecol[2 * l + 1], emax_im);
        __syncthreads();
        {
            const int e0 = ecol[2 * l], e1 = ecol[2 * l + 1];
            for (int c = 0; c < 2; ++c) {
                const int col = 2 * l + c;
                const int e = c ? e1 : e0;
                // slices of 8 consecutive k packed pairwise into 32-bit words
                uint32_t w[kSlices][8];
#pragma unroll
                for (int q = 0; q < 16; q += 2) {
                    float s0[kSlices], s1[kSlices];
                    split4(c ? v[q].y : v[q].x, e, s0);
                    split4(c ? v[q + 1].y : v[q + 1].x, e, s1);
#pragma unroll
                    for (int i = 0; i < kSlices; ++i) {
                        const __nv_bfloat162 b2 = __floats2bfloat162_rn(s0[i], s1[i]);   // .x = k, .y = k + 1
                        w[i][q >> 1] = *reinterpret_cast<const uint32_t *>(&b2);
                    }
                }
#pragma unroll
                for (int i = 0; i < kSlices; ++i)
#pragma unroll
                    for (int h = 0; h < 2; ++h)
                        *reinterpret_cast<uint4 *>(Bs + i * kDataSliceBytes + core_off(col, kb * 16 + h * 8)) =
                            make_uint4(w[i][4 * h], w[i][4 * h + 1], w[i][4 * h + 2], w[i][4 * h + 3]);
            }
        }
        asm volatile("cp.async.wait_all;\n" ::);
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");

        if (tid == 0) {
            const unsigned a0 = smem_u32(As), b0 = smem_u32(Bs);
            const unsigned sbo = (kMxK / 8) * 128;   // next 8-row group
            for (int lv = 0; lv < kLevels; ++lv) {
                const int Lsum = lv + 2;
                bool first = true;
                for (int i = 1; i <= kSlices; ++i) {
                    const int j = Lsum - i;
                    if (j < 1 || j > kSlices) continue;
                    for (int ks = 0; ks < kMxK / 16; ++ks) {
                        const uint64_t da = umma_desc(a0 + (i - 1) * kOpSliceBytes + ks * 256, 128, sbo);
                        const uint64_t db = umma_desc(b0 + (j - 1) * kDataSliceBytes + ks * 256, 128, sbo);
                        mma_bf16(tbase + lv * kMxN, da, db, first ? 0u : 1u);
                        first = false;
                    }
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n"
                         :: "r"(smem_u32(bar)) : "memory");
        }
        bool ok = false;
        for (unsigned it = 0; it < kSpinLimit; ++it) {
            if (mbar_try_wait(bar, phase)) { ok = true; break; }
            if (it > 64) __nanosleep(32);
        }
        ok = __all_sync(0xffffffffu, ok);   // tcgen05.ld below is warp-collective
        phase ^= 1u;
        if (!ok) {
            atomicExch(p.err, 1);
            failed = true;
        } else {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            // epilogue: warp w -> TMEM lanes 32 (w % 4).., columns 32 (w / 4)..
            const int qd = warp & 3, half = warp >> 2;
            const int o = qd * 32 + lane;
            float acc[kLevels][32];
#pragma unroll
            for (int lv = 0; lv < kLevels; ++lv) {
                float t0[16], t1[16];
                const uint32_t ta = tbase + ((uint32_t)(qd * 32) << 16) + lv * kMxN + half * 32;
                tmem_ld16(ta, t0);
                tmem_ld16(ta + 16, t1);
#pragma unroll
                for (int i = 0; i < 16; ++i) { acc[lv][i] = t0[i]; acc[lv][16 + i] = t1[i]; }
            }
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
            if (o < n) {
                const double lam = p.lam[F.plane0 + plane];
                const bool singular = (F.sing_io >= 0) && fabs(lam) <= 1.0e-10;
                const bool im0 = p.zero_im_mode0 && F.mode0 && plane == 0;
                const int eo = F.Aexp[o];
                const double* addp = F.add ? F.add + (long long)plane * p.plane_stride : nullptr;
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    const int lq = half * 16 + q;
                    if (lq >= L) continue;
                    const int lg = l0 + lq;
                    double val[2];
#pragma unroll
                    for (int c = 0; c < 2; ++c) {
                        const int cc = 2 * q + c;
                        double s = (double)acc[3][cc] * 0x1p-35;
                        s += (double)acc[2][cc] * 0x1p-28;
                        s += (double)acc[1][cc] * 0x1p-21;
                        s += (double)acc[0][cc] * 0x1p-14;
                        val[c] = s * pow2(eo + ecol[2 * lq + c]);
                    }
                    if (p.divide) {
                        if (singular && o == F.sing_io && lg == F.sing_io) {
                            val[0] = val[1] = 0.0;
                        } else {
                            const double den = (F.E[o] + F.E[lg]) - lam;
                            val[0] /= den;
                            val[1] /= den;
                        }
                    }
                    const long long off = 2 * ((long long)(o + 1) * sk + (long long)(lg + 1) * sl);
                    if (addp) {
                        const double2 a = *reinterpret_cast<const double2 *>(addp + off);
                        val[0] += a.x;
                        val[1] += a.y;
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
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" :: "r"(tbase), "r"(kTmemCols));
}

// ---- operator slicing (setup) --------------------------------------------
// Per-row exponents and kSlices BF16 slices of an n x n column-major operator
// padded to 128 x 128, in the core-matrix layout k_pass_mixed copies as is.
__global__ void k_split_operator(int n, const double *A, uint8_t *slices, int *rexp)
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
    for (int k = threadIdx.x; k < kMxK; k += blockDim.x) {
        const double x = (o < n && k < n) ? A[o + (size_t)n * k] : 0.0;
        float s[kSlices];
        split4(x, e, s);
        for (int i = 0; i < kSlices; ++i)
            *reinterpret_cast<__nv_bfloat16 *>(slices + i * kOpSliceBytes + core_off(o, k)) = __float2bfloat16_rn(s[i]);
    }
}

int split_operator(ductgpu_ctx ctx, int n, const double *A, uint8_t **slices, int **rexp)
{
    if (!*slices) DUCT_CUDA(ctx, cudaMalloc(slices, kSlices * kOpSliceBytes));
    if (!*rexp) DUCT_CUDA(ctx, cudaMalloc(rexp, kMxM * sizeof(int)));
    {
        LaunchScope ls(ctx, DUCTGPU_K_OTHER);
        k_split_operator<<<kMxM, 128, 0, ctx->stream>>>(n, A, *slices, *rexp);
    }
    return check_cuda(ctx, cudaGetLastError(), "k_split_operator");
}

static size_t mixed_smem_bytes()
{
    return (size_t)kSlices * (kOpSliceBytes + kDataSliceBytes) + kMxN * sizeof(int) + 64;
}

int mixed_pass(ductgpu_ctx ctx, const MixedParams &mp, int tiles)
{
    const size_t smem = mixed_smem_bytes();
    DUCT_CUDA(ctx, cudaFuncSetAttribute(k_pass_mixed, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int grid = tiles < ctx->num_sms ? tiles : ctx->num_sms;   // one CTA per SM (shared memory)
    {
        LaunchScope ls(ctx, DUCTGPU_K_MIXED_GEMM);
        k_pass_mixed<<<grid, 256, smem, ctx->stream>>>(mp);
    }
    return check_cuda(ctx, cudaGetLastError(), "k_pass_mixed");
}

// One split-precision solve of every task: src -> dst through w1, w2
// (interior only; walls untouched).  add (per task) is added to the result.
int mixed_solve_interior(ductgpu_ctx ctx, const FieldTask *tasks, int ntasks, double *const *srcs,
                         double *const *dsts, double *const *adds, double *w1, double *w2)
{
    const int m = ctx->my, n = m - 2;
    const long long ps = 2LL * m * m;
    MixedParams mp{};
    mp.nf = ntasks;
    mp.lam = ctx->lam;
    mp.plane_stride = ps;
    mp.n = n;
    mp.nchunks = (n + kMxLines - 1) / kMxLines;
    mp.err = ctx->dev_err;
    int cta = 0;
    for (int i = 0; i < ntasks; ++i) {
        mp.cta_start[i] = cta;
        cta += tasks[i].nmodes * mp.nchunks;
        mp.f[i].nmodes = tasks[i].nmodes;
        mp.f[i].mode0 = tasks[i].mode0;
        mp.f[i].plane0 = tasks[i].plane0;
        mp.f[i].sing_io = (tasks[i].bound == 'n') ? ctx->neu.iofzero - 1 : -1;
    }
    mp.cta_start[ntasks] = cta;
    for (int pass = 0; pass < 4; ++pass) {
        long long off = 0;
        for (int i = 0; i < ntasks; ++i) {
            const BoundOps &b = (tasks[i].bound == 'n') ? ctx->neu : ctx->dir;
            double *a1 = w1 + off * ps, *a2 = w2 + off * ps;
            off += tasks[i].nmodes;
            const bool useP = (pass >= 2);
            mp.f[i].Aslices = useP ? b.Pslices : b.Qslices;
            mp.f[i].Aexp = useP ? b.Pexp : b.Qexp;
            mp.f[i].E = b.E;
            mp.f[i].add = nullptr;
            switch (pass) {
            case 0: mp.f[i].src = srcs[i]; mp.f[i].dst = a1; break;
            case 1: mp.f[i].src = a1; mp.f[i].dst = a2; break;
            case 2: mp.f[i].src = a2; mp.f[i].dst = a1; break;
            default: mp.f[i].src = a1; mp.f[i].dst = dsts[i]; mp.f[i].add = adds ? adds[i] : nullptr; break;
            }
        }
        const bool ypass = (pass == 0 || pass == 3);
        mp.sk = ypass ? 1 : m;
        mp.sl = ypass ? m : 1;
        mp.divide = (pass == 1);
        mp.zero_im_mode0 = (pass == 3);
        int rc = mixed_pass(ctx, mp, cta);
        if (rc) return rc;
    }
    return DUCTGPU_OK;
}

// Remove the singular eigen-component (iofzero, iofzero) of a Neumann
// kx=0 residual in FP64: R <- R - (q^T R q) p p^T with q = row iofzero of
// P^-1 and p = column iofzero of P.  The reference's solve drops exactly
// this component of its right-hand side (src/solvediag.f90:180); removing
// it before the low-precision solve keeps the incompatible part of the data
// from leaking into the correction.  One CTA per plane.
struct ProjField {
    double *R;
    int plane0;
};
struct ProjParams {
    ProjField f[kMaxFields];
    int cta_start[kMaxFields + 1];
    int nf;
    const double *lam, *p, *q;
    long long plane_stride;
    int m, n;
};

__global__ void __launch_bounds__(256) k_project_null(const __grid_constant__ ProjParams pp)
{
    __shared__ double red[2 * 8];
    int fi = 0;
    while (fi + 1 < pp.nf && (int)blockIdx.x >= pp.cta_start[fi + 1]) ++fi;
    const int plane = blockIdx.x - pp.cta_start[fi];
    const double lam = pp.lam[pp.f[fi].plane0 + plane];
    if (!(fabs(lam) <= 1.0e-10)) return;
    const int m = pp.m, n = pp.n;
    double2 *R = reinterpret_cast<double2 *>(pp.f[fi].R + (long long)plane * pp.plane_stride);
    double s0 = 0.0, s1 = 0.0;
    for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
        const int i = idx % n, j = idx / n;
        const double w = pp.q[i] * pp.q[j];
        const double2 r = R[(i + 1) + (long long)m * (j + 1)];
        s0 += w * r.x;
        s1 += w * r.y;
    }
    for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { red[2 * warp] = s0; red[2 * warp + 1] = s1; }
    __syncthreads();
    double c0 = 0.0, c1 = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { c0 += red[2 * w]; c1 += red[2 * w + 1]; }
    for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
        const int i = idx % n, j = idx / n;
        const double w = pp.p[i] * pp.p[j];
        double2 &r = R[(i + 1) + (long long)m * (j + 1)];
        r = make_double2(r.x - c0 * w, r.y - c1 * w);
    }
}

// Split-precision solve with FP64 iterative refinement (refine_steps steps):
//   U = S(F);  repeat: R = F - (B U + U B^T - lam U);  U = U + S(R)
// S: the four tcgen05 passes above; the residual uses the reference's own
// FP64 interior operator B (D2 block, Dirichlet or Neumann-eliminated) on
// the DMMA pass, so the refined result converges to the reference's
// discrete solution.  The singular kx=0 pin, the Neumann walls/corners and
// the Dirichlet walls follow as in the FP64 path.
int solve_mixed(ductgpu_ctx ctx, const FieldTask *tasks, int ntasks)
{
    if (ntasks < 1 || ntasks > kMaxFields)
        return set_error(ctx, DUCTGPU_EARG, "solve: %d fields (1..%d)", ntasks, kMaxFields);
    const int m = ctx->my, n = m - 2;
    if (n > 127)
        return set_error(ctx, DUCTGPU_EARG, "split-precision path supports my <= 129 (got %d)", m);
    const long long ps = 2LL * m * m;
    int planes = 0;
    for (int i = 0; i < ntasks; ++i) planes += tasks[i].nmodes;
    int rc = ensure(ctx, ctx->work, (size_t)3 * planes * ps * sizeof(double));
    if (rc) return rc;
    double *w1 = ctx->work.buf, *w2 = w1 + (size_t)planes * ps, *w3 = w2 + (size_t)planes * ps;
    double *srcs[kMaxFields], *dsts[kMaxFields], *adds[kMaxFields];
    for (int i = 0; i < ntasks; ++i) {
        srcs[i] = tasks[i].rhs;
        dsts[i] = tasks[i].sol;
        adds[i] = nullptr;
    }
    // U0 = S(F) into sol
    if ((rc = mixed_solve_interior(ctx, tasks, ntasks, srcs, dsts, nullptr, w1, w2))) return rc;
    FieldTask sub[kMaxFields];
    for (int step = 0; step < ctx->refine_steps; ++step) {
        // the fields that still refine at this step, keeping their offsets
        // into the work buffers
        long long suboff[kMaxFields];
        int ns = 0;
        long long o0 = 0;
        for (int i = 0; i < ntasks; ++i) {
            if (tasks[i].refine > step) { sub[ns] = tasks[i]; suboff[ns] = o0; ++ns; }
            o0 += tasks[i].nmodes;
        }
        if (!ns) break;
        // residual R -> w3: y-pass T = (B x I) U -> w1, z-pass with the
        // residual epilogue R = F - T - (I x B) U + lam U
        PassParams pp{};
        pp.nf = ns;
        pp.lam = ctx->lam;
        int cta = 0;
        for (int i = 0; i < ns; ++i) {
            const long long off = suboff[i];
            const BoundOps &b = (sub[i].bound == 'n') ? ctx->neu : ctx->dir;
            pp.f[i].nmodes = sub[i].nmodes;
            pp.f[i].mode0 = sub[i].mode0;
            pp.f[i].plane0 = sub[i].plane0;
            pp.f[i].sing_io = -1;
            pp.f[i].sing_l = -1;
            pp.f[i].A = b.Bpack;
            pass_geometry(pp.f[i], b, b.E, n, 1, m, ps);
            pp.cta_start[i] = cta;
            cta += sub[i].nmodes * pp.f[i].nchunks;
            pp.f[i].src = sub[i].sol;
            pp.f[i].dst = w1 + off * ps;
            pp.f[i].resF = sub[i].rhs;
            pp.f[i].resT = w1 + off * ps;
            pp.f[i].resU = sub[i].sol;
        }
        pp.cta_start[ns] = cta;
        pp.divide = 0; pp.zero_im_mode0 = 0; pp.residual = 0;
        if ((rc = fp64_pass(ctx, pp, cta))) return rc;
        for (int i = 0; i < ns; ++i) {
            pp.f[i].dst = w3 + suboff[i] * ps;
            pp.f[i].sk = m;
            pp.f[i].sl = 1;
        }
        pp.residual = 1;
        if ((rc = fp64_pass(ctx, pp, cta))) return rc;
        // drop the singular component of Neumann kx=0 residuals
        ProjParams pj{};
        int pcta = 0;
        for (int i = 0; i < ns; ++i) {
            if (sub[i].bound == 'n' && ctx->neu.qrow) {
                pj.f[pj.nf].R = w3 + suboff[i] * ps;
                pj.f[pj.nf].plane0 = sub[i].plane0;
                pj.cta_start[pj.nf] = pcta;
                pcta += sub[i].nmodes;
                pj.nf++;
            }
        }
        if (pj.nf) {
            pj.cta_start[pj.nf] = pcta;
            pj.lam = ctx->lam;
            pj.p = ctx->neu.pcol;
            pj.q = ctx->neu.qrow;
            pj.plane_stride = ps;
            pj.m = m;
            pj.n = n;
            {
                LaunchScope ls(ctx, DUCTGPU_K_RESIDUAL);
                k_project_null<<<pcta, 256, 0, ctx->stream>>>(pj);
            }
            if ((rc = check_cuda(ctx, cudaGetLastError(), "k_project_null"))) return rc;
        }
        // U = U + S(R); w1/w2 are free again, indexed from the sub-list start
        for (int i = 0; i < ns; ++i) {
            srcs[i] = w3 + suboff[i] * ps;
            dsts[i] = sub[i].sol;
            adds[i] = sub[i].sol;
        }
        if ((rc = mixed_solve_interior(ctx, sub, ns, srcs, dsts, adds, w1, w2))) return rc;
    }
    if ((rc = zero_walls(ctx, tasks, ntasks))) return rc;
    return neumann_fill(ctx, tasks, ntasks);
}

}  // namespace duct
