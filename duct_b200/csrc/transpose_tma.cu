// transpose_tma.cu -- the pencil transposes (cxyz2yzx / cyzx2xyz / chx2z /
// chz2x, src/parallel.F:1-208, 476-529 on one rank) as TMA tile loads:
// out(q, a) = in(a, q) for an A x Q column-major array of complex elements.
//
// A persistent CTA walks 32 x 32 complex tiles.  Each tile arrives as four
// TMA boxes of 32 rows (q) x 8 complex (a) = 128 bytes, stored with the
// 128-byte swizzle (the 16-byte chunk c of row q lands at chunk c ^ (q & 7)),
// so a warp that reads one column a across 32 rows q hits 32 distinct banks;
// the warp then writes 32 consecutive q of out(., a) (512 contiguous bytes).
// Two tile buffers alternate: the next tile's boxes are in flight while the
// current one is transposed.  Ragged edges come from the tensor map (zero
// fill beyond the array on load, bounds checks on store).  Every wait on an
// mbarrier is bounded; running out sets the context's error word.
#include "internal.h"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <string.h>

namespace duct {

namespace {

constexpr int kTile = 32;                            // complex a x q per tile
constexpr int kBoxA = 8;                             // complex per box row: 128 bytes, the swizzle span
constexpr int kBoxBytes = kTile * kBoxA * 16;        // 4 KB
constexpr int kTileBytes = 4 * kBoxBytes;            // 16 KB
constexpr int kTThreads = 256;
constexpr unsigned kTSpin = 1u << 22;
constexpr size_t kTSmem = 2 * kTileBytes + 64 + 1024;   // two tiles, two mbarriers, alignment slack

__device__ __forceinline__ unsigned smem_addr(const void *p)
{
    return (unsigned)__cvta_generic_to_shared(p);
}

__global__ void __launch_bounds__(kTThreads) k_transpose_tma(const __grid_constant__ CUtensorMap in_map,
                                                             double2 *__restrict__ out, long long A, long long Q,
                                                             long long ta_n, long long tiles, int *err)
{
    extern __shared__ unsigned char t_raw[];
    // the 128-byte swizzle repeats every 1024 bytes of the shared address
    // space: the boxes start on a 1024-byte boundary of it
    unsigned char *base = t_raw + ((1024u - (smem_addr(t_raw) & 1023u)) & 1023u);
    double2 *stage0 = reinterpret_cast<double2 *>(base);
    uint64_t *bar = reinterpret_cast<uint64_t *>(base + 2 * kTileBytes);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_addr(bar)));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_addr(bar + 1)));
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();

    // thread 0: the four boxes of tile t into buffer s
    auto issue = [&](long long t, int s) {
        const long long ta = t % ta_n, tq = t / ta_n;
        const unsigned b = smem_addr(bar + s);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(b), "r"(kTileBytes) : "memory");
        const int y = (int)(tq * kTile);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            // inner coordinate in doubles: 2 (32 ta + 8 k), a multiple of 16 bytes
            const int x = (int)(ta * 2 * kTile) + 2 * kBoxA * k;
            const unsigned dst = smem_addr(base + (size_t)s * kTileBytes + (size_t)k * kBoxBytes);
            asm volatile(
                "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n"
                ::"r"(dst), "l"(reinterpret_cast<uint64_t>(&in_map)), "r"(x), "r"(y), "r"(b)
                : "memory");
        }
    };

    unsigned phase[2] = {0u, 0u};
    int s = 0;
    long long t = blockIdx.x;
    if (tid == 0 && t < tiles) issue(t, 0);
    for (; t < tiles; t += gridDim.x) {
        const long long tn = t + gridDim.x;
        if (tid == 0 && tn < tiles) {
            // buffer s ^ 1 was read before the barrier that closed the
            // previous tile: order those reads before the TMA writes
            asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
            issue(tn, s ^ 1);
        }
        bool ok = false;
        const unsigned b = smem_addr(bar + s);
        for (unsigned it = 0; it < kTSpin && !ok; ++it) {
            unsigned r;
            asm volatile("{\n\t.reg .pred p;\n\t"
                         "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                         "selp.u32 %0, 1, 0, p;\n\t}\n"
                         : "=r"(r) : "r"(b), "r"(phase[s]) : "memory");
            ok = r != 0;
        }
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicExch(err, 1);
            return;
        }
        phase[s] ^= 1u;
        const long long ta = t % ta_n, tq = t / ta_n;
        const long long a0 = ta * kTile, q0 = tq * kTile;
        const double2 *tile = stage0 + (size_t)s * (kTileBytes / 16);
        const int q = lane;
#pragma unroll
        for (int i = 0; i < kTile / 8; ++i) {
            const int a = warp + 8 * i, k = a >> 3, c = a & 7;
            const double2 v = tile[k * (kTile * kBoxA) + q * kBoxA + (c ^ (q & 7))];
            const long long ag = a0 + a, qg = q0 + q;
            if (ag < A && qg < Q) out[qg + Q * ag] = v;
        }
        __syncthreads();   // buffer s read: the tile after next may refill it
        s ^= 1;
    }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_tiled()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            cudaGetLastError();
    }
    return fn;
}

} // namespace

// DUCTGPU_OK, an error status, or -1 when the tensor map cannot describe the
// arrays (the caller then runs the plain tiled kernel).
int transpose_tma(ductgpu_ctx ctx, const double *in, double *out, long long A, long long Q)
{
    PFN_cuTensorMapEncodeTiled_v12000 enc = encode_tiled();
    if (!enc || A < 1 || Q < 1) return -1;
    if ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15) return -1;
    // tensor coordinates are signed 32-bit: the last tile's must fit
    if (2 * A + 2 * kTile > 0x7fffffffll || Q + kTile > 0x7fffffffll || 16 * A >= (1ll << 40)) return -1;
    static_assert(sizeof(CUtensorMap) == sizeof(ctx->tma_maps[0].map), "tensor map size");
    CUtensorMap map;
    int hit = -1;
    for (int i = 0; i < ductgpu_ctx_s::kTmaMaps; ++i)
        if (ctx->tma_maps[i].in == in && ctx->tma_maps[i].A == A && ctx->tma_maps[i].Q == Q) hit = i;
    if (hit >= 0) {
        memcpy(&map, ctx->tma_maps[hit].map, sizeof map);
    } else {
        const cuuint64_t dims[2] = {(cuuint64_t)(2 * A), (cuuint64_t)Q};
        const cuuint64_t strides[1] = {(cuuint64_t)(16 * A)};
        const cuuint32_t box[2] = {(cuuint32_t)(2 * kBoxA), (cuuint32_t)kTile};
        const cuuint32_t estr[2] = {1, 1};
        if (enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double *>(in), dims, strides, box, estr,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return -1;
        ductgpu_ctx_s::TmaMap &slot = ctx->tma_maps[ctx->tma_next];
        ctx->tma_next = (ctx->tma_next + 1) % ductgpu_ctx_s::kTmaMaps;
        slot.in = in;
        slot.A = A;
        slot.Q = Q;
        memcpy(slot.map, &map, sizeof map);
    }
    const long long ta_n = (A + kTile - 1) / kTile, tiles = ta_n * ((Q + kTile - 1) / kTile);
    // resident CTAs per SM: asked once per context (a call is ~16 us of
    // device time at a config-4 field, so host work per call shows)
    if (ctx->tma_tr_per_sm == 0) {
        int per_sm = 0;
        DUCT_CUDA(ctx, cudaFuncSetAttribute(k_transpose_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTSmem));
        DUCT_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_transpose_tma, kTThreads, kTSmem));
        ctx->tma_tr_per_sm = per_sm > 0 ? per_sm : -1;
    }
    const int per_sm = ctx->tma_tr_per_sm;
    if (per_sm < 1) return -1;
    const long long grid = std::min<long long>(tiles, (long long)per_sm * ctx->num_sms);
    {
        LaunchScope ls(ctx, DUCTGPU_K_TRANSPOSE);
        k_transpose_tma<<<(unsigned)grid, kTThreads, kTSmem, ctx->stream>>>(map, reinterpret_cast<double2 *>(out),
                                                                           A, Q, ta_n, tiles, ctx->dev_err);
    }
    return check_cuda(ctx, cudaGetLastError(), "k_transpose_tma");
}

} // namespace duct
