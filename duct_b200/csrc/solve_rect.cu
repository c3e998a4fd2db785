// solve_rect.cu -- the rectangular / general-wall-condition solve of the
// reference's temperature path: helm3d_temp -> int2d3d_temp ->
// solvediag_temp (src/helm3d_temp.f90:2-46, src/int2d3d_temp.f90:51-88,
// src/solvediag_temp.f90:1-351), batched over modes, fields and duct
// shapes.
//
//   F' = F_interior + mod_term_FTy + mod_term_FTz   (non-homogeneous walls)
//   U  = PY [ (PY^-1 F' PZ^-T) / (EY_i + EZ_j - lambda) ] PZ^T
//   walls from edge_value_y / edge_value_z, corners kept from the input.
//
// The four GEMM passes are the FP64 DMMA passes of solve_fp64.cu with
// per-field geometry, so fields of differently shaped ducts (operator
// slots) share each launch.  The reference divides by zero for the
// singular all-Neumann mode at lambda = 0 (its guard
// `abs(den).eq.1.d-12` never fires, src/solvediag_temp.f90:52); here the
// eigen-coefficient of the smallest |EY| x |EZ| pair is set to zero, which
// fixes the additive constant (GAUGE_MEAN then shifts it to zero mean).
#include <math.h>

#include "internal.h"

namespace duct {

struct RectKField {
    const double *rhs;
    double *dst;         // corrected interior (bc kernel) or solution (edges)
    double *sol;
    const double *bcy, *bcz;
    int my, mz, mode0, plane0, slot;
    long long plane_stride;
    // slot data
    const double *DY, *D2Y, *DZ, *D2Z, *wy, *wz;
    char by1, by2, bz1, bz2;
    int allneu;
};

struct RectKParams {
    RectKField f[kMaxFields];
    int cta_start[kMaxFields + 1];
    int nf;
    const double *lam;
    int gauge;
};

__device__ __forceinline__ int rect_field(const RectKParams &p)
{
    int fi = 0;
    while (fi + 1 < p.nf && (int)blockIdx.x >= p.cta_start[fi + 1]) ++fi;
    return fi;
}

// mod_term_FTy / mod_term_FTz (src/solvediag_temp.f90:86-239) added to the
// interior of the right-hand side; the same real wall values serve the real
// and the imaginary part (src/int2d3d_temp.f90:71-83).
__global__ void __launch_bounds__(256) k_rect_bc(const __grid_constant__ RectKParams p)
{
    const int fi = rect_field(p);
    const RectKField &F = p.f[fi];
    const int plane = blockIdx.x - p.cta_start[fi];
    const int my = F.my, mz = F.mz;
    const double2 *R = reinterpret_cast<const double2 *>(F.rhs + (long long)plane * F.plane_stride);
    double2 *O = reinterpret_cast<double2 *>(F.dst + (long long)plane * F.plane_stride);
    const double *bcy = F.bcy ? F.bcy + (long long)2 * mz * plane : nullptr;
    const double *bcz = F.bcz ? F.bcz + (long long)2 * my * plane : nullptr;
    const double *DY = F.DY, *D2Y = F.D2Y, *DZ = F.DZ, *D2Z = F.D2Z;
    const double y11 = DY[0], y1m = DY[(long long)my * (my - 1)], ym1 = DY[my - 1], ymm = DY[(my - 1) + (long long)my * (my - 1)];
    const double z11 = DZ[0], z1m = DZ[(long long)mz * (mz - 1)], zm1 = DZ[mz - 1], zmm = DZ[(mz - 1) + (long long)mz * (mz - 1)];
    for (int idx = threadIdx.x; idx < (my - 2) * (mz - 2); idx += blockDim.x) {
        const int i = idx % (my - 2) + 1, j = idx / (my - 2) + 1;
        double v = 0.0, h = 0.0;
        if (bcy) {
            const double c1 = bcy[j], c2 = bcy[j + mz];
            const double a1 = D2Y[i], a2 = D2Y[i + (long long)my * (my - 1)];
            if (F.by1 == 'd' && F.by2 == 'd') v = -a1 * c1 - a2 * c2;
            else if (F.by1 == 'd') v = -a1 * c1 - a2 * (c2 - ym1 * c1) / ymm;
            else if (F.by2 == 'd') v = -a1 * (c1 - y1m * c2) / y11 - a2 * c2;
            else {
                const double det = y11 * ymm - y1m * ym1;
                v = a1 * (y1m * c2 - ymm * c1) / det + a2 * (ym1 * c1 - y11 * c2) / det;
            }
        }
        if (bcz) {
            const double c1 = bcz[i], c2 = bcz[i + my];
            const double a1 = D2Z[j], a2 = D2Z[j + (long long)mz * (mz - 1)];
            if (F.bz1 == 'd' && F.bz2 == 'd') h = -a1 * c1 - a2 * c2;
            else if (F.bz1 == 'd') h = -a1 * c1 - a2 * (c2 - zm1 * c1) / zmm;
            else if (F.bz2 == 'd') h = -a1 * (c1 - z1m * c2) / z11 - a2 * c2;
            else {
                const double det = z11 * zmm - z1m * zm1;
                h = a1 * (z1m * c2 - zmm * c1) / det + a2 * (zm1 * c1 - z11 * c2) / det;
            }
        }
        const double2 r = R[i + (long long)my * j];
        O[i + (long long)my * j] = make_double2(r.x + v + h, r.y + v + h);
    }
}

// edge_value_y / edge_value_z (src/solvediag_temp.f90:241-351), corners
// copied from the input plane, mode 0 real, optional zero-mean gauge of the
// singular all-Neumann mode.  One CTA per plane.
__global__ void __launch_bounds__(256) k_rect_edges(const __grid_constant__ RectKParams p)
{
    __shared__ double red[2 * 8];
    const int fi = rect_field(p);
    const RectKField &F = p.f[fi];
    const int plane = blockIdx.x - p.cta_start[fi];
    const int my = F.my, mz = F.mz;
    const double2 *R = reinterpret_cast<const double2 *>(F.rhs + (long long)plane * F.plane_stride);
    double2 *U = reinterpret_cast<double2 *>(F.sol + (long long)plane * F.plane_stride);
    const double *bcy = F.bcy ? F.bcy + (long long)2 * mz * plane : nullptr;
    const double *bcz = F.bcz ? F.bcz + (long long)2 * my * plane : nullptr;
    const double *DY = F.DY, *DZ = F.DZ;
    const double y11 = DY[0], y1m = DY[(long long)my * (my - 1)], ym1 = DY[my - 1], ymm = DY[(my - 1) + (long long)my * (my - 1)];
    const double z11 = DZ[0], z1m = DZ[(long long)mz * (mz - 1)], zm1 = DZ[mz - 1], zmm = DZ[(mz - 1) + (long long)mz * (mz - 1)];
    const bool mode0 = F.mode0 && plane == 0;
    // y walls U(1,j), U(my,j) of the interior columns: one warp per column
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int j = 1 + warp; j < mz - 1; j += nw) {
        double a[2] = {0, 0}, b[2] = {0, 0};
        for (int i = 1 + lane; i < my - 1; i += 32) {
            const double2 v = U[i + (long long)my * j];
            const double d1 = DY[(long long)my * i], dm = DY[(my - 1) + (long long)my * i];
            a[0] += d1 * v.x; a[1] += d1 * v.y; b[0] += dm * v.x; b[1] += dm * v.y;
        }
        for (int o = 16; o > 0; o >>= 1)
            for (int c = 0; c < 2; ++c) {
                a[c] += __shfl_xor_sync(0xffffffffu, a[c], o);
                b[c] += __shfl_xor_sync(0xffffffffu, b[c], o);
            }
        if (lane == 0) {
            const double c1 = bcy ? bcy[j] : 0.0, c2 = bcy ? bcy[j + mz] : 0.0;
            double lo[2], hi[2];
            for (int c = 0; c < 2; ++c) {
                if (F.by1 == 'd' && F.by2 == 'd') { lo[c] = c1; hi[c] = c2; }
                else if (F.by1 == 'd') { lo[c] = c1; hi[c] = (c2 - ym1 * lo[c] - b[c]) / ymm; }
                else if (F.by2 == 'd') { hi[c] = c2; lo[c] = (c1 - y1m * hi[c] - a[c]) / y11; }
                else {
                    const double det = y11 * ymm - y1m * ym1;
                    lo[c] = (ymm * (c1 - a[c]) - y1m * (c2 - b[c])) / det;
                    hi[c] = (-ym1 * (c1 - a[c]) + y11 * (c2 - b[c])) / det;
                }
            }
            U[(long long)my * j] = make_double2(lo[0], mode0 ? 0.0 : lo[1]);
            U[(my - 1) + (long long)my * j] = make_double2(hi[0], mode0 ? 0.0 : hi[1]);
        }
    }
    // z walls U(i,1), U(i,mz) of the interior rows: one thread per row
    for (int i = 1 + threadIdx.x; i < my - 1; i += blockDim.x) {
        double a[2] = {0, 0}, b[2] = {0, 0};
        for (int j = 1; j < mz - 1; ++j) {
            const double2 v = U[i + (long long)my * j];
            const double d1 = DZ[(long long)mz * j], dm = DZ[(mz - 1) + (long long)mz * j];
            a[0] += d1 * v.x; a[1] += d1 * v.y; b[0] += dm * v.x; b[1] += dm * v.y;
        }
        const double c1 = bcz ? bcz[i] : 0.0, c2 = bcz ? bcz[i + my] : 0.0;
        double lo[2], hi[2];
        for (int c = 0; c < 2; ++c) {
            if (F.bz1 == 'd' && F.bz2 == 'd') { lo[c] = c1; hi[c] = c2; }
            else if (F.bz1 == 'd') { lo[c] = c1; hi[c] = (c2 - zm1 * lo[c] - b[c]) / zmm; }
            else if (F.bz2 == 'd') { hi[c] = c2; lo[c] = (c1 - z1m * hi[c] - a[c]) / z11; }
            else {
                const double det = z11 * zmm - z1m * zm1;
                lo[c] = (zmm * (c1 - a[c]) - z1m * (c2 - b[c])) / det;
                hi[c] = (-zm1 * (c1 - a[c]) + z11 * (c2 - b[c])) / det;
            }
        }
        U[i] = make_double2(lo[0], mode0 ? 0.0 : lo[1]);
        U[i + (long long)my * (mz - 1)] = make_double2(hi[0], mode0 ? 0.0 : hi[1]);
    }
    if (threadIdx.x < 4) {
        const long long c = (threadIdx.x & 1 ? my - 1 : 0) + (long long)my * (threadIdx.x & 2 ? mz - 1 : 0);
        const double2 r = R[c];
        U[c] = make_double2(r.x, mode0 ? 0.0 : r.y);
    }
    const double lam = p.lam[F.plane0 + plane];
    if (F.allneu && p.gauge == DUCTGPU_GAUGE_MEAN && fabs(lam) <= 1.0e-10) {
        __syncthreads();
        double s[2] = {0.0, 0.0};
        for (int idx = threadIdx.x; idx < my * mz; idx += blockDim.x) {
            const int i = idx % my, j = idx / my;
            const double w = F.wy[i] * F.wz[j];
            const double2 v = U[idx];
            s[0] += w * v.x;
            s[1] += w * v.y;
        }
        for (int o = 16; o > 0; o >>= 1)
            for (int c = 0; c < 2; ++c) s[c] += __shfl_xor_sync(0xffffffffu, s[c], o);
        if (lane == 0) { red[2 * warp] = s[0]; red[2 * warp + 1] = s[1]; }
        __syncthreads();
        double t0 = 0.0, t1 = 0.0;
        for (int w = 0; w < nw; ++w) { t0 += red[2 * w]; t1 += red[2 * w + 1]; }
        // area of [-sy,sy] x [-sz,sz] = sum of the weights
        double area = 0.0;
        for (int i = 0; i < my; ++i) area += F.wy[i];
        double az = 0.0;
        for (int j = 0; j < mz; ++j) az += F.wz[j];
        area *= az;
        for (int idx = threadIdx.x; idx < my * mz; idx += blockDim.x)
            U[idx] = make_double2(U[idx].x - t0 / area, U[idx].y - t1 / area);
    }
}

int solve_rect(ductgpu_ctx ctx, const RectTask *tasks, int ntasks)
{
    if (ntasks < 1 || ntasks > kMaxFields)
        return set_error(ctx, DUCTGPU_EARG, "solve: %d fields (1..%d)", ntasks, kMaxFields);
    long long offs[kMaxFields + 1];
    offs[0] = 0;
    bool any_bc = false;
    for (int i = 0; i < ntasks; ++i) {
        const RectSlot &r = ctx->rect[tasks[i].slot];
        offs[i + 1] = offs[i] + (long long)tasks[i].nmodes * 2 * r.my * r.mz;
        any_bc |= (tasks[i].bcy || tasks[i].bcz);
    }
    const long long total = offs[ntasks];
    int rc = ensure(ctx, ctx->work, (size_t)(any_bc ? 3 : 2) * total * sizeof(double));
    if (rc) return rc;
    double *w1 = ctx->work.buf, *w2 = w1 + total, *w3 = w2 + total;

    RectKParams kp{};
    kp.nf = ntasks;
    kp.lam = ctx->lam;
    kp.gauge = ctx->gauge;
    int kcta = 0;
    for (int i = 0; i < ntasks; ++i) {
        const RectSlot &r = ctx->rect[tasks[i].slot];
        RectKField &f = kp.f[i];
        f.rhs = tasks[i].rhs;
        f.dst = w3 + offs[i];
        f.sol = tasks[i].sol;
        f.bcy = tasks[i].bcy;
        f.bcz = tasks[i].bcz;
        f.my = r.my; f.mz = r.mz;
        f.mode0 = tasks[i].mode0;
        f.plane0 = tasks[i].plane0;
        f.slot = tasks[i].slot;
        f.plane_stride = 2LL * r.my * r.mz;
        f.DY = r.DY; f.D2Y = r.D2Y; f.DZ = r.DZ; f.D2Z = r.D2Z; f.wy = r.wy; f.wz = r.wz;
        f.by1 = r.by1; f.by2 = r.by2; f.bz1 = r.bz1; f.bz2 = r.bz2;
        f.allneu = (r.by1 == 'n' && r.by2 == 'n' && r.bz1 == 'n' && r.bz2 == 'n');
        kp.cta_start[i] = kcta;
        kcta += tasks[i].nmodes;
    }
    kp.cta_start[ntasks] = kcta;
    if (any_bc) {
        LaunchScope ls(ctx, DUCTGPU_K_OTHER);
        k_rect_bc<<<kcta, 256, 0, ctx->stream>>>(kp);
    }
    if ((rc = check_cuda(ctx, cudaGetLastError(), "k_rect_bc"))) return rc;

    // the flip-symmetric half blocks when every field's two directions have them
    bool fold = ctx->rect_fold != 0;
    for (int i = 0; i < ntasks && fold; ++i) {
        const RectSlot &r = ctx->rect[tasks[i].slot];
        fold = r.y.fold_ok && r.z.fold_ok;
    }
    if (fold) {
        // field i of pass `pass` on the half blocks
        auto folded_field = [&](PassField &f, int pass, int i) {
            const RectSlot &r = ctx->rect[tasks[i].slot];
            const bool ypass = (pass == 0 || pass == 3);
            const BoundOps &b = ypass ? r.y : r.z;
            const long long ps = 2LL * r.my * r.mz;
            pass_geometry(f, b, ypass ? r.z.E : r.y.E, ypass ? r.z.n : r.y.n, ypass ? 1 : r.my, ypass ? r.my : 1,
                          ps);
            f.nmodes = tasks[i].nmodes;
            f.mode0 = tasks[i].mode0;
            f.plane0 = tasks[i].plane0;
            const double *src0 = (tasks[i].bcy || tasks[i].bcz) ? w3 + offs[i] : tasks[i].rhs;
            switch (pass) {
            case 0: f.src = src0; f.dst = w1 + offs[i]; break;
            case 1: f.src = w1 + offs[i]; f.dst = w2 + offs[i]; break;
            case 2: f.src = w2 + offs[i]; f.dst = w1 + offs[i]; break;
            default: f.src = w1 + offs[i]; f.dst = tasks[i].sol; break;
            }
            fold_field(f, b, (pass < 2) ? 1 : 2, (pass < 2) ? b.Qfold : b.Pfold, false);
            // eigenvalues along the pass and along the lines, both in the
            // even-first order; the all-Neumann singular pair in it
            f.E = b.Eperm;
            f.El = ypass ? r.z.Eperm : r.y.Eperm;
            const bool allneu = kp.f[i].allneu;
            f.sing_io = allneu ? (ypass ? r.sing_yp : r.sing_zp) : -1;
            f.sing_l = allneu ? (ypass ? r.sing_zp : r.sing_yp) : -1;
        };
        auto pass_flags = [](PassParams &pp, int pass) {
            pp.divide = (pass == 1);
            pp.zero_im_mode0 = (pass == 3);
            pp.residual = 0;
        };
        // fields grouped by the half-block sizes of their two directions:
        // groups are independent, so with several of them each group's four
        // passes run on a stream of its own (forked from and joined to the
        // context's stream; a captured graph gets parallel branches), and
        // the small launches of one group fill the tails of the others'
        int grp[kMaxFields], ng = 0, gy[kMaxFields], gz[kMaxFields];
        for (int i = 0; i < ntasks; ++i) {
            const RectSlot &r = ctx->rect[tasks[i].slot];
            int g = 0;
            while (g < ng && !(gy[g] == r.y.hpad && gz[g] == r.z.hpad)) ++g;
            if (g == ng) {
                gy[ng] = r.y.hpad;
                gz[ng] = r.z.hpad;
                ++ng;
            }
            grp[i] = g;
        }
        bool streams = ctx->rect_fold == 1 && ng > 1 && ng <= 1 + ductgpu_ctx_s::kSideStreams;
        if (streams && !ctx->side[ng - 2]) {
            if (ctx->capturing) {
                streams = false;        // created outside a capture only: one stream then
            } else {
                if (!ctx->side_fork) DUCT_CUDA(ctx, cudaEventCreateWithFlags(&ctx->side_fork, cudaEventDisableTiming));
                for (int k = 0; k < ng - 1; ++k)
                    if (!ctx->side[k]) {
                        DUCT_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->side[k], cudaStreamNonBlocking));
                        DUCT_CUDA(ctx, cudaEventCreateWithFlags(&ctx->side_join[k], cudaEventDisableTiming));
                    }
            }
        }
        if (streams) {
            cudaStream_t main = ctx->stream;
            DUCT_CUDA(ctx, cudaEventRecord(ctx->side_fork, main));
            int rcg = DUCTGPU_OK;
            for (int g = 0; g < ng; ++g) {
                cudaStream_t st = g ? ctx->side[g - 1] : main;
                if (g) DUCT_CUDA(ctx, cudaStreamWaitEvent(st, ctx->side_fork, 0));
                ctx->stream = st;
                for (int pass = 0; pass < 4 && !rcg; ++pass) {
                    PassParams pp{};
                    pp.lam = ctx->lam;
                    int cta = 0, nf = 0;
                    for (int i = 0; i < ntasks; ++i) {
                        if (grp[i] != g) continue;
                        folded_field(pp.f[nf], pass, i);
                        pp.cta_start[nf] = cta;
                        cta += tasks[i].nmodes * pp.f[nf].nchunks;
                        ++nf;
                    }
                    pp.cta_start[nf] = cta;
                    pp.nf = nf;
                    pass_flags(pp, pass);
                    rcg = fp64_pass(ctx, pp, cta);
                }
                ctx->stream = main;
                if (g) {
                    // joined even after an error, so that a capture stays whole
                    cudaEventRecord(ctx->side_join[g - 1], st);
                    cudaStreamWaitEvent(main, ctx->side_join[g - 1], 0);
                }
            }
            if (rcg) return rcg;
        } else if (ctx->rect_fold == 2) {
            // one persistent launch for the four passes of every field, any
            // mix of half-block sizes
            PassParams pp[4] = {};
            for (int pass = 0; pass < 4; ++pass) {
                pp[pass].lam = ctx->lam;
                pp[pass].nf = ntasks;
                pass_flags(pp[pass], pass);
                for (int i = 0; i < ntasks; ++i) folded_field(pp[pass].f[i], pass, i);
            }
            if ((rc = fp64_pass_queue(ctx, pp))) return rc;
        } else {
            // a launch per pass and half-block size of the pass direction
            for (int pass = 0; pass < 4; ++pass) {
                const bool ypass = (pass == 0 || pass == 3);
                bool done[kMaxFields] = {};
                for (int lead = 0; lead < ntasks; ++lead) {
                    if (done[lead]) continue;
                    const int hp = ypass ? ctx->rect[tasks[lead].slot].y.hpad : ctx->rect[tasks[lead].slot].z.hpad;
                    PassParams pp{};
                    pp.lam = ctx->lam;
                    int cta = 0, nf = 0;
                    for (int i = lead; i < ntasks; ++i) {
                        const RectSlot &r = ctx->rect[tasks[i].slot];
                        const BoundOps &b = ypass ? r.y : r.z;
                        if (done[i] || b.hpad != hp) continue;
                        done[i] = true;
                        PassField &f = pp.f[nf];
                        folded_field(f, pass, i);
                        pp.cta_start[nf] = cta;
                        cta += tasks[i].nmodes * f.nchunks;
                        ++nf;
                    }
                    pp.cta_start[nf] = cta;
                    pp.nf = nf;
                    pass_flags(pp, pass);
                    if ((rc = fp64_pass(ctx, pp, cta))) return rc;
                }
            }
        }
        {
            LaunchScope ls(ctx, DUCTGPU_K_NEUMANN);
            k_rect_edges<<<kcta, 256, 0, ctx->stream>>>(kp);
        }
        return check_cuda(ctx, cudaGetLastError(), "k_rect_edges");
    }

    PassParams pp{};
    pp.lam = ctx->lam;
    for (int pass = 0; pass < 4; ++pass) {
        int cta = 0;
        for (int i = 0; i < ntasks; ++i) {
            const RectSlot &r = ctx->rect[tasks[i].slot];
            PassField &f = pp.f[i];
            const long long ps = 2LL * r.my * r.mz;
            const bool ypass = (pass == 0 || pass == 3);
            const BoundOps &b = ypass ? r.y : r.z;
            pass_geometry(f, b, ypass ? r.z.E : r.y.E, ypass ? r.z.n : r.y.n, ypass ? 1 : r.my,
                          ypass ? r.my : 1, ps);
            f.nmodes = tasks[i].nmodes;
            f.mode0 = tasks[i].mode0;
            f.plane0 = tasks[i].plane0;
            const bool allneu = kp.f[i].allneu;
            f.sing_io = allneu ? r.sing_z : -1;   // used in pass 2: o along z, lines along y
            f.sing_l = allneu ? r.sing_y : -1;
            const double *src0 = (tasks[i].bcy || tasks[i].bcz) ? w3 + offs[i] : tasks[i].rhs;
            switch (pass) {
            case 0: f.src = src0; f.dst = w1 + offs[i]; f.A = r.y.Qpack; break;
            case 1: f.src = w1 + offs[i]; f.dst = w2 + offs[i]; f.A = r.z.Qpack; break;
            case 2: f.src = w2 + offs[i]; f.dst = w1 + offs[i]; f.A = r.z.Ppack; break;
            default: f.src = w1 + offs[i]; f.dst = tasks[i].sol; f.A = r.y.Ppack; break;
            }
            pp.cta_start[i] = cta;
            cta += tasks[i].nmodes * f.nchunks;
        }
        pp.cta_start[ntasks] = cta;
        pp.nf = ntasks;
        pp.divide = (pass == 1);
        pp.zero_im_mode0 = (pass == 3);
        pp.residual = 0;
        if ((rc = fp64_pass(ctx, pp, cta))) return rc;
    }
    {
        LaunchScope ls(ctx, DUCTGPU_K_NEUMANN);
        k_rect_edges<<<kcta, 256, 0, ctx->stream>>>(kp);
    }
    return check_cuda(ctx, cudaGetLastError(), "k_rect_edges");
}

}  // namespace duct
