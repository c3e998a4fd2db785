// adjoint.cu -- the adjoint (transpose) of the FP64 helm3d solve map
// rhs -> sol of solve_fp64.cu, for reverse-mode gradients through the
// implicit step.  The forward map of one real plane is
//   Dirichlet:  sol = E_int L R_int rhs
//   Neumann:    sol = Mean o Corners o Walls o Pin o E_int L R_int rhs
// with L F = P [(P^-1 F P^-T) ./ D] P^T on the interior (D_ij = E_i + E_j -
// lambda, the singular (io,io) coefficient zeroed at lambda = 0), Pin the
// kx=0 point gauge U += c p p^T (src/solvediag.f90:195-206), Walls and
// Corners the Neumann fill from DC and AM1 (src/solvediag.f90:250-322) and
// Mean the optional zero-mean gauge.  Its transpose applied to a cotangent
// G of sol is
//   R_int^T L^T (Pin^T Walls^T Corners^T Mean^T G)_int,
//   L^T G = P^-T [(P^T G P) ./ D] P^-1,
// i.e. the same four batched DMMA passes with P^T, P^-T in place of P^-1,
// P (the transposed eigenbasis), after one kernel that folds the wall and
// corner cotangents of the Neumann planes back into their interiors.  Wall
// entries of the result are zero (the forward map ignores rhs walls), and
// mode 0 has a zero imaginary part (its forward imaginary output is zero).
#include "internal.h"

namespace duct {

struct AdjFillParams {
    const double *g[kMaxFields];
    double *w[kMaxFields];
    int plane0[kMaxFields];
    int cta_start[kMaxFields + 1];
    int nf;
    const double *DC, *AM1, *ccw, *pcol, *lam;
    int m, io, gauge;
    long long plane_stride;
};

__device__ __forceinline__ void adj_block_sum2(double &x, double &y, double *red)
{
    for (int o = 16; o > 0; o >>= 1) {
        x += __shfl_xor_sync(0xffffffffu, x, o);
        y += __shfl_xor_sync(0xffffffffu, y, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    __syncthreads();
    if (lane == 0) { red[2 * warp] = x; red[2 * warp + 1] = y; }
    __syncthreads();
    x = 0.0;
    y = 0.0;
    for (int w = 0; w < nw; ++w) { x += red[2 * w]; y += red[2 * w + 1]; }
    __syncthreads();
}

// Neumann planes: W_int = Pin^T (G' + Walls^T(G'_walls + Corners^T G'_corners))
// with G' = Mean^T G.  One CTA per complex plane.
__global__ void __launch_bounds__(1024) k_neumann_fill_adj(const __grid_constant__ AdjFillParams p)
{
    extern __shared__ double2 wl[];   // 4 wall lines of cotangents: z0, zm, y0, ym
    __shared__ double red[64];
    __shared__ double2 fbar[4];
    int fi = 0;
    while (fi + 1 < p.nf && (int)blockIdx.x >= p.cta_start[fi + 1]) ++fi;
    const int plane = blockIdx.x - p.cta_start[fi];
    const int m = p.m, n = m - 2;
    const double2 *G = reinterpret_cast<const double2 *>(p.g[fi] + (long long)plane * p.plane_stride);
    double2 *W = reinterpret_cast<double2 *>(p.w[fi] + (long long)plane * p.plane_stride);
    double2 *gz0 = wl, *gzm = wl + m, *gy0 = wl + 2 * m, *gym = wl + 3 * m;
    const double lam = p.lam[p.plane0[fi] + plane];
    const bool singular = fabs(lam) <= 1.0e-10;
    const double *DC = p.DC;

    // Mean^T: G' = G - (sum G)/4 w_i w_j
    double sx = 0.0, sy = 0.0;
    if (singular && p.gauge == DUCTGPU_GAUGE_MEAN) {
        for (int idx = threadIdx.x; idx < m * m; idx += blockDim.x) {
            const double2 v = G[idx];
            sx += v.x;
            sy += v.y;
        }
        adj_block_sum2(sx, sy, red);
    }
    auto gp = [&](int i, int j) -> double2 {
        const double2 v = G[i + (long long)m * j];
        const double w = 0.25 * p.ccw[i] * p.ccw[j];
        return make_double2(v.x - w * sx, v.y - w * sy);
    };
    // Corners^T: Fbar = AM1^T cbar, corners (1,1), (m,1), (m,m), (1,m)
    if (threadIdx.x < 4) {
        const int r = threadIdx.x;
        const double2 c[4] = {gp(0, 0), gp(m - 1, 0), gp(m - 1, m - 1), gp(0, m - 1)};
        double2 f = make_double2(0.0, 0.0);
        for (int k = 0; k < 4; ++k) {
            const double a = p.AM1[k + 4 * r];
            f.x += a * c[k].x;
            f.y += a * c[k].y;
        }
        fbar[r] = f;
    }
    __syncthreads();
    // wall cotangents of the interior wall points
    for (int i = 1 + threadIdx.x; i < m - 1; i += blockDim.x) {
        const double a = DC[(long long)m * i], b = DC[(m - 1) + (long long)m * i];
        const double2 f0 = fbar[0], f1 = fbar[1], f2 = fbar[2], f3 = fbar[3];
        const double2 z0 = gp(i, 0), y0 = gp(0, i), ym = gp(m - 1, i), zm = gp(i, m - 1);
        gz0[i] = make_double2(z0.x - a * f0.x + b * f1.x, z0.y - a * f0.y + b * f1.y);
        gy0[i] = make_double2(y0.x - a * f0.x + b * f3.x, y0.y - a * f0.y + b * f3.y);
        gym[i] = make_double2(ym.x - a * f1.x - b * f2.x, ym.y - a * f1.y - b * f2.y);
        gzm[i] = make_double2(zm.x - b * f2.x - a * f3.x, zm.y - b * f2.y - a * f3.y);
    }
    __syncthreads();
    // Walls^T into the interior
    const double d11 = DC[0], d1m = DC[(long long)m * (m - 1)];
    const double dm1 = DC[m - 1], dmm = DC[(m - 1) + (long long)m * (m - 1)];
    const double idet = 1.0 / (d11 * dmm - d1m * dm1);
    for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
        const int i = 1 + idx % n, j = 1 + idx / n;
        const double a_j = DC[(long long)m * j], b_j = DC[(m - 1) + (long long)m * j];
        const double a_i = DC[(long long)m * i], b_i = DC[(m - 1) + (long long)m * i];
        const double2 v = gp(i, j);
        const double2 z0 = gz0[i], zm = gzm[i], y0 = gy0[j], ym = gym[j];
        const double cz0 = (-dmm * a_j + d1m * b_j) * idet, czm = (dm1 * a_j - d11 * b_j) * idet;
        const double cy0 = (-dmm * a_i + d1m * b_i) * idet, cym = (dm1 * a_i - d11 * b_i) * idet;
        W[i + (long long)m * j] = make_double2(v.x + cz0 * z0.x + czm * zm.x + cy0 * y0.x + cym * ym.x,
                                               v.y + cz0 * z0.y + czm * zm.y + cy0 * y0.y + cym * ym.y);
    }
    // Pin^T: W(io,io) -= (p^T W p) / p_io^2
    if (singular && p.io >= 0) {
        __syncthreads();
        double px = 0.0, py = 0.0;
        for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
            const int i = idx % n, j = idx / n;
            const double w = p.pcol[i] * p.pcol[j];
            const double2 v = W[(i + 1) + (long long)m * (j + 1)];
            px += w * v.x;
            py += w * v.y;
        }
        adj_block_sum2(px, py, red);
        if (threadIdx.x == 0) {
            const double pio = p.pcol[p.io];
            double2 &u = W[(p.io + 1) + (long long)m * (p.io + 1)];
            u = make_double2(u.x - px / (pio * pio), u.y - py / (pio * pio));
        }
    }
}

// Wall lines of the result are zero (one CTA per plane).
struct AdjWallParams {
    double *out[kMaxFields];
    int cta_start[kMaxFields + 1];
};
__global__ void k_adj_walls(const __grid_constant__ AdjWallParams p, int nf, int m, long long ps)
{
    const int *cta_start = p.cta_start;
    double *const *outs = p.out;
    int fi = 0;
    while (fi + 1 < nf && (int)blockIdx.x >= cta_start[fi + 1]) ++fi;
    double2 *U = reinterpret_cast<double2 *>(outs[fi] + (long long)(blockIdx.x - cta_start[fi]) * ps);
    for (int i = threadIdx.x; i < 4 * m; i += blockDim.x) {
        const int side = i / m, q = i % m;
        long long off;
        if (side == 0) off = q;
        else if (side == 1) off = q + (long long)m * (m - 1);
        else if (side == 2) off = (long long)m * q;
        else off = (m - 1) + (long long)m * q;
        U[off] = make_double2(0.0, 0.0);
    }
}

int solve_adjoint(ductgpu_ctx ctx, const FieldTask *tasks, int ntasks)
{
    const int m = ctx->my, n = m - 2;
    const long long ps = 2LL * m * m;
    int planes = 0, nneu = 0;
    for (int i = 0; i < ntasks; ++i) {
        planes += tasks[i].nmodes;
        if (tasks[i].bound == 'n') nneu += tasks[i].nmodes;
    }
    int rc;
    if ((rc = pack_transposed(ctx, ctx->dir))) return rc;
    if ((rc = pack_transposed(ctx, ctx->neu))) return rc;
    if ((rc = ensure(ctx, ctx->work, (size_t)(2 * planes + nneu) * ps * sizeof(double)))) return rc;
    double *w1 = ctx->work.buf, *w2 = w1 + (size_t)planes * ps, *w0 = w2 + (size_t)planes * ps;

    // Neumann planes: fold wall and corner cotangents into the interior (w0)
    const double *src0[kMaxFields];
    {
        AdjFillParams fp{};
        int cta = 0, fn = 0;
        long long off = 0;
        for (int i = 0; i < ntasks; ++i) {
            src0[i] = tasks[i].rhs;
            if (tasks[i].bound != 'n') continue;
            fp.g[fn] = tasks[i].rhs;
            fp.w[fn] = w0 + off * ps;
            src0[i] = fp.w[fn];
            fp.plane0[fn] = tasks[i].plane0;
            fp.cta_start[fn] = cta;
            cta += tasks[i].nmodes;
            off += tasks[i].nmodes;
            ++fn;
        }
        if (fn) {
            fp.cta_start[fn] = cta;
            fp.nf = fn;
            fp.DC = ctx->DC; fp.AM1 = ctx->AM1; fp.ccw = ctx->ccw; fp.pcol = ctx->neu.pcol; fp.lam = ctx->lam;
            fp.m = m;
            fp.io = ctx->neu.pcol ? pin_index(ctx) : -1;
            fp.gauge = ctx->gauge;
            fp.plane_stride = ps;
            LaunchScope ls(ctx, DUCTGPU_K_NEUMANN);
            k_neumann_fill_adj<<<cta, 1024, 4 * m * sizeof(double2), ctx->stream>>>(fp);
        }
    }
    // L^T: y with P^T, z with P^T + divide, z with P^-T, y with P^-T.  On the
    // flip-symmetric operators (when the forward solve uses them) the
    // transpose of an unfolded P pass is a folded pass with the blocks
    // transposed, and that of a folded P^-1 pass an unfolded one.
    const bool fold = use_fold(ctx, tasks, ntasks);
    PassParams pp{};
    pp.lam = ctx->lam;
    for (int pass = 0; pass < 4; ++pass) {
        long long off = 0;
        int cta = 0;
        const bool ypass = (pass == 0 || pass == 3);
        for (int i = 0; i < ntasks; ++i) {
            const BoundOps &b = (tasks[i].bound == 'n') ? ctx->neu : ctx->dir;
            PassField &f = pp.f[i];
            double *a1 = w1 + off * ps, *a2 = w2 + off * ps;
            off += tasks[i].nmodes;
            pass_geometry(f, b, b.E, n, ypass ? 1 : m, ypass ? m : 1, ps);
            f.nmodes = tasks[i].nmodes;
            f.mode0 = tasks[i].mode0;
            f.plane0 = tasks[i].plane0;
            f.sing_io = (tasks[i].bound == 'n') ? ctx->neu.iofzero - 1 : -1;
            f.sing_l = f.sing_io;
            switch (pass) {
            case 0: f.src = src0[i]; f.dst = a1; f.A = b.PTpack; break;
            case 1: f.src = a1; f.dst = a2; f.A = b.PTpack; break;
            case 2: f.src = a2; f.dst = a1; f.A = b.QTpack; break;
            default: f.src = a1; f.dst = tasks[i].sol; f.A = b.QTpack; break;
            }
            if (fold)
                fold_field(f, b, (pass < 2) ? 1 : 2, (pass < 2) ? b.PfoldT : b.QfoldT, tasks[i].bound == 'n');
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
    AdjWallParams wp{};
    int cta = 0;
    for (int i = 0; i < ntasks; ++i) {
        wp.out[i] = tasks[i].sol;
        wp.cta_start[i] = cta;
        cta += tasks[i].nmodes;
    }
    wp.cta_start[ntasks] = cta;
    {
        LaunchScope ls(ctx, DUCTGPU_K_WALLS);
        k_adj_walls<<<cta, 256, 0, ctx->stream>>>(wp, ntasks, m, ps);
    }
    return check_cuda(ctx, cudaGetLastError(), "solve_adjoint");
}

}  // namespace duct
