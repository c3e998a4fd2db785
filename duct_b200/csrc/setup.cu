// setup.cu -- one-time FP64 operator setup on the GPU: the reference's
// pseudomat('d',m) and pseudomat('n',m) (src/pseudomat.f90:2-312).
//
// Collocation nodes, the CHQZ derivative matrix, D2 = D*D, the Dirichlet
// interior block and the Neumann-eliminated block are built by small FP64
// kernels; the non-symmetric eigen-decomposition (the reference's dgeev) is
// cuSOLVER's Xgeev and the inverse (dgetrf/dgetri) is getrf + getrs against
// the identity, all on the device.  Only iofzero (an argmin over n values)
// and the 4x4 corner matrix AM1 are finished on the host.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "internal.h"

namespace duct {

// src/pseudomat.f90:72-107: nodes x_j = -cos(pi j/(m-1)) and
// DC(l,j) = dd(l)/dd(j) (-1)^(l+j) / (x_l - x_j), diagonal per CHQZ; every
// entry times `scale` (1/half-width, src/pseudomat_temp.f90:77).
__global__ void k_build_dc(int m, double *x, double *DC, double scale = 1.0)
{
    const double pi = 3.14159265358979323846;
    const int n = m - 1;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < m * m;
         idx += gridDim.x * blockDim.x) {
        const int l = idx % m, j = idx / m;
        const double xl = -cos(pi * (double)l / (double)n);
        const double xj = -cos(pi * (double)j / (double)n);
        if (j == 0) x[l] = xl;
        double v;
        if (l == j) {
            if (l == 0) v = -(2.0 * (double)n * (double)n + 1.0) / 6.0;
            else if (l == m - 1) v = (2.0 * (double)n * (double)n + 1.0) / 6.0;
            else v = -0.5 * xl / (1.0 - xl * xl);
        } else {
            const double ddl = (l == 0 || l == m - 1) ? 2.0 : 1.0;
            const double ddj = (j == 0 || j == m - 1) ? 2.0 : 1.0;
            const double sgn = ((l + j) & 1) ? -1.0 : 1.0;
            v = ddl / ddj * sgn / (xl - xj);
        }
        DC[l + (size_t)m * j] = v * scale;
    }
}

// Interior block of D2 for a wall-condition pair (b1 at -s, b2 at +s),
// src/pseudomat_temp.f90:89-137.
__global__ void k_block_bc(int m, char b1, char b2, const double *D, const double *D2, double *B)
{
    const int n = m - 2;
    const double d11 = D[0], d1m = D[(size_t)m * (m - 1)];
    const double dm1 = D[m - 1], dmm = D[(m - 1) + (size_t)m * (m - 1)];
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n * n; idx += gridDim.x * blockDim.x) {
        const int i = idx % n + 1, j = idx / n + 1;
        double v = D2[i + (size_t)m * j];
        if (b1 == 'n' && b2 == 'n') {
            const double det = d11 * dmm - d1m * dm1;
            v = D2[i] * (d1m * D[(m - 1) + (size_t)m * j] - dmm * D[(size_t)m * j]) / det + v +
                D2[i + (size_t)m * (m - 1)] * (dm1 * D[(size_t)m * j] - d11 * D[(m - 1) + (size_t)m * j]) / det;
        } else if (b1 == 'd' && b2 == 'n') {
            v = v - D2[i + (size_t)m * (m - 1)] * D[(m - 1) + (size_t)m * j] / dmm;
        } else if (b1 == 'n' && b2 == 'd') {
            v = v - D2[i] * D[(size_t)m * j] / d11;
        }
        B[(i - 1) + (size_t)n * (j - 1)] = v;
    }
}

// C = A*B, m x m column-major (src/pseudomat.f90:110, D2 = DC*DC).
__global__ void k_matmul(int m, const double *A, const double *B, double *C)
{
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < m * m;
         idx += gridDim.x * blockDim.x) {
        const int i = idx % m, j = idx / m;
        double s = 0.0;
        for (int k = 0; k < m; ++k) s = fma(A[i + (size_t)m * k], B[k + (size_t)m * j], s);
        C[idx] = s;
    }
}

// Dirichlet interior block D2(2:m-1,2:m-1) (src/pseudomat.f90:232-240) or the
// Neumann-eliminated block (src/pseudomat.f90:116-128).
__global__ void k_block(int m, int neumann, const double *DC, const double *D2,
                        double *B)
{
    const int n = m - 2;
    const double d11 = DC[0], d1m = DC[(size_t)m * (m - 1)];
    const double dm1 = DC[m - 1], dmm = DC[(m - 1) + (size_t)m * (m - 1)];
    const double det = d11 * dmm - d1m * dm1;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n * n;
         idx += gridDim.x * blockDim.x) {
        const int ii = idx % n, jj = idx / n;
        const int i = ii + 1, j = jj + 1;
        double v = D2[i + (size_t)m * j];
        if (neumann) {
            const double ter1 = D2[i] * (d1m * DC[(m - 1) + (size_t)m * j] -
                                         dmm * DC[(size_t)m * j]) / det;
            const double ter3 = D2[i + (size_t)m * (m - 1)] *
                                (dm1 * DC[(size_t)m * j] -
                                 d11 * DC[(m - 1) + (size_t)m * j]) / det;
            v = ter1 + v + ter3;
        }
        B[ii + (size_t)n * jj] = v;
    }
}

__global__ void k_identity(int n, double *I)
{
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n * n;
         idx += gridDim.x * blockDim.x)
        I[idx] = (idx % n == idx / n) ? 1.0 : 0.0;
}

// Real parts of the complex eigenvalues W (interleaved) into E.
__global__ void k_real_part(int n, const double *W, double *E)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        E[i] = W[2 * i];
}

// Pack an n x n column-major matrix A into the A-operand fragment order of
// mma.sync m16n8k16 f64: element (row g + 8*(v&1), col t + 4*(v>>1)) of
// 16x16 tile (mt, ks) goes to lane g*4+t, value v (0..7), stored at
// ((ks*mtiles + mt)*4 + v/2)*64 + lane*2 + v%2 -- the value pair outermost,
// so that a warp's 16-byte loads of one pair are consecutive (no shared
// memory bank conflicts, one 512-byte run from global memory).  Outside
// n x n the packing is zero.
__global__ void k_pack_a(int n, int kpad, int mtiles, const double *A, double *out)
{
    const int total = (kpad / 16) * mtiles * 256;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += gridDim.x * blockDim.x) {
        int row, col;
        pack_slot(idx, mtiles, row, col);
        out[idx] = (row < n && col < n) ? A[row + (size_t)n * col] : 0.0;
    }
}

__global__ void k_copy_col(int n, const double *P, int col, double *out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = P[i + (size_t)n * col];
}

__global__ void k_copy_row(int n, const double *Q, int row, double *out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = Q[row + (size_t)n * i];
}

static int blocks_for(long n) { return (int)((n + 255) / 256 < 1184 ? (n + 255) / 256 : 1184); }

// The same packing of A^T (the adjoint solve applies P^T and P^-T).
__global__ void k_pack_at(int n, int kpad, int mtiles, const double *A, double *out)
{
    const int total = (kpad / 16) * mtiles * 256;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += gridDim.x * blockDim.x) {
        int row, col;
        pack_slot(idx, mtiles, row, col);
        out[idx] = (row < n && col < n) ? A[col + (size_t)n * row] : 0.0;
    }
}

int pack_transposed(ductgpu_ctx ctx, BoundOps &b)
{
    if (b.PTpack && b.QTpack) return DUCTGPU_OK;
    const size_t packed = (size_t)(b.kpad / 16) * b.mtiles * 256;
    if (!b.PTpack) DUCT_CUDA(ctx, cudaMalloc(&b.PTpack, packed * sizeof(double)));
    if (!b.QTpack) DUCT_CUDA(ctx, cudaMalloc(&b.QTpack, packed * sizeof(double)));
    k_pack_at<<<blocks_for((long)packed), 256, 0, ctx->stream>>>(b.n, b.kpad, b.mtiles, b.P, b.PTpack);
    k_pack_at<<<blocks_for((long)packed), 256, 0, ctx->stream>>>(b.n, b.kpad, b.mtiles, b.PM1, b.QTpack);
    ctx->launches += 2;
    return check_cuda(ctx, cudaGetLastError(), "pack_transposed");
}

void free_bound(BoundOps &b)
{
    cudaFree(b.E); cudaFree(b.P); cudaFree(b.PM1);
    cudaFree(b.Ppack); cudaFree(b.Qpack); cudaFree(b.pcol); cudaFree(b.qrow);
    cudaFree(b.D2B); cudaFree(b.Bpack); cudaFree(b.PTpack); cudaFree(b.QTpack);
    cudaFree(b.Pslices); cudaFree(b.Qslices); cudaFree(b.Pexp); cudaFree(b.Qexp);
    cudaFree(b.Pi8); cudaFree(b.Qi8); cudaFree(b.Pexp8); cudaFree(b.Qexp8);
    cudaFree(b.Pfold); cudaFree(b.Qfold); cudaFree(b.PfoldT); cudaFree(b.QfoldT); cudaFree(b.Eperm);
    b = BoundOps();
}

int pack_operators(ductgpu_ctx ctx, BoundOps &b)
{
    const int n = b.n;
    b.kpad = (n + 31) / 32 * 32;
    // 4 warps along M, each owning mtiles/4 tiles of 16 rows.
    const int mt_per_warp = (n + 63) / 64;
    b.mtiles = 4 * mt_per_warp;
    const size_t packed = (size_t)(b.kpad / 16) * b.mtiles * 256;
    cudaFree(b.Ppack);
    cudaFree(b.Qpack);
    cudaFree(b.PTpack);   // the transposed packs follow the operators: rebuilt on next use
    cudaFree(b.QTpack);
    b.Ppack = b.Qpack = b.PTpack = b.QTpack = nullptr;
    DUCT_CUDA(ctx, cudaMalloc(&b.Ppack, packed * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(&b.Qpack, packed * sizeof(double)));
    k_pack_a<<<blocks_for((long)packed), 256, 0, ctx->stream>>>(n, b.kpad, b.mtiles, b.P, b.Ppack);
    k_pack_a<<<blocks_for((long)packed), 256, 0, ctx->stream>>>(n, b.kpad, b.mtiles, b.PM1, b.Qpack);
    ctx->launches += 2;
    if (b.D2B) {
        if (!b.Bpack) DUCT_CUDA(ctx, cudaMalloc(&b.Bpack, packed * sizeof(double)));
        k_pack_a<<<blocks_for((long)packed), 256, 0, ctx->stream>>>(n, b.kpad, b.mtiles, b.D2B, b.Bpack);
        ctx->launches += 1;
    }
    // BF16 slices for the split-precision path (operators up to 128 rows)
    if (n <= 127) {
        int rc = split_operator(ctx, n, b.P, &b.Pslices, &b.Pexp);
        if (rc) return rc;
        if ((rc = split_operator(ctx, n, b.PM1, &b.Qslices, &b.Qexp))) return rc;
        if ((rc = split_operator_i8(ctx, n, b.P, &b.Pi8, &b.Pexp8))) return rc;
        if ((rc = split_operator_i8(ctx, n, b.PM1, &b.Qi8, &b.Qexp8))) return rc;
    }
    if (b.iofzero > 0) {
        if (!b.pcol) DUCT_CUDA(ctx, cudaMalloc(&b.pcol, n * sizeof(double)));
        k_copy_col<<<1, 256, 0, ctx->stream>>>(n, b.P, b.iofzero - 1, b.pcol);
        if (!b.qrow) DUCT_CUDA(ctx, cudaMalloc(&b.qrow, n * sizeof(double)));
        k_copy_row<<<1, 256, 0, ctx->stream>>>(n, b.PM1, b.iofzero - 1, b.qrow);
        ctx->launches += 2;
    }
    return check_cuda(ctx, cudaGetLastError(), "pack_operators");
}

// Packs the two half blocks of a flip-symmetric operator b: Ue (he x he)
// and Uo (ho x ho) are the eigenvectors of the even and odd blocks on the
// first-half points, Ie and Io their inverses acting on the folded input
// (in_k + in_{n-1-k} for the even block, in_k - in_{n-1-k} for the odd one,
// in_mid alone at the middle), Ee and Eo the eigenvalues.
static int store_fold(ductgpu_ctx ctx, BoundOps &b, const std::vector<double> &Ue, const std::vector<double> &Ie,
                      const std::vector<double> &Ee, const std::vector<double> &Uo, const std::vector<double> &Io,
                      const std::vector<double> &Eo)
{
    const int n = b.n, he = (n + 1) / 2, ho = n / 2;
    const int hpad = (he + 31) / 32 * 32;
    // the two half blocks stacked, 2 hpad x hpad, in the fragment order of k_pack_a
    const int mtiles = 2 * hpad / 16;
    const size_t packed = (size_t)(hpad / 16) * mtiles * 256;
    std::vector<double> Pf(packed), Qf(packed), PfT(packed), QfT(packed), Ep(n);
    for (size_t idx = 0; idx < packed; ++idx) {
        int row, col;
        pack_slot((int)idx, mtiles, row, col);
        double pv = 0.0, qv = 0.0, pt = 0.0, qt = 0.0;
        if (row < hpad) {
            if (row < he && col < he) {
                pv = Ue[row + (size_t)he * col];
                qv = Ie[row + (size_t)he * col] * ((col < ho) ? 0.5 : 1.0);
                pt = Ue[col + (size_t)he * row];
                qt = Ie[col + (size_t)he * row] * ((row < ho) ? 0.5 : 1.0);
            }
        } else if (row - hpad < ho && col < ho) {
            const int r = row - hpad;
            pv = Uo[r + (size_t)ho * col];
            qv = Io[r + (size_t)ho * col] * 0.5;
            pt = Uo[col + (size_t)ho * r];
            qt = Io[col + (size_t)ho * r] * 0.5;
        }
        Pf[idx] = pv;
        Qf[idx] = qv;
        PfT[idx] = pt;
        QfT[idx] = qt;
    }
    for (int r = 0; r < he; ++r) Ep[r] = Ee[r];
    for (int r = 0; r < ho; ++r) Ep[he + r] = Eo[r];
    // the pinned (singular) mode: first index of the smallest |E|, the
    // rule of the full operators (src/pseudomat.f90:146-152)
    int sing = -1;
    if (b.iofzero > 0) {
        double emin = 1.0e300;
        for (int r = 0; r < n; ++r)
            if (fabs(Ep[r]) < emin) { emin = fabs(Ep[r]); sing = r; }
    }
    DUCT_CUDA(ctx, cudaMalloc(&b.Pfold, packed * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(&b.Qfold, packed * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(&b.PfoldT, packed * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(&b.QfoldT, packed * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(&b.Eperm, n * sizeof(double)));
    DUCT_CUDA(ctx, cudaMemcpyAsync(b.Pfold, Pf.data(), packed * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    DUCT_CUDA(ctx, cudaMemcpyAsync(b.Qfold, Qf.data(), packed * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    DUCT_CUDA(ctx, cudaMemcpyAsync(b.PfoldT, PfT.data(), packed * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    DUCT_CUDA(ctx, cudaMemcpyAsync(b.QfoldT, QfT.data(), packed * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    DUCT_CUDA(ctx, cudaMemcpyAsync(b.Eperm, Ep.data(), n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    DUCT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    b.he = he;
    b.ho = ho;
    b.hpad = hpad;
    b.sing_perm = sing;
    b.fold_ok = true;
    return DUCTGPU_OK;
}

// Flip symmetry of the wall-normal operators.  With the same condition on
// both walls the interior operator B commutes with the reflection J (point
// k <-> n-1-k, the Gauss-Lobatto nodes being symmetric), so B maps even
// vectors to even ones and odd to odd.  On the first-half values of an even
// vector (points 0..he-1, he = ceil(n/2), the middle point included when n
// is odd) B acts as Be(r,k) = B(r,k) + B(r,n-1-k) (B(r,mid) at the middle),
// on those of an odd vector (0..ho-1, ho = floor(n/2)) as
// Bo(r,k) = B(r,k) - B(r,n-1-k).  Be and Bo are decomposed on their own
// (half-size eigen problems whose eigenvectors are exactly even / odd), and
// with the modes ordered even first every pass becomes block diagonal:
//   P^-1 pass: even coefficients = Ue^-1 u, u_k = (in_k + in_{n-1-k}) / 2
//              (in_mid at the middle); odd = Uo^-1 v, v_k = (in_k - in_{n-1-k}) / 2
//   P pass:    out_o = (Ue c_e)_o + (Uo c_o)_o, out_{n-1-o} = (Ue c_e)_o - (Uo c_o)_o
// -- half the flops of a pass.  The result is the diagonalisation solve
// with another, equally valid, FP64 eigen-decomposition of B (its accuracy
// against the exact discrete solution is the same as the full one's).
// Built only for the library's own operators (ductgpu_pseudomat): operators
// imported with ductgpu_set_operators are applied exactly as given.  B must
// be flip-symmetric to rounding (|B - JBJ| <= 1e-12 max|B|), both blocks'
// spectra real, and n <= 191; otherwise fold_ok stays false and the solve
// uses the full operators.  The (symmetric part of) B is folded on the host.
int fold_operators(ductgpu_ctx ctx, BoundOps &b)
{
    b.fold_ok = false;
    cudaFree(b.Pfold);
    cudaFree(b.Qfold);
    cudaFree(b.PfoldT);
    cudaFree(b.QfoldT);
    cudaFree(b.Eperm);
    b.Pfold = b.Qfold = b.PfoldT = b.QfoldT = b.Eperm = nullptr;
    const int n = b.n, he = (n + 1) / 2, ho = n / 2;
    const int hpad = (he + 31) / 32 * 32;   // 32 rows per M warp of each half block
    if (n < 2 || hpad > 96 || !b.D2B) return DUCTGPU_OK;
    const size_t nn = (size_t)n * n;
    std::vector<double> B(nn);
    DUCT_CUDA(ctx, cudaMemcpyAsync(B.data(), b.D2B, nn * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    DUCT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    auto ba = [&](int r, int c) { return B[r + (size_t)n * c]; };
    double bmax = 0.0, asym = 0.0;
    for (int c = 0; c < n; ++c)
        for (int r = 0; r < n; ++r) {
            bmax = fmax(bmax, fabs(ba(r, c)));
            asym = fmax(asym, fabs(ba(r, c) - ba(n - 1 - r, n - 1 - c)));
        }
    if (!(asym <= 1.0e-12 * bmax)) return DUCTGPU_OK;
    auto bs = [&](int r, int c) { return 0.5 * (ba(r, c) + ba(n - 1 - r, n - 1 - c)); };
    std::vector<double> Be((size_t)he * he), Bo((size_t)ho * ho);
    for (int c = 0; c < he; ++c)
        for (int r = 0; r < he; ++r) Be[r + (size_t)he * c] = (c < ho) ? bs(r, c) + bs(r, n - 1 - c) : bs(r, c);
    for (int c = 0; c < ho; ++c)
        for (int r = 0; r < ho; ++r) Bo[r + (size_t)ho * c] = bs(r, c) - bs(r, n - 1 - c);

    BoundOps be, bo;
    be.n = he;
    bo.n = ho;
    double *dB = nullptr;
    int rc = DUCTGPU_OK;
    std::vector<double> Ue, Ie, Ee, Uo, Io, Eo;
    auto half = [&](BoundOps &h, std::vector<double> &M, std::vector<double> &U, std::vector<double> &I,
                    std::vector<double> &E) {
        const int k = h.n;
        const size_t kk = (size_t)k * k;
        int r = DUCTGPU_OK;
        if ((r = check_cuda(ctx, cudaMalloc(&h.E, k * sizeof(double)), "fold E"))) return r;
        if ((r = check_cuda(ctx, cudaMalloc(&h.P, kk * sizeof(double)), "fold P"))) return r;
        if ((r = check_cuda(ctx, cudaMalloc(&h.PM1, kk * sizeof(double)), "fold PM1"))) return r;
        if ((r = check_cuda(ctx, cudaMemcpyAsync(dB, M.data(), kk * sizeof(double), cudaMemcpyHostToDevice, ctx->stream), "fold B"))) return r;
        if ((r = eigen_gpu(ctx, k, dB, h))) return r;
        U.resize(kk);
        I.resize(kk);
        E.resize(k);
        if ((r = check_cuda(ctx, cudaMemcpyAsync(U.data(), h.P, kk * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream), "fold U"))) return r;
        if ((r = check_cuda(ctx, cudaMemcpyAsync(I.data(), h.PM1, kk * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream), "fold U^-1"))) return r;
        if ((r = check_cuda(ctx, cudaMemcpyAsync(E.data(), h.E, k * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream), "fold E"))) return r;
        return check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "fold sync");
    };
    if (!(rc = check_cuda(ctx, cudaMalloc(&dB, (size_t)he * he * sizeof(double)), "fold B")))
        if (!(rc = half(be, Be, Ue, Ie, Ee))) rc = half(bo, Bo, Uo, Io, Eo);
    cudaFree(dB);
    free_bound(be);
    free_bound(bo);
    if (rc == DUCTGPU_ESOLVER) return DUCTGPU_OK;   // a block with a complex pair: full operators
    if (rc) return rc;

    return store_fold(ctx, b, Ue, Ie, Ee, Uo, Io, Eo);
}

// 4x4 inverse by Gauss-Jordan with partial pivoting (the reference inverts
// AM1 with dgetrf/dgetri, src/pseudomat.f90:177-178).
static bool invert4(double *A)
{
    double a[4][8];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            a[r][c] = A[r + 4 * c];
            a[r][c + 4] = (r == c) ? 1.0 : 0.0;
        }
    for (int c = 0; c < 4; ++c) {
        int p = c;
        for (int r = c + 1; r < 4; ++r)
            if (fabs(a[r][c]) > fabs(a[p][c])) p = r;
        if (a[p][c] == 0.0) return false;
        if (p != c)
            for (int k = 0; k < 8; ++k) { double t = a[p][k]; a[p][k] = a[c][k]; a[c][k] = t; }
        const double inv = 1.0 / a[c][c];
        for (int k = 0; k < 8; ++k) a[c][k] *= inv;
        for (int r = 0; r < 4; ++r)
            if (r != c) {
                const double f = a[r][c];
                for (int k = 0; k < 8; ++k) a[r][k] -= f * a[c][k];
            }
    }
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) A[r + 4 * c] = a[r][c + 4];
    return true;
}

// Eigen-decomposition of the n x n block B (destroyed) into b.E, b.P, b.PM1.
int eigen_gpu(ductgpu_ctx ctx, int n, double *B, BoundOps &b)
{
    cusolverDnHandle_t h = ctx->solver;
    cusolverDnParams_t params = nullptr;
    if (cusolverDnCreateParams(&params) != CUSOLVER_STATUS_SUCCESS)
        return set_error(ctx, DUCTGPU_ESOLVER, "cusolverDnCreateParams failed");
    double *W = nullptr, *dbuf = nullptr;
    int *dinfo = nullptr, *ipiv = nullptr;
    void *hbuf = nullptr;
    size_t dws = 0, hws = 0;
    int rc = DUCTGPU_OK;
    std::vector<double> Wh(2 * (size_t)n);
    int info = 0;
    cusolverStatus_t st;
    if ((rc = check_cuda(ctx, cudaMalloc(&W, 2 * (size_t)n * sizeof(double)), "malloc W"))) goto out;
    if ((rc = check_cuda(ctx, cudaMalloc(&dinfo, sizeof(int)), "malloc info"))) goto out;
    st = cusolverDnXgeev_bufferSize(h, params, CUSOLVER_EIG_MODE_NOVECTOR, CUSOLVER_EIG_MODE_VECTOR,
                                    n, CUDA_R_64F, B, n, CUDA_C_64F, W, CUDA_R_64F, nullptr, 1,
                                    CUDA_R_64F, b.P, n, CUDA_R_64F, &dws, &hws);
    if (st != CUSOLVER_STATUS_SUCCESS) { rc = set_error(ctx, DUCTGPU_ESOLVER, "Xgeev_bufferSize status %d", (int)st); goto out; }
    if ((rc = check_cuda(ctx, cudaMalloc(&dbuf, dws + 16), "malloc geev work"))) goto out;
    hbuf = malloc(hws + 16);
    if (!hbuf) { rc = set_error(ctx, DUCTGPU_EALLOC, "host workspace"); goto out; }
    st = cusolverDnXgeev(h, params, CUSOLVER_EIG_MODE_NOVECTOR, CUSOLVER_EIG_MODE_VECTOR, n,
                         CUDA_R_64F, B, n, CUDA_C_64F, W, CUDA_R_64F, nullptr, 1, CUDA_R_64F,
                         b.P, n, CUDA_R_64F, dbuf, dws, hbuf, hws, dinfo);
    if (st != CUSOLVER_STATUS_SUCCESS) { rc = set_error(ctx, DUCTGPU_ESOLVER, "Xgeev status %d", (int)st); goto out; }
    if ((rc = check_cuda(ctx, cudaMemcpyAsync(&info, dinfo, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream), "info"))) goto out;
    if ((rc = check_cuda(ctx, cudaMemcpyAsync(Wh.data(), W, 2 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream), "W"))) goto out;
    if ((rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "geev sync"))) goto out;
    if (info != 0) { rc = set_error(ctx, DUCTGPU_ESOLVER, "Xgeev info %d", info); goto out; }
    {
        // The Chebyshev D2 blocks have real spectra; a complex pair would mean
        // a packed eigenvector layout this solver does not use.
        double emax = 0.0, imax = 0.0;
        for (int i = 0; i < n; ++i) {
            emax = fmax(emax, fabs(Wh[2 * i]));
            imax = fmax(imax, fabs(Wh[2 * i + 1]));
        }
        if (imax > 1e-6 * emax) { rc = set_error(ctx, DUCTGPU_ESOLVER, "complex eigenvalues (|im| %.3e)", imax); goto out; }
        double emin = emax;
        for (int i = 0; i < n; ++i) emin = fmin(emin, fabs(Wh[2 * i]));
        b.emin = emin;
        b.emax = emax;
    }
    k_real_part<<<blocks_for(n), 256, 0, ctx->stream>>>(n, W, b.E);
    // inverse of P: getrf + getrs(P, I)
    {
        int lwork = 0;
        if (cusolverDnDgetrf_bufferSize(h, n, n, B, n, &lwork) != CUSOLVER_STATUS_SUCCESS) {
            rc = set_error(ctx, DUCTGPU_ESOLVER, "getrf_bufferSize"); goto out;
        }
        cudaFree(dbuf); dbuf = nullptr;
        if ((rc = check_cuda(ctx, cudaMalloc(&dbuf, ((size_t)lwork + 16) * sizeof(double)), "getrf work"))) goto out;
        if ((rc = check_cuda(ctx, cudaMalloc(&ipiv, (size_t)n * sizeof(int)), "ipiv"))) goto out;
        if ((rc = check_cuda(ctx, cudaMemcpyAsync(B, b.P, (size_t)n * n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream), "copy P"))) goto out;
        k_identity<<<blocks_for((long)n * n), 256, 0, ctx->stream>>>(n, b.PM1);
        ctx->launches += 2;
        if (cusolverDnDgetrf(h, n, n, B, n, dbuf, ipiv, dinfo) != CUSOLVER_STATUS_SUCCESS) {
            rc = set_error(ctx, DUCTGPU_ESOLVER, "getrf"); goto out;
        }
        if (cusolverDnDgetrs(h, CUBLAS_OP_N, n, n, B, n, ipiv, b.PM1, n, dinfo) != CUSOLVER_STATUS_SUCCESS) {
            rc = set_error(ctx, DUCTGPU_ESOLVER, "getrs"); goto out;
        }
        if ((rc = check_cuda(ctx, cudaMemcpyAsync(&info, dinfo, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream), "info"))) goto out;
        if ((rc = check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "getrs sync"))) goto out;
        if (info != 0) { rc = set_error(ctx, DUCTGPU_ESOLVER, "getrf/getrs info %d", info); goto out; }
    }
    // iofzero: first index of the smallest |E| (src/pseudomat.f90:146-152)
    {
        double eigmin = 1.0e6;
        b.iofzero = 0;
        for (int i = 0; i < n; ++i) {
            const double e = fmin(eigmin, fabs(Wh[2 * i]));
            if (e != eigmin) { b.iofzero = i + 1; eigmin = e; }
        }
    }
out:
    cudaFree(W); cudaFree(dbuf); cudaFree(dinfo); cudaFree(ipiv);
    free(hbuf);
    cusolverDnDestroyParams(params);
    return rc;
}

void free_rect(RectSlot &r)
{
    free_bound(r.y);
    free_bound(r.z);
    cudaFree(r.DY); cudaFree(r.D2Y); cudaFree(r.DZ); cudaFree(r.D2Z); cudaFree(r.wy); cudaFree(r.wz);
    r = RectSlot();
}

static void cc_weights(int m, double scale, std::vector<double> &w)
{
    w.assign(m, 0.0);
    const int N = m - 1;
    const double pi = 3.14159265358979323846;
    for (int j = 0; j <= N; ++j) {
        double s = 0.0;
        for (int k = 1; k <= N / 2; ++k) {
            const double bk = (2 * k == N) ? 1.0 : 2.0;
            s += bk * cos(2.0 * pi * (double)k * (double)j / (double)N) / (4.0 * k * k - 1.0);
        }
        const double cj = (j == 0 || j == N) ? 1.0 : 2.0;
        w[j] = scale * cj / (double)N * (1.0 - s);
    }
}

// One direction of pseudomaty_temp / pseudomatz_temp on the GPU.
static int rect_direction(ductgpu_ctx ctx, int m, double s, char b1, char b2, BoundOps &b, double **D,
                          double **D2, double **w)
{
    const int n = m - 2;
    double *x = nullptr, *blk = nullptr;
    DUCT_CUDA(ctx, cudaMalloc(D, (size_t)m * m * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(D2, (size_t)m * m * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(&x, m * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(&blk, (size_t)n * n * sizeof(double)));
    b.n = n;
    DUCT_CUDA(ctx, cudaMalloc(&b.D2B, (size_t)n * n * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(&b.E, n * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(&b.P, (size_t)n * n * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(&b.PM1, (size_t)n * n * sizeof(double)));
    k_build_dc<<<blocks_for((long)m * m), 256, 0, ctx->stream>>>(m, x, *D, 1.0 / s);
    k_matmul<<<blocks_for((long)m * m), 256, 0, ctx->stream>>>(m, *D, *D, *D2);
    k_block_bc<<<blocks_for((long)n * n), 256, 0, ctx->stream>>>(m, b1, b2, *D, *D2, blk);
    ctx->launches += 3;
    DUCT_CUDA(ctx, cudaMemcpyAsync(b.D2B, blk, (size_t)n * n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    int rc = eigen_gpu(ctx, n, blk, b);
    cudaFree(blk);
    cudaFree(x);
    if (rc) return rc;
    b.iofzero = 0;
    if ((rc = pack_operators(ctx, b))) return rc;
    std::vector<double> wh;
    cc_weights(m, s, wh);
    DUCT_CUDA(ctx, cudaMalloc(w, m * sizeof(double)));
    DUCT_CUDA(ctx, cudaMemcpyAsync(*w, wh.data(), m * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    return DUCTGPU_OK;
}

int rect_setup(ductgpu_ctx ctx, int slot, int my, int mz, double sy, double sz, char by1, char by2,
               char bz1, char bz2)
{
    if (slot < 0 || slot >= kMaxRect) return set_error(ctx, DUCTGPU_EARG, "rectangular slot %d (0..%d)", slot, kMaxRect - 1);
    if (my < 5 || mz < 5 || my - 2 > kMaxN || mz - 2 > kMaxN)
        return set_error(ctx, DUCTGPU_EARG, "pseudomat_temp: my=%d mz=%d outside [5,%d]", my, mz, kMaxN + 2);
    for (char c : {by1, by2, bz1, bz2})
        if (c != 'd' && c != 'n') return set_error(ctx, DUCTGPU_EARG, "wall condition '%c' is neither 'd' nor 'n'", c);
    if (!(sy > 0.0) || !(sz > 0.0)) return set_error(ctx, DUCTGPU_EARG, "half-widths must be positive");
    RectSlot &r = ctx->rect[slot];
    cudaStreamSynchronize(ctx->stream);
    free_rect(r);
    r.my = my; r.mz = mz; r.sy = sy; r.sz = sz;
    r.by1 = by1; r.by2 = by2; r.bz1 = bz1; r.bz2 = bz2;
    int rc = rect_direction(ctx, my, sy, by1, by2, r.y, &r.DY, &r.D2Y, &r.wy);
    if (!rc) rc = rect_direction(ctx, mz, sz, bz1, bz2, r.z, &r.DZ, &r.D2Z, &r.wz);
    if (rc) { free_rect(r); return rc; }
    // singular pair of the all-Neumann operator: smallest |E| per direction
    std::vector<double> ey(r.y.n), ez(r.z.n);
    DUCT_CUDA(ctx, cudaMemcpyAsync(ey.data(), r.y.E, r.y.n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    DUCT_CUDA(ctx, cudaMemcpyAsync(ez.data(), r.z.E, r.z.n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    DUCT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    r.sing_y = 0;
    for (int i = 1; i < r.y.n; ++i) if (fabs(ey[i]) < fabs(ey[r.sing_y])) r.sing_y = i;
    r.sing_z = 0;
    for (int i = 1; i < r.z.n; ++i) if (fabs(ez[i]) < fabs(ez[r.sing_z])) r.sing_z = i;
    // flip-symmetric half blocks of a direction whose two walls match (the
    // operator then commutes with the reflection of the nodes; fold_operators
    // checks it), and the singular mode's place in their even-first order
    auto fold_dir = [&](BoundOps &b, char w1, char w2, int &sing) -> int {
        sing = -1;
        if (w1 != w2) return DUCTGPU_OK;
        int rc2 = fold_operators(ctx, b);
        if (rc2 || !b.fold_ok) return rc2;
        std::vector<double> ep(b.n);
        DUCT_CUDA(ctx, cudaMemcpy(ep.data(), b.Eperm, b.n * sizeof(double), cudaMemcpyDeviceToHost));
        sing = 0;
        for (int i = 1; i < b.n; ++i) if (fabs(ep[i]) < fabs(ep[sing])) sing = i;
        return DUCTGPU_OK;
    };
    if ((rc = fold_dir(r.y, by1, by2, r.sing_yp)) || (rc = fold_dir(r.z, bz1, bz2, r.sing_zp))) {
        free_rect(r);
        return rc;
    }
    r.ready = true;
    return DUCTGPU_OK;
}

int pseudomat_gpu(ductgpu_ctx ctx, int m, bool eigen)
{
    if (m < 5 || m - 2 > kMaxN)
        return set_error(ctx, DUCTGPU_EARG, "pseudomat: my=%d outside [5,%d]", m, kMaxN + 2);
    const int n = m - 2;
    cudaFree(ctx->xcol); cudaFree(ctx->DC); cudaFree(ctx->D2); cudaFree(ctx->AM1); cudaFree(ctx->ccw);
    cudaFree(ctx->dcr);
    ctx->xcol = ctx->DC = ctx->D2 = ctx->AM1 = ctx->ccw = ctx->dcr = nullptr;
    free_bound(ctx->dir);
    free_bound(ctx->neu);
    ctx->ready = false;
    ctx->grid_ready = false;
    ctx->ops_set = 0;
    ctx->pin_point = 0;
    DUCT_CUDA(ctx, cudaMalloc(&ctx->xcol, m * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(&ctx->DC, (size_t)m * m * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(&ctx->D2, (size_t)m * m * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(&ctx->AM1, 16 * sizeof(double)));
    DUCT_CUDA(ctx, cudaMalloc(&ctx->ccw, m * sizeof(double)));
    for (BoundOps *b : {&ctx->dir, &ctx->neu}) {
        b->n = n;
        DUCT_CUDA(ctx, cudaMalloc(&b->D2B, (size_t)n * n * sizeof(double)));
        DUCT_CUDA(ctx, cudaMalloc(&b->E, n * sizeof(double)));
        DUCT_CUDA(ctx, cudaMalloc(&b->P, (size_t)n * n * sizeof(double)));
        DUCT_CUDA(ctx, cudaMalloc(&b->PM1, (size_t)n * n * sizeof(double)));
    }
    double *blk = nullptr;
    DUCT_CUDA(ctx, cudaMalloc(&blk, (size_t)n * n * sizeof(double)));
    k_build_dc<<<blocks_for((long)m * m), 256, 0, ctx->stream>>>(m, ctx->xcol, ctx->DC);
    DUCT_CUDA(ctx, cudaMalloc(&ctx->dcr, 2 * (size_t)m * sizeof(double)));
    k_copy_row<<<1, 256, 0, ctx->stream>>>(m, ctx->DC, 0, ctx->dcr);
    k_copy_row<<<1, 256, 0, ctx->stream>>>(m, ctx->DC, m - 1, ctx->dcr + m);
    if (!ctx->pin_cc) DUCT_CUDA(ctx, cudaMalloc(&ctx->pin_cc, 2 * 64 * sizeof(double)));
    ctx->launches += 2;
    k_matmul<<<blocks_for((long)m * m), 256, 0, ctx->stream>>>(m, ctx->DC, ctx->DC, ctx->D2);
    k_block<<<blocks_for((long)n * n), 256, 0, ctx->stream>>>(m, 0, ctx->DC, ctx->D2, blk);
    ctx->launches += 3;
    DUCT_CUDA(ctx, cudaMemcpyAsync(ctx->dir.D2B, blk, (size_t)n * n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    int rc = eigen ? eigen_gpu(ctx, n, blk, ctx->dir) : DUCTGPU_OK;
    if (rc == DUCTGPU_OK) {
        k_block<<<blocks_for((long)n * n), 256, 0, ctx->stream>>>(m, 1, ctx->DC, ctx->D2, blk);
        ctx->launches += 1;
        DUCT_CUDA(ctx, cudaMemcpyAsync(ctx->neu.D2B, blk, (size_t)n * n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
        if (eigen) rc = eigen_gpu(ctx, n, blk, ctx->neu);
    }
    cudaFree(blk);
    if (rc) return rc;
    ctx->dir.iofzero = 0;  // only the Neumann operator pins a point
    // AM1 (src/pseudomat.f90:158-178) from the four corner entries of DC.
    double c4[4];
    DUCT_CUDA(ctx, cudaMemcpyAsync(&c4[0], ctx->DC, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    DUCT_CUDA(ctx, cudaMemcpyAsync(&c4[1], ctx->DC + (size_t)m * (m - 1), sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    DUCT_CUDA(ctx, cudaMemcpyAsync(&c4[2], ctx->DC + (m - 1), sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    DUCT_CUDA(ctx, cudaMemcpyAsync(&c4[3], ctx->DC + (m - 1) + (size_t)m * (m - 1), sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    DUCT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    const double d11 = c4[0], d1m = c4[1], dm1 = c4[2], dmm = c4[3];
    double A[16] = {2.0 * d11, -dm1, 0.0, -dm1,
                    d1m, d11 - dmm, dm1, 0.0,
                    0.0, d1m, 2.0 * dmm, d1m,
                    d1m, 0.0, dm1, d11 - dmm};
    if (!invert4(A)) return set_error(ctx, DUCTGPU_ESOLVER, "AM1 singular");
    // Clenshaw-Curtis weights of the CGL nodes (for the zero-mean gauge):
    // w_j = c_j/N (1 - sum_{k=1}^{N/2} b_k cos(2 pi k j/N)/(4k^2-1)).
    std::vector<double> w(m);
    {
        const int N = m - 1;
        const double pi = 3.14159265358979323846;
        for (int j = 0; j <= N; ++j) {
            double s = 0.0;
            for (int k = 1; k <= N / 2; ++k) {
                const double bk = (2 * k == N) ? 1.0 : 2.0;
                s += bk * cos(2.0 * pi * (double)k * (double)j / (double)N) / (4.0 * k * k - 1.0);
            }
            const double cj = (j == 0 || j == N) ? 1.0 : 2.0;
            w[j] = cj / (double)N * (1.0 - s);
        }
    }
    DUCT_CUDA(ctx, cudaMemcpyAsync(ctx->AM1, A, 16 * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    DUCT_CUDA(ctx, cudaMemcpyAsync(ctx->ccw, w.data(), m * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    ctx->my = ctx->mz = m;
    ctx->grid_ready = true;
    if (!eigen) {
        // the eigen-decompositions come from ductgpu_set_operators
        DUCT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        return DUCTGPU_OK;
    }
    if ((rc = pack_operators(ctx, ctx->dir))) return rc;
    if ((rc = pack_operators(ctx, ctx->neu))) return rc;
    if ((rc = fold_operators(ctx, ctx->dir))) return rc;
    if ((rc = fold_operators(ctx, ctx->neu))) return rc;
    DUCT_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->ops_set = 3;
    ctx->ready = true;
    return DUCTGPU_OK;
}

}  // namespace duct
