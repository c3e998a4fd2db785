// internal.h -- context and shared declarations of libductgpu (not part of
// the C-ABI).  The context replaces the reference's module globals of the
// solver (fulldiagdir, fulldiagneu, chebystuff, gpudevice; src/mod.f90:
// 277-343, 409-483) with device-resident state owned by one handle.
#pragma once

#include <cuda_runtime.h>
#include <cusolverDn.h>
#include <stdarg.h>
#include <stdio.h>

#include <cstdint>
#include <vector>

#include "../../include/ductgpu.h"

namespace duct {

constexpr int kMaxFields = 16;  // fields per batched launch (4 ducts x u, v, w, p)
constexpr int kMaxN = 191;      // largest interior size (my-2) supported
constexpr int kNumEvents = 16;
constexpr int kMaxRect = 8;     // rectangular operator slots (duct shapes)

// Interior operators of one boundary condition ('d' or 'n').
// default GEMM-pass kernel per operator size class (n <= 63, <= 127, <= 191)
constexpr int kPassDefault[3] = {DUCTGPU_PASS_PARITY, DUCTGPU_PASS_PARITY, DUCTGPU_PASS_PARITY};

struct BoundOps {
    int n = 0;                 // interior points, my-2
    int kpad = 0;              // n rounded up to the K chunk (32)
    int mtiles = 0;            // 16-row tiles of the padded M extent
    double *E = nullptr;       // [n] eigenvalues
    double *P = nullptr;       // [n*n] eigenvectors, column-major
    double *PM1 = nullptr;     // [n*n] inverse
    double *Ppack = nullptr;   // P in DMMA A-fragment order, zero padded
    double *Qpack = nullptr;   // PM1 in DMMA A-fragment order
    double *pcol = nullptr;    // [n] column iofzero of P (Neumann pin)
    double *qrow = nullptr;    // [n] row iofzero of P^-1 (null-space projection)
    int iofzero = 0;           // 1-based, Neumann only
    double emin = 0.0, emax = 0.0;   // smallest / largest |eigenvalue| (host)
    double *D2B = nullptr;     // [n*n] the interior operator block itself
    double *Bpack = nullptr;   // D2B in DMMA A-fragment order (residual)
    double *PTpack = nullptr, *QTpack = nullptr;  // P^T, P^-T packed (adjoint; built on first use)
    uint8_t *Pslices = nullptr, *Qslices = nullptr;  // BF16 slices (mixed)
    int *Pexp = nullptr, *Qexp = nullptr;            // per-row exponents
    int8_t *Pi8 = nullptr, *Qi8 = nullptr;          // int8 slices (int8-emulated FP64)
    int *Pexp8 = nullptr, *Qexp8 = nullptr;
    // flip-symmetric form (setup.cu fold_operators): modes reordered even
    // first (he of them) then odd (ho); Qfold / Pfold are the two half
    // blocks stacked (2 hpad rows x hpad columns) in DMMA A-fragment order
    bool fold_ok = false;
    int he = 0, ho = 0, hpad = 0;
    int sing_perm = -1;        // position of iofzero - 1 in the reordered modes
    double *Pfold = nullptr, *Qfold = nullptr;
    double *PfoldT = nullptr, *QfoldT = nullptr;   // the blocks transposed (adjoint)
    double *Eperm = nullptr;   // [n] eigenvalues in the reordered mode order
};

// Operators of one rectangular duct shape (src/pseudomat_temp.f90): y and z
// directions with their own points, half-widths and wall conditions.
struct RectSlot {
    bool ready = false;
    int my = 0, mz = 0;
    double sy = 1.0, sz = 1.0;
    char by1 = 'd', by2 = 'd', bz1 = 'd', bz2 = 'd';
    BoundOps y, z;
    double *DY = nullptr, *D2Y = nullptr, *DZ = nullptr, *D2Z = nullptr;  // device
    double *wy = nullptr, *wz = nullptr;   // Clenshaw-Curtis weights (scaled)
    int sing_y = -1, sing_z = -1;          // argmin |E| per direction
    int sing_yp = -1, sing_zp = -1;        // the same in the flip-symmetric (even-first) mode order
};

// Shen-Legendre operators of one wall condition (src/preshen.f90)
struct ShenOps {
    bool ready = false;
    int m = 0;
    char bound = 'd';
    BoundOps leg;        // P = A (Chebyshev -> Legendre), PM1 = B = A^-1, n = m
    BoundOps eig;        // P = eigenvectors, PM1 = P^-1 S^-1, E = rho, n = m-2
    double *Md = nullptr, *Mo = nullptr, *Sm = nullptr;   // mass diag, mass (k,k+2), makeMS stiffness
    double *bk = nullptr;   // b_k
};

struct Workspace {
    double *buf = nullptr;
    size_t bytes = 0;
};

}  // namespace duct

namespace duct { struct DnsAux; }

struct ductgpu_ctx_s {
    int device = 0;
    int num_sms = 148;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    cusolverDnHandle_t solver = nullptr;
    char err[512] = {0};

    int my = 0, mz = 0;
    bool ready = false;        // grid and both eigen-decompositions set up
    bool grid_ready = false;   // grid, D, D2, blocks, AM1 (ductgpu_pseudomat[_ex])
    int ops_set = 0;           // eigen-decompositions present: 1 Dirichlet, 2 Neumann
    int pin_point = 0;         // kx=0 Neumann gauge point (1-based interior index; 0: iofzero)
    double *xcol = nullptr;    // [my]
    double *DC = nullptr;      // [my*my]
    double *dcr = nullptr;     // [2*my] rows 1 and my of DC, contiguous (Neumann walls)
    double *pin_cc = nullptr;  // [2*64] point-gauge coefficients of singular planes
    double *D2 = nullptr;      // [my*my]
    double *AM1 = nullptr;     // [16] device copy
    double *ccw = nullptr;     // [my] Clenshaw-Curtis weights on the nodes
    double wanted = 0.0;
    int gauge = DUCTGPU_GAUGE_POINT;
    int refine_steps = 2;      // FP64 refinement steps of the split-precision path
    int parity_ws = 1;         // flip-symmetric passes at hpad 32 / 64: warp-specialised persistent kernel
    int i8_kernel = 1;         // int8-emulated passes: 0 sequential, 1 warp-specialised pipeline
    int rect_fold = 1;         // rectangular solves on the flip-symmetric half blocks where both walls match
    // GEMM-pass kernel per operator size class (n <= 63, <= 127, <= 191),
    // one of DUCTGPU_PASS_* (ductgpu_set_pass_kernel, ductgpu_autotune);
    // defaults (kPassDefault) from measurements on B200 at n = 31, 63, 127,
    // 191; ductgpu_autotune re-picks them by timing
    int pass_variant[3] = {duct::kPassDefault[0], duct::kPassDefault[1], duct::kPassDefault[2]};
    duct::BoundOps dir, neu;

    duct::RectSlot rect[duct::kMaxRect];
    duct::ShenOps shen_d, shen_n;
    // Galerkin-basis Neumann operators (pseudopois): EN, PN, PNM1 and the
    // wall vectors r_-, r_+ = B^-T phi(-+1) [2 (my-2)]
    duct::BoundOps pois;
    double *pois_r = nullptr;
    int pois_m = 0;
    // constant mass-flow-rate forcing (precomp_mass_flow): premassfu
    // (my,my,mf_mrk) real, premassf[mf_mrk], the last measured flow rate
    double *mf_u = nullptr, *mf_f = nullptr, *mf_sum = nullptr;
    int mf_mrk = 0, mf_my = 0;
    double mf_aspect = 1.0;
    // captured solves (CUDA graphs), each with its own lambda array
    static constexpr int kMaxGraphs = 16;
    cudaGraphExec_t graph_exec[kMaxGraphs] = {};
    double *graph_lam[kMaxGraphs] = {};
    bool capturing = false;
    duct::Workspace work;      // pass intermediates
    duct::Workspace io;        // device copies for host entries
    // copy streams and events of the pipelined host helm3d
    static constexpr int kPipeChunks = 8;
    cudaStream_t cp_in = nullptr, cp_out = nullptr;
    cudaEvent_t ev_in[kPipeChunks] = {}, ev_out[kPipeChunks] = {};
    // W_L twiddle tables of the register-FFT transforms, one per length
    static constexpr int kTwTables = 24;
    int tw_len[kTwTables] = {};
    void *tw_tab[kTwTables] = {};
    int *dev_err = nullptr;    // device error word (bounded waits)
    int tma_tr_per_sm = 0;     // resident TMA-transpose CTAs per SM (0: not asked yet, -1: none)
    // the last tensor maps of the TMA transpose (a map describes an address
    // and sizes, not a context), encoded once: calls take ~16 us on a
    // config-4 field, so per-call host work shows
    struct TmaMap {
        const void *in = nullptr;
        long long A = 0, Q = 0;
        alignas(64) unsigned char map[128];
    };
    static constexpr int kTmaMaps = 8;
    TmaMap tma_maps[kTmaMaps];
    int tma_next = 0;
    int *pq_ctr = nullptr;     // counters of the queued flip-symmetric passes
    size_t pq_cap = 0;
    // side streams of a rectangular batch's independent field groups
    static constexpr int kSideStreams = 4;
    cudaStream_t side[kSideStreams] = {};
    cudaEvent_t side_fork = nullptr, side_join[kSideStreams] = {};
    duct::DnsAux *dns_aux = nullptr;   // buffers of the DNS operator entries (dns.cu)
    // derivative lines on the FP64 tensor cores (dlines.cu): the folded,
    // packed collocation matrices per line length
    static constexpr int kDlineSlots = 12;
    int dl_nn[kDlineSlots] = {};
    double *dl_ops[kDlineSlots] = {};
    int dlines = 1;            // 1: derivative lines by DMMA where supported, 0: the FFT kernel
    double *lam = nullptr;     // per-plane lambda (device)
    double *lam_host = nullptr;// pinned staging
    int lam_cap = 0;

    cudaEvent_t ev[duct::kNumEvents] = {};
    long long launches = 0;

    // per-kernel profiling (events around launches)
    bool prof_on = false;
    static constexpr int kProfSlots = 4096;
    cudaEvent_t prof_ev[2 * kProfSlots] = {};
    int prof_kind[kProfSlots] = {};
    int prof_used = 0;
    double prof_ms[DUCTGPU_K_COUNT] = {};
    long long prof_n[DUCTGPU_K_COUNT] = {};
    double prof_bytes[DUCTGPU_K_COUNT] = {};   // algorithmic bytes of the launches (kernels that count them)
    double prof_flops[DUCTGPU_K_COUNT] = {};   // executed tensor-core flops (kernels that count them)
};

namespace duct {

int set_error(ductgpu_ctx ctx, int code, const char *fmt, ...);
// 0-based interior index of the kx=0 Neumann gauge point: the caller's
// (ductgpu_set_gauge_point), else the position of the smallest |eigenvalue|
// in the operator's own order (the reference's iofzero rule)
inline int pin_index(ductgpu_ctx c) { return (c->pin_point > 0 ? c->pin_point : c->neu.iofzero) - 1; }
int check_cuda(ductgpu_ctx ctx, cudaError_t e, const char *what);
int ensure(ductgpu_ctx ctx, Workspace &w, size_t bytes);
// noalloc.cu: looks up the fixed scratch of the no-allocation entry point
// on the context's GPU (at context creation)
void noalloc_reserve(ductgpu_ctx ctx);
// h5io.cu: the metadata of a uvwp_NNNN.h5 file (everything before the four
// fields' data), the fields' file offsets and the end-of-file address
struct H5Layout {
    std::vector<uint8_t> meta;
    uint64_t field_off[4] = {}, field_bytes = 0, eof = 0;
};
void h5_layout(const ductgpu_h5_header *hdr, H5Layout &L);
// h5io.cu: a statistics_NNNN.h5 file from host copies of the accumulators
struct H5Stats {
    int mgalx = 0, my = 0, mz = 0, nmodes = 0, nstat = 0;
    double timef = 0.0, time = 0.0, fnu = 0.0, alp = 0.0, aspect = 1.0;
    const double *mean = nullptr, *prod = nullptr, *ppb = nullptr, *spec = nullptr, *om2 = nullptr;
};
int h5_write_statistics(ductgpu_ctx ctx, const char *filename, const H5Stats &st);

// Brackets one kernel launch with profiling events when enabled and
// counts it.  Use: { LaunchScope ls(ctx, DUCTGPU_K_...); kernel<<<>>>(); }
struct LaunchScope {
    ductgpu_ctx c;
    int slot = -1;
    LaunchScope(ductgpu_ctx ctx, int kind);
    ~LaunchScope();
};
void profile_drain(ductgpu_ctx ctx);

// setup.cu
// eigen false: grid, D, D2, interior blocks and AM1 only; the
// eigen-decompositions are then imported with ductgpu_set_operators
int pseudomat_gpu(ductgpu_ctx ctx, int m, bool eigen = true);
int pack_operators(ductgpu_ctx ctx, BoundOps &b);
// flip-symmetric half operators of b (fold_ok false when b lacks the symmetry)
int fold_operators(ductgpu_ctx ctx, BoundOps &b);
int pack_transposed(ductgpu_ctx ctx, BoundOps &b);
// Real eigen-decomposition of the n x n device matrix B (destroyed) into
// b.E, b.P, b.PM1 (allocated by the caller), with emin/emax and iofzero.
int eigen_gpu(ductgpu_ctx ctx, int n, double *B, BoundOps &b);
// Ainv = A^-1 for an n x n device matrix (getrf/getrs; synchronises).
int invert_dev(ductgpu_ctx ctx, int n, const double *A, double *Ainv);
void free_bound(BoundOps &b);

// solve_fp64.cu
struct FieldTask {
    double *rhs;
    double *sol;
    int nmodes;
    int mode0;        // 1: first plane is Fourier mode 0
    char bound;
    int plane0;       // index of the first plane in ctx->lam
    int refine;       // FP64 refinement steps for the split-precision path
};
int solve_fp64(ductgpu_ctx ctx, const FieldTask *tasks, int ntasks);
// emulate: every GEMM pass as int8 slice products on tcgen05 (solve_i8.cu)
int solve_fp64_ex(ductgpu_ctx ctx, const FieldTask *tasks, int ntasks, bool emulate);
// adjoint.cu: the transpose of solve_fp64's map rhs -> sol; task.rhs is the
// cotangent of sol (read only), task.sol receives the cotangent of rhs
int solve_adjoint(ductgpu_ctx ctx, const FieldTask *tasks, int ntasks);

// One batched FP64 GEMM pass (k_pass_fp64), usable by other solvers.
struct PassField {
    const double *src;
    double *dst;
    const double *A;     // packed operator (n x n, fragment order)
    const int8_t *Ai8;   // int8 operator slices (int8-emulated passes), or null
    const int *Aexp;     // per-row exponents of Ai8
    const double *E;     // eigenvalues along the pass direction (divide)
    const double *El;    // eigenvalues along the line direction (divide)
    int nmodes;
    int mode0;
    int plane0;
    int sing_io;         // 0-based singular index along the pass, else -1
    int sing_l;          // 0-based singular index along the lines
    // geometry of this field's planes for this pass
    int n;               // operator size (interior points along the pass)
    int nlines;          // interior lines (points along the other direction)
    int nchunks;         // ceil(nlines / kPassLines)
    int kpad, mtiles;    // padded K and 16-row tiles of the packed operator
    int sk, sl;          // complex strides of (k, line)
    int off;             // first point/line: 1 (interior) or 0 (full plane)
    long long plane_stride;  // doubles per complex plane
    // residual epilogue: dst = resF - resT - acc + lam * resU
    const double *resF, *resT, *resU;
    // flip-symmetric pass (k_pass_fp64s): 1 folds a physical input into
    // even / odd halves, 2 unfolds the two halves into a physical output;
    // kpad is then the half extent hpad and the mode order is even first
    int par;
    int he, ho;
};
struct PassParams {
    PassField f[kMaxFields];
    int cta_start[kMaxFields + 1];
    int nf;
    const double *lam;
    int divide;
    int zero_im_mode0;
    int residual;
};
constexpr int kPassLines = 32;
int fp64_pass(ductgpu_ctx ctx, const PassParams &pp, int grid);
// the four flip-symmetric passes of a batched solve in one persistent launch
int fp64_pass_queue(ductgpu_ctx ctx, const PassParams *pp);
// solve_fp64ws.cu: the flip-symmetric pass as a warp-specialised persistent
// kernel (hpad 32 or 64, every field folded, no residual epilogue)
cudaError_t fp64_pass_ws(ductgpu_ctx ctx, const PassParams &pp, int hpad);
// one CTA whose bounded wait runs out after `polls` polls (failure-path self-test)
cudaError_t wait_selftest(ductgpu_ctx ctx, unsigned polls);
// Whether a solve (or its adjoint) over these fields runs the flip-symmetric
// passes: DUCTGPU_PASS_PARITY selected for the size class and every field's
// operators have the folded form.  The forward and adjoint take the same
// decision, so the adjoint is the transpose of the map the forward applies.
bool use_fold(ductgpu_ctx ctx, const FieldTask *tasks, int ntasks);
// Turns a pass field into a flip-symmetric one: par 1 folds the input,
// par 2 unfolds the output, A is the matching folded pack of b.
void fold_field(PassField &f, const BoundOps &b, int par, const double *A, bool neumann);
// Sets the geometry of one field of a pass: operator b along a direction
// with stride sk (complex elements), nlines lines of stride sl.
void pass_geometry(PassField &f, const BoundOps &b, const double *El, int nlines, int sk, int sl,
                   long long plane_stride);

// setup.cu (rectangular)
int rect_setup(ductgpu_ctx ctx, int slot, int my, int mz, double sy, double sz, char by1, char by2,
               char bz1, char bz2);
void free_rect(RectSlot &r);

// shen.cu
void free_shen(ShenOps &s);
int shen_setup(ductgpu_ctx ctx, int m, char bound);
struct ShenTask {
    double *rhs, *sol;
    int nmodes, mode0, plane0;
    char bound;
};
int solve_shen(ductgpu_ctx ctx, const ShenTask *tasks, int ntasks);

// pois.cu
int pois_setup(ductgpu_ctx ctx, int m);
int solve_pois(ductgpu_ctx ctx, const FieldTask *tasks, int ntasks);

// solve_rect.cu
struct RectTask {
    double *rhs, *sol;
    const double *bcy, *bcz;   // device wall values (mz,2,nmodes), (my,2,nmodes) or null
    int nmodes, mode0, plane0, slot;
};
int solve_rect(ductgpu_ctx ctx, const RectTask *tasks, int ntasks);

// solve_mixed.cu
int split_operator(ductgpu_ctx ctx, int n, const double *A, uint8_t **slices, int **rexp);
// solve_i8.cu
int split_operator_i8(ductgpu_ctx ctx, int n, const double *A, int8_t **slices, int **rexp);
int i8_pass(ductgpu_ctx ctx, const PassParams &pp, int grid);
int solve_mixed(ductgpu_ctx ctx, const FieldTask *tasks, int ntasks);
int zero_walls(ductgpu_ctx ctx, const FieldTask *tasks, int ntasks);
int neumann_fill(ductgpu_ctx ctx, const FieldTask *tasks, int ntasks);

// transforms.cu
int transyz_dev(ductgpu_ctx ctx, double *f, int my, int mz, int nmodes, char cdir, int iopt);
int derivyz_dev(ductgpu_ctx ctx, const double *u, double *du, int my, int mz, int nmodes, char cdir,
                int ider, double scal, char what, double aspect);
int transpose_dev(ductgpu_ctx ctx, const double *in, double *out, long long A, long long Q);
// transpose_tma.cu: the same by TMA tile loads; -1 when not applicable
int transpose_tma(ductgpu_ctx ctx, const double *in, double *out, long long A, long long Q);

// cheb_lines.cu: fused Chebyshev derivative lines with a pointwise epilogue
// (see the file's header).  One output:
//   out = sigma * (beta * out + fac * D^order(in) + sum_t (xc0_t + xc1_t i kx
//                  + xc2_t (i kx)^2) xs_t + [mode 0] m0)
// with D the reference's derivyz between transyz -1 / +1 along the launch's
// direction (fac already divided by aspect^order for z).  maxabs (device,
// or null): atomic max of |out| over the interior points.  No output of a
// launch may write, or read (as an x-term), the field that another output
// of the launch writes: the kernels order an element's loads only before
// its own store (lines_launch checks).
constexpr int kLineXTerms = 5;
constexpr int kMaxLineOut = 3;
constexpr int kMaxLineJobs = 4;
struct LineOut {
    double *out = nullptr;
    const double *xs[kLineXTerms] = {};
    double xc0[kLineXTerms] = {}, xc1[kLineXTerms] = {}, xc2[kLineXTerms] = {};
    double fac = 1.0, beta = 0.0, sigma = 1.0, m0 = 0.0;
    double *maxabs = nullptr;
    int order = 0;
};
struct LineJob {
    const double *in = nullptr;
    int nout = 0;
    LineOut o[kMaxLineOut];
};
struct LineParams {
    LineJob job[kMaxLineJobs];
    int njobs = 0;
    int my = 0, mz = 0, nmodes = 0;
    char dir = 'y';
    const double *xalp = nullptr;   // device [nmodes]
    int real0 = 0;                  // 1: mode 0 of every input is real -> derivative terms of mode 0 real
    int ctas_per_job = 0;           // set by lines_launch
};
int lines_launch(ductgpu_ctx ctx, const LineParams &p);
// dns.cu
void free_dns_aux(ductgpu_ctx ctx);

// Position (row, col) of element idx of an operator packed in the DMMA
// A-fragment order used by every FP64 pass (m16n8k16: tiles of 16 x 16,
// m-tile fastest; inside a tile the value pair outermost, then the lane,
// so that a warp's 16-byte loads are consecutive).
__host__ __device__ __forceinline__ void pack_slot(int idx, int mtiles, int &row, int &col)
{
    const int tile = idx >> 8, h = (idx >> 6) & 3, lane = (idx >> 1) & 31, v = 2 * h + (idx & 1);
    const int mt = tile % mtiles, ks = tile / mtiles;
    const int g = lane >> 2, t = lane & 3;
    row = mt * 16 + g + 8 * (v & 1);
    col = ks * 16 + t + 4 * (v >> 1);
}

// dlines.cu: the derivative lines on the FP64 tensor cores (flip-symmetric
// half blocks of the collocation matrices of k_lines)
bool dlines_supported(int nn);
int dlines_launch(ductgpu_ctx ctx, const LineParams &p);
void free_dlines(ductgpu_ctx ctx);
bool lines_supported(int nn);
const double2 *twiddle_table(ductgpu_ctx ctx, int L);

}  // namespace duct

#define DUCT_CUDA(ctx, call)                                         \
    do {                                                             \
        cudaError_t e_ = (call);                                     \
        if (e_ != cudaSuccess) return duct::check_cuda(ctx, e_, #call); \
    } while (0)
