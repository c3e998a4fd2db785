/*
 * ductgpu.h -- C-ABI of libductgpu, the B200 (sm_100a) implementation of the
 * duct per-Fourier-mode 2D Helmholtz/Poisson diagonalisation solve, its
 * Chebyshev transforms and pencil transposes.
 *
 * Plain C types only: pointers, sizes, doubles, chars.  Every entry returns
 * an int status (DUCTGPU_OK = 0); the message of the last failure is read
 * with ductgpu_last_error().  No entry aborts the process.
 *
 * Array conventions are the reference's: column-major (Fortran) order, y
 * fastest; a complex field rhs(my,mz,ib:ie) is my*mz*(ie-ib+1) interleaved
 * (re, im) doubles.  "host" entries take host arrays and copy them to and
 * from the GPU inside the call; "_dev" entries take device pointers.
 *
 * A context is bound to one device and one CUDA stream; calls on one
 * context are serialised by the caller (not re-entrant); separate contexts
 * may be driven from separate threads.
 */
#ifndef DUCTGPU_H
#define DUCTGPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ductgpu_ctx_s *ductgpu_ctx;

/* status codes */
#define DUCTGPU_OK 0
#define DUCTGPU_EARG 1       /* bad size, bound character, null pointer     */
#define DUCTGPU_ESTATE 2     /* operators not set up (pseudomat not called)  */
#define DUCTGPU_ECUDA 3      /* CUDA runtime error                           */
#define DUCTGPU_ESOLVER 4    /* eigen-decomposition / inversion failure      */
#define DUCTGPU_ENONFINITE 5 /* NaN/Inf in a result                          */
#define DUCTGPU_ETIMEOUT 6   /* a bounded device-side wait ran out           */
#define DUCTGPU_EALLOC 7     /* device or host allocation failure            */

/* arithmetic of the solve */
#define DUCTGPU_PREC_FP64 0  /* plain FP64 (DMMA tensor cores): the drop-in  */
#define DUCTGPU_PREC_MIXED 1 /* BF16 split GEMMs + FP64 refinement           */
#define DUCTGPU_PREC_INT8 2  /* FP64-accurate: every GEMM pass as 7 x 7 int8   
                                slices on tcgen05, exact int32 sums (my<=129) */

/* gauge of the singular kx=0 Neumann (pressure) mode */
#define DUCTGPU_GAUGE_POINT 0 /* reference: U(iofzero+1,iofzero+1)=wanted=0 */
#define DUCTGPU_GAUGE_MEAN 1  /* zero mean over the duct cross-section      */

/* ---- context --------------------------------------------------------- */
/* Replaces the gpudevice module state (src/mod.f90:409-483) and the
 * cuBLAS/cuSPARSE handle creation of src/pseudomat.f90:265-298.           */
int ductgpu_create(int device, ductgpu_ctx *out);
int ductgpu_destroy(ductgpu_ctx ctx);
/* Copies the message of the last failure (NUL-terminated) into buf.       */
int ductgpu_last_error(ductgpu_ctx ctx, char *buf, int len);
/* Launch all work of ctx on this cudaStream_t (NULL: the context's own).  */
int ductgpu_set_stream(ductgpu_ctx ctx, void *cuda_stream);
/* Returns the stream work is launched on (for events around a call).      */
void *ductgpu_get_stream(ductgpu_ctx ctx);
int ductgpu_synchronize(ductgpu_ctx ctx);
/* Self-test of the device-side failure path (no counterpart in the
 * reference, whose GPU code has no bounded waits): one CTA waits, with the
 * bounded wait of the pipelined pass kernels, on a barrier that nothing
 * completes; after about `polls` polls (clamped to 1..1<<20, well under a
 * second) it gives up and raises the context's error word.  The call itself
 * returns DUCTGPU_OK; the next ductgpu_synchronize returns DUCTGPU_ETIMEOUT
 * and clears the word, and the context stays usable.                      */
int ductgpu_selftest_wait_timeout(ductgpu_ctx ctx, unsigned polls);

/* ---- setup (one-time) ------------------------------------------------- */
/* pseudomat('d',my) then pseudomat('n',my) (src/pseudomat.f90:2-312, called
 * from helm3d with ipro<=0, src/helm3d.f90:36-46), computed on the GPU in
 * FP64: collocation nodes and derivative matrix, D2=D*D, Dirichlet interior
 * block and Neumann-eliminated block, their eigen-decomposition, inverses,
 * iofzero and the 4x4 corner matrix AM1.  my must equal mz (the square
 * solver stops otherwise, src/helm3d.f90:37-41).                          */
int ductgpu_pseudomat(ductgpu_ctx ctx, int my, int mz);

/* pseudomat with options.  DUCTGPU_SETUP_NO_EIGEN builds the grid, D, D2,
 * the interior blocks, AM1 and the quadrature weights but no
 * eigen-decomposition: both bounds' (E, P, PM1) then come from
 * ductgpu_set_operators, e.g. from the host code's own LAPACK pseudomat
 * (src/pseudomat.f90:131-205), and solves are accepted once 'd' and 'n'
 * are both set.                                                            */
#define DUCTGPU_SETUP_NO_EIGEN 1
int ductgpu_pseudomat_ex(ductgpu_ctx ctx, int my, int mz, int flags);

/* Read back the operators of bound 'd' or 'n' (n = my-2):  E[n] eigenvalues,
 * P[n*n] eigenvectors, PM1[n*n] inverse (column-major), iofzero (1-based,
 * Neumann).  Any output pointer may be NULL.  Bound 'p' reads the
 * Galerkin-basis Neumann operators of ductgpu_pseudopois.                 */
int ductgpu_get_operators(ductgpu_ctx ctx, char bound, double *E, double *P,
                          double *PM1, int *iofzero);

/* Replace the eigen-decomposition of bound 'd' or 'n' with host data, e.g.
 * the LAPACK results of the reference's own pseudomat.  Requires a prior
 * ductgpu_pseudomat[_ex] for the grid.  iofzero <= 0 recomputes it from E.
 * Imported operators are applied as given, on the full (not the
 * flip-symmetric half-size) passes: the solve then restates the reference
 * arithmetic to rounding.  Bound 'p' replaces the pseudopois operators
 * (after ductgpu_pseudopois).                                              */
int ductgpu_set_operators(ductgpu_ctx ctx, char bound, const double *E,
                          const double *P, const double *PM1, int iofzero);

/* *folded = 1 when the solves of bound 'd' or 'n' run the flip-symmetric
 * half-size passes, 0 when they run the full operators.                    */
int ductgpu_get_fold(ductgpu_ctx ctx, char bound, int *folded);

/* Gauge point of the singular kx=0 Neumann mode.  The reference pins
 * U(iofzero+1, iofzero+1) = 0 (src/solvediag.f90:195-206), iofzero being the
 * position of the smallest |eigenvalue| in the order its host LAPACK dgeev
 * returned (src/pseudomat.f90:141-152).  That order is particular to the
 * LAPACK build and cannot be derived from another eigen-solver, so a caller
 * that wants the kx=0 pressure with the reference's additive constant
 * passes its own iofzero here (1-based interior index, 1..my-2).  0
 * restores the default: the position of the smallest |eigenvalue| in the
 * order of the operators in use (the library's own, or imported ones).
 * Reset by ductgpu_pseudomat.                                              */
int ductgpu_set_gauge_point(ductgpu_ctx ctx, int iofzero);

/* Gauge of the singular kx=0 Neumann mode (reference default: POINT).     */
int ductgpu_set_gauge(ductgpu_ctx ctx, int gauge);

/* FP64 iterative-refinement steps of DUCTGPU_PREC_MIXED (0..4, default 2):
 * each step is one FP64 residual of the reference's interior operator and
 * one more split-precision solve.                                          */
int ductgpu_set_refinement(ductgpu_ctx ctx, int steps);

/* ---- the 2D solve ------------------------------------------------------ */
/* helm3d(rhs,sol,work,ipro,bound,cvar,a,b,alambda), src/helm3d.f90:2-76,
 * for one field on host arrays: solves lap(u) - (alambda + xalp(i)^2) u = f
 * for every mode i = ib..ie (xalp[i-ib] = kx of mode i).  Same observable
 * effects as the reference: rhs walls zeroed in place for bound 'd', mode
 * 0 returns a real solution (src/int2d3d.f90:43,91-96), Neumann walls and
 * corners filled (src/solvediag.f90:250-322), kx=0 Neumann mode pinned.
 * ipro <= 0 runs the setup first; ipro == -1 only runs the setup.         */
int ductgpu_helm3d(ductgpu_ctx ctx, double *rhs, double *sol, int ipro,
                   char bound, double alambda, int my, int mz, int ib,
                   int ie, const double *xalp, int precision);

/* The helm3d calls of one substep (u, v, w and p: src/main1.f90:617-619,
 * 643) in one call on host arrays: per field the same effects as
 * ductgpu_helm3d, with each field (the first and the last in two mode
 * ranges) copied in while the previous one is solved and the one before
 * copied back (pinned host memory from ductgpu_host_alloc makes the
 * copies asynchronous).  rhs[i], sol[i]: complex (my,mz,ie-ib+1) host
 * arrays; bounds[i] 'd' or 'n'; alambdas[i]; one xalp for all fields.    */
int ductgpu_helm3d_batch(ductgpu_ctx ctx, int nfields, double *const *rhs, double *const *sol,
                         const char *bounds, const double *alambdas, int my, int mz, int ib,
                         int ie, const double *xalp, int precision);

/* One field of a batched device-resident solve. */
typedef struct {
    double *rhs;         /* device, complex (my,mz,nmodes); walls zeroed in
                            place for bound 'd' like helm3d               */
    double *sol;         /* device, complex (my,mz,nmodes)                 */
    const double *xalp;  /* HOST, nmodes wavenumbers                       */
    double alambda;
    int ib;              /* mode number of the first plane (0: real only)  */
    int nmodes;
    char bound;          /* 'd' or 'n'                                     */
} ductgpu_field;

/* All fields (each a helm3d call of the reference, e.g. u, v, w and the
 * pressure of one RK substep, src/main1.f90:617-619,643) in one batched
 * launch sequence on the context's stream, 1..16 fields.  Asynchronous:
 * returns once the work is queued.                                         */
int ductgpu_solve_fields_dev(ductgpu_ctx ctx, const ductgpu_field *fields,
                             int nfields, int precision);

/* GEMM-pass kernels of the FP64 solve (and of the residual passes):
 * STAGED streams the operator through shared memory in 16-wide K chunks;
 * REGISTER stages the data lines once and streams the operator from L2
 * into registers with no CTA barrier in the K loop.  Chosen per operator
 * size class (0: n <= 63, 1: n <= 127, 2: n <= 191); class -1 sets all.
 * ductgpu_autotune picks them by timing.                                  */
#define DUCTGPU_PASS_STAGED 0
#define DUCTGPU_PASS_REGISTER 1
#define DUCTGPU_PASS_STAGED16 2   /* STAGED with 16 lines per CTA (3 CTAs/SM) */
#define DUCTGPU_PASS_PERSIST 3    /* persistent, operator in registers (n <= 127) */
#define DUCTGPU_PASS_PARITY 4     /* STAGED on the flip-symmetric half operators: even and
                                     odd eigenvectors in two blocks of half size, half the
                                     flops (n <= 191; operators without the symmetry, e.g.
                                     from ductgpu_set_operators, run STAGED)            */
#define DUCTGPU_PASS_PARITY_QUEUE 5 /* PARITY with the four passes of a solve in ONE
                                     persistent launch: tiles taken in pass order, a
                                     plane's pass waiting on per-plane counters of its
                                     earlier passes (bounded waits)                     */
/* kernel -1 restores the library's defaults for the size class(es).      */
int ductgpu_set_pass_kernel(ductgpu_ctx ctx, int size_class, int kernel);
/* Rectangular solves (ductgpu_helm3d_temp, ductgpu_solve_rect_fields_dev)
 * on the flip-symmetric half blocks wherever both walls of each direction
 * match: 1 (the default) the fields grouped by their half-block sizes, each
 * group's four passes on a stream of its own (forked from and joined to
 * the context's stream; parallel branches in a captured graph); 2 the
 * four passes of every field as ONE persistent launch (tiles taken in pass
 * order, a plane's pass waiting on per-plane counters of its earlier
 * passes, any mix of half-block sizes; measured slower on the config-2
 * batch, 0.59 against 0.42 ms); 0 the full operators.                    */
int ductgpu_set_rect_fold(ductgpu_ctx ctx, int on);
/* Kernel of the y / z derivative lines of the DNS operators: 1 (default)
 * the collocation matrices' flip-symmetric half blocks on the FP64 tensor
 * cores, 8 lines per CTA (odd line lengths 17..257; operators built in
 * long double), 2 the same with 16 lines per CTA, 0 the FFT-based transyz
 * + derivyz + transyz chain in one kernel (its half-length DCT-I carries a
 * few 1e-12 of relative error at 129 and 193 points, the tensor-core form
 * a few 1e-13).                                                           */
int ductgpu_set_line_kernel(ductgpu_ctx ctx, int kernel);
/* The real n x n matrix (column-major, 3 <= n <= 1025 points, order 1 or
 * 2) of the reference's derivative along one Chebyshev direction --
 * transyz -1, derivyz, transyz +1 (src/tchebw.f:62-192,
 * src/chebyshev.f90:1-295) -- computed in long double and rounded to FP64;
 * the operators the tensor-core line kernel applies (as flip-symmetric half
 * blocks).  For order 1 it is -cheb_colloc_deriv1 of
 * src/cheb_collocation.F (the chain differentiates along the ascending
 * coordinate), for order 2 the square of that.  Host only: no context, no
 * GPU; O(n^3) work.                                                      */
int ductgpu_cheb_deriv_matrix(int n, int order, double *D);
/* Autotuner: times the FP64 batched solve of these device fields with each
 * pass kernel (reps runs each, after one warm-up; the fields' sol arrays
 * are overwritten and Dirichlet rhs walls zeroed, as by the solve itself)
 * and keeps the fastest for the current grid's size class; *chosen (may be
 * NULL) receives it.  Not during graph capture.                            */
int ductgpu_autotune(ductgpu_ctx ctx, const ductgpu_field *fields, int nfields, int reps,
                     int *chosen);

/* No counterpart in the reference.  ductgpu_solve_fields_dev (FP64) for
 * callers that cannot allocate device memory -- a host code whose own pool
 * allocator has reserved the device, or one that runs several streams and
 * cannot let cudaFree wait for the whole device.  It allocates nothing: its
 * scratch is a fixed 32 MiB array per GPU inside the library (held until
 * the process exits).  A call may hold at most 4096 planes (sum of nmodes)
 * and needs 2 * planes * 2 * my * my doubles of that scratch (my = 129: 62
 * planes); larger calls return DUCTGPU_EARG.  The array is shared by all
 * calls on a GPU: calls that overlap on one GPU race on it -- serialise
 * them.  Nothing in it needs clearing first.  The array's address is looked
 * up (cudaGetSymbolAddress) when the first context is created on a GPU,
 * which under CUDA's default lazy module loading is also when its 32 MiB
 * is taken (under CUDA_MODULE_LOADING=EAGER: when the library's code is
 * loaded on the GPU, whether or not this entry is ever called); create the
 * context before a pool allocator reserves the device and before any
 * stream capture.  Under lazy loading the solve's kernels take device
 * memory for their code at their first launch: set
 * CUDA_MODULE_LOADING=EAGER, or make one call before the pool reserves the
 * device.  Operators must be set up (ductgpu_pseudomat) beforehand.        */
int ductgpu_solve_fields_dev_noalloc(ductgpu_ctx ctx, const ductgpu_field *fields,
                                     int nfields);

/* ---- adjoint (backward) solve ------------------------------------------ */
/* The transpose of the FP64 helm3d map rhs -> sol (of every mode and field,
 * walls, the Neumann wall/corner fill and the kx=0 gauge included), for
 * reverse-mode gradients through the implicit step: given the cotangent
 * gsol of sol it returns grhs = S^T gsol, so <gsol, S f> = <grhs, f> for
 * every f.  Computed in the transposed eigenbasis, P^-T[(P^T G P)./D]P^-1,
 * with the same batched DMMA passes.  The reference has no adjoint; it is
 * checked against the transpose of the oracle's dense helm3d matrix.
 * Fields as in ductgpu_solve_fields_dev with rhs = gsol (read only) and
 * sol = grhs (walls zero; mode 0 real).                                   */
int ductgpu_solve_adjoint_fields_dev(ductgpu_ctx ctx, const ductgpu_field *fields,
                                     int nfields);
/* The same for one field on host arrays (gsol, grhs complex (my,mz,nmodes)). */
int ductgpu_helm3d_adjoint(ductgpu_ctx ctx, const double *gsol, double *grhs, char bound,
                           double alambda, int my, int mz, int ib, int ie, const double *xalp);

/* ---- rectangular ducts, general wall conditions (temperature path) ---- */
/* pseudomaty_temp + pseudomatz_temp (src/pseudomat_temp.f90:2-320) on the
 * GPU for operator slot `slot` (0..7, one per duct shape): my x mz points on
 * [-sy,sy] x [-sz,sz]; wall conditions by1 (y=-sy), by2 (y=+sy), bz1, bz2,
 * each 'd' (Dirichlet) or 'n' (Neumann).                                   */
int ductgpu_pseudomat_temp(ductgpu_ctx ctx, int slot, int my, int mz, double sy, double sz,
                           char by1, char by2, char bz1, char bz2);

/* helm3d_temp(rhs,sol,work,ipro,cvar,a,b,alambda,bcco),
 * src/helm3d_temp.f90:2-46, on host arrays with operator slot 0: solves
 * lap(u) - (alambda + xalp^2) u = f with wall values bcy(mz,2,nmodes) (at
 * y = -a, +a) and bcz(my,2,nmodes) (z = -b, +b), real, the same for the
 * real and the imaginary part as in src/int2d3d_temp.f90:71-83 (NULL: zero
 * walls).  ipro <= 0 runs the setup first (ipro == -1: setup only).  The
 * singular all-Neumann mode at lambda = 0, which the reference divides by
 * zero, gets the zero-eigen-coefficient gauge (GAUGE_MEAN: zero mean).     */
int ductgpu_helm3d_temp(ductgpu_ctx ctx, double *rhs, double *sol, int ipro, double a,
                        double b, double alambda, int my, int mz, int ib, int ie,
                        const double *xalp, const double *bcy, const double *bcz,
                        char by1, char by2, char bz1, char bz2);

/* One field of a batched rectangular solve (device arrays). */
typedef struct {
    double *rhs;         /* device, complex (my,mz,nmodes) of the slot      */
    double *sol;         /* device, complex (my,mz,nmodes)                  */
    const double *xalp;  /* HOST, nmodes wavenumbers                        */
    const double *bcy;   /* device (mz,2,nmodes) wall values, or NULL       */
    const double *bcz;   /* device (my,2,nmodes) wall values, or NULL       */
    double alambda;
    int ib;
    int nmodes;
    int slot;            /* operator slot (duct shape)                      */
} ductgpu_rect_field;

/* Fields of several duct shapes (slots) solved together: each of the four
 * GEMM passes is one launch over all fields, modes and shapes.           */
int ductgpu_solve_rect_fields_dev(ductgpu_ctx ctx, const ductgpu_rect_field *fields,
                                  int nfields);

/* ---- Shen-Legendre Galerkin solver (HELM_SHEN build) ----------------- */
/* preshen(eigv,psm1,bound) + leg_cheb_mat, src/preshen.f90:2-535 and
 * src/legendre.f90:3-110: the Legendre-Chebyshev matrices and the
 * generalized eigen-decomposition M x = rho S x of bound 'd' or 'n' for a
 * square my x my grid (my odd, 5..191, my-1 = 2^a 3^b for the transform). */
int ductgpu_preshen(ductgpu_ctx ctx, int my, char bound);
/* helm3d_shen(rhs,sol,work,ipro,bound,cvar,a,b,alambda),
 * src/helm_shen.f90:2-85 -> int2d3d -> solveshen (src/solveshen.f90:5-94):
 * solves -lap(u) + (alambda + xalp^2) u = rhs in the Shen basis on host
 * arrays.  As in the reference, rhs is overwritten with its Chebyshev
 * coefficients (transyz y and z, iopt -1); ipro <= 0 runs preshen first,
 * ipro = -1 only that.  Mode 0 (ib = 0) has a real solution.              */
int ductgpu_helm3d_shen(ductgpu_ctx ctx, double *rhs, double *sol, int ipro, char bound,
                        double alambda, int my, int mz, int ib, int ie, const double *xalp);
/* Batched device-resident form: every field's `bound` selects its preshen
 * operators; all fields share my (= mz).  rhs is overwritten as above.    */
int ductgpu_solve_shen_fields_dev(ductgpu_ctx ctx, const ductgpu_field *fields, int nfields);

/* ---- Galerkin-basis Neumann (pressure) solver ------------------------- */
/* pseudopois(m), src/pseudopois.f90:2-104: the Neumann operator in the basis
 * phi_j = T_j - j^2/(j+2)^2 T_{j+2} (B2 B^-1 on the interior nodes), its
 * eigen-decomposition and iofzero, on the GPU; my = 5..193.               */
int ductgpu_pseudopois(ductgpu_ctx ctx, int my);
/* solvepois(U,F,FT,wk1,wk2,xlambda,m), src/solvepois.f90:1-170, on one real
 * host plane U (my,my): interior = rhs in, solution (walls and corners from
 * the basis, kx=0 point pinned to 0 when |xlambda| <= 1e-10) out.         */
int ductgpu_solvepois(ductgpu_ctx ctx, double *U, double xlambda, int my);
/* Batched complex fields (bound 'n'), as ductgpu_solve_fields_dev.       */
int ductgpu_solve_pois_fields_dev(ductgpu_ctx ctx, const ductgpu_field *fields, int nfields);

/* ---- constant mass-flow-rate forcing ---------------------------------- */
/* precomp_mass_flow(dtp,alphak,work,nwk), src/operators.F:2205-2289 (square
 * build; needs ductgpu_pseudomat): for RK index k = 1..mrk solves
 * (dyy+dzz)u - u/(alphak[k-1] dtp fnu) = 1 with zero walls and keeps the
 * solution premassfu(:,:,k) and its flow rate premassf[k-1] (integral over
 * the cross-section times aspect) in the context.  premassf (mrk) and
 * premassfu (my*my*mrk, real) are optional host outputs (NULL: skipped).  */
int ductgpu_precomp_mass_flow(ductgpu_ctx ctx, double dtp, const double *alphak, int mrk,
                              double fnu, double aspect, double *premassf, double *premassfu);
/* impose_mass_flow(csum,krk,u,work,nwk,iflag), src/operators.F:2291-2344, on
 * the first (mode 0) plane of the device field u (complex (my,my,...)):
 * iflag 0 stores its flow rate in *csum (synchronises); iflag 1 adds
 * (*csum - flow)/premassf(krk) * premassfu(:,:,krk) to its real part
 * (krk 1-based), asynchronously, in one kernel.                          */
int ductgpu_impose_mass_flow_dev(ductgpu_ctx ctx, double *csum, int krk, double *u, int iflag);
/* The same on a host field (only its mode 0 plane is copied).             */
int ductgpu_impose_mass_flow(ductgpu_ctx ctx, double *csum, int krk, double *u, int iflag);

/* ---- captured solves (CUDA graphs) ------------------------------------ */
/* Capture one batched solve -- kind 0: `fields` is a ductgpu_field array
 * (square path, `precision` as in ductgpu_solve_fields_dev); kind 1: a
 * ductgpu_rect_field array; kind 2: a ductgpu_field array of the Shen
 * solver (ductgpu_solve_shen_fields_dev) -- as a CUDA graph bound to the fields' device
 * pointers and wavenumbers, e.g. the four solves of an RK3/CN substep.  The
 * solve runs once uncaptured first (workspaces, checks).  Replays with
 * ductgpu_graph_launch cost one launch.                                   */
int ductgpu_graph_create(ductgpu_ctx ctx, int kind, const void *fields, int nfields,
                         int precision, int *graph_id);
int ductgpu_graph_launch(ductgpu_ctx ctx, int graph_id);
int ductgpu_graph_destroy(ductgpu_ctx ctx, int graph_id);

/* ---- Chebyshev transforms, derivatives, pencil transposes ------------ */
/* transyz(cheb,cdir,iopt), src/chebyshev.f90:458-540 with tcheb_fftw,
 * src/tchebw.f:62-192: DCT-I of every line of a complex (my,mz,nmodes)
 * field along cdir = 'y' or 'z', in place.  iopt < 0: physical ->
 * Chebyshev (ends scaled 1/(2(n-1)), interior 1/(n-1)); iopt >= 0: the
 * inverse.  The line length minus one must be 2^a 3^b (as the reference's
 * FFTW plans assume, src/tchebw.f:11-12).                                 */
int ductgpu_transyz_dev(ductgpu_ctx ctx, double *field, int my, int mz, int nmodes,
                        char cdir, int iopt);
int ductgpu_transyz(ductgpu_ctx ctx, double *field, int my, int mz, int nmodes,
                    char cdir, int iopt);

/* derivyz(u,du,aux,cdir,ider,scal,what), src/chebyshev.f90:1-295: first or
 * second derivative (ider = 1, 2) of a Chebyshev-space complex field along
 * cdir; z derivatives carry 1/aspect^ider.  what = 'n' overwrites du,
 * anything else accumulates into it.  u and du must not overlap.         */
int ductgpu_derivyz_dev(ductgpu_ctx ctx, const double *u, double *du, int my, int mz,
                        int nmodes, char cdir, int ider, double scal, char what,
                        double aspect);
int ductgpu_derivyz(ductgpu_ctx ctx, const double *u, double *du, int my, int mz,
                    int nmodes, char cdir, int ider, double scal, char what,
                    double aspect);

/* Local pencil transposes of one rank, src/parallel.F:476-529 (complex):
 * cxyz2yzx: phys(0:mx1,my,nz) -> phys2(my,nz,0:mx1)
 * cyzx2xyz: phys2(my,nz,0:mx1) -> phys(0:mx1,my,nz)                       */
int ductgpu_cxyz2yzx_dev(ductgpu_ctx ctx, const double *phys, double *phys2,
                         int nmodes, int my, int nz);
int ductgpu_cyzx2xyz_dev(ductgpu_ctx ctx, double *phys, const double *phys2,
                         int nmodes, int my, int nz);
/* chx2z(xy,xz,wk2) and chz2x(xz,xy,wk2) on one rank, src/parallel.F:1-208:
 * chx2z: xz <- xy (y,z,x layout), xy <- x-fastest transpose of it;
 * chz2x: the inverse (xy <- y-fastest transpose of xz, xz <- xy).  The
 * reference's chz2x returns before its transpose on one rank
 * (src/parallel.F:132); this is the inverse of chx2z it documents.        */
int ductgpu_chx2z_dev(ductgpu_ctx ctx, double *xy, double *xz, int my, int mz, int nmodes);
int ductgpu_chz2x_dev(ductgpu_ctx ctx, double *xz, double *xy, int my, int mz, int nmodes);

/* ---- operators of the DNS time step (x-cut complex (my,mz,nmodes) device
 * fields, wavenumbers xalp[nmodes] on the host) ------------------------
 * The y / z derivatives are the reference's transyz(-1) -> derivyz ->
 * transyz(+1) round trip, computed per line in one pass (my-1 and mz-1 one
 * of 16, 24, 32, 48, 64, 96, 128, 144, 192, 256); x derivatives are i kx.
 * The reference transforms some inputs in place and back (changing them by
 * rounding); here inputs are left untouched.  Asynchronous on the context
 * stream unless stated.                                                   */
/* derivx(u,du,ider,scal,what), src/fourier.F:120-188:
 * du = [du +] scal (i kx)^ider u (what = 'n' overwrites).                 */
int ductgpu_derivx_dev(ductgpu_ctx ctx, const double *u, double *du, int my, int mz, int nmodes,
                       const double *xalp, int ider, double scal, char what);
/* laplacian3d(u,flap,tmp,tmpyz,scal,what), src/operators.F:278-347:
 * flap = [flap +] scal (-kx^2 u + u_yy + u_zz / aspect^2).               */
int ductgpu_laplacian3d_dev(ductgpu_ctx ctx, const double *u, double *flap, int my, int mz,
                            int nmodes, const double *xalp, double aspect, double scal, char what);
/* grad3d(u,dxu,dyu,dzu,tmp,tmpyz,scal,what), src/operators.F:349-425.     */
int ductgpu_grad3d_dev(ductgpu_ctx ctx, const double *u, double *dxu, double *dyu, double *dzu,
                       int my, int mz, int nmodes, const double *xalp, double aspect, double scal,
                       char what);
/* div3d(u,v,w,div,tmp,tmpyz,scal), src/operators.F:427-501:
 * div = scal (i kx u + v_y + w_z / aspect).                               */
int ductgpu_div3d_dev(ductgpu_ctx ctx, const double *u, const double *v, const double *w, double *div,
                      int my, int mz, int nmodes, const double *xalp, double aspect, double scal);
/* update_uvwp(u,v,w,p,phi,rhsphi,tmp,tmpyz,akk,bkk), src/operators.F:503-605
 * (no FILTER): p += phi - (akk+bkk) dt fnu lap(phi); (u,v,w) -= dt
 * (akk+bkk) grad(phi).  The reference's rhsphi work array is not produced. */
int ductgpu_update_uvwp_dev(ductgpu_ctx ctx, double *u, double *v, double *w, double *p,
                            const double *phi, int my, int mz, int nmodes, const double *xalp,
                            double aspect, double akk, double bkk, double dt, double fnu);
/* advection3d(u,v,w,adv1,adv2,adv3,...), src/operators.F:9-276, with the
 * x transforms of fourx/pack_fftw/fill (src/fourier.F:1-118, 2/3 rule:
 * nmodes = mx/2, mx = 2 (mgalx/3); mgalx one of 16, 64, 144, 256) and the
 * pencil transposes folded into the addressing.  work: 5 fields of the same
 * size (the products uv, uw, vv, vw, ww).  stats2 (device (my,mz,6) or
 * NULL): statistics_fou2 (src/operators.F:1957-2004) -- the x-means of uu,
 * vv, ww, uv, uw, vw added.                                              */
int ductgpu_advection3d_dev(ductgpu_ctx ctx, const double *u, const double *v, const double *w,
                            double *adv1, double *adv2, double *adv3, double *work, int my, int mz,
                            int nmodes, int mgalx, const double *xalp, double aspect, double *stats2);
/* max_3din(u,divmax), src/operators.F:2524-2550: max |u| over the interior
 * points of every mode (synchronises).                                    */
int ductgpu_max_3din_dev(ductgpu_ctx ctx, const double *u, int my, int mz, int nmodes, double *divmax);
/* wallstressx(u,tmpyz,stress4), src/operators.F:676-710 with
 * cheb2_wallstress_circum (src/chebyshev.f90:642-690): the wall stress of
 * the x-mean of u per wall (host stress4[4]; synchronises).               */
int ductgpu_wallstressx_dev(ductgpu_ctx ctx, const double *u, int my, int mz, double aspect,
                            double *stress4);
/* energy_fou(u,energy,energy2), src/operators.F:907-973 (one rank):
 * sqrt(sum_{i>=1} 2|u_i|^2 dy dz / area) and the same with mode 0
 * (synchronises).                                                         */
int ductgpu_energy_fou_dev(ductgpu_ctx ctx, const double *u, int my, int mz, int nmodes, double aspect,
                           double *energy, double *energy2);
/* vorticity(u,v,w,vort,tmp,iflag), src/operators.F:810-905: component
 * iflag of the vorticity, 1 om_x = dw/dy - dv/dz, 2 om_y = du/dz - dw/dx,
 * 3 om_z = dv/dx - du/dy, of device x-cut fields (vort distinct from u, v,
 * w; xalp on the host).                                                   */
int ductgpu_vorticity_dev(ductgpu_ctx ctx, const double *u, const double *v, const double *w, double *vort,
                          int my, int mz, int nmodes, const double *xalp, double aspect, int iflag);
/* statistics_fou(u,v,w,p,1), src/operators.F:1608-1765 (one rank): adds
 * to the device accumulators mean (my,mz,4) the mode-0 real parts of u, v,
 * w, p, ppb (my,mz) the x-mean of p^2, spec (nmodes,7,4) the streamwise
 * spectra at the reference's seven points (synchronises).                 */
int ductgpu_statistics_fou_dev(ductgpu_ctx ctx, const double *u, const double *v, const double *w,
                               const double *p, int my, int mz, int nmodes, double *mean, double *ppb,
                               double *spec);

/* ---- the RK3/Crank-Nicolson DNS step, device resident ------------------
 * The substep of src/main1.f90:384-723 (square duct, no temperature,
 * DT_FIXED): advection (i), (ii); statistics at the first substep of a
 * recorded step; the explicit right-hand side (iii)-(vii); the implicit
 * helm3d 'd' solves of u, v, w (viii); the pseudo-pressure Poisson solve
 * (ix), (x); update_uvwp (xi); impose_mass_flow with CMASSFLOW; the
 * divergence check max_3din.  Needs a context set up with
 * ductgpu_pseudomat at my = mz.  cmassflow 1 holds the flow rate of the
 * initial u (set by ductgpu_dns_set_fields); 0 drives the flow with the
 * mean pressure gradient dpdx.  precision: DUCTGPU_PREC_* of the solves.
 * hist_cap: rows of the per-step diagnostics history kept on the device.
 * After the first use of each RK index, a substep runs as one CUDA graph
 * launch.                                                                 */
typedef struct ductgpu_dns_s *ductgpu_dns;
int ductgpu_dns_create(ductgpu_ctx ctx, int mgalx, double alp, double fnu, double dt, double aspect,
                       int cmassflow, double dpdx, int precision, int hist_cap, ductgpu_dns *out);
int ductgpu_dns_destroy(ductgpu_dns dns);
/* u, v, w, p: complex (my,my,nmodes) host or device arrays (copied).      */
int ductgpu_dns_set_fields(ductgpu_dns dns, const double *u, const double *v, const double *w,
                           const double *p);
/* NULL outputs are skipped; host or device destinations.  Synchronises.   */
int ductgpu_dns_get_fields(ductgpu_dns dns, double *u, double *v, double *w, double *p);
/* Device pointer of the resident field which = 0 u, 1 v, 2 w, 3 p.        */
int ductgpu_dns_field(ductgpu_dns dns, int which, double **dev);
/* Graph replay of substeps on (1, the default) or off.                    */
int ductgpu_dns_set_graphs(ductgpu_dns dns, int on);
/* One substep krk = 1..3 (stats: gather the step's statistics, krk 1).    */
int ductgpu_dns_substep(ductgpu_dns dns, int krk, int stats);
/* nsteps RK3 steps, statistics every stats_every-th step (0: none).       */
int ductgpu_dns_steps(ductgpu_dns dns, int nsteps, int stats_every);
/* Accumulated statistics to the host (NULL outputs skipped): mean
 * (my,my,4), prod (my,my,6) (uu, vv, ww, uv, uw, vw), ppb (my,my), spec
 * (nmodes,7,4); hist rows (10 doubles: stress4[4], energy[3] of u, v, w,
 * energy2[3]); nstat recorded steps; nhist rows; divmax3 the divergence
 * after each substep of the last step.  Synchronises.                    */
int ductgpu_dns_statistics(ductgpu_dns dns, double *mean, double *prod, double *ppb, double *spec,
                           double *hist, int *nstat, int *nhist, double *divmax3);
/* The time-step and slip checks that advection3d makes at the first
 * substep of every step (determine_step, src/operators.F:608-672, and
 * slip_velocity_3d, 2552-2608), taken by the x-FFT kernel on the physical
 * velocities: cfl = dt max(|u| alp mgalx/(2 pi), |v|/dy, |w|/dz) of the
 * last step (the CFL number of the fixed step; the reference stops above
 * 100, src/main1.f90:426-434), slip = the largest velocity component on
 * the walls of the last step, cfl_max = the largest cfl since the previous
 * call (reset by the call).  0 before the first step.  NULL outputs are
 * skipped.  Synchronises.                                                  */
int ductgpu_dns_cfl(ductgpu_dns dns, double *cfl, double *slip, double *cfl_max);
/* The vorticity diagnostics of the recorded steps (src/main1.f90:453-466):
 * om2 (my,my,3) the accumulators omx2, omy2, omz2 of statistics_omg2_fou
 * (src/operators.F:1859-1955); hist rows of 16 doubles per recorded step,
 * in the order of ductgpu_dns_statistics' rows: energy_fou_zero_sector of
 * om_x (energomx4[5], :1018-1099), integral_abs_zero_sector of om_x
 * (energomxb4[5], :1462-1541), energy_fou of om_x, om_y, om_z (energomx,
 * energomy, energomz) and the same with mode 0 (energomxb, energomyb,
 * energomzb).  NULL outputs are skipped.  Synchronises.                   */
int ductgpu_dns_statistics_omg(ductgpu_dns dns, double *om2, double *hist, int *nhist);
/* Body force f = (f1, f2, f3) (complex (my,my,nmodes) fields, host or
 * device; copied): it enters the substep's right-hand side like the
 * pressure gradient and the reference's forcings (src/main1.f90 (vi-b),
 * force_global / add_puff_forcing with -(akk+bkk)): h += (akk+bkk) f.
 * All NULL removes it.                                                    */
int ductgpu_dns_set_forcing(ductgpu_dns dns, const double *f1, const double *f2, const double *f3);
/* J = the wall stress of u summed over the four walls (wallstressx,
 * src/operators.F:676-710) after nsteps RK3 steps from the current state;
 * the state is left as it was.                                            */
int ductgpu_dns_wallstress_after(ductgpu_dns dns, int nsteps, double *J);
/* Reverse mode through one RK3/CN step from the current state (left as it
 * was): J as above after one step, and fbar = dJ/df (3 complex fields,
 * host or device; the gradient in the coefficient inner product
 * Re sum conj(a) b, i.e. dJ/dRe f + i dJ/dIm f per coefficient).  The
 * discrete adjoint of the GPU step: adjoint solves (transposed eigenbasis),
 * transposed derivative matrices, the transposed advection products
 * linearised at the substeps' entry velocities (in-memory checkpoints of
 * the forward sweep), the mass-flow correction transposed.  Synchronises.
 * No counterpart in the reference (it has no adjoint).                    */
int ductgpu_dns_grad_wallstress(ductgpu_dns dns, double *J, double *fbar);

/* ---- field checkpoint files uvwp_NNNN.h5 --------------------------------
 * The reference's restart / output file (src/readwrite_hdf5.f90): datasets
 * u, v, w, p of HDF5 shape (mx1+1, mz, my, 2), big-endian doubles (the
 * Fortran (2, my, mz, mx1+1) view of a complex (my, mz, mx1+1) field), and
 * writeheader_hdf5's scalars in the root group.  Written in the HDF5 file
 * format without an HDF5 library (version 0 superblock, symbol-table root
 * group, contiguous storage: what libhdf5 writes with its default format
 * bounds); read back from that subset.  File errors return DUCTGPU_EARG
 * with the reason in ductgpu_last_error.                                  */
typedef struct {
    int nparams;        /* 7: no temperature fields (read back; written as 7) */
    int numerop;        /* ranks of the run (written as given, 1 if <= 0)      */
    int mgalx, my, mz, mx1;
    double alp, aspect, time, fnu, cfl, dtfixed, cmassflow;
    double slip;        /* dataset SLIP-VELOCITY                               */
    double divergence;  /* dataset DIVERGENCE                                  */
} ductgpu_h5_header;
/* concat5b(fuvwpout,'uvwp_',5,ext,4,'.',1,'h5',2,filename) with ext the
 * i4.4 of iimag (src/readwrite_hdf5.f90:326-330, src/concat.F:74-87): the
 * prefix up to its first blank + "uvwp_NNNN.h5".  cap: bytes of out.     */
int ductgpu_uvwp_filename(const char *fuvwpout, int iimag, char *out, int cap);
/* save_4fields_fou_hdf5(u,v,w,p,iimag,'r8') on one rank
 * (src/readwrite_hdf5.f90:276-386, h5dump_parallel :650-722,
 * writeheader_hdf5 :851-920): u, v, w, p are DEVICE complex
 * (my, mz, mx1+1) fields; the header gives the sizes and the scalars.
 * The fields are converted to big-endian on the GPU (in stream order after
 * the work already on the context's stream).  Synchronises.               */
int ductgpu_save_4fields_fou_hdf5_dev(ductgpu_ctx ctx, const char *filename, const double *u,
                                      const double *v, const double *w, const double *p,
                                      const ductgpu_h5_header *hdr);
/* readheader_hdf5 (src/readwrite_hdf5.f90:799-849); without mx1 in the file
 * mx1 = 2 (mgalx/3)/2 - 1 as there.  ctx may be NULL (no error text).     */
int ductgpu_read_hdf5_header(ductgpu_ctx ctx, const char *filename, ductgpu_h5_header *hdr);
/* read_4fields_fou_hdf5(u,v,w,p,filename,'r8') (src/readwrite_hdf5.f90:5-197
 * with h5load_parallel :199-273) into DEVICE complex (my, mz, nmodes)
 * fields: the file's modes beyond nmodes are dropped and missing ones are
 * zero, as there; a file of another my AND mz is re-interpolated as the
 * reference does (cheb_interp, src/chebyshev.f90:725-765: the first
 * min(20, myr) x min(20, mzr) Chebyshev coefficients of each plane summed
 * at the new nodes; myr - 1 and mzr - 1 of the form 2^a 3^b), a file with
 * only one of them different is refused.  hdr_out (may be NULL) receives
 * the file's header.  Synchronises.                                        */
int ductgpu_read_4fields_fou_hdf5_dev(ductgpu_ctx ctx, const char *filename, double *u, double *v,
                                      double *w, double *p, int my, int mz, int nmodes,
                                      ductgpu_h5_header *hdr_out);
/* The stepper's state to / from such a file (src/main1.f90:735-752 saves
 * every nimag steps; irestart reads it back at start-up).  save: header
 * from the stepper (mgalx, my = mz, mx1 = modes - 1, alp, aspect, fnu,
 * dtfixed = dt, cmassflow = the held flow rate, DIVERGENCE = the last
 * substep's max_3din) plus the caller's time, cfl and slip (NaN: the wall
 * slip measured at the last step, as the reference saves).  load: the
 * fields as ductgpu_dns_set_fields takes them, the file's time to *time
 * (may be NULL); with cmassflow the file's cmassflow is the flow rate held
 * (that of the loaded u when the file's is 0), so a restart repeats the
 * saved run bit for bit.                                                   */
int ductgpu_dns_save_hdf5(ductgpu_dns dns, const char *filename, double time, double cfl, double slip);
/* write_statistics_hdf5 (src/readwrite_hdf5.f90:388-648, one rank, no
 * temperature): the stepper's accumulated statistics as the reference
 * writes them -- mgalx, my, mz, nstat (32-bit ints), timef, time, fnu,
 * alp, aspect (doubles), the (my, mz) sums um, vm, wm, pm, uub, uvb, uwb,
 * vvb, vwb, wwb, ppb, ox2, oy2, oz2, the (mx1+1, nspec) spectra uust,
 * vvst, wwst, ppst and the spectra points jinco, kinco (nspec = 7).
 * timef: the reference's timef (the caller's value).  Synchronises.       */
int ductgpu_dns_write_statistics_hdf5(ductgpu_dns dns, const char *filename, double time, double timef);
/* The reference's statistics file name: the prefix (up to its first blank)
 * + "statistics_NNNN.h5" with the first NNNN = 0001, 0002, ... that does
 * not exist yet (src/readwrite_hdf5.f90:446-456).  DUCTGPU_EARG when all
 * 9999 exist or cap is too small.                                          */
int ductgpu_statistics_filename(const char *fuvwpout, char *out, int cap);
int ductgpu_dns_load_hdf5(ductgpu_dns dns, const char *filename, double *time);

/* ---- the reference's own GPU entry points (src/mytranspose_cuda.cu) --- */
/* transpose_gpu_(handle,Nx,Ny,alpha,devPtrA,devPtrC) and
 * mat_invdiag_gpu_(handle,Nx,Ny,xlam,devPtrF,devPtrED,devPtrC) with the
 * reference's Fortran argument convention (pointers to integers, device
 * addresses as size_t handles; src/mytranspose_cuda.cu:132-196).  Unlike the
 * reference (grid(N/32,N/32), defect for N not a multiple of 32) every size
 * is handled.  C(j,i) = A(i,j) for an Nx x Ny column-major A;
 * C = F / (ED - xlam) elementwise.  They run on the legacy default stream;
 * handle and alpha are accepted and unused, as in the reference.          */
int transpose_gpu_(size_t *handle, const int *Nx, const int *Ny, const double *alpha,
                   const size_t *devPtrA, size_t *devPtrC);
int mat_invdiag_gpu_(size_t *handle, const int *Nx, const int *Ny, const double *xlam,
                     const size_t *devPtrF, const size_t *devPtrED, size_t *devPtrC);

/* ---- memory helpers (for callers without a CUDA toolchain, e.g. Fortran
 * hosts that keep fields resident on the device between time steps) ---- */
int ductgpu_device_alloc(ductgpu_ctx ctx, size_t bytes, void **ptr);
int ductgpu_device_free(ductgpu_ctx ctx, void *ptr);
/* pinned host memory: host<->device copies from it run at full link speed */
int ductgpu_host_alloc(ductgpu_ctx ctx, size_t bytes, void **ptr);
int ductgpu_host_free(ductgpu_ctx ctx, void *ptr);
/* asynchronous copies on the context stream (kind: 1 = H2D, 2 = D2H,
 * 3 = D2D, as cudaMemcpyKind)                                              */
int ductgpu_copy(ductgpu_ctx ctx, void *dst, const void *src, size_t bytes, int kind);

/* ---- timing helpers for benchmarks (CUDA events on the ctx stream) ---- */
int ductgpu_event_record(ductgpu_ctx ctx, int slot);
/* milliseconds between two recorded slots (synchronises on the later). */
int ductgpu_event_elapsed(ductgpu_ctx ctx, int slot0, int slot1, float *ms);

/* Count of kernels this library launched on ctx since creation.           */
long long ductgpu_launch_count(ductgpu_ctx ctx);

/* Per-kernel device time: with profiling on, every launch of the library is
 * bracketed by CUDA events on the ctx stream.  ductgpu_profile_read
 * synchronises and returns, for kernel class `kind` (DUCTGPU_K_*), the
 * summed milliseconds and launch count since the last reset.               */
#define DUCTGPU_K_PASS_FP64 0   /* FP64 DMMA GEMM pass                      */
#define DUCTGPU_K_NEUMANN 1     /* Neumann walls/corners/pin                */
#define DUCTGPU_K_WALLS 2       /* Dirichlet wall zeroing                   */
#define DUCTGPU_K_MIXED_GEMM 3  /* split-precision tcgen05 GEMM pass        */
#define DUCTGPU_K_RESIDUAL 4    /* FP64 refinement residual                 */
#define DUCTGPU_K_TRANSFORM 5   /* Chebyshev transforms / derivatives       */
#define DUCTGPU_K_TRANSPOSE 6   /* pencil transposes                        */
#define DUCTGPU_K_OTHER 7
#define DUCTGPU_K_LINES 8      /* fused Chebyshev line derivative + epilogue */
#define DUCTGPU_K_ADVECTION 9  /* x-direction Fourier products (advection)  */
#define DUCTGPU_K_STATS 10     /* statistics / diagnostics reductions     */
#define DUCTGPU_K_COUNT 11
int ductgpu_profile_enable(ductgpu_ctx ctx, int on);
int ductgpu_profile_reset(ductgpu_ctx ctx);
int ductgpu_profile_read(ductgpu_ctx ctx, int kind, double *ms, long long *launches);
/* Algorithmic bytes (each field element read or written once) of the
 * launches of class `kind` since the last reset, counted on the host for
 * the kernels that report them (DUCTGPU_K_LINES, DUCTGPU_K_ADVECTION);
 * with profiling on only.                                                 */
int ductgpu_profile_bytes(ductgpu_ctx ctx, int kind, double *bytes);
/* Tensor-core flops executed (padded tiles included) by the launches of
 * class `kind` since the last reset, for the kernels that report them
 * (DUCTGPU_K_LINES on the FP64 tensor cores); with profiling on only.     */
int ductgpu_profile_flops(ductgpu_ctx ctx, int kind, double *flops);

#ifdef __cplusplus
}
#endif
#endif
