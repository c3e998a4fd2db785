/*
 * duct_oracle.h -- CPU FP64 restatement of the duct reference hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path
 * and the timed CPU baseline.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py load it.  The product library (libductgpu)
 * never links, loads or calls it.
 *
 * Parity pin: the reference is Fortran + MPI + FFTW + HDF5 and cannot be
 * built in this image (no Fortran compiler), so no output of the reference
 * itself is available.  The restatement is pinned by the reference's own
 * known-answer data -- the laminar duct table of get_dpdx
 * (src/operators.F:2496-2507, "-(dyy+dzz)U=dpval -> max(U)=1", aspect
 * ratios 1..10) -- by the classical series for the laminar duct flow rate
 * and by exact manufactured polynomial solutions.  (CMASSFLOW in
 * utils/gen_tsd2hdf5.py:10 is a run's flow rate, not the laminar integral,
 * which is 1.9081638750 for aspect 1.)  Parity is therefore "partially
 * pinned": known answers, not reference outputs.
 *
 * Conventions follow the reference: column-major arrays, y fastest, complex
 * fields stored as interleaved (re, im) doubles, 1-based index names in the
 * comments map to 0-based C indices.
 */
#ifndef DUCT_ORACLE_H
#define DUCT_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Operators of one square collocation grid: the contents of the reference's
 * modules chebystuff, fulldiagdir and fulldiagneu (src/mod.f90:277-343),
 * filled by orc_pseudomat (src/pseudomat.f90:2-312).                       */
typedef struct {
    int m;              /* my = mz, collocation points incl. walls           */
    double *xcol;       /* m      CGL nodes  -cos(pi j/(m-1))                */
    double *DC;         /* m*m    first-derivative matrix (CHQZ p.69)         */
    double *D2;         /* m*m    DC*DC                                       */
    /* Dirichlet ('d') interior eigen-decomposition of D2(2:m-1,2:m-1)        */
    double *ED, *EDim;  /* n      eigenvalues (real, imaginary) n = m-2       */
    double *PD, *PDM1;  /* n*n    right eigenvectors and their inverse        */
    /* Neumann ('n') eigen-decomposition of the boundary-eliminated block     */
    double *EN, *ENim;
    double *PN, *PNM1;
    int iofzero;        /* 1-based index of the smallest |EN|                 */
    double wanted;      /* pinned value of U(iofzero+1,iofzero+1), 0         */
    double AM1[16];     /* 4x4 inverse corner matrix, column-major            */
    double *D2Bd;       /* n*n    Dirichlet block (kept for residual checks)  */
    double *D2Bn;       /* n*n    Neumann-eliminated block                    */
} orc_ops;

/* pseudomat('d',m) followed by pseudomat('n',m).  Returns LAPACK info != 0 or
 * -1 on a bad size.  */
int  orc_pseudomat(int m, orc_ops *ops);
void orc_ops_free(orc_ops *ops);

/* solvediag(U,F,FT,bound,xlambda), src/solvediag.f90:2-330, CPU branch.
 * U is m*m real, in: rhs in the interior (+ Dirichlet values on the walls),
 * out: solution.  Returns 0, or -1 for a bad bound.                        */
int  orc_solvediag(double *U, const orc_ops *ops, char bound, double xlambda);

/* helm3d(rhs,sol,work,1,bound,...) for modes ib..ie (src/helm3d.f90:2-76 and
 * int2d3d src/int2d3d.f90:2-53).  rhs, sol: complex (my,mz,nmodes)
 * interleaved; xalp[i] = kx of local mode i (mode number ib+i).  rhs walls
 * are zeroed in place for bound='d'.  nthreads > 1 spreads modes over
 * OpenMP threads (the reference spreads them over MPI ranks).               */
int  orc_helm3d(double *rhs, double *sol, int my, int mz, int ib, int ie,
                const double *xalp, char bound, double alambda,
                const orc_ops *ops, int nthreads);

/* tcheb_fftw(cr,ise,isa,m,cdir,iopt), src/tchebw.f:62-192, with FFTW's
 * REDFT00 evaluated directly in FP64.  nn = transform length.               */
void orc_tcheb(double *cr, long ise, long isa, long nlines, int nn, int iopt);

/* transyz(cheb,cdir,iopt), src/chebyshev.f90:458-540 on a complex field
 * (my,mz,nmodes).                                                            */
void orc_transyz(double *cheb, int my, int mz, int nmodes, char cdir, int iopt);

/* transyz_plane(cheb,iopt), src/chebyshev.f90:542-595, real (my,mz) plane. */
void orc_transyz_plane(double *cheb, int my, int mz, int iopt);

/* derivyz(u,du,aux,cdir,ider,scal,what), src/chebyshev.f90:1-295, complex
 * c-c-f field (my,mz,nmodes).  what='n' overwrites du, else accumulates.   */
void orc_derivyz(const double *u, double *du, int my, int mz, int nmodes,
                 char cdir, int ider, double scal, char what, double aspect);

/* cheb2_integral(u,1,aspect,sum,ny,nz), src/chebyshev.f90:692-723.         */
double orc_cheb2_integral(const double *u, int ny, int nz, double aspect);

/* Local pencil transposes of one rank, src/parallel.F:476-529.
 * cxyz2yzx: phys(0:mx1,my,nz) -> phys2(my,nz,0:mx1)
 * cyzx2xyz: phys2(my,nz,0:mx1) -> phys(0:mx1,my,nz)                       */
void orc_cxyz2yzx(const double *phys, double *phys2, int nmodes, int my, int nz);
void orc_cyzx2xyz(double *phys, const double *phys2, int nmodes, int my, int nz);

/* ---- rectangular / general-BC solver (temperature path) --------------- */
/* One direction of pseudomaty_temp / pseudomatz_temp
 * (src/pseudomat_temp.f90:2-150, 152-320): D scaled by 1/s, D2 = D*D, the
 * interior block for the BC pair (b1 at -s, b2 at +s; 'd' or 'n'), its
 * eigen-decomposition and inverse.                                         */
typedef struct {
    int m;
    double s;
    char b1, b2;
    double *D, *D2;          /* m*m                                          */
    double *E, *P, *PM1;     /* n, n*n, n*n (n = m-2)                        */
    double *B;               /* n*n interior block                           */
} orc_dir;

int  orc_pseudomat_temp(int m, double s, char b1, char b2, orc_dir *d);
void orc_dir_free(orc_dir *d);

/* solvediag_temp(U,F,FT,...,xlambda,bcy,bcz), src/solvediag_temp.f90:1-84
 * with mod_term_FTy/z (:86-239) and edge_value_y/z (:241-351).  U is
 * (my,mz) real; bcy (mz,2), bcz (my,2) wall values (NULL = zero).  The
 * reference has no rule for the singular n/n mode at lambda = 0 (its guard
 * abs(den).eq.1e-12 never fires, src/solvediag_temp.f90:52); this
 * restatement zeroes the eigen-coefficient of the smallest |Ey|+|Ez| pair
 * there (sing != 0), the gauge the CUDA path uses.                          */
int orc_solvediag_temp(double *U, const orc_dir *y, const orc_dir *z, double xlambda,
                       const double *bcy, const double *bcz, int sing);

/* helm3d_temp over modes ib..ie (src/helm3d_temp.f90:2-46,
 * src/int2d3d_temp.f90:51-88): the same real wall values bcy(:,:,i),
 * bcz(:,:,i) serve the real and the imaginary solve of mode i; mode 0 is
 * real.  bcy: (mz,2,nmodes), bcz: (my,2,nmodes), or NULL.                  */
int orc_helm3d_temp(const double *rhs, double *sol, int my, int mz, int ib, int ie,
                    const double *xalp, double alambda, const orc_dir *y, const orc_dir *z,
                    const double *bcy, const double *bcz, int nthreads);

/* ---- Shen-Legendre Galerkin solver (HELM_SHEN build) ------------------ */
/* preshen(bound) + makeMS + precomeigen (src/preshen.f90:2-535) and
 * leg_cheb_mat (src/legendre.f90:3-110) for m (odd) points, n = m-2:
 * b[m] basis coefficients, M, S [n*n] mass and stiffness (precomeigen),
 * E[n], P[n*n] generalized eigen-pairs of M x = E S x, PSM1 = P^-1 S^-1,
 * A [m*m] Chebyshev -> Legendre, B = A^-1.                                 */
typedef struct {
    int m;
    char bound;
    double *b, *M, *S, *E, *P, *PSM1, *A, *B;
} orc_shen;

int    orc_shen_setup(int m, char bound, orc_shen *s);
void   orc_shen_free(orc_shen *s);
/* largest parity-mixing entry the reference's even/odd split drops, relative */
double orc_shen_parity_leak(const orc_shen *s);
/* solveshen on one real (m,m) plane of Chebyshev coefficients, in place
 * (src/solveshen.f90:5-94 with src/legendre.f90:195-660, :96-546).       */
int    orc_solveshen(double *U, const orc_shen *s, double xlambda);
/* helm3d_shen over modes ib..ie (src/helm_shen.f90:2-85): rhs (physical)
 * is transformed to Chebyshev coefficients in place, like the reference. */
int    orc_helm3d_shen(double *rhs, double *sol, int my, int mz, int ib, int ie,
                       const double *xalp, double alambda, const orc_shen *s, int nthreads);

/* ---- Galerkin-basis Neumann (pressure) solver, pseudopois/solvepois --- */
typedef struct {
    int m;
    double *EN, *PN, *PNM1;  /* n, n*n, n*n (n = m-2): eigen-pairs of B2 B^-1 */
    double *PNT;             /* n*n  B^-1 (basis coefficients from interior) */
    int iofzero;             /* 1-based, smallest |EN|                       */
    double wanted;
} orc_pois;
/* pseudopois(m), src/pseudopois.f90:2-104.                                 */
int  orc_pseudopois(int m, orc_pois *p);
void orc_pois_free(orc_pois *p);
/* solvepois(U,F,FT,wk1,wk2,xlambda,m), src/solvepois.f90:1-170: U real
 * (m,m), interior in, solution with walls and corners out.                */
int  orc_solvepois(double *U, const orc_pois *p, double xlambda);

/* precomp_mass_flow / impose_mass_flow, src/operators.F:2205-2344 (square
 * build).  premassfu: (my,my,mrk) real, premassf: mrk.                     */
int    orc_precomp_mass_flow(const orc_ops *o, double dtp, const double *alphak, int mrk,
                             double fnu, double aspect, double *premassfu, double *premassf);
double orc_impose_mass_flow(double *csum, int krk, double *u, int my, int mz, double aspect,
                            const double *premassfu, const double *premassf, int iflag);

void orc_set_blas_threads(int n);

#ifdef __cplusplus
}
#endif

/* ---- DNS time step around the solve (duct_oracle_dns.c) ---------------- */
/* Statistics of one step (src/operators.F:1608-2004, 676-973).            */
typedef struct {
    double *mean;       /* 4 my mz: um, vm, wm, pm (x-means, accumulated)   */
    double *prod;       /* 6 my mz: uub, vvb, wwb, uvb, uwb, vwb            */
    double *ppb;        /* my mz                                            */
    double *spec;       /* 4 x 7 x M streamwise spectra at (jinco, kinco)    */
    double stress4[4];  /* wallstressx of the step's u                      */
    double energy[3], energy2[3];   /* energy_fou of u, v, w               */
    int nstat;
    /* vorticity diagnostics (src/main1.f90:453-466); om2 NULL: not gathered */
    double *om2;        /* 3 my mz: omx2, omy2, omz2 (statistics_omg2_fou)   */
    double omg[16];     /* the step's energomx4[5], energomxb4[5], energy_fou
                           of om_x, om_y, om_z, the same with mode 0         */
    double cfl2[2];     /* the step's remx (determine_step), slipmx          */
} orc_dns_stats;

void orc_fourx(double *fou, double *phys, int mx1, int mgalx, int my, int nz, int iopt);
void orc_derivx(const double *u, double *du, int my, int mz, int nmodes, const double *xalp, int ider,
                double scal, char what);
void orc_chx2z(double *f, int my, int mz, int M);
void orc_chz2x(double *f, int my, int mz, int M);
void orc_advection3d(const double *u, const double *v, const double *w, double *adv1, double *adv2,
                     double *adv3, int my, int mz, int M, int mgalx, const double *xalp, double aspect,
                     double *stats2);
void orc_vorticity(double *u, double *v, double *w, double *vort, double *tmp, int my, int mz, int M,
                   const double *xalp, double aspect, int iflag);
void orc_statistics_omg2_fou(const double *fou, int my, int mz, int M, double *om2);
void orc_energy_fou_zero_sector(const double *u, int my, int mz, double aspect, double energy[5]);
void orc_integral_abs_zero_sector(const double *u, int my, int mz, double aspect, double energy[5]);
void orc_advection3d_ex(const double *u, const double *v, const double *w, double *adv1, double *adv2,
                        double *adv3, int my, int mz, int M, int mgalx, const double *xalp, double aspect,
                        double *stats2, double *cfl2);
void orc_laplacian3d(double *u, double *flap, int my, int mz, int M, const double *xalp, double aspect,
                     double scal, char what);
void orc_grad3d(double *u, double *dxu, double *dyu, double *dzu, int my, int mz, int M, const double *xalp,
                double aspect, double scal, char what);
void orc_div3d(const double *u, double *v, double *w, double *div, int my, int mz, int M, const double *xalp,
               double aspect, double scal);
void orc_update_uvwp(double *u, double *v, double *w, double *p, double *phi, double *rhsphi, int my, int mz,
                     int M, const double *xalp, double aspect, double akk, double bkk, double dt, double fnu);
double orc_max_3din(const double *u, int my, int mz, int M);
void orc_wallstressx(const double *u, int my, int mz, double aspect, double stress4[4]);
void orc_energy_fou(const double *u, int my, int mz, int M, double aspect, double *energy, double *energy2);
void orc_statistics_fou(const double *u, const double *v, const double *w, const double *p, int my, int mz,
                        int M, double *mean, double *ppb, double *spec);
void orc_rk_coefficients(double *a, double *b, double *g, double *r);
double orc_dns_substep(double *u, double *v, double *w, double *p, double *adv1, double *adv2, double *adv3,
                       double *h1, double *h2, double *h3, int my, int mz, int M, int mgalx, const double *xalp,
                       double aspect, double fnu, double dt, int krk, const orc_ops *ops, int cmassflow,
                       double csum, const double *premassfu, const double *premassf, double dpdx,
                       orc_dns_stats *stats, int nthreads, const double *force);

#endif
