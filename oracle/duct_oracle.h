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
 * (src/operators.F:2496-2507, "-(dyy+dzz)U=dpval -> max(U)=1") and the
 * laminar mass flow CMASSFLOW=1.92783343620839 (utils/gen_tsd2hdf5.py:10) --
 * and by exact manufactured polynomial solutions.  Parity is therefore
 * "partially pinned": known answers, not reference outputs.
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
/* Same, but the Neumann block/eigen solve is skipped when want_neumann=0.   */
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

void orc_set_blas_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
