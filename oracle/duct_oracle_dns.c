/*
 * duct_oracle_dns.c -- CPU FP64 restatement of the duct DNS time step around
 * the 2D solve: the x-direction Fourier transform with 2/3 de-aliasing, the
 * advection products, the operators of the fractional-step RK3/CN substep,
 * and the statistics and wall diagnostics.
 *
 * TEST INFRASTRUCTURE ONLY (checker and CPU baseline).  Each function cites
 * the reference routine it restates, in the reference's order of
 * operations (including the in-place transyz round trips that leave their
 * input changed by rounding).  Two documented departures:
 *  * chz2x on one rank is the inverse of chx2z (the transpose back to the
 *    x-cut); the reference returns before its transpose when numerop = 1
 *    (src/parallel.F:132);
 *  * FFTW's r2c/c2r are restated from their definitions (orc_fft.h).
 * Layouts (complex interleaved, column-major):
 *  x-cut  fou(my, mz, 0:mx1)          (the reference's u(my,mz,ib:ie))
 *  z-cut  fou(0:mx1, my, mz)          (after chx2z)
 *  phys   fis(mgalx+2, my, mz) real   (the fourx work array)
 */
#include "duct_oracle.h"
#include "orc_fft.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define CPLX(a, i) ((a)[2 * (size_t)(i)])
#define CPLXI(a, i) ((a)[2 * (size_t)(i) + 1])

/* ---- fourx (src/fourier.F:1-68) with pack_fftw (:70-95) and fill (:97-118)
 * iopt >= 0: fou (z-cut) -> phys, the modes above mx1 zero-filled
 *            (fill), FFTW c2r (imaginary parts of the 0 and N/2 modes
 *            ignored, as FFTW does);
 * iopt < 0:  phys -> fou, FFTW r2c, modes 0..mx1 kept and scaled by 1/mgalx
 *            (pack_fftw).                                                    */
void orc_fourx(double *fou, double *phys, int mx1, int mgalx, int my, int nz, int iopt)
{
    const int N = mgalx, nl = my * nz, M = mx1 + 1;
    orc_fft_plan plan;
    orc_fft_plan_init(&plan, N);
#pragma omp parallel
    {
        double *a = (double *)malloc(sizeof(double) * 2 * (size_t)N);
        double *b = (double *)malloc(sizeof(double) * 2 * (size_t)N);
#pragma omp for
        for (int l = 0; l < nl; ++l) {
            double *f = fou + 2 * (size_t)l * M;
            double *x = phys + (size_t)l * (N + 2);
            if (iopt >= 0) {
                /* Hermitian spectrum of length N from modes 0..mx1 */
                memset(a, 0, sizeof(double) * 2 * (size_t)N);
                a[0] = f[0];                       /* Im of mode 0 ignored */
                for (int k = 1; k < M && k <= N / 2; ++k) {
                    if (2 * k == N) { a[2 * k] = f[2 * k]; continue; }   /* Nyquist: real */
                    a[2 * k] = f[2 * k];
                    a[2 * k + 1] = f[2 * k + 1];
                    a[2 * (N - k)] = f[2 * k];
                    a[2 * (N - k) + 1] = -f[2 * k + 1];
                }
                orc_fft(&plan, a, b, 1);
                for (int n = 0; n < N; ++n) x[n] = b[2 * n];
                x[N] = 0.0;
                x[N + 1] = 0.0;
            } else {
                for (int n = 0; n < N; ++n) { a[2 * n] = x[n]; a[2 * n + 1] = 0.0; }
                orc_fft(&plan, a, b, 0);
                const double sca = 1.0 / (double)N;
                for (int k = 0; k < M; ++k) {
                    f[2 * k] = sca * b[2 * k];
                    f[2 * k + 1] = sca * b[2 * k + 1];
                }
            }
        }
        free(a);
        free(b);
    }
    orc_fft_plan_free(&plan);
}

/* mult(ntot,u,v,s,'n','+'), src/mult.F:11-45 */
static void mult_nplus(long ntot, const double *u, const double *v, double *s)
{
#pragma omp parallel for
    for (long i = 0; i < ntot; ++i) s[i] = u[i] * v[i];
}

/* derivx(u,du,ider,scal,what), src/fourier.F:120-188: x-cut fields
 * (my,mz,nmodes); du = du? + cii*xalp*u*scal (ider 1) or -xalp^2*u*scal. */
void orc_derivx(const double *u, double *du, int my, int mz, int nmodes, const double *xalp, int ider,
                double scal, char what)
{
    const long pl = (long)my * mz;
#pragma omp parallel for
    for (int i = 0; i < nmodes; ++i) {
        const double a = xalp[i];
        for (long q = 0; q < pl; ++q) {
            const long e = (long)i * pl + q;
            const double ur = CPLX(u, e), ui = CPLXI(u, e);
            double dr, di;
            if (ider == 1) { dr = (-(a * ui)) * scal; di = (a * ur) * scal; }
            else { const double c = -(a * a); dr = (c * ur) * scal; di = (c * ui) * scal; }
            if (what == 'n') { CPLX(du, e) = dr; CPLXI(du, e) = di; }
            else { CPLX(du, e) += dr; CPLXI(du, e) += di; }
        }
    }
}

/* chx2z / chz2x on one rank (src/parallel.F:1-208): x-cut (my,mz,M) <->
 * z-cut (M,my,mz), in place through a temporary.                           */
void orc_chx2z(double *f, int my, int mz, int M)
{
    const size_t n = 2 * (size_t)my * mz * M;
    double *t = (double *)malloc(sizeof(double) * n);
    memcpy(t, f, sizeof(double) * n);
    orc_cyzx2xyz(f, t, M, my, mz);
    free(t);
}

void orc_chz2x(double *f, int my, int mz, int M)
{
    const size_t n = 2 * (size_t)my * mz * M;
    double *t = (double *)malloc(sizeof(double) * n);
    orc_cxyz2yzx(f, t, M, my, mz);
    memcpy(f, t, sizeof(double) * n);
    free(t);
}

static void daxpy_(long n, double a, const double *x, double *y)
{
#pragma omp parallel for
    for (long i = 0; i < n; ++i) y[i] = y[i] + a * x[i];
}

/* y = x + d/dcdir(x) composite of the reference: transyz(x,cdir,-1),
 * derivyz(x,out,cdir,ider,scal,'n'), transyz(out,cdir,+1), transyz(x,cdir,+1)
 * (x restored up to rounding, as in the reference). */
static void dphys(double *x, double *out, int my, int mz, int M, char cdir, int ider, double scal, double aspect,
                  int restore)
{
    orc_transyz(x, my, mz, M, cdir, -1);
    orc_derivyz(x, out, my, mz, M, cdir, ider, scal, 'n', aspect);
    orc_transyz(out, my, mz, M, cdir, 1);
    if (restore) orc_transyz(x, my, mz, M, cdir, 1);
}

/* advection3d(u,v,w,adv1,adv2,adv3,...), src/operators.F:9-276, on x-cut
 * fields.  stats2 (6 my mz, or NULL): statistics_fou2 (src/operators.F:
 * 1957-2004) of the six products, the x-mean (mode-0 real part) added to
 * uub, vvb, wwb, uvb, uwb, vwb.                                             */
static void cfl_slip(const double *ufis, const double *vfis, const double *wfis, int my, int mz, int mgalx,
                     double alp, double aspect, double *cfl2);

void orc_advection3d(const double *u, const double *v, const double *w, double *adv1, double *adv2, double *adv3,
                     int my, int mz, int M, int mgalx, const double *xalp, double aspect, double *stats2)
{
    orc_advection3d_ex(u, v, w, adv1, adv2, adv3, my, mz, M, mgalx, xalp, aspect, stats2, NULL);
}

/* advection3d with, when cfl2 is not NULL, its first-substep checks on the
 * physical velocities (src/operators.F:71-75): cfl2[0] = the remx of
 * determine_step, cfl2[1] = the slipmx of slip_velocity_3d. */
void orc_advection3d_ex(const double *u, const double *v, const double *w, double *adv1, double *adv2, double *adv3,
                        int my, int mz, int M, int mgalx, const double *xalp, double aspect, double *stats2,
                        double *cfl2)
{
    const size_t nf = 2 * (size_t)my * mz * M;        /* doubles of a fou field */
    const size_t ns = (size_t)(mgalx + 2) * my * mz;   /* doubles of a fis field */
    const long pl = (long)my * mz;
    double *tmp1 = (double *)malloc(sizeof(double) * ns);
    double *ufis = (double *)malloc(sizeof(double) * ns);
    double *vfis = (double *)malloc(sizeof(double) * ns);
    double *wfis = (double *)malloc(sizeof(double) * ns);
    double *tmp2 = (double *)calloc(nf, sizeof(double));
    double *tmp3 = (double *)calloc(nf, sizeof(double));
    double *tq = (double *)calloc(nf, sizeof(double));
    memcpy(adv1, u, sizeof(double) * nf);
    memcpy(adv2, v, sizeof(double) * nf);
    memcpy(adv3, w, sizeof(double) * nf);
    orc_chx2z(adv1, my, mz, M);
    orc_chx2z(adv2, my, mz, M);
    orc_chx2z(adv3, my, mz, M);
    orc_fourx(adv1, ufis, M - 1, mgalx, my, mz, 1);
    orc_fourx(adv2, vfis, M - 1, mgalx, my, mz, 1);
    orc_fourx(adv3, wfis, M - 1, mgalx, my, mz, 1);
    if (cfl2) cfl_slip(ufis, vfis, wfis, my, mz, mgalx, M > 1 ? xalp[1] : 0.0, aspect, cfl2);
#define STAT2(f, s)                                                                  \
    if (stats2)                                                                      \
        for (long q = 0; q < pl; ++q) stats2[(size_t)(s) * pl + q] += (f)[2 * q];
    /* (1) u*u -> d/dx -> adv1 */
    mult_nplus((long)ns, ufis, ufis, tmp1);
    orc_fourx(adv1, tmp1, M - 1, mgalx, my, mz, -1);
    orc_chz2x(adv1, my, mz, M);
    STAT2(adv1, 0);
    orc_derivx(adv1, adv1, my, mz, M, xalp, 1, 1.0, 'n');
    /* (2) v*v -> d/dy -> adv2 */
    mult_nplus((long)ns, vfis, vfis, tmp1);
    orc_fourx(adv2, tmp1, M - 1, mgalx, my, mz, -1);
    orc_chz2x(adv2, my, mz, M);
    STAT2(adv2, 1);
    dphys(adv2, tmp2, my, mz, M, 'y', 1, 1.0, aspect, 0);
    memcpy(adv2, tmp2, sizeof(double) * nf);
    /* (3) w*w -> d/dz -> adv3 */
    mult_nplus((long)ns, wfis, wfis, tmp1);
    orc_fourx(adv3, tmp1, M - 1, mgalx, my, mz, -1);
    orc_chz2x(adv3, my, mz, M);
    STAT2(adv3, 2);
    dphys(adv3, tmp2, my, mz, M, 'z', 1, 1.0, aspect, 0);
    memcpy(adv3, tmp2, sizeof(double) * nf);
    /* (4) u*v: d/dx -> ++adv2, d/dy -> ++adv1 */
    mult_nplus((long)ns, ufis, vfis, tmp1);
    orc_fourx(tmp2, tmp1, M - 1, mgalx, my, mz, -1);
    orc_chz2x(tmp2, my, mz, M);
    STAT2(tmp2, 3);
    orc_derivx(tmp2, adv2, my, mz, M, xalp, 1, 1.0, '+');
    dphys(tmp2, tq, my, mz, M, 'y', 1, 1.0, aspect, 0);
    daxpy_((long)nf, 1.0, tq, adv1);
    /* (5) u*w: d/dx -> ++adv3, d/dz -> ++adv1 */
    mult_nplus((long)ns, ufis, wfis, tmp1);
    orc_fourx(tmp2, tmp1, M - 1, mgalx, my, mz, -1);
    orc_chz2x(tmp2, my, mz, M);
    STAT2(tmp2, 4);
    orc_derivx(tmp2, adv3, my, mz, M, xalp, 1, 1.0, '+');
    dphys(tmp2, tq, my, mz, M, 'z', 1, 1.0, aspect, 0);
    daxpy_((long)nf, 1.0, tq, adv1);
    /* (6) v*w: d/dy -> ++adv3, d/dz -> ++adv2 */
    mult_nplus((long)ns, vfis, wfis, tmp1);
    orc_fourx(tmp2, tmp1, M - 1, mgalx, my, mz, -1);
    orc_chz2x(tmp2, my, mz, M);
    STAT2(tmp2, 5);
    memcpy(tmp3, tmp2, sizeof(double) * nf);
    dphys(tmp2, tq, my, mz, M, 'y', 1, 1.0, aspect, 0);
    daxpy_((long)nf, 1.0, tq, adv3);
    dphys(tmp3, tq, my, mz, M, 'z', 1, 1.0, aspect, 0);
    daxpy_((long)nf, 1.0, tq, adv2);
#undef STAT2
    free(tmp1); free(ufis); free(vfis); free(wfis); free(tmp2); free(tmp3); free(tq);
}

/* laplacian3d(u,flap,tmp,tmpyz,scal,what), src/operators.F:278-347.  u is
 * transformed in place and back (changed by rounding, as in the reference). */
void orc_laplacian3d(double *u, double *flap, int my, int mz, int M, const double *xalp, double aspect,
                     double scal, char what)
{
    const size_t nf = 2 * (size_t)my * mz * M;
    double *tmp = (double *)malloc(sizeof(double) * nf);
    orc_derivx(u, flap, my, mz, M, xalp, 2, scal, what);
    dphys(u, tmp, my, mz, M, 'y', 2, scal, aspect, 1);
    daxpy_((long)nf, 1.0, tmp, flap);
    dphys(u, tmp, my, mz, M, 'z', 2, scal, aspect, 1);
    daxpy_((long)nf, 1.0, tmp, flap);
    free(tmp);
}

/* grad3d(u,dxu,dyu,dzu,tmp,tmpyz,scal,what), src/operators.F:349-425. */
void orc_grad3d(double *u, double *dxu, double *dyu, double *dzu, int my, int mz, int M, const double *xalp,
                double aspect, double scal, char what)
{
    const size_t nf = 2 * (size_t)my * mz * M;
    double *tmp = (double *)malloc(sizeof(double) * nf);
    orc_derivx(u, dxu, my, mz, M, xalp, 1, scal, what);
    dphys(u, tmp, my, mz, M, 'y', 1, scal, aspect, 1);
    if (what == 'n') memcpy(dyu, tmp, sizeof(double) * nf);
    else daxpy_((long)nf, 1.0, tmp, dyu);
    dphys(u, tmp, my, mz, M, 'z', 1, scal, aspect, 1);
    if (what == 'n') memcpy(dzu, tmp, sizeof(double) * nf);
    else daxpy_((long)nf, 1.0, tmp, dzu);
    free(tmp);
}

/* div3d(u,v,w,div,tmp,tmpyz,scal), src/operators.F:427-501 (v, w
 * transformed in place and back). */
void orc_div3d(const double *u, double *v, double *w, double *div, int my, int mz, int M, const double *xalp,
               double aspect, double scal)
{
    const size_t nf = 2 * (size_t)my * mz * M;
    double *tmp = (double *)malloc(sizeof(double) * nf);
    orc_derivx(u, div, my, mz, M, xalp, 1, scal, 'n');
    dphys(v, tmp, my, mz, M, 'y', 1, scal, aspect, 1);
    daxpy_((long)nf, 1.0, tmp, div);
    dphys(w, tmp, my, mz, M, 'z', 1, scal, aspect, 1);
    daxpy_((long)nf, 1.0, tmp, div);
    free(tmp);
}

/* update_uvwp(u,v,w,p,phi,rhsphi,tmp,tmpyz,akk,bkk), src/operators.F:503-605
 * (no FILTER): p += phi - (akk+bkk) dt nu lap(phi); u -= dt (akk+bkk) grad
 * phi.  phi is left in Chebyshev-z space (the reference skips the last
 * back transform), rhsphi overwritten. */
void orc_update_uvwp(double *u, double *v, double *w, double *p, double *phi, double *rhsphi, int my, int mz,
                     int M, const double *xalp, double aspect, double akk, double bkk, double dt, double fnu)
{
    const size_t nf = 2 * (size_t)my * mz * M;
    double *tmp = (double *)malloc(sizeof(double) * nf);
    double scal = (akk + bkk) * dt * fnu;
    orc_laplacian3d(phi, rhsphi, my, mz, M, xalp, aspect, scal, 'n');
    for (size_t i = 0; i < nf; ++i) p[i] = p[i] + phi[i] - rhsphi[i];
    scal = -dt * (akk + bkk);
    orc_derivx(phi, u, my, mz, M, xalp, 1, scal, '+');
    dphys(phi, tmp, my, mz, M, 'y', 1, scal, aspect, 1);
    daxpy_((long)nf, 1.0, tmp, v);
    dphys(phi, tmp, my, mz, M, 'z', 1, scal, aspect, 0);
    daxpy_((long)nf, 1.0, tmp, w);
    free(tmp);
}

/* max_3din(u,divmax), src/operators.F:2524-2550: max |u| over the interior. */
double orc_max_3din(const double *u, int my, int mz, int M)
{
    double fmax = -1.0e300;
    for (int i = 0; i < M; ++i)
        for (int k = 1; k < mz - 1; ++k)
            for (int j = 1; j < my - 1; ++j) {
                const size_t e = (size_t)j + (size_t)my * (k + (size_t)mz * i);
                const double a = hypot(CPLX(u, e), CPLXI(u, e));
                if (a > fmax) fmax = a;
            }
    return fmax;
}

/* cheb2_wallstress_circum(u,1,aspect,sum,ny,nz), src/chebyshev.f90:642-690,
 * of a real (ny,nz) plane of Chebyshev coefficients.                       */
static void cheb2_wallstress_circum(const double *u, double aspect, double sum[4], int ny, int nz)
{
    for (int i = 0; i < 4; ++i) sum[i] = 0.0;
    for (int k = 0; k < nz; k += 2)
        for (int j = 0; j < ny; ++j) {
            const double c = u[j + (size_t)ny * k];
            const double f = 2.0 * aspect * (double)(j * j) / (double)(k * k - 1);
            sum[0] = sum[0] - c * f;
            sum[1] = sum[1] + c * (((j + 1) & 1) ? -1.0 : 1.0) * f;
        }
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; j += 2) {
            const double c = u[j + (size_t)ny * k];
            const double f = 2.0 / aspect * (double)(k * k) / (double)(j * j - 1);
            sum[2] = sum[2] - c * f;
            sum[3] = sum[3] + c * (((k + 1) & 1) ? -1.0 : 1.0) * f;
        }
    for (int i = 0; i < 4; ++i) sum[i] = sum[i] / (4.0 + 4.0 * aspect);
}

/* wallstressx(u,tmpyz,stress4), src/operators.F:676-710: the wall stress of
 * the x-mean (mode-0 real part) of u, per wall. */
void orc_wallstressx(const double *u, int my, int mz, double aspect, double stress4[4])
{
    double *t = (double *)malloc(sizeof(double) * (size_t)my * mz);
    for (long q = 0; q < (long)my * mz; ++q) t[q] = u[2 * q];
    orc_transyz_plane(t, my, mz, -1);
    cheb2_wallstress_circum(t, aspect, stress4, my, mz);
    free(t);
}

/* Mesh-size weights of src/ininewc.f90:102-112 on the nodes x (n points). */
static void mesh_weights(const double *x, int n, double *d)
{
    d[0] = (x[1] - x[0]) * 0.5;
    for (int j = 1; j < n - 1; ++j) d[j] = (x[j + 1] - x[j - 1]) * 0.5;
    d[n - 1] = (x[n - 1] - x[n - 2]) * 0.5;
}

static void cgl_nodes(int n, double s, double *x)
{
    const double pi = 4.0 * atan(1.0);
    for (int j = 0; j < n; ++j) x[j] = -s * cos(pi * (double)j / (double)(n - 1));
}

/* determine_step (src/operators.F:608-672): remx = max over the physical
 * points of |u| alp mgalx/(2 pi), |v|/dy, |w|/dz; slip_velocity_3d
 * (2552-2608): the largest u, v or w on the y = +-1 and z = +-aspect walls.
 * Physical fields (mgalx+2, my, mz), points i < mgalx. */
static void cfl_slip(const double *ufis, const double *vfis, const double *wfis, int my, int mz, int mgalx,
                     double alp, double aspect, double *cfl2)
{
    const double pi = 4.0 * atan(1.0);
    double *y = (double *)malloc(sizeof(double) * my), *z = (double *)malloc(sizeof(double) * mz);
    double *dy = (double *)malloc(sizeof(double) * my), *dz = (double *)malloc(sizeof(double) * mz);
    cgl_nodes(my, 1.0, y);
    cgl_nodes(mz, aspect, z);
    mesh_weights(y, my, dy);
    mesh_weights(z, mz, dz);
    const double hxalp = alp * (double)mgalx / (2.0 * pi);
    double reig = 0.0, fmx = -1.0e308;
    for (int k = 0; k < mz; ++k)
        for (int j = 0; j < my; ++j) {
            const size_t o = (size_t)(mgalx + 2) * (j + (size_t)my * k);
            const int wall = (j == 0 || j == my - 1 || k == 0 || k == mz - 1);
            for (int i = 0; i < mgalx; ++i) {
                const double uu = ufis[o + i], vv = vfis[o + i], ww = wfis[o + i];
                reig = fmax(reig, fabs(uu * hxalp));
                reig = fmax(reig, fabs(vv / dy[j]));
                reig = fmax(reig, fabs(ww / dz[k]));
                if (wall) fmx = fmax(fmx, fmax(uu, fmax(vv, ww)));
            }
        }
    cfl2[0] = reig;
    cfl2[1] = fmx;
    free(y); free(z); free(dy); free(dz);
}

/* energy_fou(u,energy,energy2), src/operators.F:907-973 (one rank):
 * energy = sqrt(sum_{i>=1} 2|u_i|^2 dy dz / area), energy2 with mode 0. */
void orc_energy_fou(const double *u, int my, int mz, int M, double aspect, double *energy, double *energy2)
{
    double *y = (double *)malloc(sizeof(double) * my), *z = (double *)malloc(sizeof(double) * mz);
    double *dy = (double *)malloc(sizeof(double) * my), *dz = (double *)malloc(sizeof(double) * mz);
    cgl_nodes(my, 1.0, y);
    cgl_nodes(mz, aspect, z);
    mesh_weights(y, my, dy);
    mesh_weights(z, mz, dz);
    double e = 0.0, e2 = 0.0;
    for (int k = 0; k < mz; ++k)
        for (int j = 0; j < my; ++j) {
            double ue = 0.0;
            for (int i = 1; i < M; ++i) {
                const size_t q = (size_t)j + (size_t)my * (k + (size_t)mz * i);
                ue = ue + (CPLX(u, q) * CPLX(u, q) + CPLXI(u, q) * CPLXI(u, q)) * 2.0;
            }
            e = e + ue * dy[j] * dz[k];
        }
    for (int k = 0; k < mz; ++k)
        for (int j = 0; j < my; ++j) {
            const size_t q = (size_t)j + (size_t)my * k;
            e2 = e2 + (CPLX(u, q) * CPLX(u, q) + CPLXI(u, q) * CPLXI(u, q)) * dy[j] * dz[k];
        }
    const double area = 4.0 * aspect;
    *energy = sqrt(e / area);
    *energy2 = sqrt((e + e2) / area);
    free(y); free(z); free(dy); free(dz);
}

/* vorticity(u,v,w,vort,tmp,iflag), src/operators.F:810-905: om_x = w,y -
 * v,z (1), om_y = u,z - w,x (2), om_z = v,x - u,y (3), with the reference's
 * transyz / derivyz / transyz sequence (u, v, w go through its in-place
 * round trips, so they come back to rounding, as there). */
void orc_vorticity(double *u, double *v, double *w, double *vort, double *tmp, int my, int mz, int M,
                   const double *xalp, double aspect, int iflag)
{
    const long n = 2L * my * mz * M;
    if (iflag == 1) {
        dphys(w, vort, my, mz, M, 'y', 1, 1.0, aspect, 1);
        dphys(v, tmp, my, mz, M, 'z', 1, 1.0, aspect, 1);
    } else if (iflag == 2) {
        dphys(u, vort, my, mz, M, 'z', 1, 1.0, aspect, 1);
        orc_derivx(w, tmp, my, mz, M, xalp, 1, 1.0, 'n');
    } else {
        orc_derivx(v, vort, my, mz, M, xalp, 1, 1.0, 'n');
        dphys(u, tmp, my, mz, M, 'y', 1, 1.0, aspect, 1);
    }
    daxpy_(n, -1.0, tmp, vort);
}

/* statistics_omg2_fou(fou,iflag), src/operators.F:1859-1955 (one rank):
 * om2[my mz] += |fou_0|^2 + sum_{i>=1} 2 |fou_i|^2 (mode 0 first, as there). */
void orc_statistics_omg2_fou(const double *fou, int my, int mz, int M, double *om2)
{
    const long pl = (long)my * mz;
    for (long q = 0; q < pl; ++q) om2[q] = om2[q] + (CPLX(fou, q) * CPLX(fou, q) + CPLXI(fou, q) * CPLXI(fou, q));
    for (int i = 1; i < M; ++i)
        for (long q = 0; q < pl; ++q) {
            const size_t e = (size_t)i * pl + q;
            om2[q] = om2[q] + (CPLX(fou, e) * CPLX(fou, e) + CPLXI(fou, e) * CPLXI(fou, e)) * 2.0;
        }
}

/* The sector of point (j, k), 1-based, of energy_fou_zero_sector and
 * integral_abs_zero_sector (0-based sector index; 4 = on a diagonal). */
static int zero_sector(int j, int k, int mz)
{
    if (j < k && j < mz + 1 - k) return 0;
    if (j < k && j > mz + 1 - k) return 1;
    if (j > k && j > mz + 1 - k) return 2;
    if (j > k && j < mz + 1 - k) return 3;
    return 4;
}

/* energy_fou_zero_sector(u,energy), src/operators.F:1018-1099 (one rank):
 * energy[s] = sum over sector s of |u_0|^2 dy dz / area. */
void orc_energy_fou_zero_sector(const double *u, int my, int mz, double aspect, double energy[5])
{
    double *y = (double *)malloc(sizeof(double) * my), *z = (double *)malloc(sizeof(double) * mz);
    double *dy = (double *)malloc(sizeof(double) * my), *dz = (double *)malloc(sizeof(double) * mz);
    cgl_nodes(my, 1.0, y);
    cgl_nodes(mz, aspect, z);
    mesh_weights(y, my, dy);
    mesh_weights(z, mz, dz);
    for (int s = 0; s < 5; ++s) energy[s] = 0.0;
    for (int k = 1; k <= mz; ++k)
        for (int j = 1; j <= my; ++j) {
            const size_t q = (size_t)(j - 1) + (size_t)my * (k - 1);
            const double ue = CPLX(u, q) * CPLX(u, q) + CPLXI(u, q) * CPLXI(u, q);
            const int s = zero_sector(j, k, mz);
            energy[s] = energy[s] + ue * dy[j - 1] * dz[k - 1];
        }
    for (int s = 0; s < 5; ++s) energy[s] = energy[s] / (4.0 * aspect);
    free(y); free(z); free(dy); free(dz);
}

/* integral_abs_zero_sector(u,energy), src/operators.F:1462-1541 (one rank):
 * energy[s] = sum over sector s of |Re u_0| dy dz / area. */
void orc_integral_abs_zero_sector(const double *u, int my, int mz, double aspect, double energy[5])
{
    double *y = (double *)malloc(sizeof(double) * my), *z = (double *)malloc(sizeof(double) * mz);
    double *dy = (double *)malloc(sizeof(double) * my), *dz = (double *)malloc(sizeof(double) * mz);
    cgl_nodes(my, 1.0, y);
    cgl_nodes(mz, aspect, z);
    mesh_weights(y, my, dy);
    mesh_weights(z, mz, dz);
    for (int s = 0; s < 5; ++s) energy[s] = 0.0;
    for (int k = 1; k <= mz; ++k)
        for (int j = 1; j <= my; ++j) {
            const size_t q = (size_t)(j - 1) + (size_t)my * (k - 1);
            const int s = zero_sector(j, k, mz);
            energy[s] = energy[s] + fabs(CPLX(u, q)) * dy[j - 1] * dz[k - 1];
        }
    for (int s = 0; s < 5; ++s) energy[s] = energy[s] / (4.0 * aspect);
    free(y); free(z); free(dy); free(dz);
}

/* statistics_fou(u,v,w,p,1), src/operators.F:1608-1765 (one rank):
 * mean[4 my mz] += mode-0 real parts of u, v, w, p; ppb[my mz] += the
 * x-mean of p^2 (|p_0|^2 + sum 2|p_i|^2); spec[4][7][M] += the streamwise
 * spectra of u, v, w, p at the seven points (jinco, kinco). */
void orc_statistics_fou(const double *u, const double *v, const double *w, const double *p, int my, int mz, int M,
                        double *mean, double *ppb, double *spec)
{
    const long pl = (long)my * mz;
    const double *f[4] = {u, v, w, p};
    for (int c = 0; c < 4; ++c)
        for (long q = 0; q < pl; ++q) mean[c * pl + q] += f[c][2 * q];
    for (int i = 1; i < M; ++i)
        for (long q = 0; q < pl; ++q) {
            const size_t e = (size_t)i * pl + q;
            ppb[q] = ppb[q] + (CPLX(p, e) * CPLX(p, e) + CPLXI(p, e) * CPLXI(p, e)) * 2.0;
        }
    for (long q = 0; q < pl; ++q) ppb[q] = ppb[q] + (CPLX(p, q) * CPLX(p, q) + CPLXI(p, q) * CPLXI(p, q));
    const int jin[7] = {my / 16, my / 8, my / 4, my / 2, my / 16, my / 8, my / 4};
    const int kin[7] = {mz / 2, mz / 2, mz / 2, mz / 2, mz / 16, mz / 8, mz / 4};
    for (int c = 0; c < 4; ++c)
        for (int s = 0; s < 7; ++s) {
            const long q = (long)(jin[s] - 1) + (long)my * (kin[s] - 1);   /* 1-based indices */
            for (int i = 0; i < M; ++i) {
                const size_t e = (size_t)i * pl + q;
                const double a = CPLX(f[c], e) * CPLX(f[c], e) + CPLXI(f[c], e) * CPLXI(f[c], e);
                spec[((size_t)c * 7 + s) * M + i] += (i == 0) ? a : a * 2.0;
            }
        }
}

/* ---- one RK3/CN substep of src/main1.f90:384-723 --------------------- */
/* Runge-Kutta coefficients, src/mod.f90:52-55 */
static const double akkc[3] = {29.0 / 96.0, -3.0 / 40.0, 1.0 / 6.0};
static const double bkkc[3] = {37.0 / 160.0, 5.0 / 24.0, 1.0 / 6.0};
static const double gkkc[3] = {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};
static const double rkkc[3] = {0.0, -17.0 / 60.0, -5.0 / 12.0};

void orc_rk_coefficients(double *a, double *b, double *g, double *r)
{
    for (int i = 0; i < 3; ++i) { a[i] = akkc[i]; b[i] = bkkc[i]; g[i] = gkkc[i]; r[i] = rkkc[i]; }
}

/* The substep krk (1..3) on the state: velocities u, v, w, pressure p,
 * advection terms adv[3] (kept from the previous substep), work h[3]
 * (x-cut, complex (my,mz,M) each).  cmassflow: 1 imposes the flow rate
 * *csum with premassfu / premassf (CMASSFLOW build), 0 adds the mean
 * pressure gradient dpdx to mode 0 of the x-momentum (icase 1).  stats
 * (NULL or the accumulators, see orc_dns_stats) gathers the statistics of
 * the step at krk = 1.  Returns the divergence max_3din after the update. */
double orc_dns_substep(double *u, double *v, double *w, double *p, double *adv1, double *adv2, double *adv3,
                       double *h1, double *h2, double *h3, int my, int mz, int M, int mgalx, const double *xalp,
                       double aspect, double fnu, double dt, int krk, const orc_ops *ops, int cmassflow,
                       double csum, const double *premassfu, const double *premassf, double dpdx,
                       orc_dns_stats *stats, int nthreads, const double *force)
{
    const size_t nf = 2 * (size_t)my * mz * M;
    const int k = krk - 1;
    double *adv[3] = {adv1, adv2, adv3}, *h[3] = {h1, h2, h3}, *vel[3] = {u, v, w};
    /* (i) h = -rho_k adv(u^{k-2}) */
    for (int c = 0; c < 3; ++c) {
        if (krk > 1) {
            const double s = -rkkc[k];
            for (size_t i = 0; i < nf; ++i) h[c][i] = adv[c][i] * s;
        } else {
            memset(h[c], 0, sizeof(double) * nf);
        }
    }
    /* (ii) adv(u^{k-1}) */
    orc_advection3d_ex(u, v, w, adv1, adv2, adv3, my, mz, M, mgalx, xalp, aspect,
                       (stats && krk == 1) ? stats->prod : NULL, (stats && krk == 1) ? stats->cfl2 : NULL);
    if (stats && krk == 1) {
        orc_wallstressx(u, my, mz, aspect, stats->stress4);
        orc_energy_fou(u, my, mz, M, aspect, &stats->energy[0], &stats->energy2[0]);
        orc_energy_fou(v, my, mz, M, aspect, &stats->energy[1], &stats->energy2[1]);
        orc_energy_fou(w, my, mz, M, aspect, &stats->energy[2], &stats->energy2[2]);
        if (stats->om2) {
            /* src/main1.f90:453-466: each vorticity component, its second
             * moments and energies; the zero-mode sectors of om_x */
            double *vort = (double *)malloc(sizeof(double) * nf), *tmp = (double *)malloc(sizeof(double) * nf);
            const size_t pl = (size_t)my * mz;
            for (int c = 0; c < 3; ++c) {
                orc_vorticity(u, v, w, vort, tmp, my, mz, M, xalp, aspect, c + 1);
                orc_statistics_omg2_fou(vort, my, mz, M, stats->om2 + c * pl);
                orc_energy_fou(vort, my, mz, M, aspect, &stats->omg[10 + c], &stats->omg[13 + c]);
                if (c == 0) {
                    orc_energy_fou_zero_sector(vort, my, mz, aspect, stats->omg);
                    orc_integral_abs_zero_sector(vort, my, mz, aspect, stats->omg + 5);
                }
            }
            free(vort);
            free(tmp);
        }
        orc_statistics_fou(u, v, w, p, my, mz, M, stats->mean, stats->ppb, stats->spec);
        stats->nstat += 1;
    }
    /* (iii) h += -gamma_k adv */
    for (int c = 0; c < 3; ++c) daxpy_((long)nf, -gkkc[k], adv[c], h[c]);
    /* (iv) h += alpha_k nu lap(u) */
    for (int c = 0; c < 3; ++c) orc_laplacian3d(vel[c], h[c], my, mz, M, xalp, aspect, fnu * akkc[k], '+');
    /* (v) h += u / dt */
    for (int c = 0; c < 3; ++c) daxpy_((long)nf, 1.0 / dt, vel[c], h[c]);
    /* (vi) h += -(alpha_k + beta_k) grad p */
    orc_grad3d(p, h1, h2, h3, my, mz, M, xalp, aspect, -(akkc[k] + bkkc[k]), '+');
    /* (vi-b) a body force f (3 fields, or NULL) enters like the pressure
     * gradient and the reference's forcings (force_global / add_puff_forcing
     * with scale -(akk+bkk)): h += (akk+bkk) f */
    if (force)
        for (int c = 0; c < 3; ++c) daxpy_((long)nf, akkc[k] + bkkc[k], force + (size_t)c * nf, h[c]);
    /* (vi-b) mean pressure gradient on mode 0 of x-momentum (not CMASSFLOW) */
    if (!cmassflow) {
        const double t = -(akkc[k] + bkkc[k]) * dpdx;
        for (long q = 0; q < (long)my * mz; ++q) h1[2 * q] = h1[2 * q] + 1.0 * t;
    }
    /* (vii) h *= -1/(nu beta_k) */
    for (int c = 0; c < 3; ++c) {
        const double s = -1.0 / (fnu * bkkc[k]);
        for (size_t i = 0; i < nf; ++i) h[c][i] = h[c][i] * s;
    }
    /* (viii) predictor: helm3d 'd' with helco = 1/(beta_k nu dt) */
    const double helco = 1.0 / (bkkc[k] * fnu * dt);
    for (int c = 0; c < 3; ++c) orc_helm3d(h[c], vel[c], my, mz, 0, M - 1, xalp, 'd', helco, ops, nthreads);
    /* (ix) rhs of the pseudo-pressure */
    orc_div3d(u, v, w, h1, my, mz, M, xalp, aspect, 1.0 / ((akkc[k] + bkkc[k]) * dt));
    /* (x) Poisson 'n' -> phi (h2) */
    orc_helm3d(h1, h2, my, mz, 0, M - 1, xalp, 'n', 0.0, ops, nthreads);
    /* (xi) update */
    orc_update_uvwp(u, v, w, p, h2, h1, my, mz, M, xalp, aspect, akkc[k], bkkc[k], dt, fnu);
    if (cmassflow) {
        double cs = csum;
        orc_impose_mass_flow(&cs, krk, u, my, mz, aspect, premassfu, premassf, 1);
    }
    /* divergence check (h2 <- div u) */
    memset(h2, 0, sizeof(double) * nf);
    orc_div3d(u, v, w, h2, my, mz, M, xalp, aspect, 1.0);
    return orc_max_3din(h2, my, mz, M);
}
