/*
 * orc_fft.h -- complex FFT of any length for the CPU oracle (test
 * infrastructure only).
 *
 * The reference transforms with FFTW (src/tchebw.f:38-56 REDFT00 plans,
 * src/ininewc.f90:47-48 r2c/c2r plans); FFTW is not vendored and its version
 * is not pinned, so this file restates the published discrete Fourier
 * transform it computes:
 *   forward  X_k = sum_n x_n exp(-2 pi i n k / N),
 *   backward x_n = sum_k X_k exp(+2 pi i n k / N)   (unnormalised, as FFTW).
 * Algorithm: recursive mixed-radix decimation in time (Cooley-Tukey) over
 * the prime factors of N, the prime-length butterflies as direct sums;
 * twiddles exp(-2 pi i t / N) from a table of exact-angle cosines/sines.
 */
#ifndef ORC_FFT_H
#define ORC_FFT_H

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int n;
    int nf;          /* number of factors */
    int f[32];       /* prime factors of n, 4 merged from 2x2 */
    double *tw;      /* 2n: cos, -sin of 2 pi t / n */
} orc_fft_plan;

static inline void orc_fft_plan_init(orc_fft_plan *p, int n)
{
    p->n = n;
    p->nf = 0;
    int r = n;
    while (r % 4 == 0) { p->f[p->nf++] = 4; r /= 4; }
    while (r % 2 == 0) { p->f[p->nf++] = 2; r /= 2; }
    for (int q = 3; (long)q * q <= r; q += 2)
        while (r % q == 0) { p->f[p->nf++] = q; r /= q; }
    if (r > 1) p->f[p->nf++] = r;
    p->tw = (double *)malloc(sizeof(double) * 2 * (size_t)(n > 0 ? n : 1));
    const double pi = 4.0 * atan(1.0);
    for (int t = 0; t < n; ++t) {
        /* exact-angle reduction: angle 2 pi t/n in the first octant form */
        const double a = 2.0 * pi * (double)t / (double)n;
        p->tw[2 * t] = cos(a);
        p->tw[2 * t + 1] = -sin(a);
    }
}

static inline void orc_fft_plan_free(orc_fft_plan *p)
{
    free(p->tw);
    p->tw = NULL;
}

/* out[k*os] = sum_{j<m} in[j*is] w^(jk), w = exp(-2 pi i/m)*sign, m = product of
 * factors f[level..]; tstride = n/m (index into the n-point table).        */
static void orc_fft_rec(const orc_fft_plan *p, int level, const double *in, long is, double *out, int m,
                        int tstride, int inv)
{
    if (m == 1) {
        out[0] = in[0];
        out[1] = in[1];
        return;
    }
    const int R = p->f[level], M = m / R;
    /* sub-transforms of the R decimated sequences into out[q*M .. ] */
    for (int q = 0; q < R; ++q)
        orc_fft_rec(p, level + 1, in + 2 * (long)q * is, is * R, out + 2 * (long)q * M, M, tstride * R, inv);
    double tmp[2 * 64];
    double *t = (R <= 64) ? tmp : (double *)malloc(sizeof(double) * 2 * (size_t)R);
    for (int k = 0; k < M; ++k) {
        /* twiddled inputs of the radix-R butterfly at output k */
        for (int q = 0; q < R; ++q) {
            const double xr = out[2 * ((long)q * M + k)], xi = out[2 * ((long)q * M + k) + 1];
            const long ti = ((long)q * k * tstride) % p->n;
            const double c = p->tw[2 * ti], s = inv ? -p->tw[2 * ti + 1] : p->tw[2 * ti + 1];
            t[2 * q] = xr * c - xi * s;
            t[2 * q + 1] = xr * s + xi * c;
        }
        for (int r = 0; r < R; ++r) {
            double ar = 0.0, ai = 0.0;
            for (int q = 0; q < R; ++q) {
                const long ti = ((long)q * r % R) * (p->n / R);
                const double c = p->tw[2 * ti], s = inv ? -p->tw[2 * ti + 1] : p->tw[2 * ti + 1];
                ar += t[2 * q] * c - t[2 * q + 1] * s;
                ai += t[2 * q] * s + t[2 * q + 1] * c;
            }
            out[2 * ((long)r * M + k)] = ar;
            out[2 * ((long)r * M + k) + 1] = ai;
        }
    }
    if (t != tmp) free(t);
}

/* out = DFT(in) (complex interleaved, length p->n); inv 1: the backward sign. */
static inline void orc_fft(const orc_fft_plan *p, const double *in, double *out, int inv)
{
    orc_fft_rec(p, 0, in, 1, out, p->n, 1, inv);
}

#endif
