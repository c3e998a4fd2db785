// fft.cuh -- small FFT building blocks shared by the Chebyshev line
// kernels (transforms.cu, cheb_lines.cu) and the x-direction Fourier
// kernels (dns.cu): complex multiply, register DFTs of 2, 3 and 4 points,
// compile-time Stockham sequences of them for register-resident DFTs of
// 2^a 3^b points, and the cp.async staging helpers.  All FP64.
#pragma once

#include <cuda_runtime.h>

namespace duct {

__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// In-place DFT of R points (R = 2, 3, 4), forward sign exp(-2 pi i jk/R).
template <int R>
__device__ __forceinline__ void dft(double2 (&v)[4])
{
    if (R == 2) {
        const double2 a = v[0], b = v[1];
        v[0] = make_double2(a.x + b.x, a.y + b.y);
        v[1] = make_double2(a.x - b.x, a.y - b.y);
    } else if (R == 3) {
        const double s = 0.86602540378443864676;  // sqrt(3)/2
        const double2 a = v[0], b = v[1], c = v[2];
        const double2 t = make_double2(b.x + c.x, b.y + c.y);
        const double2 d = make_double2(b.x - c.x, b.y - c.y);
        v[0] = make_double2(a.x + t.x, a.y + t.y);
        const double2 m = make_double2(a.x - 0.5 * t.x, a.y - 0.5 * t.y);
        // -i s d
        v[1] = make_double2(m.x + s * d.y, m.y - s * d.x);
        v[2] = make_double2(m.x - s * d.y, m.y + s * d.x);
    } else {
        const double2 a = v[0], b = v[1], c = v[2], d = v[3];
        const double2 s0 = make_double2(a.x + c.x, a.y + c.y), s1 = make_double2(a.x - c.x, a.y - c.y);
        const double2 s2 = make_double2(b.x + d.x, b.y + d.y), s3 = make_double2(b.x - d.x, b.y - d.y);
        v[0] = make_double2(s0.x + s2.x, s0.y + s2.y);
        v[2] = make_double2(s0.x - s2.x, s0.y - s2.y);
        // s1 - i s3, s1 + i s3
        v[1] = make_double2(s1.x + s3.y, s1.y - s3.x);
        v[3] = make_double2(s1.x - s3.y, s1.y + s3.x);
    }
}

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem));
}
__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.commit_group;\n" ::);
    asm volatile("cp.async.wait_group 0;\n" ::);
}

// Register-resident DFT of R points (R = 2^a 3^b), forward sign, as a
// compile-time sequence of radix-4, 3, 2 Stockham stages; the twiddles
// W_(NS P)^(r k) are read from a table tw[t] = exp(-2 pi i t / L) of a
// length L that R divides.
template <int R>
__host__ __device__ constexpr int reg_nstages()
{
    int n = 0, r = R;
    while (r % 4 == 0) { r /= 4; ++n; }
    while (r % 3 == 0) { r /= 3; ++n; }
    while (r % 2 == 0) { r /= 2; ++n; }
    return n;
}
template <int R>
__host__ __device__ constexpr int reg_radix(int s)
{
    int r = R;
    while (r % 4 == 0) { if (s == 0) return 4; r /= 4; --s; }
    while (r % 3 == 0) { if (s == 0) return 3; r /= 3; --s; }
    while (r % 2 == 0) { if (s == 0) return 2; r /= 2; --s; }
    return 1;
}

template <int R, int S, int NS>
__device__ __forceinline__ void reg_fft(double2 (&x)[R], const double2 *tw, int L)
{
    if constexpr (S < reg_nstages<R>()) {
        constexpr int P = reg_radix<R>(S);
        constexpr int NB = R / P;
        double2 y[R];
        const int tstep = L / (NS * P);
#pragma unroll
        for (int j = 0; j < NB; ++j) {
            const int k = j % NS;
            double2 v[4];
#pragma unroll
            for (int r = 0; r < P; ++r) v[r] = x[j + r * NB];
            if (NS > 1) {
#pragma unroll
                for (int r = 1; r < P; ++r) v[r] = cmul(v[r], tw[r * k * tstep]);
            }
            dft<P>(v);
            const int d = (j / NS) * NS * P + k;
#pragma unroll
            for (int r = 0; r < P; ++r) y[d + r * NS] = v[r];
        }
#pragma unroll
        for (int i = 0; i < R; ++i) x[i] = y[i];
        reg_fft<R, S + 1, NS * P>(x, tw, L);
    }
}


}  // namespace duct
