// Counter-based random numbers for the fluctuated forward.
//
// Philox-4x32-10: J. K. Salmon, M. A. Moraes, R. O. Dror, D. E. Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11.  Every draw is a pure
// function of (key, counter), so a kernel can regenerate the same variate in
// another pass, in any order, on any thread.
//
// Binomial variates (IRandom::binomial, iface/inc/WireCellIface/IRandom.h;
// gen/src/Random.cxx draws them with std::binomial_distribution):
//   * n * min(p, 1-p) < 10: inversion by sequential search from 0 using
//     f(x+1) = f(x) * (n - x) / (x + 1) * p / (1 - p);
//   * otherwise: transformed rejection with squeeze, algorithm BTRS of
//     W. Hormann, "The generation of binomial random variates", J. Statist.
//     Comput. Simul. 46 (1993) 101-110: accept k when
//     log(v * alpha / (a / us^2 + b)) <= log f(k) - log f(m), m the mode,
//     with log x! = (x + 1/2) log(x + 1) - (x + 1) + log(2 pi) / 2 + fc(x),
//     fc the Stirling correction (exact values below 10, the series
//     1/12 (x+1)^-1 - 1/360 (x+1)^-3 + 1/1260 (x+1)^-5 above).
// Both are exact samplers (up to floating-point rounding).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace wctb200 {

struct Philox {
    uint32_t c[4];
    uint32_t k[2];
    uint32_t out[4];
    int used;  // 64-bit words taken from out (0..2)

    __device__ __forceinline__ void block()
    {
        uint32_t x0 = c[0], x1 = c[1], x2 = c[2], x3 = c[3];
        uint32_t k0 = k[0], k1 = k[1];
#pragma unroll
        for (int r = 0; r < 10; ++r) {
            const uint32_t lo0 = 0xD2511F53u * x0, hi0 = __umulhi(0xD2511F53u, x0);
            const uint32_t lo1 = 0xCD9E8D57u * x2, hi1 = __umulhi(0xCD9E8D57u, x2);
            const uint32_t y0 = hi1 ^ x1 ^ k0, y2 = hi0 ^ x3 ^ k1;
            x0 = y0;
            x1 = lo1;
            x2 = y2;
            x3 = lo0;
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        out[0] = x0;
        out[1] = x1;
        out[2] = x2;
        out[3] = x3;
        ++c[3];  // the last counter word numbers the blocks of one stream
        used = 0;
    }

    // Stream (key0, key1) x (ctr0, ctr1, ctr2); the fourth counter word counts blocks.
    __device__ __forceinline__ void init(uint32_t key0, uint32_t key1, uint32_t ctr0, uint32_t ctr1, uint32_t ctr2)
    {
        k[0] = key0;
        k[1] = key1;
        c[0] = ctr0;
        c[1] = ctr1;
        c[2] = ctr2;
        c[3] = 0;
        used = 2;
    }

    // Uniform double in the open interval (0, 1), 53 random bits.
    __device__ __forceinline__ double uniform()
    {
        if (used == 2) block();
        const uint64_t hi = out[2 * used], lo = out[2 * used + 1];
        ++used;
        const uint64_t x = ((hi << 32) | lo) >> 11;
        return ((double)x + 0.5) * 1.1102230246251565404e-16;  // 2^-53
    }
};

// Stirling correction fc(x) = log x! - [(x + 1/2) log(x + 1) - (x + 1) + log(2 pi)/2].
__device__ __forceinline__ double stirling_fc(int x)
{
    if (x < 10) {
        const double t[10] = {0.08106146679532733,  0.041340695955409457, 0.027677925684997717,
                              0.020790672103765839, 0.016644691189821259, 0.013876128823072875,
                              0.011896709945893313, 0.010411265261973668, 0.0092554621827094508,
                              0.0083305634333594725};
        return t[x];
    }
    const double r = 1.0 / ((double)x + 1.0), r2 = r * r;
    return r * (1.0 / 12.0 - r2 * (1.0 / 360.0 - r2 * (1.0 / 1260.0)));
}

// log x! up to the terms that cancel in the ratios below: (x + 1/2) log(x + 1) + fc(x).
__device__ __forceinline__ double logfact_part(int x)
{
    return ((double)x + 0.5) * log((double)x + 1.0) + stirling_fc(x);
}

// Binomial(n, p) for 0 <= p <= 1/2.
__device__ __forceinline__ int binomial_low(int n, double p, Philox& g)
{
    const double q = 1.0 - p;
    const double np = (double)n * p;
    if (np < 10.0) {
        const double s = p / q;
        const double f0 = exp((double)n * log1p(-p));  // q^n, >= exp(-10 * 1.39)
        for (int attempt = 0; attempt < 64; ++attempt) {
            double u = g.uniform();
            double f = f0;
            int x = 0;
            // at most n steps; the tail below one part in 2^53 ends the search
            while (u > f && x < n) {
                u -= f;
                f *= s * (double)(n - x) / (double)(x + 1);
                ++x;
                if (f < 1e-300) break;
            }
            if (u <= f || x == n) return x;
            // rounding left u above the remaining mass: draw again
        }
        return (int)floor(np);
    }
    // BTRS
    const double spq = sqrt(np * q);
    const double b = 1.15 + 2.53 * spq;
    const double a = -0.0873 + 0.0248 * b + 0.01 * p;
    const double c = np + 0.5;
    const double vr = 0.92 - 4.2 / b;
    const double alpha = (2.83 + 5.1 / b) * spq;
    const double lpq = log(p / q);
    const int m = (int)floor((double)(n + 1) * p);
    const double lfm = logfact_part(m) + logfact_part(n - m);
    for (int attempt = 0; attempt < 1000; ++attempt) {
        const double u = g.uniform() - 0.5;
        const double v = g.uniform();
        const double us = 0.5 - fabs(u);
        const int k = (int)floor((2.0 * a / us + b) * u + c);
        if (k < 0 || k > n) continue;
        if (us >= 0.07 && v <= vr) return k;  // squeeze
        const double lv = log(v * alpha / (a / (us * us) + b));
        // log f(k) - log f(m); the -(x+1) and log(2 pi)/2 terms of the four factorials cancel
        const double lratio = lfm - logfact_part(k) - logfact_part(n - k) + (double)(k - m) * lpq;
        if (lv <= lratio) return k;
    }
    return m;  // not reached in practice (acceptance probability per try is above 0.5)
}

// Binomial(n, p); p >= 1 gives n (GaussianDiffusion.cxx:196-198), p <= 0 gives 0.
__device__ __forceinline__ int binomial(int n, double p, Philox& g)
{
    if (n <= 0 || !(p > 0.0)) return 0;
    if (p >= 1.0) return n;
    if (p <= 0.5) return binomial_low(n, p, g);
    return n - binomial_low(n, 1.0 - p, g);
}

// Counter-stream tags (first counter word's top bits are the plane, the
// drift uses its own tag).
constexpr uint32_t kRngDriftTag = 0xFFFFu;
constexpr uint32_t kRngSampleTag = 0xFFFEu;  // bulk draws of the sampling entry point

}  // namespace wctb200
