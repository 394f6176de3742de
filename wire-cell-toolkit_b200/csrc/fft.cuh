// Block-cooperative mixed-radix FFTs in shared memory (Stockham autosort,
// radices 2, 3, 4, 5, 7, 8), plus the half-length packing used for
// real-to-complex and complex-to-real transforms along the time axis.
//
// Conventions follow the reference IDFT interface
// (iface/inc/WireCellIface/IDFT.h:10-80): forward transforms are
// unnormalised, inverse transforms carry 1/n.
//
// Packed real spectra: a real row of even length N = 2M is transformed into
// M complex bins; bin 0 holds (X[0], X[M]) -- the DC and Nyquist values,
// both real -- and bins 1..M-1 hold X[1..M-1].  Every linear operation on
// the spectrum treats bin 0 component-wise.
#pragma once

#include "common.cuh"

namespace wctb200 {

constexpr int kFftMaxStages = 16;

struct FftDesc {
    int M;                       // complex length
    int nst;                     // number of stages
    int radix[kFftMaxStages];    // radix of each stage
    const float2* tw;            // [M]  exp(-2 pi i m / M)
    const float2* twh;           // [M]  exp(-2 pi i k / (2M))  (real packing)
};

namespace fftk {

constexpr float kS2 = 0.70710678118654752f;  // sqrt(1/2)
constexpr float kS3 = 0.86602540378443865f;  // sqrt(3)/2
// cos/sin(2 pi m / R) for m = 1..(R-1)/2, R = 5, 7 (folded to literals
// once the butterfly loops are unrolled).
template <int R>
__device__ __forceinline__ float root_cos(int m)
{
    if (R == 5) return m == 1 ? 0.30901699437494745f : -0.80901699437494734f;
    return m == 1 ? 0.62348980185873359f : (m == 2 ? -0.22252093395631434f : -0.90096886790241903f);
}
template <int R>
__device__ __forceinline__ float root_sin(int m)
{
    if (R == 5) return m == 1 ? 0.95105651629515353f : 0.58778525229247314f;
    return m == 1 ? 0.78183148246802981f : (m == 2 ? 0.97492791218182362f : 0.43388373911755823f);
}

template <int SIGN>
__device__ __forceinline__ void bfly2(float2* v)
{
    float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
}

template <int SIGN>
__device__ __forceinline__ void bfly4(float2& v0, float2& v1, float2& v2, float2& v3)
{
    float2 t0 = cadd(v0, v2), t1 = csub(v0, v2);
    float2 t2 = cadd(v1, v3), t3 = cmul_i<SIGN>(csub(v1, v3));
    v0 = cadd(t0, t2);
    v2 = csub(t0, t2);
    v1 = cadd(t1, t3);
    v3 = csub(t1, t3);
}

template <int SIGN>
__device__ __forceinline__ void bfly3(float2* v)
{
    float2 s = cadd(v[1], v[2]);
    float2 d = csub(v[1], v[2]);
    float2 m = make_float2(v[0].x - 0.5f * s.x, v[0].y - 0.5f * s.y);
    float2 id = cmul_i<SIGN>(make_float2(kS3 * d.x, kS3 * d.y));  // SIGN*i*(sqrt3/2)*d
    v[0] = cadd(v[0], s);
    v[1] = cadd(m, id);
    v[2] = csub(m, id);
}

// Odd radix R = 2h+1 with the symmetric pairing
//   y_a = A_a + SIGN i B_a,  y_{R-a} = A_a - SIGN i B_a,
//   A_a = v0 + sum_b cos(2 pi ab/R)(v_b + v_{R-b}),  B_a = sum_b sin(2 pi ab/R)(v_b - v_{R-b}).
template <int R, int SIGN>
__device__ __forceinline__ void bfly_odd(float2* v)
{
    constexpr int h = (R - 1) / 2;
    float2 p[h], q[h];
#pragma unroll
    for (int b = 1; b <= h; ++b) {
        p[b - 1] = cadd(v[b], v[R - b]);
        q[b - 1] = csub(v[b], v[R - b]);
    }
    float2 y0 = v[0];
#pragma unroll
    for (int b = 0; b < h; ++b) y0 = cadd(y0, p[b]);
    float2 out[R];
    out[0] = y0;
#pragma unroll
    for (int a = 1; a <= h; ++a) {
        float2 A = v[0], B = make_float2(0.f, 0.f);
#pragma unroll
        for (int b = 1; b <= h; ++b) {
            const int mab = (a * b) % R;
            const float c = mab <= h ? root_cos<R>(mab) : root_cos<R>(R - mab);
            const float s = mab <= h ? root_sin<R>(mab) : -root_sin<R>(R - mab);
            A.x += c * p[b - 1].x;
            A.y += c * p[b - 1].y;
            B.x += s * q[b - 1].x;
            B.y += s * q[b - 1].y;
        }
        float2 iB = cmul_i<SIGN>(B);
        out[a] = cadd(A, iB);
        out[R - a] = csub(A, iB);
    }
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = out[r];
}

template <int SIGN>
__device__ __forceinline__ void bfly8(float2* v)
{
    // split into two radix-4 DFTs over even and odd inputs
    float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    float2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    bfly4<SIGN>(e0, e1, e2, e3);
    bfly4<SIGN>(o0, o1, o2, o3);
    // twiddles w8^k, k = 1..3, w8 = exp(SIGN i pi/4)
    float2 t1 = cmul(o1, make_float2(kS2, SIGN * kS2));
    float2 t2 = cmul_i<SIGN>(o2);
    float2 t3 = cmul(o3, make_float2(-kS2, SIGN * kS2));
    v[0] = cadd(e0, o0);
    v[4] = csub(e0, o0);
    v[1] = cadd(e1, t1);
    v[5] = csub(e1, t1);
    v[2] = cadd(e2, t2);
    v[6] = csub(e2, t2);
    v[3] = cadd(e3, t3);
    v[7] = csub(e3, t3);
}

template <int R, int SIGN>
__device__ __forceinline__ void bfly(float2* v)
{
    if constexpr (R == 2) bfly2<SIGN>(v);
    else if constexpr (R == 3) bfly3<SIGN>(v);
    else if constexpr (R == 4) bfly4<SIGN>(v[0], v[1], v[2], v[3]);
    else if constexpr (R == 5) bfly_odd<5, SIGN>(v);
    else if constexpr (R == 7) bfly_odd<7, SIGN>(v);
    else if constexpr (R == 8) bfly8<SIGN>(v);
}

// Bank swizzle of the intermediate stage buffers (float2 index; used when M
// is a multiple of 16): the low four bits are XORed with bits 3..6, a
// bijection inside every aligned block of 16.  Stockham stages with short
// sub-transforms (Ns = 1, 8) write with a stride of R or R*Ns elements, which
// in natural order puts up to 16 lanes of a half-warp on one bank pair;
// swizzled, those writes and the contiguous reads of the next stage both
// spread over all 32 banks.
__device__ __forceinline__ int swz(int i) { return i ^ ((i >> 3) & 15); }

// j mod Ns without a division: q = floor(j / Ns) as the high word of
// j * ceil(2^32 / Ns), exact for j, Ns < 2^16 (the error term j * (m Ns - 2^32)
// stays below 2^32).
struct FastMod {
    unsigned m;
    int d;
    __device__ __forceinline__ explicit FastMod(int ns) : m(0xffffffffu / (unsigned)ns + 1u), d(ns) {}
    __device__ __forceinline__ int operator()(int j) const
    {
        return d == 1 ? 0 : j - (int)__umulhi((unsigned)j, m) * d;
    }
};

// One Stockham stage: sub-transforms of length Ns grow to Ns*R.  SWI / SWO:
// src / dst hold the swizzled order.
template <int R, int SIGN, bool SWI, bool SWO>
__device__ __forceinline__ void stage(const float2* __restrict__ src, float2* __restrict__ dst, int M, int Ns,
                                      const float2* __restrict__ tw, int tid, int nth)
{
    const int nR = M / R;
    const int step = M / (Ns * R);
    const FastMod mod(Ns);
    for (int j = tid; j < nR; j += nth) {
        const int k = mod(j);
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int i = j + r * nR;
            v[r] = src[SWI ? swz(i) : i];
        }
        if (k) {
            // w^1 and w^2 from the table, higher powers as products of them
            // (two loads per item instead of R - 1; at most five factors)
            float2 w[R];
            w[1] = __ldg(tw + k * step);
            if (R > 2) w[2] = __ldg(tw + 2 * k * step);
            if (R > 3) w[3] = cmul(w[1], w[2]);
            if (R > 4) w[4] = cmul(w[2], w[2]);
            if (R > 5) w[5] = cmul(w[2], w[3]);
            if (R > 6) w[6] = cmul(w[3], w[3]);
            if (R > 7) w[7] = cmul(w[3], w[4]);
#pragma unroll
            for (int r = 1; r < R; ++r) {
                float2 wr = w[r];
                if (SIGN > 0) wr.y = -wr.y;
                v[r] = cmul(v[r], wr);
            }
        }
        bfly<R, SIGN>(v);
        const int base = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int i = base + r * Ns;
            dst[SWO ? swz(i) : i] = v[r];
        }
    }
}

template <int R, int SIGN>
__device__ __forceinline__ void stage_any(const float2* __restrict__ src, float2* __restrict__ dst, int M, int Ns,
                                          const float2* __restrict__ tw, int tid, int nth, bool swi, bool swo)
{
    if (swi) {
        if (swo) stage<R, SIGN, true, true>(src, dst, M, Ns, tw, tid, nth);
        else stage<R, SIGN, true, false>(src, dst, M, Ns, tw, tid, nth);
    }
    else {
        if (swo) stage<R, SIGN, false, true>(src, dst, M, Ns, tw, tid, nth);
        else stage<R, SIGN, false, false>(src, dst, M, Ns, tw, tid, nth);
    }
}

}  // namespace fftk

// Complex FFT of length d.M held in smem buffer a; b is scratch of the same
// size.  All threads of the block must call it (it synchronises between
// stages).  Returns the buffer that holds the result.
template <int SIGN>
__device__ float2* fft_c2c(float2* a, float2* b, const FftDesc& d, int tid, int nth)
{
    // input and result in natural order; a stage's output swizzled where its
    // writes are strided (Ns < 16) and another stage reads it
    const bool sw = (d.M & 15) == 0;
    int Ns = 1;
    bool swi = false;
    for (int s = 0; s < d.nst; ++s) {
        const int R = d.radix[s];
        const bool swo = sw && s + 1 < d.nst && Ns < 16;
        switch (R) {
            case 2: fftk::stage_any<2, SIGN>(a, b, d.M, Ns, d.tw, tid, nth, swi, swo); break;
            case 3: fftk::stage_any<3, SIGN>(a, b, d.M, Ns, d.tw, tid, nth, swi, swo); break;
            case 4: fftk::stage_any<4, SIGN>(a, b, d.M, Ns, d.tw, tid, nth, swi, swo); break;
            case 5: fftk::stage_any<5, SIGN>(a, b, d.M, Ns, d.tw, tid, nth, swi, swo); break;
            case 7: fftk::stage_any<7, SIGN>(a, b, d.M, Ns, d.tw, tid, nth, swi, swo); break;
            default: fftk::stage_any<8, SIGN>(a, b, d.M, Ns, d.tw, tid, nth, swi, swo); break;
        }
        __syncthreads();
        float2* t = a;
        a = b;
        b = t;
        Ns *= R;
        swi = swo;
    }
    return a;
}

// Real-to-complex post-processing: Z = FFT_M(x[2m] + i x[2m+1]) -> packed X.
__device__ __forceinline__ float2 r2c_bin(const float2* Z, int k, int M, const float2* __restrict__ twh)
{
    const float2 zk = Z[k];
    if (k == 0) return make_float2(zk.x + zk.y, zk.x - zk.y);
    const float2 zm = cconj(Z[M - k]);
    const float2 E = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y + zm.y));
    const float2 D = make_float2(0.5f * (zk.x - zm.x), 0.5f * (zk.y - zm.y));
    const float2 O = make_float2(D.y, -D.x);  // -i * D
    return cadd(E, cmul(__ldg(twh + k), O));
}

// Complex-to-real pre-processing: packed X -> Z with x = IFFT_M(Z)/M interleaved.
__device__ __forceinline__ float2 c2r_bin(const float2* X, int k, int M, const float2* __restrict__ twh)
{
    const float2 xk = X[k];
    if (k == 0) {
        const float E = 0.5f * (xk.x + xk.y), O = 0.5f * (xk.x - xk.y);
        return make_float2(E, O);
    }
    const float2 xm = cconj(X[M - k]);
    const float2 E = make_float2(0.5f * (xk.x + xm.x), 0.5f * (xk.y + xm.y));
    const float2 D = make_float2(0.5f * (xk.x - xm.x), 0.5f * (xk.y - xm.y));
    const float2 O = cmulc(D, __ldg(twh + k));  // D * conj(W^k)
    return make_float2(E.x - O.y, E.y + O.x);   // E + i O
}

}  // namespace wctb200
