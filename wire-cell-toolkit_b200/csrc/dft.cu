// Kernels of the GPU IDFT (iface/inc/WireCellIface/IDFT.h): batched complex
// transforms of rows in shared memory, Bluestein's chirp-z transform for
// lengths with a prime factor above 7, and tiled matrix transposes (the
// column transforms of the 1b and 2d methods run as row transforms between
// two transposes).
//
// Bluestein (L. I. Bluestein, "A linear filtering approach to the
// computation of discrete Fourier transform", IEEE Trans. Audio
// Electroacoust. 18 (1970) 451-455): with c_n = exp(-pi i n^2 / N),
//   X_k = c_k sum_n (x_n c_n) conj(c_{k-n}),
// a circular convolution of length P >= 2N - 1 done with two length-P FFTs
// and the precomputed spectrum B = FFT_P(b), b_m = conj(c_|m|) at m mod P.
// Inverse transforms use inv(x) = conj(fwd(conj(x))) / N.
#include <algorithm>

#include "kernels.cuh"
#include "rng.cuh"

namespace wctb200 {

// One row per block: out = scale * DFT_sign(in), length d.M, in place allowed.
template <int SIGN>
__global__ void k_c2c_rows(const float2* in, long ld_in, float2* out, long ld_out, int nrows, FftDesc d, float scale)
{
    extern __shared__ float2 dsm[];
    const int row = blockIdx.x;
    if (row >= nrows) return;
    const int M = d.M, tid = threadIdx.x, nth = blockDim.x;
    float2* a = dsm;
    float2* b = dsm + M;
    const float2* x = in + (size_t)row * ld_in;
    for (int m = tid; m < M; m += nth) a[m] = x[m];
    __syncthreads();
    const float2* z = fft_c2c<SIGN>(a, b, d, tid, nth);
    float2* o = out + (size_t)row * ld_out;
    for (int m = tid; m < M; m += nth) o[m] = make_float2(z[m].x * scale, z[m].y * scale);
}

// One row per block, Bluestein: length N through FFTs of length dP.M.
// INV: the inverse transform (conjugated input and output).
template <bool INV>
__global__ void k_bluestein_rows(const float2* in, long ld_in, float2* out, long ld_out, int nrows, int N, FftDesc dP,
                                 const float2* __restrict__ chirp, const float2* __restrict__ bhat, float scale)
{
    extern __shared__ float2 dsm[];
    const int row = blockIdx.x;
    if (row >= nrows) return;
    const int P = dP.M, tid = threadIdx.x, nth = blockDim.x;
    float2* a = dsm;
    float2* b = dsm + P;
    const float2* x = in + (size_t)row * ld_in;
    for (int m = tid; m < P; m += nth) {
        float2 v = make_float2(0.f, 0.f);
        if (m < N) {
            float2 xv = x[m];
            if (INV) xv.y = -xv.y;
            v = cmul(xv, chirp[m]);
        }
        a[m] = v;
    }
    __syncthreads();
    float2* z = fft_c2c<-1>(a, b, dP, tid, nth);
    for (int m = tid; m < P; m += nth) z[m] = cmul(z[m], bhat[m]);
    __syncthreads();
    const float2* y = fft_c2c<+1>(z, z == a ? b : a, dP, tid, nth);
    const float s = scale / (float)P;
    float2* o = out + (size_t)row * ld_out;
    for (int k = tid; k < N; k += nth) {
        float2 v = cmul(y[k], chirp[k]);
        if (INV) v.y = -v.y;
        o[k] = make_float2(v.x * s, v.y * s);
    }
}

// b_m = conj(c_|m|) for |m| < N at m mod P, zero elsewhere.
__global__ void k_bluestein_b(const float2* __restrict__ chirp, float2* __restrict__ b, int N, int P)
{
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < P; m += gridDim.x * blockDim.x) {
        float2 v = make_float2(0.f, 0.f);
        if (m < N) v = chirp[m];
        else if (m > P - N) v = chirp[P - m];
        b[m] = make_float2(v.x, -v.y);
    }
}

// out[c][r] = in[r][c] for an nrows x ncols input (32 x 32 tiles); a batch
// of matrices along blockIdx.z, each nrows * ncols elements apart.
template <typename T>
__global__ void k_transpose(const T* __restrict__ in, T* __restrict__ out, int nrows, int ncols)
{
    __shared__ T tile[32][33];
    const size_t boff = (size_t)blockIdx.z * nrows * ncols;
    in += boff;
    out += boff;
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int r = r0 + k, c = c0 + threadIdx.x;
        if (r < nrows && c < ncols) tile[k][threadIdx.x] = in[(size_t)r * ncols + c];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int c = c0 + k, r = r0 + threadIdx.x;
        if (r < nrows && c < ncols) out[(size_t)c * nrows + r] = tile[threadIdx.x][k];
    }
}

// Real rows (n values, row stride ld) packed two per complex row of length
// nfft: Z[p][k] = rows[2p][k] + i rows[2p+1][k] for k < n, zero beyond.
__global__ void k_pack_rows(const float* __restrict__ rows, long ld, int nrows, int n, float2* __restrict__ Z,
                            int nfft)
{
    const int p = blockIdx.y;
    const float* r0 = rows + (size_t)(2 * p) * ld;
    const bool has1 = 2 * p + 1 < nrows;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nfft; k += gridDim.x * blockDim.x) {
        float2 v = make_float2(0.f, 0.f);
        if (k < n) v = make_float2(r0[k], has1 ? r0[ld + k] : 0.f);
        Z[(size_t)p * nfft + k] = v;
    }
}

// The inverse of k_pack_rows for the first n values of each row.
__global__ void k_unpack_rows(const float2* __restrict__ Z, int nfft, float* __restrict__ rows, long ld, int nrows,
                              int n)
{
    const int p = blockIdx.y;
    float* r0 = rows + (size_t)(2 * p) * ld;
    const bool has1 = 2 * p + 1 < nrows;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const float2 v = Z[(size_t)p * nfft + k];
        r0[k] = v.x;
        if (has1) r0[ld + k] = v.y;
    }
}

// Z[p][k] *= L[k] (or conj(L[k])).
__global__ void k_cmul_rows(float2* __restrict__ Z, int nfft, const float2* __restrict__ L, int conj)
{
    const int p = blockIdx.y;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nfft; k += gridDim.x * blockDim.x) {
        float2 l = L[k];
        if (conj) l.y = -l.y;
        Z[(size_t)p * nfft + k] = cmul(Z[(size_t)p * nfft + k], l);
    }
}

void launch_pack_rows(const float* rows, long ld, int nrows, int n, float2* Z, int nfft, cudaStream_t s)
{
    if (nrows <= 0) return;
    const dim3 grid(std::min((nfft + 255) / 256, 64), (nrows + 1) / 2);
    k_pack_rows<<<grid, 256, 0, s>>>(rows, ld, nrows, n, Z, nfft);
}

void launch_unpack_rows(const float2* Z, int nfft, float* rows, long ld, int nrows, int n, cudaStream_t s)
{
    if (nrows <= 0) return;
    const dim3 grid(std::min((n + 255) / 256, 64), (nrows + 1) / 2);
    k_unpack_rows<<<grid, 256, 0, s>>>(Z, nfft, rows, ld, nrows, n);
}

void launch_cmul_rows(float2* Z, int nfft, int nz, const float2* L, bool conj, cudaStream_t s)
{
    if (nz <= 0) return;
    const dim3 grid(std::min((nfft + 255) / 256, 64), nz);
    k_cmul_rows<<<grid, 256, 0, s>>>(Z, nfft, L, conj ? 1 : 0);
}

// Four-step FFT twiddles: Z[b][n2][k1] *= exp(sign 2 pi i n2 k1 / (N1 N2)),
// the phase reduced in integers and evaluated in double precision.
__global__ void k_twiddle4(float2* __restrict__ Z, long long count, int N1, int N2, int sign)
{
    const long long N = (long long)N1 * N2;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < count;
         e += (long long)gridDim.x * blockDim.x) {
        const long long in_b = e % N;
        const int n2 = (int)(in_b / N1), k1 = (int)(in_b - (long long)n2 * N1);
        const long long q = ((long long)n2 * k1) % N;
        double sn, cs;
        sincospi(2.0 * (double)q / (double)N, &sn, &cs);
        const float2 w = make_float2((float)cs, (float)(sign * sn));
        Z[e] = cmul(Z[e], w);
    }
}

// Bluestein in global memory (lengths whose FFT exceeds shared memory):
// Z[r][m] = x_m c_m (conjugated input for the inverse) for m < N, 0 up to P;
// then out[r][k] = scale * c_k Z[r][k] (conjugated for the inverse).
__global__ void k_blue_pre(const float2* __restrict__ in, long ld_in, float2* __restrict__ Z, int N, int P,
                           const float2* __restrict__ chirp, int inv)
{
    const int r = blockIdx.y;
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < P; m += gridDim.x * blockDim.x) {
        float2 v = make_float2(0.f, 0.f);
        if (m < N) {
            float2 x = in[(size_t)r * ld_in + m];
            if (inv) x.y = -x.y;
            v = cmul(x, chirp[m]);
        }
        Z[(size_t)r * P + m] = v;
    }
}

__global__ void k_blue_post(const float2* __restrict__ Z, int P, float2* __restrict__ out, long ld_out, int N,
                            const float2* __restrict__ chirp, int inv, float scale)
{
    const int r = blockIdx.y;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
        float2 v = cmul(Z[(size_t)r * P + k], chirp[k]);
        if (inv) v.y = -v.y;
        out[(size_t)r * ld_out + k] = make_float2(v.x * scale, v.y * scale);
    }
}

void launch_twiddle4(float2* Z, long long count, int N1, int N2, int sign, cudaStream_t s)
{
    if (count <= 0) return;
    const long long blocks = std::min<long long>((count + 255) / 256, 148LL * 16);
    k_twiddle4<<<(unsigned)blocks, 256, 0, s>>>(Z, count, N1, N2, sign);
}

void launch_blue_pre(const float2* in, long ld_in, float2* Z, int nrows, int N, int P, const float2* chirp, bool inv,
                     cudaStream_t s)
{
    if (nrows <= 0) return;
    const dim3 grid(std::min((P + 255) / 256, 64), nrows);
    k_blue_pre<<<grid, 256, 0, s>>>(in, ld_in, Z, N, P, chirp, inv ? 1 : 0);
}

void launch_blue_post(const float2* Z, int P, float2* out, long ld_out, int nrows, int N, const float2* chirp,
                      bool inv, float scale, cudaStream_t s)
{
    if (nrows <= 0) return;
    const dim3 grid(std::min((N + 255) / 256, 64), nrows);
    k_blue_post<<<grid, 256, 0, s>>>(Z, P, out, ld_out, N, chirp, inv ? 1 : 0, scale);
}

static int dft_threads(int M) { return M >= 2048 ? 512 : 256; }

void launch_c2c_rows(const float2* in, long ld_in, float2* out, long ld_out, int nrows, const FftDesc& d, int sign,
                     float scale, cudaStream_t s)
{
    if (nrows <= 0) return;
    const size_t sm = 2 * sizeof(float2) * (size_t)d.M;
    if (sign < 0) {
        cudaFuncSetAttribute((const void*)k_c2c_rows<-1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k_c2c_rows<-1><<<nrows, dft_threads(d.M), sm, s>>>(in, ld_in, out, ld_out, nrows, d, scale);
    }
    else {
        cudaFuncSetAttribute((const void*)k_c2c_rows<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k_c2c_rows<1><<<nrows, dft_threads(d.M), sm, s>>>(in, ld_in, out, ld_out, nrows, d, scale);
    }
}

void launch_bluestein_rows(const float2* in, long ld_in, float2* out, long ld_out, int nrows, int N, const FftDesc& dP,
                           const float2* chirp, const float2* bhat, int sign, float scale, cudaStream_t s)
{
    if (nrows <= 0) return;
    const size_t sm = 2 * sizeof(float2) * (size_t)dP.M;
    if (sign < 0) {
        cudaFuncSetAttribute((const void*)k_bluestein_rows<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sm);
        k_bluestein_rows<false><<<nrows, dft_threads(dP.M), sm, s>>>(in, ld_in, out, ld_out, nrows, N, dP, chirp,
                                                                       bhat, scale);
    }
    else {
        cudaFuncSetAttribute((const void*)k_bluestein_rows<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sm);
        k_bluestein_rows<true><<<nrows, dft_threads(dP.M), sm, s>>>(in, ld_in, out, ld_out, nrows, N, dP, chirp,
                                                                      bhat, scale);
    }
}

void launch_bluestein_b(const float2* chirp, float2* b, int N, int P, cudaStream_t s)
{
    k_bluestein_b<<<std::min((P + 255) / 256, 1024), 256, 0, s>>>(chirp, b, N, P);
}

void launch_transpose_c(const float2* in, float2* out, int nrows, int ncols, cudaStream_t s, int batch)
{
    if (nrows <= 0 || ncols <= 0 || batch <= 0) return;
    const dim3 grid((ncols + 31) / 32, (nrows + 31) / 32, batch), block(32, 8);
    k_transpose<float2><<<grid, block, 0, s>>>(in, out, nrows, ncols);
}

void launch_transpose_r(const float* in, float* out, int nrows, int ncols, cudaStream_t s)
{
    if (nrows <= 0 || ncols <= 0) return;
    const dim3 grid((ncols + 31) / 32, (nrows + 31) / 32), block(32, 8);
    k_transpose<float><<<grid, block, 0, s>>>(in, out, nrows, ncols);
}

// ---------------------------------------------------------------------------
// Digitizer (gen/src/Digitizer.cxx:82-141): per sample, voltage = gain * value
// + baseline of the row's plane (a float, as the reference reads it), then
// Digitizer::digitize (:82-97): 0 at or below fullscale[0], 2^resolution - 1
// at or above fullscale[1], otherwise (v - fs0) / (fs1 - fs0) * max rounded
// (half away from zero) or floored.  Double arithmetic with explicit
// rounding (no fused multiply-add), as the reference computes it on the CPU.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float digitize_one(float x, double gain, double base, double fs0, double fs1, double span,
                                              double maxv, int rnd)
{
    const double v = __dadd_rn(__dmul_rn(gain, (double)x), base);
    double adc;
    if (v <= fs0) adc = 0.0;
    else if (v >= fs1) adc = maxv;
    else {
        const double fp = __dmul_rn(__ddiv_rn(__dsub_rn(v, fs0), span), maxv);
        adc = rnd ? round(fp) : floor(fp);
    }
    return (float)adc;
}

// VEC: four samples per thread (16-byte aligned rows), four independent
// divisions in flight instead of one.
template <bool VEC>
__global__ void k_digitize(const float* __restrict__ in, long ld_in, float* __restrict__ out, long ld_out, int nrows,
                           int ncols, const float* __restrict__ row_baseline, double gain, double fs0, double fs1,
                           int resolution, int rnd)
{
    const int r = blockIdx.y;
    if (r >= nrows) return;
    const double maxv = (double)((1 << resolution) - 1);
    const double base = (double)row_baseline[r];
    const double span = __dsub_rn(fs1, fs0);
    const float* x = in + (size_t)r * ld_in;
    float* y = out + (size_t)r * ld_out;
    int c0 = 0;
    if (VEC) {
        const int n4 = ncols / 4;
        const float4* x4 = reinterpret_cast<const float4*>(x);
        float4* y4 = reinterpret_cast<float4*>(y);
        for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n4; c += gridDim.x * blockDim.x) {
            const float4 a = __ldcs(x4 + c);
            float4 b;
            b.x = digitize_one(a.x, gain, base, fs0, fs1, span, maxv, rnd);
            b.y = digitize_one(a.y, gain, base, fs0, fs1, span, maxv, rnd);
            b.z = digitize_one(a.z, gain, base, fs0, fs1, span, maxv, rnd);
            b.w = digitize_one(a.w, gain, base, fs0, fs1, span, maxv, rnd);
            __stcs(y4 + c, b);
        }
        c0 = n4 * 4;
    }
    for (int c = c0 + blockIdx.x * blockDim.x + threadIdx.x; c < ncols; c += gridDim.x * blockDim.x)
        y[c] = digitize_one(x[c], gain, base, fs0, fs1, span, maxv, rnd);
}

void launch_digitize(const float* in, long ld_in, float* out, long ld_out, int nrows, int ncols,
                     const float* row_baseline, double gain, double fs0, double fs1, int resolution, bool rnd,
                     cudaStream_t s)
{
    if (nrows <= 0 || ncols <= 0) return;
    const bool vec = ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15) == 0 &&
                     ld_in % 4 == 0 && ld_out % 4 == 0;
    if (vec) {
        const dim3 grid(std::min((ncols / 4 + 127) / 128, 32), nrows);
        k_digitize<true><<<grid, 128, 0, s>>>(in, ld_in, out, ld_out, nrows, ncols, row_baseline, gain, fs0, fs1,
                                              resolution, rnd ? 1 : 0);
    }
    else {
        const dim3 grid(std::min((ncols + 255) / 256, 32), nrows);
        k_digitize<false><<<grid, 256, 0, s>>>(in, ld_in, out, ld_out, nrows, ncols, row_baseline, gain, fs0, fs1,
                                               resolution, rnd ? 1 : 0);
    }
}

// ---------------------------------------------------------------------------
// Noise (gen/src/AddNoise.cxx:44-100 IncoherentAddNoise, :102-160
// CoherentAddNoise; the waveform of aux/src/NoiseTools.cxx GeneratorN::spec
// and ::wave): for a channel spectrum S of N bins, sigma_k = S_k *
// sqrt(2 / 3.141592) (the reference's constant), bins 0 .. N/2 get
// sigma_k (n_k, n_{k + N/2}) from one list of normals n (the two index
// ranges overlap as in the reference), DC and Nyquist take their modulus,
// the spectrum is made Hermitian and transformed back (1/N): the noise
// waveform, added to the row's first min(N, ncols) samples.  Normals come
// from a counter-based stream per row: the channel's (incoherent) or the
// group's (coherent, so every channel of a group gets the same waveform).
// One row per block; N even, N/2 a supported FFT length.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float noise_normal(unsigned k0, unsigned k1, unsigned stream, unsigned model, int i)
{
    Philox g;
    g.init(k0, k1, stream, model, (unsigned)i);
    const double u1 = g.uniform(), u2 = g.uniform();
    double sn, cs;
    sincospi(2.0 * u2, &sn, &cs);
    return (float)(sqrt(-2.0 * log(u1)) * cs);  // Box-Muller
}

__global__ void k_add_noise(float* frame, long ld, int ncols, const float* __restrict__ spectra, int nspec,
                            const int* __restrict__ row_spec, const int* __restrict__ row_stream, unsigned k0,
                            unsigned k1, unsigned model, FftDesc d)
{
    extern __shared__ float2 nsm[];
    const int row = blockIdx.x;
    const int sp = row_spec[row];
    if (sp < 0) return;
    const unsigned stream = (unsigned)row_stream[row];
    const float* S = spectra + (size_t)sp * nspec;
    const int M = d.M, N = 2 * M, nhalf = M;
    const int tid = threadIdx.x, nth = blockDim.x;
    const float s2opi = sqrtf(2.0f / 3.141592f);
    float2* a = nsm;
    float2* b = nsm + M;
    // packed half spectrum: bin 0 = (|X_0|, |X_M|), bins 1 .. M-1 = X_k
    for (int k = tid; k < M; k += nth) {
        float2 v;
        if (k == 0) {
            const float m0 = S[0] * s2opi, mh = S[nhalf] * s2opi;
            const float2 x0 = make_float2(m0 * noise_normal(k0, k1, stream, model, 0),
                                          m0 * noise_normal(k0, k1, stream, model, nhalf));
            const float2 xh = make_float2(mh * noise_normal(k0, k1, stream, model, nhalf),
                                          mh * noise_normal(k0, k1, stream, model, 2 * nhalf));
            v = make_float2(sqrtf(x0.x * x0.x + x0.y * x0.y), sqrtf(xh.x * xh.x + xh.y * xh.y));
        }
        else {
            const float m = S[k] * s2opi;
            v = make_float2(m * noise_normal(k0, k1, stream, model, k),
                            m * noise_normal(k0, k1, stream, model, k + nhalf));
        }
        b[k] = v;
    }
    __syncthreads();
    for (int k = tid; k < M; k += nth) a[k] = c2r_bin(b, k, M, d.twh);
    __syncthreads();
    const float2* z = fft_c2c<+1>(a, b, d, tid, nth);
    const float sc = 1.0f / (float)M;  // with the halves of c2r_bin: the inverse's 1/N
    float* f = frame + (size_t)row * ld;
    for (int m = tid; m < M; m += nth) {
        const int c0 = 2 * m;
        if (c0 < ncols && c0 < N) f[c0] += z[m].x * sc;
        if (c0 + 1 < ncols && c0 + 1 < N) f[c0 + 1] += z[m].y * sc;
    }
}

void launch_add_noise(float* frame, long ld, int nrows, int ncols, const float* spectra, int nspec,
                      const int* row_spec, const int* row_stream, unsigned k0, unsigned k1, unsigned model,
                      const FftDesc& d, cudaStream_t s)
{
    if (nrows <= 0) return;
    const size_t sm = 2 * sizeof(float2) * (size_t)d.M;
    cudaFuncSetAttribute((const void*)k_add_noise, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_add_noise<<<nrows, dft_threads(d.M), sm, s>>>(frame, ld, ncols, spectra, nspec, row_spec, row_stream, k0, k1,
                                                     model, d);
}

}  // namespace wctb200
