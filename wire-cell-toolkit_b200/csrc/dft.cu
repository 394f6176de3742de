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

// out[c][r] = in[r][c] for an nrows x ncols input (32 x 32 tiles).
template <typename T>
__global__ void k_transpose(const T* __restrict__ in, T* __restrict__ out, int nrows, int ncols)
{
    __shared__ T tile[32][33];
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

void launch_transpose_c(const float2* in, float2* out, int nrows, int ncols, cudaStream_t s)
{
    if (nrows <= 0 || ncols <= 0) return;
    const dim3 grid((ncols + 31) / 32, (nrows + 31) / 32), block(32, 8);
    k_transpose<float2><<<grid, block, 0, s>>>(in, out, nrows, ncols);
}

void launch_transpose_r(const float* in, float* out, int nrows, int ncols, cudaStream_t s)
{
    if (nrows <= 0 || ncols <= 0) return;
    const dim3 grid((ncols + 31) / 32, (nrows + 31) / 32), block(32, 8);
    k_transpose<float><<<grid, block, 0, s>>>(in, out, nrows, ncols);
}

}  // namespace wctb200
