// DepoTransform forward kernels for sm_100a.
//
// Pipeline for one plane of one event (all on one stream):
//   k_drift        Drifter::insert per depo               gen/src/Drifter.cxx:127-196
//   k_prep         BinnedDiffusion_transform::add + the    gen/src/BinnedDiffusion_transform.cxx:37-92
//                  patch window (sample_bin_range) and     gen/src/GaussianDiffusion.cxx:116-149
//                  the event window reduction              gen/src/BinnedDiffusion_transform.cxx:416-464
//   k_raster       erf-integrated patches, linear impact   gen/src/GaussianDiffusion.cxx:30-229
//                  weights, scatter into impact groups     gen/src/BinnedDiffusion_transform.cxx:227-391
//   k_rfft_rows    real FFT along time of each group row   gen/src/ImpactTransform.cxx:149-151,237
//   k_wire_conv    wire-direction convolution with the     gen/src/ImpactTransform.cxx:153-212,242-300
//                  per-group response spectra (direct taps)
//   k_irfft_rows   inverse FFT along time, frame write     gen/src/ImpactTransform.cxx:303-347
//
// The 2-D FFT convolution of the reference is replaced by an exactly
// equivalent (no wrap-around) real FFT along time plus a direct
// (2*npad+1)-tap convolution along wires in the frequency domain.
//
// Index arithmetic that decides bins (drift, pitch distance, rejection,
// sample_bin_range, window min/max) is written with explicit _rn intrinsics
// so that no multiply-add is contracted and results are bit-identical to the
// reference's IEEE double arithmetic.

#include "kernels.cuh"

#include <cfloat>

namespace wctb200 {

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ int bin_of(double v, double lo, double bs)
{
    return __double2int_rz(__ddiv_rn(__dsub_rn(v, lo), bs));  // Binning::bin, Binning.h:75
}
__device__ __forceinline__ double edge_of(int i, double lo, double bs)
{
    return __dadd_rn(lo, __dmul_rn((double)i, bs));  // Binning::edge, Binning.h:88
}
__device__ __forceinline__ double gdistance(double x, double c, double s)
{
    return s != 0.0 ? __ddiv_rn(__dsub_rn(x, c), s) : __dsub_rn(x, c);  // GaussianDiffusion.h:34-44
}

template <typename T, typename Op>
__device__ __forceinline__ T warp_reduce(T v, Op op)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = op(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// ---------------------------------------------------------------------------
// Drift: Drifter::insert without fluctuation (gen/src/Drifter.cxx:127-196).
// ---------------------------------------------------------------------------
__global__ void k_drift(const double* __restrict__ in, int n, DriftDev dd, int do_drift, double* __restrict__ out,
                        unsigned char* __restrict__ valid)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double* p = in + 7 * (size_t)i;
    double t = p[0], q = p[1], x = p[2], y = p[3], z = p[4], el = p[5], et = p[6];
    unsigned char ok = 1;
    if (do_drift) {
        if (q == 0.0) ok = 0;
        else {
            int found = -1;
            double dir = 0.0;
            for (int r = 0; r < dd.nxr; ++r) {
                const double a = dd.xr[r][0], rp = dd.xr[r][1];
                if ((a < x && x < rp) || (rp < x && x < a)) { found = r; dir = -1.0; break; }
            }
            if (found < 0)
                for (int r = 0; r < dd.nxr; ++r) {
                    const double rp = dd.xr[r][1], c = dd.xr[r][2];
                    if ((rp < x && x < c) || (c < x && x < rp)) { found = r; dir = 1.0; break; }
                }
            if (found < 0) ok = 0;
            else {
                const double respx = dd.xr[found][1];
                const double dt = fabs(__ddiv_rn(__dsub_rn(respx, x), dd.speed));
                if (dir > 0) {
                    const double absorb = __dsub_rn(1.0, exp(__ddiv_rn(-dt, dd.lifetime)));
                    const double dQ = __dmul_rn(q, absorb);
                    q = __dsub_rn(q, dQ);
                    el = __dsqrt_rn(__dadd_rn(__dmul_rn(__dmul_rn(2.0, dd.DL), dt), __dmul_rn(el, el)));
                    et = __dsqrt_rn(__dadd_rn(__dmul_rn(__dmul_rn(2.0, dd.DT), dt), __dmul_rn(et, et)));
                }
                t = __dadd_rn(__dadd_rn(t, __dmul_rn(dir, dt)), dd.toffset);
                x = respx;
            }
        }
    }
    double* o = out + 7 * (size_t)i;
    o[0] = t; o[1] = q; o[2] = x; o[3] = y; o[4] = z; o[5] = el; o[6] = et;
    valid[i] = ok;
}

void launch_drift(const double* depos, int n, const DriftDev& dd, int do_drift, double* out, unsigned char* valid,
                  cudaStream_t s)
{
    if (n <= 0) return;
    k_drift<<<(n + 255) / 256, 256, 0, s>>>(depos, n, dd, do_drift, out, valid);
}

// ---------------------------------------------------------------------------
// Prep: sensitive-volume cut (aux/src/DepoTools.cxx:110-123,
// util/src/BoundingBox.cxx:37-56), BinnedDiffusion_transform::add rejection,
// GaussianDiffusion sample ranges, and the per-plane window reduction.
// ---------------------------------------------------------------------------
__global__ void k_prep(const double* __restrict__ dep, const unsigned char* __restrict__ valid, int n, PlaneDev pl,
                       TimeDev tb, double drift_speed, double nsigma, PatchRec* __restrict__ rec,
                       WindowDev* __restrict__ win)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long kpmin = ~0ull, kpmax = 0ull, ktmin = ~0ull, ktmax = 0ull;
    int nadd = 0, nout_t = 0, nout_p = 0, nover = 0;
    if (i < n) {
        PatchRec r;
        r.toff = r.poff = 0;
        r.nt = r.np = 0;
        r.tcr = r.pcr = r.st = r.sp = r.q = 0.f;
        if (valid[i]) {
            const double* p = dep + 7 * (size_t)i;
            const double t = p[0], q = p[1], x = p[2], y = p[3], z = p[4], el = p[5], et = p[6];
            bool inbb = true;
            if (pl.have_bb) {
                const double pp[3] = {x, y, z};
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const double b1 = pl.bb_lo[k], b2 = pl.bb_hi[k];
                    if (b1 < b2) { if (pp[k] < b1 || pp[k] > b2) inbb = false; }
                    else if (b2 < b1) { if (pp[k] < b2 || pp[k] > b1) inbb = false; }
                }
            }
            if (inbb) {
                const double ct = t;
                const double st = __ddiv_rn(el, drift_speed);                         // DepoTransform.cxx:185
                const double rx = __dsub_rn(x, pl.ox), ry = __dsub_rn(y, pl.oy), rz = __dsub_rn(z, pl.oz);
                const double cp = __dadd_rn(__dadd_rn(__dmul_rn(pl.ax, rx), __dmul_rn(pl.ay, ry)),
                                            __dmul_rn(pl.az, rz));                  // Pimpos.cxx:58
                const double sp = et;
                const double eff_t = st > 0 ? nsigma : 0.0;
                const double eff_p = sp > 0 ? nsigma : 0.0;
                if (gdistance(tb.tmin, ct, st) > eff_t || gdistance(tb.tmax, ct, st) < -eff_t) {
                    nout_t = 1;
                }
                else if (gdistance(pl.imp_min, cp, sp) > eff_p || gdistance(pl.imp_max, cp, sp) < -eff_p) {
                    nout_p = 1;
                }
                else {
                    nadd = 1;
                    const double tlo = __dsub_rn(ct, __dmul_rn(st, nsigma));
                    const double thi = __dadd_rn(ct, __dmul_rn(st, nsigma));
                    const double plo = __dsub_rn(cp, __dmul_rn(sp, nsigma));
                    const double phi = __dadd_rn(cp, __dmul_rn(sp, nsigma));
                    ktmin = dkey(tlo); ktmax = dkey(thi);
                    kpmin = dkey(plo); kpmax = dkey(phi);
                    const int t0 = max(bin_of(tlo, tb.tmin, tb.bs), 0);
                    const int t1 = min(bin_of(thi, tb.tmin, tb.bs) + 1, tb.nbins);
                    const int p0 = max(bin_of(plo, pl.imp_min, pl.imp_bs), 0);
                    const int p1 = min(bin_of(phi, pl.imp_min, pl.imp_bs) + 1, pl.imp_nbins);
                    if (t1 > t0 && p1 > p0) {
                        const int nt = t1 - t0, np = p1 - p0;
                        if (nt > kMaxPatchT || np > kMaxPatchP || (st == 0.0 && nt != 1) ||
                            (sp == 0.0 && np != 1)) {
                            nover = 1;
                        }
                        else {
                            r.toff = t0;
                            r.poff = p0;
                            r.nt = (unsigned short)nt;
                            r.np = (unsigned short)np;
                            r.tcr = (float)__dsub_rn(ct, edge_of(t0, tb.tmin, tb.bs));
                            r.pcr = (float)__dsub_rn(cp, edge_of(p0, pl.imp_min, pl.imp_bs));
                            r.st = (float)st;
                            r.sp = (float)sp;
                            r.q = (float)q;
                        }
                    }
                }
            }
        }
        rec[i] = r;
    }
    // block reduction, one atomic per block per quantity
    auto umin = [](unsigned long long a, unsigned long long b) { return a < b ? a : b; };
    auto umax = [](unsigned long long a, unsigned long long b) { return a > b ? a : b; };
    auto iadd = [](int a, int b) { return a + b; };
    kpmin = warp_reduce(kpmin, umin);
    ktmin = warp_reduce(ktmin, umin);
    kpmax = warp_reduce(kpmax, umax);
    ktmax = warp_reduce(ktmax, umax);
    nadd = warp_reduce(nadd, iadd);
    nout_t = warp_reduce(nout_t, iadd);
    nout_p = warp_reduce(nout_p, iadd);
    nover = warp_reduce(nover, iadd);
    __shared__ unsigned long long s_k[4][32];
    __shared__ int s_c[4][32];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        s_k[0][w] = kpmin; s_k[1][w] = kpmax; s_k[2][w] = ktmin; s_k[3][w] = ktmax;
        s_c[0][w] = nadd; s_c[1][w] = nout_t; s_c[2][w] = nout_p; s_c[3][w] = nover;
    }
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        kpmin = l < nw ? s_k[0][l] : ~0ull;
        kpmax = l < nw ? s_k[1][l] : 0ull;
        ktmin = l < nw ? s_k[2][l] : ~0ull;
        ktmax = l < nw ? s_k[3][l] : 0ull;
        nadd = l < nw ? s_c[0][l] : 0;
        nout_t = l < nw ? s_c[1][l] : 0;
        nout_p = l < nw ? s_c[2][l] : 0;
        nover = l < nw ? s_c[3][l] : 0;
        kpmin = warp_reduce(kpmin, umin);
        ktmin = warp_reduce(ktmin, umin);
        kpmax = warp_reduce(kpmax, umax);
        ktmax = warp_reduce(ktmax, umax);
        nadd = warp_reduce(nadd, iadd);
        nout_t = warp_reduce(nout_t, iadd);
        nout_p = warp_reduce(nout_p, iadd);
        nover = warp_reduce(nover, iadd);
        if (l == 0 && nadd) {
            atomicMin(&win->pmin, kpmin);
            atomicMax(&win->pmax, kpmax);
            atomicMin(&win->tmin, ktmin);
            atomicMax(&win->tmax, ktmax);
            atomicAdd(&win->nadded, nadd);
        }
        if (l == 0 && nout_t) atomicAdd(&win->out_time, nout_t);
        if (l == 0 && nout_p) atomicAdd(&win->out_pitch, nout_p);
        if (l == 0 && nover) atomicAdd(&win->oversize, nover);
    }
}

void launch_prep(const double* depos, const unsigned char* valid, int n, const PlaneDev& pl, const TimeDev& tb,
                 double drift_speed, double nsigma, PatchRec* rec, WindowDev* win, cudaStream_t s)
{
    if (n <= 0) return;
    k_prep<<<(n + 255) / 256, 256, 0, s>>>(depos, valid, n, pl, tb, drift_speed, nsigma, rec, win);
}

// ---------------------------------------------------------------------------
// Raster: one warp per depo patch.
//
// Bin integrals of the unit Gaussian are differences of erfc on the side of
// the centre the bin lies on, so tail bins keep full FP32 relative accuracy
// (0.5*(erf(b) - erf(a)) of GaussianDiffusion.cxx:30-56 loses ~4 digits there).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float edge_erfc(int k, float bs, float cr, float inv)
{
    const float x = ((float)k * bs - cr) * inv;
    return copysignf(erfcf(fabsf(x)), x);  // sign of x carried on the (non-negative) erfc value
}
__device__ __forceinline__ float bin_from_edges(float a, float b)
{
    const float ea = fabsf(a), eb = fabsf(b);
    const bool na = signbit(a), nb = signbit(b);
    if (!na) return 0.5f * (ea - eb);         // both edges at or above the centre
    if (nb) return 0.5f * (eb - ea);          // both below
    return 0.5f * ((2.0f - ea) - eb);         // bin straddles the centre
}

constexpr int kRasterWarps = 4;

__global__ void __launch_bounds__(kRasterWarps * 32) k_raster(const PatchRec* __restrict__ rec, int n, PlaneDev pl,
                                                               TimeDev tb, int G, int row0, int nrows, int col0,
                                                               int ldq, float* __restrict__ Q)
{
    __shared__ float s_e[kRasterWarps][kMaxPatchT + 1];
    __shared__ float s_t[kRasterWarps][kMaxPatchT];
    __shared__ float s_p[kRasterWarps][kMaxPatchP];
    __shared__ float s_w[kRasterWarps][kMaxPatchP];
    __shared__ int s_off[kRasterWarps][kMaxPatchP];
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int half_g = (G - 1) / 2;
    const float tbs = (float)tb.bs, pbs = (float)pl.imp_bs;
    const size_t gstride = (size_t)nrows * ldq;
    for (int i = blockIdx.x * kRasterWarps + wib; i < n; i += gridDim.x * kRasterWarps) {
        const PatchRec r = rec[i];
        const int nt = r.nt, np = r.np;
        if (np == 0 || nt == 0) continue;
        // ---- time profile
        double sum_t = 0.0;
        if (r.st > 0.f) {
            const float inv = 1.0f / (1.41421356237309505f * r.st);
            for (int k = lane; k <= nt; k += 32) s_e[wib][k] = edge_erfc(k, tbs, r.tcr, inv);
            __syncwarp();
            for (int k = lane; k < nt; k += 32) {
                const float v = bin_from_edges(s_e[wib][k], s_e[wib][k + 1]);
                s_t[wib][k] = v;
                sum_t += (double)v;
            }
        }
        else {
            if (lane == 0) { s_t[wib][0] = 1.0f; sum_t = 1.0; }
        }
        __syncwarp();
        // ---- pitch profile and linear weights (GausDesc::weight, GaussianDiffusion.cxx:61-92)
        double sum_p = 0.0;
        if (r.sp > 0.f) {
            const float inv = 1.0f / (1.41421356237309505f * r.sp);
            for (int k = lane; k <= np; k += 32) s_e[wib][k] = edge_erfc(k, pbs, r.pcr, inv);
            __syncwarp();
            const float isg = 1.0f / r.sp;
            const float c0 = r.sp / (pbs * 2.50662827463100050f);  // sigma / (step*sqrt(2 pi))
            for (int k = lane; k < np; k += 32) {
                const float v = bin_from_edges(s_e[wib][k], s_e[wib][k + 1]);
                const float x1 = (float)k * pbs - r.pcr;
                const float x2 = (float)(k + 1) * pbs - r.pcr;
                const float u1 = x1 * isg, u2 = x2 * isg;
                const float g1 = expf(-0.5f * u1 * u1), g2 = expf(-0.5f * u2 * u2);
                float w = v > 0.f ? c0 * (g2 - g1) / v + x2 / pbs : 0.0f;
                s_p[wib][k] = v;
                s_w[wib][k] = w;
                sum_p += (double)v;
            }
        }
        else {
            if (lane == 0) {
                s_p[wib][0] = 1.0f;
                s_w[wib][0] = (pbs - r.pcr) / pbs;
                sum_p = 1.0;
            }
        }
        // ---- impact bin -> (wire row, group) offsets (Pimpos.cxx:41-47)
        for (int k = lane; k < np; k += 32) {
            const int kk = r.poff + k;
            const int w = kk / pl.nimp;
            const int red = kk - (w * pl.nimp + pl.nimp / 2);
            const int g0 = red + half_g;
            s_off[wib][k] = (int)((size_t)g0 * gstride + (size_t)(w - row0) * ldq);
        }
        sum_t = warp_reduce(sum_t, [](double a, double b) { return a + b; });
        sum_p = warp_reduce(sum_p, [](double a, double b) { return a + b; });
        __syncwarp();
        const float scale = (float)((double)r.q / (sum_p * sum_t));
        const int cbase = r.toff - col0;
        // ---- scatter the patch into the two bracketing impact groups
        if (nt <= 32) {
            const int rpp = 32 / nt;
            const int li = lane / nt, lt = lane - li * nt;
            if (li < rpp) {
                const float tv = s_t[wib][lt] * scale;
                for (int ip = li; ip < np; ip += rpp) {
                    const float v = s_p[wib][ip] * tv;
                    const float w = s_w[wib][ip];
                    float* q0 = Q + s_off[wib][ip] + cbase + lt;
                    atomicAdd(q0, v * w);
                    atomicAdd(q0 + gstride, v * (1.0f - w));
                }
            }
        }
        else {
            for (int ip = 0; ip < np; ++ip) {
                const float pv = s_p[wib][ip] * scale;
                const float w = s_w[wib][ip];
                float* q0 = Q + s_off[wib][ip] + cbase;
                for (int it = lane; it < nt; it += 32) {
                    const float v = pv * s_t[wib][it];
                    atomicAdd(q0 + it, v * w);
                    atomicAdd(q0 + it + gstride, v * (1.0f - w));
                }
            }
        }
        __syncwarp();
    }
}

void launch_raster(const PatchRec* rec, int n, const PlaneDev& pl, const TimeDev& tb, int ngroups, int row0,
                   int nrows, int col0, int ldq, float* Q, WindowDev*, cudaStream_t s)
{
    if (n <= 0) return;
    int blocks = (n + kRasterWarps - 1) / kRasterWarps;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_raster<<<blocks, kRasterWarps * 32, 0, s>>>(rec, n, pl, tb, ngroups, row0, nrows, col0, ldq, Q);
}

// ---------------------------------------------------------------------------
// Real FFT of rows (forward), packed output.  One row per block.
// ---------------------------------------------------------------------------
__global__ void k_rfft_rows(const float* in, long in_ld, int in_len, float2* out, long out_ld, int nrows, FftDesc d)
{
    extern __shared__ float2 sm[];
    const int row = blockIdx.x;
    if (row >= nrows) return;
    float2* a = sm;
    float2* b = sm + d.M;
    const int M = d.M, tid = threadIdx.x, nth = blockDim.x;
    const float* x = in + (size_t)row * in_ld;
    if (in_len >= 2 * M) {
        const float2* x2 = reinterpret_cast<const float2*>(x);
        for (int m = tid; m < M; m += nth) a[m] = x2[m];
    }
    else {
        for (int m = tid; m < M; m += nth) {
            const int k = 2 * m;
            a[m] = make_float2(k < in_len ? x[k] : 0.f, k + 1 < in_len ? x[k + 1] : 0.f);
        }
    }
    __syncthreads();
    float2* Z = fft_c2c<-1>(a, b, d, tid, nth);
    float2* o = out + (size_t)row * out_ld;
    for (int k = tid; k < M; k += nth) o[k] = r2c_bin(Z, k, M, d.twh);
}

// Two complex rows of M bins in dynamic shared memory; raise the opt-in limit
// when they exceed the default 48 KB.
static void allow_smem(const void* f, size_t bytes)
{
    if (bytes > 48 * 1024) cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

void launch_rfft_rows(const float* in, long in_ld, int in_len, float2* out, long out_ld, int nrows, const FftDesc& d,
                      cudaStream_t s)
{
    if (nrows <= 0) return;
    allow_smem((const void*)k_rfft_rows, 2 * d.M * sizeof(float2));
    const int nth = d.M >= 2048 ? 512 : 256;
    k_rfft_rows<<<nrows, nth, 2 * d.M * sizeof(float2), s>>>(in, in_ld, in_len, out, out_ld, nrows, d);
}

// ---------------------------------------------------------------------------
// Inverse real FFT of rows + frame write (ImpactTransform.cxx:303-347).
// Row r of Vh is wire wire0 + r; ticks are tick0 + column.
// ---------------------------------------------------------------------------
__global__ void k_irfft_rows(const float2* __restrict__ Vh, int nrows, FftDesc d, int wire0, int wlo, int whi,
                             int tick0, int ncols, int nticks, float* __restrict__ frame)
{
    extern __shared__ float2 sm[];
    const int row = blockIdx.x;
    const int W = wire0 + row;
    if (row >= nrows || W < wlo || W >= whi) return;
    float2* a = sm;
    float2* b = sm + d.M;
    const int M = d.M, tid = threadIdx.x, nth = blockDim.x;
    const float2* v = Vh + (size_t)row * M;
    for (int k = tid; k < M; k += nth) b[k] = v[k];
    __syncthreads();
    for (int k = tid; k < M; k += nth) a[k] = c2r_bin(b, k, M, d.twh);
    __syncthreads();
    float2* z = fft_c2c<+1>(a, b, d, tid, nth);
    const float sc = 1.0f / (float)M;
    float* f = frame + (size_t)W * nticks;
    for (int m = tid; m < M; m += nth) {
        const float2 zz = z[m];
        const int c0 = 2 * m;
        const int t0 = tick0 + c0;
        if (c0 < ncols && t0 >= 0 && t0 < nticks) f[t0] = zz.x * sc;
        if (c0 + 1 < ncols && t0 + 1 >= 0 && t0 + 1 < nticks) f[t0 + 1] = zz.y * sc;
    }
}

void launch_irfft_rows(const float2* Vh, int nrows, const FftDesc& d, int wire0, int wlo, int whi, int tick0,
                       int ncols, int nticks, float* frame, cudaStream_t s)
{
    if (nrows <= 0) return;
    allow_smem((const void*)k_irfft_rows, 2 * d.M * sizeof(float2));
    const int nth = d.M >= 2048 ? 512 : 256;
    k_irfft_rows<<<nrows, nth, 2 * d.M * sizeof(float2), s>>>(Vh, nrows, d, wire0, wlo, whi, tick0, ncols, nticks,
                                                                  frame);
}

// ---------------------------------------------------------------------------
// Wire-direction convolution in the (wire, frequency) domain:
//   V[o][f] = sum_g sum_{j=-P}^{P} R_g[j][f] * Q_g[o - P - j][f]
// Input row i is wire row0 + i; output row o is wire row0 - P + o.
// Block: 32 frequencies x 8 row groups, each thread 8 consecutive output
// rows with a register sliding window over the staged input rows.
// Bin 0 (packed DC/Nyquist) is redone component-wise by k_wire_conv_dc.
// ---------------------------------------------------------------------------
constexpr int kConvRB = 8;
constexpr int kConvRG = 8;
constexpr int kConvRows = kConvRB * kConvRG;

template <int PAD>
__global__ void __launch_bounds__(32 * kConvRG) k_wire_conv(const float2* __restrict__ Qh,
                                                             const float2* __restrict__ Rh, float2* __restrict__ Vh,
                                                             int G, int nin, int nout, int M)
{
    constexpr int SROWS = kConvRows + 2 * PAD;
    __shared__ float2 Qs[SROWS][32];
    const int lane = threadIdx.x, rg = threadIdx.y;
    const int f = blockIdx.x * 32 + lane;
    const int o0 = blockIdx.y * kConvRows;
    const bool fok = f < M;
    float2 acc[kConvRB];
#pragma unroll
    for (int r = 0; r < kConvRB; ++r) acc[r] = make_float2(0.f, 0.f);
    const int rb0 = rg * kConvRB;
    for (int g = 0; g < G; ++g) {
        __syncthreads();
        for (int s = rg; s < SROWS; s += kConvRG) {
            const int i = o0 - 2 * PAD + s;
            Qs[s][lane] = (fok && i >= 0 && i < nin) ? Qh[((size_t)g * nin + i) * M + f] : make_float2(0.f, 0.f);
        }
        __syncthreads();
        if (fok) {
            const float2* Rg = Rh + (size_t)g * (2 * PAD + 1) * M + f;
            float2 win[kConvRB];
#pragma unroll
            for (int r = 0; r < kConvRB; ++r) win[r] = Qs[rb0 + r + 2 * PAD][lane];
#pragma unroll
            for (int jj = 0; jj <= 2 * PAD; ++jj) {
                const float2 rr = __ldg(Rg + (size_t)jj * M);
#pragma unroll
                for (int r = 0; r < kConvRB; ++r) {
                    acc[r].x = fmaf(rr.x, win[r].x, fmaf(-rr.y, win[r].y, acc[r].x));
                    acc[r].y = fmaf(rr.x, win[r].y, fmaf(rr.y, win[r].x, acc[r].y));
                }
                if (jj < 2 * PAD) {
#pragma unroll
                    for (int r = kConvRB - 1; r > 0; --r) win[r] = win[r - 1];
                    win[0] = Qs[rb0 + 2 * PAD - jj - 1][lane];
                }
            }
        }
    }
    if (fok) {
#pragma unroll
        for (int r = 0; r < kConvRB; ++r) {
            const int o = o0 + rb0 + r;
            if (o < nout) Vh[(size_t)o * M + f] = acc[r];
        }
    }
}

// Same convolution with a run-time pad (any response width).
__global__ void __launch_bounds__(32 * kConvRG) k_wire_conv_any(const float2* __restrict__ Qh,
                                                                 const float2* __restrict__ Rh,
                                                                 float2* __restrict__ Vh, int G, int PAD, int nin,
                                                                 int nout, int M)
{
    const int lane = threadIdx.x, rg = threadIdx.y;
    const int f = blockIdx.x * 32 + lane;
    const int o0 = blockIdx.y * kConvRows;
    if (f >= M) return;
    float2 acc[kConvRB];
#pragma unroll
    for (int r = 0; r < kConvRB; ++r) acc[r] = make_float2(0.f, 0.f);
    for (int g = 0; g < G; ++g) {
        const float2* Rg = Rh + (size_t)g * (2 * PAD + 1) * M + f;
        for (int jj = 0; jj <= 2 * PAD; ++jj) {
            const float2 rr = Rg[(size_t)jj * M];
            const int j = jj - PAD;
#pragma unroll
            for (int r = 0; r < kConvRB; ++r) {
                const int i = o0 + rg * kConvRB + r - PAD - j;
                if (i < 0 || i >= nin) continue;
                const float2 q = Qh[((size_t)g * nin + i) * M + f];
                acc[r].x = fmaf(rr.x, q.x, fmaf(-rr.y, q.y, acc[r].x));
                acc[r].y = fmaf(rr.x, q.y, fmaf(rr.y, q.x, acc[r].y));
            }
        }
    }
#pragma unroll
    for (int r = 0; r < kConvRB; ++r) {
        const int o = o0 + rg * kConvRB + r;
        if (o < nout) Vh[(size_t)o * M + f] = acc[r];
    }
}

// Bin 0 holds two real spectra (DC, Nyquist): convolve them component-wise.
__global__ void k_wire_conv_dc(const float2* __restrict__ Qh, const float2* __restrict__ Rh, float2* __restrict__ Vh,
                               int G, int PAD, int nin, int nout, int M)
{
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= nout) return;
    double ax = 0.0, ay = 0.0;
    for (int g = 0; g < G; ++g)
        for (int jj = 0; jj <= 2 * PAD; ++jj) {
            const int i = o - PAD - (jj - PAD);
            if (i < 0 || i >= nin) continue;
            const float2 r = Rh[((size_t)g * (2 * PAD + 1) + jj) * M];
            const float2 q = Qh[((size_t)g * nin + i) * M];
            ax += (double)r.x * q.x;
            ay += (double)r.y * q.y;
        }
    Vh[(size_t)o * M] = make_float2((float)ax, (float)ay);
}

void launch_wire_conv(const float2* Qh, const float2* Rh, float2* Vh, int ngroups, int npad, int nrows_in,
                      int nrows_out, int M, cudaStream_t s)
{
    if (nrows_out <= 0) return;
    dim3 grid((M + 31) / 32, (nrows_out + kConvRows - 1) / kConvRows);
    dim3 block(32, kConvRG);
    if (npad == 10) k_wire_conv<10><<<grid, block, 0, s>>>(Qh, Rh, Vh, ngroups, nrows_in, nrows_out, M);
    else if (npad == 21) k_wire_conv<21><<<grid, block, 0, s>>>(Qh, Rh, Vh, ngroups, nrows_in, nrows_out, M);
    else k_wire_conv_any<<<grid, block, 0, s>>>(Qh, Rh, Vh, ngroups, npad, nrows_in, nrows_out, M);
    k_wire_conv_dc<<<(nrows_out + 127) / 128, 128, 0, s>>>(Qh, Rh, Vh, ngroups, npad, nrows_in, nrows_out, M);
}

}  // namespace wctb200
