// DepoFluxSplat (gen/src/DepoFluxSplat.cxx:247-390): the truth frame of the
// depos' diffused charge on (wire, tick), no response.  One thread per depo,
// the planes in order as the reference visits them: a depo whose time span
// misses the window skips the plane, one whose pitch span misses the wire
// plane skips the remaining planes (the reference's `break`).  The patch is
// GaussianDiffusion::set_sampling (gen/src/GaussianDiffusion.cxx:116-182) on
// the window's tick binning and the plane's wire (region) binning
// (util/src/Pimpos.cxx:5-30): double erf bin integrals (GausDesc::binint,
// :30-56), float cells p_k t_j scaled by (float)(Q / sum), the absolute
// value added (double atomics) at row wire, tick toffset + tick offset + j.
#include <algorithm>

#include "kernels.cuh"

namespace wctb200 {

namespace {
__device__ __forceinline__ int sbin(double v, double lo, double bs)
{
    return __double2int_rz(__ddiv_rn(__dsub_rn(v, lo), bs));  // Binning::bin
}
__device__ __forceinline__ double sedge(int i, double lo, double bs)
{
    return __dadd_rn(lo, __dmul_rn((double)i, bs));  // Binning::edge
}
__device__ __forceinline__ double sdist(double x, double c, double s)
{
    return s != 0.0 ? __ddiv_rn(__dsub_rn(x, c), s) : __dsub_rn(x, c);  // GausDesc::distance
}
// GausDesc::binint value of bin k (k < n) from edges start + step * k.
__device__ __forceinline__ double sbinint(double start, double step, int k, double c, double s)
{
    if (s == 0.0) return 1.0;
    const double d = __dmul_rn(1.41421356237309515, s);  // sqrt(2.0) rounded to double
    const double x0 = __ddiv_rn(__dsub_rn(__dadd_rn(start, __dmul_rn(step, (double)k)), c), d);
    const double x1 = __ddiv_rn(__dsub_rn(__dadd_rn(start, __dmul_rn(step, (double)(k + 1))), c), d);
    return __dsub_rn(__dmul_rn(0.5, erf(x1)), __dmul_rn(0.5, erf(x0)));
}
}  // namespace

__global__ void __launch_bounds__(256) k_splat(const double* __restrict__ dep, int n, PlaneSet ps, SplatParams sp,
                                               double* __restrict__ acc)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double* p = dep + 7 * (size_t)i;
    const double t = p[0], q = p[1], x = p[2], y = p[3], z = p[4], el = p[5], et = p[6];
    // a depo with a NaN or infinite value is dropped, as the transform drops it:
    // its bin arithmetic is undefined and it would put NaNs in the frame
    if (!(isfinite(t) && isfinite(q) && isfinite(x) && isfinite(y) && isfinite(z) && isfinite(el) && isfinite(et)))
        return;
    if (ps.nplanes > 0 && ps.p[0].have_bb) {  // the face's sensitive volume
        const double pp[3] = {x, y, z};
        for (int k = 0; k < 3; ++k) {
            const double b1 = ps.p[0].bb_lo[k], b2 = ps.p[0].bb_hi[k];
            if (b1 < b2) { if (pp[k] < b1 || pp[k] > b2) return; }
            else if (b2 < b1) { if (pp[k] < b2 || pp[k] > b1) return; }
        }
    }
    const double nominal = __dadd_rn(t, sp.time_shift);
    const TimeDev& tb = sp.tb;
    for (int ip = 0; ip < ps.nplanes; ++ip) {
        const PlaneDev& pl = ps.p[ip];
        const SplatPlane& spl = sp.pl[ip];
        double sL = el;
        if (spl.smear_long > 0) {
            const double extra = __dmul_rn(__dmul_rn(spl.smear_long, tb.bs), sp.speed);
            sL = __dsqrt_rn(__dadd_rn(__dmul_rn(sL, sL), __dmul_rn(extra, extra)));
        }
        const double st = __ddiv_rn(sL, sp.speed);
        const double eff_t = el > 0 ? sp.nsigma : 0.0;
        if (sdist(tb.tmin, nominal, st) > eff_t || sdist(tb.tmax, nominal, st) < -eff_t) continue;
        const double rlo = pl.imp_min, rhi = pl.imp_max;
        const double rbs = __ddiv_rn(__dsub_rn(rhi, rlo), (double)pl.nwires);
        double sT = et;
        if (spl.smear_tran > 0) {
            const double extra = __dmul_rn(spl.smear_tran, rbs);
            sT = __dsqrt_rn(__dadd_rn(__dmul_rn(sT, sT), __dmul_rn(extra, extra)));
        }
        const double cp = __dadd_rn(__dadd_rn(__dmul_rn(pl.ax, __dsub_rn(x, pl.ox)), __dmul_rn(pl.ay, __dsub_rn(y, pl.oy))),
                                    __dmul_rn(pl.az, __dsub_rn(z, pl.oz)));
        const double eff_p = et > 0 ? sp.nsigma : 0.0;
        if (sdist(rlo, cp, sT) > eff_p || sdist(rhi, cp, sT) < -eff_p) break;
        // set_sampling windows (Binning::sample_bin_range)
        const int t0 = max(sbin(__dsub_rn(nominal, __dmul_rn(st, sp.nsigma)), tb.tmin, tb.bs), 0);
        const int t1 = min(sbin(__dadd_rn(nominal, __dmul_rn(st, sp.nsigma)), tb.tmin, tb.bs) + 1, tb.nbins);
        const int p0 = max(sbin(__dsub_rn(cp, __dmul_rn(sT, sp.nsigma)), rlo, rbs), 0);
        const int p1 = min(sbin(__dadd_rn(cp, __dmul_rn(sT, sp.nsigma)), rlo, rbs) + 1, pl.nwires);
        if (t1 <= t0 || p1 <= p0) continue;
        const int nt = st == 0.0 ? 1 : t1 - t0, np = sT == 0.0 ? 1 : p1 - p0;
        const double ts = sedge(t0, tb.tmin, tb.bs), ps0 = sedge(p0, rlo, rbs);
        double raw = 0.0;
        for (int a = 0; a < np; ++a) {
            const double pv = sbinint(ps0, rbs, a, cp, sT);
            for (int k = 0; k < nt; ++k) raw = __dadd_rn(raw, __dmul_rn(pv, sbinint(ts, tb.bs, k, nominal, st)));
        }
        const float scale = (float)__ddiv_rn(q, raw);
        const int tstart = (int)((double)t0 + spl.tick_offset);
        for (int a = 0; a < np; ++a) {
            const int pbin = p0 + a;
            if (pbin < 0 || pbin >= pl.nwires) continue;
            const double pv = sbinint(ps0, rbs, a, cp, sT);
            double* row = acc + (size_t)(pl.wire_base + pbin) * tb.nbins;
            for (int k = 0; k < nt; ++k) {
                const int tick = tstart + k;
                if (tick < 0 || tick >= tb.nbins) continue;
                const float v = (float)__dmul_rn(pv, sbinint(ts, tb.bs, k, nominal, st)) * scale;
                atomicAdd(row + tick, (double)fabsf(v));
            }
        }
    }
}

__global__ void k_splat_finish(const double* __restrict__ acc, float* __restrict__ frame, long long count)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < count;
         e += (long long)gridDim.x * blockDim.x)
        frame[e] = (float)acc[e];
}

void launch_splat_face(const double* depos, int n, const PlaneSet& ps, const SplatParams& sp, double* acc,
                       cudaStream_t s)
{
    if (n > 0 && ps.nplanes > 0) k_splat<<<(n + 255) / 256, 256, 0, s>>>(depos, n, ps, sp, acc);
}

void launch_splat_finish(const double* acc, float* frame, long long count, cudaStream_t s)
{
    if (count <= 0) return;
    const long long blocks = std::min<long long>((count + 255) / 256, 148LL * 32);
    k_splat_finish<<<(unsigned)blocks, 256, 0, s>>>(acc, frame, count);
}

}  // namespace wctb200
