// DepoTransform forward kernels for sm_100a.
//
// Pipeline for one event (all on one stream):
//   k_prep_all     drift + sensitive cut + BinnedDiffusion_transform::add +
//                  patch sample ranges + event window reduction + per-wire
//                  visit counts, all planes, one thread per depo
//   k_scan/k_fill  per-wire visit lists (CSR)
//   k_raster_wires erf-integrated patches with linear impact weights,
//                  accumulated per wire row in shared memory, written as the
//                  impact-group x tick charge grids       gen/src/BinnedDiffusion_transform.cxx:227-391
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
#include "gauss.cuh"
#include "rng.cuh"

#include <algorithm>
#include <cfloat>
#include <climits>

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
// Drift, sensitive volume, rejection, patch window and visit counting for
// every plane, one thread per depo.
//
//   Drifter::insert without fluctuation          gen/src/Drifter.cxx:127-196
//   sensitive-volume cut                          aux/src/DepoTools.cxx:110-123,
//                                                 util/src/BoundingBox.cxx:37-56
//   BinnedDiffusion_transform::add rejection      gen/src/BinnedDiffusion_transform.cxx:37-92
//   GaussianDiffusion sample ranges               gen/src/GaussianDiffusion.cxx:116-149
//   window reduction (impact/time_bin_range)      gen/src/BinnedDiffusion_transform.cxx:416-464
//
// Bin integrals of the unit Gaussian are differences of erfc on the side of
// the centre the bin lies on, so tail bins keep full FP32 relative accuracy
// (0.5*(erf(b) - erf(a)) of GaussianDiffusion.cxx:30-56 loses ~4 digits there).
// ---------------------------------------------------------------------------
// Visit keys of one patch: (wire, tick tile) pairs for the wires
// [w0, w0 + wspan) and tiles [k0, k0 + kspan); key = wire * ntiles + tile.
// Warp-aggregated increment of the per-key visit counters.
__device__ __forceinline__ void count_visits(int* cnt, int wbase, int w0, int wspan, int k0, int kspan, int ntiles)
{
    const int span = wspan * kspan;
    int maxspan = span;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) maxspan = max(maxspan, __shfl_xor_sync(0xffffffffu, maxspan, o));
    const int lane = threadIdx.x & 31;
    for (int k = 0; k < maxspan; ++k) {
        int key = -1;
        if (k < span) {
            const int dw = k / kspan, dk = k - dw * kspan;
            key = (wbase + w0 + dw) * ntiles + k0 + dk;
        }
        const unsigned act = __ballot_sync(0xffffffffu, key >= 0);
        if (key >= 0) {
            const unsigned m = __match_any_sync(act, key);
            if (lane == __ffs(m) - 1) atomicAdd(cnt + key, __popc(m));
        }
    }
}

// Magnitude bound of one visit's contribution to any cell: |q| * max bin
// fraction in pitch * max bin fraction in time * 2 (two bracketing groups).
__device__ __forceinline__ float visit_bound(float qn, float sp, float st, float pbs, float tbs)
{
    const float k = 0.39894228040143268f;  // 1/sqrt(2 pi)
    const float pm = sp > 0.f ? fminf(1.0f, k * pbs / sp) : 1.0f;
    const float tm = st > 0.f ? fminf(1.0f, k * tbs / st) : 1.0f;
    return 2.0f * fabsf(qn) * pm * tm * 1.0001f;
}

// Unit bin integral of bin k of a patch (edges at k*bs - cr and (k+1)*bs - cr
// from the centre), with explicitly rounded operations and not inlined, so
// every kernel that calls it gets the same value bit for bit.
__device__ __noinline__ float unit_bin(int k, float bs, float cr, float sigma)
{
    if (!(sigma > 0.f)) return 1.0f;  // point: its single bin holds everything
    const float inv = __frcp_rn(__fmul_rn(1.41421356237309505f, sigma));
    const float x1 = __fmul_rn(__fsub_rn(__fmul_rn((float)k, bs), cr), inv);
    const float x2 = __fmul_rn(__fsub_rn(__fmul_rn((float)(k + 1), bs), cr), inv);
    return bin_from_edges(copysignf(erfc_nr(fabsf(x1)), x1), copysignf(erfc_nr(fabsf(x2)), x2));
}

// 1 / (sum of the patch's unit bin integrals in pitch * in time), edge to edge.
__device__ __noinline__ float patch_inv_norm(const PatchRec& r, float pbs, float tbs)
{
    float sp = 1.f, st = 1.f;
    if (r.sp > 0.f) {
        const float inv = __frcp_rn(__fmul_rn(1.41421356237309505f, r.sp));
        const float x1 = __fmul_rn(__fsub_rn(0.f, r.pcr), inv);
        const float x2 = __fmul_rn(__fsub_rn(__fmul_rn((float)r.np, pbs), r.pcr), inv);
        sp = bin_from_edges(copysignf(erfc_nr(fabsf(x1)), x1), copysignf(erfc_nr(fabsf(x2)), x2));
    }
    if (r.st > 0.f) {
        const float inv = __frcp_rn(__fmul_rn(1.41421356237309505f, r.st));
        const float x1 = __fmul_rn(__fsub_rn(0.f, r.tcr), inv);
        const float x2 = __fmul_rn(__fsub_rn(__fmul_rn((float)r.nt, tbs), r.tcr), inv);
        st = bin_from_edges(copysignf(erfc_nr(fabsf(x1)), x1), copysignf(erfc_nr(fabsf(x2)), x2));
    }
    return __frcp_rn(__fmul_rn(sp, st));
}

// Event of a prep/fill block: blocks never straddle events.
__device__ __forceinline__ int event_of_block(const EventTable& et, int b)
{
    int lo = 0, hi = et.nev - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (et.blk0[mid] <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Frame ident of event ev of the launch: the key of its random streams.
__device__ __forceinline__ int fluc_ident(const FlucParams& fp, int ev)
{
    return (fp.ident_base ? *fp.ident_base : 0) + fp.ident0 + ev;
}

// One thread per (depo, plane) of every event of the table (plane =
// blockIdx.y; each plane's threads drift the depo again, which is cheaper
// than serialising the planes' FP64 chains in one thread); per-event window
// statistics, visit counters and bounds (nkeys keys per event); patch
// records [plane][depo]; plane 0's threads also write the drifted charge and
// the time profiles indexed by the depo's position in the concatenated depo
// array.
__global__ void __launch_bounds__(256, 4) k_prep_all(const double* __restrict__ dep, EventTable evt, int nkeys,
                                                  DriftDev dd, int do_drift, PlaneSet ps, TimeDev tb,
                                                  double drift_speed, double nsigma, PatchRec* __restrict__ rec,
                                                  WindowDev* __restrict__ win_all, int* __restrict__ cnt_all,
                                                  float* __restrict__ tprof, unsigned long long* __restrict__ kb_all,
                                                  FlucParams fp, double* __restrict__ fq,
                                                  unsigned char* __restrict__ wide_all, int blk_offset,
                                                  const double* __restrict__ qscale)
{
    const int bid = blockIdx.x + blk_offset;  // a launch may cover a range of the table's blocks
    const int ev = event_of_block(evt, bid);
    const int i = evt.dep0[ev] + (bid - evt.blk0[ev]) * blockDim.x + threadIdx.x;
    const int n = evt.dep0[evt.nev];  // record stride: all depos of the table
    const bool in = i < evt.dep0[ev + 1];
    WindowDev* win = win_all + (size_t)ev * ps.nplanes;
    int* wire_cnt = cnt_all + (size_t)ev * nkeys;
    unsigned long long* key_bound = kb_all + (size_t)ev * nkeys * kTileBlocks;
    double t = 0, q = 0, x = 0, y = 0, z = 0, el = 0, et = 0;
    bool ok = false;
    if (in) {
        const double* p = dep + 7 * (size_t)i;
        t = p[0]; q = p[1]; x = p[2]; y = p[3]; z = p[4]; el = p[5]; et = p[6];
        // a depo with a NaN or infinite value is dropped: the reference's
        // bin-index arithmetic is undefined for it, and its extents would
        // otherwise reach the event window's min/max reduction
        ok = isfinite(t) && isfinite(q) && isfinite(x) && isfinite(y) && isfinite(z) && isfinite(el) && isfinite(et);
        if (ok && do_drift) {
            if (q == 0.0) ok = false;
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
                if (found < 0) ok = false;
                else {
                    const double respx = dd.xr[found][1];
                    const double dt = fabs(__ddiv_rn(__dsub_rn(respx, x), dd.speed));
                    if (dir > 0) {
                        const double absorb = __dsub_rn(1.0, exp(__ddiv_rn(-dt, dd.lifetime)));
                        if (fp.on_drift) {
                            // Binomial(|Q|, absorb) electrons absorbed (Drifter.cxx:179-185)
                            Philox g;
                            g.init(fp.key0, fp.key1 + 0x9E3779B9u * (unsigned)fluc_ident(fp, ev),
                                   (unsigned)(i - evt.dep0[ev]), kRngDriftTag, 0u);
                            const int nabs = binomial((int)fabs(q), absorb, g);
                            q = __dsub_rn(q, q < 0 ? -(double)nabs : (double)nabs);
                        }
                        else q = __dsub_rn(q, __dmul_rn(q, absorb));
                        el = __dsqrt_rn(__dadd_rn(__dmul_rn(__dmul_rn(2.0, dd.DL), dt), __dmul_rn(el, el)));
                        et = __dsqrt_rn(__dadd_rn(__dmul_rn(__dmul_rn(2.0, dd.DT), dt), __dmul_rn(et, et)));
                    }
                    t = __dadd_rn(__dadd_rn(t, __dmul_rn(dir, dt)), dd.toffset);
                    x = respx;
                }
            }
        }
    }
    const int ip = blockIdx.y;
    // DepoTransform::modify_depo (DepoTransform.h:33-35, applied before
    // BinnedDiffusion_transform::add at DepoTransform.cxx:182) as a per-plane
    // charge scale, [depo][plane]
    if (qscale && in) q = __dmul_rn(q, qscale[(size_t)i * ps.nplanes + ip]);
    if (fq && in) fq[(size_t)ip * n + i] = q;  // the plane's charge: trial count of its fluctuated patch
    // The time profile depends on the depo only (GaussianDiffusion.cxx:124-136):
    // compute it once here for every plane's raster.
    if (ok && ip == 0) {
        const double st = __ddiv_rn(el, drift_speed);
        const double tlo = __dsub_rn(t, __dmul_rn(st, nsigma));
        const double thi = __dadd_rn(t, __dmul_rn(st, nsigma));
        const int t0 = max(bin_of(tlo, tb.tmin, tb.bs), 0);
        const int t1 = min(bin_of(thi, tb.tmin, tb.bs) + 1, tb.nbins);
        const int nt = t1 - t0;
        if (nt > kTprof) atomicAdd(&win[0].wide_ticks, (unsigned long long)nt);
        if (nt > 0 && nt <= kTprof) {
            float* tp = tprof + (size_t)i * kTprof;
            if (st > 0) {
                const float fst = (float)st;
                const float tcr = (float)__dsub_rn(t, edge_of(t0, tb.tmin, tb.bs));
                const float inv = 1.0f / (1.41421356237309505f * fst);
                const float tbs = (float)tb.bs;
                float e1 = edge_erfc(0.f, tbs, tcr, inv);
                for (int k = 0; k < nt; ++k) {
                    const float e2 = edge_erfc((float)(k + 1), tbs, tcr, inv);
                    tp[k] = bin_from_edges(e1, e2);
                    e1 = e2;
                }
            }
            else {
                tp[0] = 1.0f;
            }
        }
    }
    __shared__ unsigned long long s_k[4][8];
    __shared__ int s_c[5][8];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    auto umin = [](unsigned long long a, unsigned long long b) { return a < b ? a : b; };
    auto umax = [](unsigned long long a, unsigned long long b) { return a > b ? a : b; };
    auto iadd = [](int a, int b) { return a + b; };
    unsigned long long myvis = 0;
    {
        const PlaneDev& pl = ps.p[ip];
        unsigned long long kpmin = ~0ull, kpmax = 0ull, ktmin = ~0ull, ktmax = 0ull;
        int nadd = 0, nout_t = 0, nout_p = 0, nover = 0, nbig = 0;
        PatchRec r;
        r.toff = r.poff = 0;
        r.nt = r.np = 0;
        r.tcr = r.pcr = r.st = r.sp = r.qn = 0.f;
        bool inbb = ok;
        if (ok && pl.have_bb) {
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
                    if (nt > kMaxPatchT || np > kMaxPatchP || (st == 0.0 && nt != 1) || (sp == 0.0 && np != 1)) {
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
                        // normalisation to the full charge (GaussianDiffusion.cxx:176-182) with the
                        // sums of the unit bin integrals taken edge to edge
                        float sum_t = 1.f, sum_p = 1.f;
                        if (st > 0) {
                            const float inv = 1.0f / (1.41421356237309505f * r.st);
                            sum_t = bin_from_edges(edge_erfc(0.f, (float)tb.bs, r.tcr, inv),
                                                   edge_erfc((float)nt, (float)tb.bs, r.tcr, inv));
                        }
                        if (sp > 0) {
                            const float inv = 1.0f / (1.41421356237309505f * r.sp);
                            sum_p = bin_from_edges(edge_erfc(0.f, (float)pl.imp_bs, r.pcr, inv),
                                                   edge_erfc((float)np, (float)pl.imp_bs, r.pcr, inv));
                        }
                        r.qn = (float)(q / ((double)sum_t * (double)sum_p));
                    }
                }
            }
        }
        if (in) rec[(size_t)ip * n + i] = r;
        const int w0 = r.np ? r.poff / pl.nimp : 0;
        const int span = r.np ? (r.poff + r.np - 1) / pl.nimp - w0 + 1 : 0;
        const int k0 = r.toff / kTile;
        const int kspan = r.np ? (r.toff + r.nt - 1) / kTile - k0 + 1 : 0;
        count_visits(wire_cnt, pl.wire_base, w0, span, k0, kspan, ps.ntiles);
        myvis += (unsigned long long)span * (unsigned long long)kspan;
        if (r.nt > kTprof) {  // keys that hold a long patch: their raster block spreads visits over warps
            unsigned char* wk = wide_all + (size_t)ev * nkeys;
            for (int ww = 0; ww < span; ++ww)
                for (int kk = 0; kk < kspan; ++kk) wk[(pl.wire_base + w0 + ww) * ps.ntiles + k0 + kk] = 1;
        }
        // fixed-point bounds of the raster: per (wire, tile, 64-tick block), summed
        // as integers in units of 2^-16 (each term rounded up), so the bound --
        // and with it the raster's scale -- does not depend on the order of the adds
        if (r.np) {
            const float b = visit_bound(r.qn, r.sp, r.st, (float)pl.imp_bs, (float)tb.bs);
            if (b > kMaxVisitBound) nbig = 1;
            const unsigned long long bu = __float2ull_ru(fminf(b, kMaxVisitBound) * 65536.0f);
            const int b0 = r.toff / kScaleBlock, b1 = (r.toff + r.nt - 1) / kScaleBlock;
            for (int ww = 0; ww < span; ++ww) {
                unsigned long long* kb = key_bound + (size_t)(pl.wire_base + w0 + ww) * ps.ntiles * kTileBlocks;
                for (int bb = b0; bb <= b1; ++bb) atomicAdd(kb + bb, bu);
            }
        }
        // block reduction, one atomic per block per quantity
        kpmin = warp_reduce(kpmin, umin);
        ktmin = warp_reduce(ktmin, umin);
        kpmax = warp_reduce(kpmax, umax);
        ktmax = warp_reduce(ktmax, umax);
        nadd = warp_reduce(nadd, iadd);
        nout_t = warp_reduce(nout_t, iadd);
        nout_p = warp_reduce(nout_p, iadd);
        nover = warp_reduce(nover, iadd);
        nbig = warp_reduce(nbig, iadd);
        if (l == 0) {
            s_k[0][w] = kpmin; s_k[1][w] = kpmax; s_k[2][w] = ktmin; s_k[3][w] = ktmax;
            s_c[0][w] = nadd; s_c[1][w] = nout_t; s_c[2][w] = nout_p; s_c[3][w] = nover; s_c[4][w] = nbig;
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
            nbig = l < nw ? s_c[4][l] : 0;
            kpmin = warp_reduce(kpmin, umin);
            ktmin = warp_reduce(ktmin, umin);
            kpmax = warp_reduce(kpmax, umax);
            ktmax = warp_reduce(ktmax, umax);
            nadd = warp_reduce(nadd, iadd);
            nout_t = warp_reduce(nout_t, iadd);
            nout_p = warp_reduce(nout_p, iadd);
            nover = warp_reduce(nover, iadd);
            nbig = warp_reduce(nbig, iadd);
            WindowDev* wd = win + ip;
            if (l == 0 && nadd) {
                atomicMin(&wd->pmin, kpmin);
                atomicMax(&wd->pmax, kpmax);
                atomicMin(&wd->tmin, ktmin);
                atomicMax(&wd->tmax, ktmax);
                atomicAdd(&wd->nadded, nadd);
            }
            if (l == 0 && nout_t) atomicAdd(&wd->out_time, nout_t);
            if (l == 0 && nout_p) atomicAdd(&wd->out_pitch, nout_p);
            if (l == 0 && nover) atomicAdd(&wd->oversize, nover);
            if (l == 0 && nbig) atomicAdd(&wd->bigcharge, nbig);
        }
    }
    // 64-bit visit total of the event (the visit lists use int offsets)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) myvis += __shfl_xor_sync(0xffffffffu, myvis, o);
    if (l == 0 && myvis) atomicAdd(&win[0].nvisits, myvis);
}

void launch_prep_all(const double* depos, const EventTable& et, int nkeys, const DriftDev& dd, int do_drift,
                     const PlaneSet& ps, const TimeDev& tb, double drift_speed, double nsigma, PatchRec* rec,
                     WindowDev* win, int* wire_cnt, float* tprof, unsigned long long* key_bound,
                     const FlucParams& fp, double* fq, unsigned char* wide, cudaStream_t s, int blk_begin,
                     int blk_end, const double* qscale)
{
    const int nb = et.blk0[et.nev];
    const int b0 = std::max(0, blk_begin), b1 = blk_end < 0 ? nb : std::min(blk_end, nb);
    if (b1 <= b0) return;
    k_prep_all<<<dim3(b1 - b0, ps.nplanes), 256, 0, s>>>(depos, et, nkeys, dd, do_drift, ps, tb, drift_speed,
                                                         nsigma, rec, win, wire_cnt, tprof, key_bound, fp, fq, wide,
                                                         b0, qscale);
}

// Exclusive scan of the per-key visit counts: block sums, a scan of the
// block sums, then per-block scans with their offsets.
constexpr int kScanBlock = 1024;

__device__ __forceinline__ int block_scan_excl(int v, int* s_warp, int& total)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[w] = x;
    __syncthreads();
    if (w == 0) {
        int t = lane < (int)(blockDim.x >> 5) ? s_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        s_warp[lane] = t;
    }
    __syncthreads();
    total = s_warp[(blockDim.x >> 5) - 1];
    const int before = w ? s_warp[w - 1] : 0;
    __syncthreads();
    return before + x - v;
}

__global__ void __launch_bounds__(kScanBlock) k_scan_sums(const int* __restrict__ cnt, int n, int* __restrict__ sums)
{
    __shared__ int s_warp[32];
    const int i = blockIdx.x * kScanBlock + threadIdx.x;
    int total = 0;
    block_scan_excl(i < n ? cnt[i] : 0, s_warp, total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanBlock) k_scan_top(int* __restrict__ sums, int nb, int* __restrict__ total_out)
{
    __shared__ int s_warp[32];
    int carry = 0;
    for (int b0 = 0; b0 < nb; b0 += kScanBlock) {
        const int i = b0 + threadIdx.x;
        int total = 0;
        const int ex = block_scan_excl(i < nb ? sums[i] : 0, s_warp, total);
        if (i < nb) sums[i] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0) *total_out = carry;
}

__global__ void __launch_bounds__(kScanBlock) k_scan_apply(const int* __restrict__ cnt, int n,
                                                           const int* __restrict__ sums, int* __restrict__ off,
                                                           int* __restrict__ cur)
{
    __shared__ int s_warp[32];
    const int i = blockIdx.x * kScanBlock + threadIdx.x;
    int total = 0;
    const int ex = block_scan_excl(i < n ? cnt[i] : 0, s_warp, total) + sums[blockIdx.x];
    if (i < n) {
        off[i] = ex;
        cur[i] = ex;
    }
}

void launch_scan(const int* wire_cnt, int nwires_total, int* wire_off, int* wire_cur, cudaStream_t s)
{
    // wire_cur[nwires_total + 1 ..] holds the block sums (the caller sizes it)
    const int n = nwires_total;
    const int nb = (n + kScanBlock - 1) / kScanBlock;
    int* sums = wire_cur + n + 1;
    k_scan_sums<<<nb, kScanBlock, 0, s>>>(wire_cnt, n, sums);
    k_scan_top<<<1, kScanBlock, 0, s>>>(sums, nb, wire_off + n);
    k_scan_apply<<<nb, kScanBlock, 0, s>>>(wire_cnt, n, sums, wire_off, wire_cur);
}

// Time profiles of the long patches, one warp per depo (its first plane with a
// patch: the time profile does not depend on the plane).
__global__ void __launch_bounds__(256) k_tprof_pool(const PatchRec* __restrict__ rec, EventTable evt, int nplanes,
                                                   float tbs, TprofPool pool, int* status)
{
    const int lane = threadIdx.x & 31;
    const int n = evt.dep0[evt.nev];
    const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (i >= n) return;  // whole warps
    PatchRec r{};
    for (int ip = 0; ip < nplanes; ++ip) {
        r = rec[(size_t)ip * n + i];
        if (r.np) break;
    }
    int off = -1;
    if (r.np && r.nt > kTprof) {
        long long off64 = 0;
        if (lane == 0) off64 = (long long)atomicAdd(pool.used, (unsigned long long)r.nt);
        off64 = __shfl_sync(0xffffffffu, off64, 0);
        off = off64 + r.nt > pool.cap ? -1 : (int)off64;  // 64-bit counter: no wrap
        if (off < 0) {
            off = -1;
            if (lane == 0 && status) atomicOr(status, kBatchPoolShort);
        }
        else
            for (int t = lane; t < r.nt; t += 32) pool.val[off + t] = unit_bin(t, tbs, r.tcr, r.st);
    }
    if (lane == 0) pool.off[i] = off;
}

void launch_tprof_pool(const PatchRec* rec, const EventTable& et, int nplanes, float tbs, const TprofPool& pool,
                       int* status, cudaStream_t s)
{
    const int n = et.dep0[et.nev];
    if (n <= 0) return;
    k_tprof_pool<<<(n + 7) / 8, 256, 0, s>>>(rec, et, nplanes, tbs, pool, status);
}

// Per-wire visit lists: wire_list[wire_off[w] ..] holds the depo indices whose
// patch covers wire w (any order).
__global__ void __launch_bounds__(256) k_fill(const PatchRec* __restrict__ rec, EventTable evt, int nkeys,
                                              PlaneSet ps, int* __restrict__ cur, Visit* __restrict__ list,
                                              long long cap)
{
    const int ev = event_of_block(evt, blockIdx.x);
    const int i = evt.dep0[ev] + (blockIdx.x - evt.blk0[ev]) * blockDim.x + threadIdx.x;
    const int n = evt.dep0[evt.nev];
    const bool in = i < evt.dep0[ev + 1];
    const int key0 = ev * nkeys;
    const int lane = threadIdx.x & 31;
    for (int ip = 0; ip < ps.nplanes; ++ip) {
        const PlaneDev& pl = ps.p[ip];
        int w0 = 0, span = 0, k0 = 0, kspan = 1;
        PatchRec r{};
        if (in) {
            r = rec[(size_t)ip * n + i];
            if (r.np) {
                w0 = r.poff / pl.nimp;
                k0 = r.toff / kTile;
                kspan = (r.toff + r.nt - 1) / kTile - k0 + 1;
                span = ((r.poff + r.np - 1) / pl.nimp - w0 + 1) * kspan;
            }
        }
        int maxspan = span;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) maxspan = max(maxspan, __shfl_xor_sync(0xffffffffu, maxspan, o));
        for (int k = 0; k < maxspan; ++k) {
            int key = -1;
            if (k < span) {
                const int dw = k / kspan, dk = k - dw * kspan;
                key = key0 + (pl.wire_base + w0 + dw) * ps.ntiles + k0 + dk;
            }
            const unsigned act = __ballot_sync(0xffffffffu, key >= 0);
            if (key >= 0) {
                const unsigned m = __match_any_sync(act, key);
                const int leader = __ffs(m) - 1;
                int base = 0;
                if (lane == leader) base = atomicAdd(cur + key, __popc(m));
                base = __shfl_sync(m, base, leader);
                const int rank = __popc(m & ((1u << lane) - 1u));
                const long long at = (long long)base + rank;
                if (at >= 0 && at < cap) list[at] = i;  // outside: the caller reports an overflow
            }
        }
    }
}

void launch_fill(const PatchRec* rec, const EventTable& et, int nkeys, const PlaneSet& ps, int* wire_cur,
                 Visit* visits, long long cap, cudaStream_t s)
{
    const int nblocks = et.blk0[et.nev];
    if (nblocks <= 0) return;
    k_fill<<<nblocks, 256, 0, s>>>(rec, et, nkeys, ps, wire_cur, visits, cap);
}

// ---------------------------------------------------------------------------
// Charge grids: one block per charge wire row of every plane.  The block
// accumulates the row's impact-group x tick grid in shared memory (one thread
// per depo visit of the wire), then writes the G rows of the plane grid with
// zero padding up to the FFT length.  Each patch bin adds weight*q to the
// group of its lower impact edge and (1-weight)*q to the next
// (BinnedDiffusion_transform.cxx:296-367, linear weights of
// GausDesc::weight, GaussianDiffusion.cxx:61-92).
//
// Accumulation is in 32-bit fixed point (native shared-memory integer
// atomics; FP32 shared atomics are compare-and-swap loops).  Every 64-tick
// block of the row has its own scale 2^30 / B, where B bounds the magnitude
// any cell of the block can reach: the sum over the visits touching the block
// of |q| * max bin fraction in pitch * max bin fraction in time * 2.  Cells
// cannot overflow and one add is resolved to ~2^-30 of that local bound.
// Integer sums are order independent (the bounds too are integer sums), so
// the grid is bit-reproducible.
// ---------------------------------------------------------------------------
constexpr int kRasterThreads = 256;
// staged per visit: 12 group coefficients, q, and 16 scaled tick values (odd stride: no bank conflicts)
constexpr int kStageQ = 12;
constexpr int kStageT = 13;
constexpr int kStageStride = 29;
constexpr int kTileLd = kTile + 8;  // fluctuated raster: row stride with an 8-word skew between groups
// Forward raster grid row stride: 4 words of skew, so eight visits scattering
// to eight consecutive group rows at the same four columns hit 32 distinct banks.
constexpr int kGridLd = kTile + 4;

size_t raster_smem_bytes(int G)
{
    return sizeof(int) * (size_t)G * kGridLd + sizeof(float) * (size_t)kRasterThreads * kStageStride +
           sizeof(int4) * (size_t)kRasterThreads;
}

// One raster work item: charge row `row` (wire start_ch + row) of plane P and
// absolute tick tile ktile.  Visit keys are key_base + wire * ntiles_abs +
// tile; at most vcap visits exist.  Called by all threads of the block;
// smem_i holds the dynamic shared memory of raster_smem_bytes(P.G).
__device__ __forceinline__ void raster_tile(const GridPlane& P, int row, int ktile, int key_base, int ntiles_abs,
                                            const PatchRec* __restrict__ rec, const float* __restrict__ tprof,
                                            const TprofPool& pool, const unsigned char* __restrict__ wide_key,
                                            const int* __restrict__ wire_cnt, const int* __restrict__ wire_off,
                                            const Visit* __restrict__ visits, long long vcap,
                                            const unsigned long long* __restrict__ key_bound,
                                            float* __restrict__ Q, int* smem_i, float* scale, float* iscale)
{
    __syncthreads();  // the previous item of a persistent block is done with the shared arrays
    const int w = P.start_ch + row;
    const int G = P.G, nimp = P.nimp;
    const int tick_lo = ktile * kTile;                      // absolute first tick of the tile
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    int* grid = smem_i;                                       // [G][kGridLd], column = tick - tick_lo
    float* stage = reinterpret_cast<float*>(smem_i + (size_t)G * kGridLd);
    int4* stagei = reinterpret_cast<int4*>(stage + (size_t)kRasterThreads * kStageStride);
    int cnt = 0;
    const Visit* list = nullptr;
    int key = -1;
    if (w >= 0 && w < P.nwires && ktile >= 0 && ktile < ntiles_abs) {
        key = key_base + (P.wire_base + w) * ntiles_abs + ktile;
        const int off = wire_off[key];
        cnt = off < 0 ? 0 : (int)min((long long)wire_cnt[key], max(0ll, vcap - off));  // no reads past the list
        list = visits + max(off, 0);
    }
    if (cnt == 0) {
        // no visit (block-uniform): the tile's G rows are zero
        const int qc0 = tick_lo - P.col0;
        for (int k = tid; k < G * kTile; k += kRasterThreads) {
            const int g = k / kTile, c = k - g * kTile;
            const int qc = qc0 + c;
            if (qc >= 0 && qc < P.N) Q[P.qoff + ((size_t)g * P.nin + row) * P.N + qc] = 0.f;
        }
        return;
    }
    const bool spread = key >= 0 && wide_key[key];
    {
        int4* g4 = reinterpret_cast<int4*>(grid);
        const int n4 = G * kGridLd / 4;
        for (int k = tid; k < n4; k += kRasterThreads) g4[k] = make_int4(0, 0, 0, 0);
        if (tid < kTileBlocks) {
            const float b = key >= 0 ? __ull2float_ru(key_bound[(size_t)key * kTileBlocks + tid]) * (1.0f / 65536.0f)
                                     : 0.f;
            scale[tid] = b > 0.f ? 1073741824.0f / b : 0.f;
            iscale[tid] = b > 0.f ? b / 1073741824.0f : 0.f;
        }
    }
    __syncthreads();
    const float pbs = P.pbs, tbs = P.tbs;
    const int wlo = w * nimp;
    // pass 2: each lane stages the group coefficients of one visit, then the
    // warp scatters its 32 staged visits, two at a time (half-warp per visit,
    // lanes over ticks, loop over the covered groups; whole warp for a pair
    // with a visit longer than 16 ticks).
    float* my = stage + (size_t)tid * kStageStride;
    const int wbase = wid * 32;
    const float inv_pbs = 1.0f / pbs;
    const int nchunks = (cnt + kRasterThreads - 1) / kRasterThreads;
    for (int ch = 0; ch < nchunks; ++ch) {
        // visit of this thread: in blocks with long patches, lanes 2k, 2k+1
        // hold consecutive visits (a pair) and consecutive pairs go to
        // different warps (the lists hold one depo kind in runs: long patches
        // would otherwise pile up on a few warps); elsewhere visits stay in
        // list order (coalesced reads, alike neighbours along a track)
        const int e = ch * kRasterThreads +
                      (spread ? (lane >> 1) * (kRasterThreads / 16) + wid * 2 + (lane & 1) : tid);
        const bool valid = e < cnt;
        int4 si = make_int4(0, 0, 0, 0);  // d, l_lo, ng, (cb << 11) | nt  (cb = toff - tick_lo, ng = 0: none)
        if (valid) {
            const int d = list[e];
            const PatchRec r = rec[P.recoff + d];
            const int rnp = r.np, rnt = r.nt;
            const int l_lo = max(r.poff, wlo) - wlo;
            const int l_hi = min(r.poff + rnp, wlo + nimp) - wlo;
            if (l_hi > l_lo) {
                const int ng = l_hi - l_lo + 1;
                if (r.sp > 0.f) {
                    const float isg = __frcp_rn(r.sp);
                    const float inv = 0.70710678118654752f * isg;            // 1/(sqrt2 sigma)
                    const float c0 = r.sp * inv_pbs * 0.39894228040143268f;  // sigma / (step*sqrt(2 pi))
                    const int k0 = wlo + l_lo - r.poff;
                    float x1 = (float)k0 * pbs - r.pcr;
                    float e1 = copysignf(erfc_nr(fabsf(x1 * inv)), x1);
                    float u1 = x1 * isg;
                    float g1 = __expf(-0.5f * u1 * u1);
                    // group lb gets p_lb * w_lb + p_(lb-1) * (1 - w_(lb-1)): the
                    // second term is carried in a register to the next bin
                    float carry = 0.f;
                    for (int lb = 0; lb < ng - 1; ++lb) {
                        const float x2 = (float)(k0 + lb + 1) * pbs - r.pcr;
                        const float e2 = copysignf(erfc_nr(fabsf(x2 * inv)), x2);
                        const float u2 = x2 * isg;
                        const float g2 = __expf(-0.5f * u2 * u2);
                        const float p = bin_from_edges(e1, e2);
                        const float wt = p > 0.f ? fmaf(c0 * (g2 - g1), __fdividef(1.0f, p), x2 * inv_pbs) : 0.0f;
                        my[lb] = carry + p * wt;
                        carry = p * (1.0f - wt);
                        e1 = e2;
                        g1 = g2;
                    }
                    my[ng - 1] = carry;
                }
                else {
                    const float wt = (pbs - r.pcr) * inv_pbs;
                    my[0] = wt;
                    my[1] = 1.0f - wt;
                }
                const int cb = r.toff - tick_lo;  // may be negative for patches starting in the previous tile
                si = make_int4(d, l_lo, ng, ((cb + 1024) << 11) | rnt);
                my[kStageQ] = r.qn;
                if (rnt <= 16) {
                    // tick values scaled to the fixed point of their 64-tick block (0 outside the tile);
                    // the whole 16-value profile row in four 128-bit loads (one L1 wavefront per
                    // lane each, against one per value with scalar loads)
                    static_assert(kTprof == 16, "profile rows are four float4");
                    const float4* tp4 = reinterpret_cast<const float4*>(tprof + (size_t)d * kTprof);
                    float tv[16];
#pragma unroll
                    for (int k4 = 0; k4 < 4; ++k4) {
                        const float4 x = __ldg(tp4 + k4);
                        tv[4 * k4] = x.x;
                        tv[4 * k4 + 1] = x.y;
                        tv[4 * k4 + 2] = x.z;
                        tv[4 * k4 + 3] = x.w;
                    }
#pragma unroll
                    for (int k = 0; k < 16; ++k) {
                        const int c = cb + k;
                        float v = 0.f;
                        if (k < rnt && c >= 0 && c < kTile) v = tv[k] * r.qn * scale[c / kScaleBlock];
                        my[kStageT + k] = v;
                    }
                }
            }
        }
        stagei[tid] = si;
        __syncwarp();
        // lanes 0 .. nv-1 of this warp hold visits (e grows with the lane)
        const int nv = __popc(__ballot_sync(0xffffffffu, valid));
        // eight visits at a time: four lanes per visit, each lane four ticks (hl + 4k)
        const int qv = lane >> 2, hl = lane & 3;
        for (int v0 = 0; v0 < nv; v0 += 8) {
            const int v = v0 + qv;
            int4 vi = make_int4(0, 0, 0, 0);
            if (v < nv) vi = stagei[wbase + v];
            const int nt = vi.w & 2047;
            const bool wide = __any_sync(0xffffffffu, nt > 16);
            if (!wide) {
                const int ng = vi.z;
                const int c0 = (vi.w >> 11) - 1024 + hl;  // tile column of this lane's first tick
                const float* vc = stage + (size_t)(wbase + min(v, 31)) * kStageStride;
                float tq[4];
                int gl[4];  // groups this lane adds at tick hl + 4k (0: tick outside the patch or tile)
                int mgl = 0;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int c = c0 + 4 * k;
                    const bool on = hl + 4 * k < nt && c >= 0 && c < kTile;
                    tq[k] = on ? vc[kStageT + hl + 4 * k] : 0.f;
                    gl[k] = on ? ng : 0;
                    mgl = max(mgl, gl[k]);
                }
                const int mg = __reduce_max_sync(0xffffffffu, mgl);
                // the eight visits start at spread-out groups and wrap around
                // (visit slot qv at group qv*ng/8): visits of one track share
                // their columns and would otherwise hit the same words together
                int gg = (qv * ng) >> 3;
                int* dst = grid + (vi.y + gg) * kGridLd + c0;
                int* const wrap = grid + vi.y * kGridLd + c0;
                int* const last = wrap + (ng - 1) * kGridLd;
                float cf = vc[gg];
                for (int g = 0; g < mg; ++g) {
                    const bool w = dst == last;
                    const int gn = w ? 0 : gg + 1;
                    const float cfn = vc[gn];  // next group's coefficient, loaded ahead
                    int v4[4];
#pragma unroll
                    for (int k = 0; k < 4; ++k) v4[k] = __float2int_rn(cf * tq[k]);
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        if (g < gl[k]) atomicAdd(dst + 4 * k, v4[k]);
                    dst = w ? wrap : dst + kGridLd;
                    gg = gn;
                    cf = cfn;
                }
            }
            else {
                // at least one of the eight has more than 16 ticks: whole warp per visit
                for (int hv = 0; hv < 8; ++hv) {
                    const int vv = v0 + hv;
                    if (vv >= nv) break;
                    const int4 wi = stagei[wbase + vv];
                    const int ng = wi.z;
                    if (ng == 0) continue;
                    const int wnt = wi.w & 2047;
                    const int cb = (wi.w >> 11) - 1024;
                    const float* vc = stage + (size_t)(wbase + vv) * kStageStride;
                    const float qn = vc[kStageQ];
                    const int tstart = max(0, -cb), tend = min(wnt, kTile - cb);  // ticks inside the tile
                    const int poff = wnt > kTprof ? __ldg(pool.off + wi.x) : -1;
                    float rtcr = 0.f, rst = 0.f;
                    if (wnt > kTprof && poff < 0) {
                        const PatchRec r = rec[P.recoff + wi.x];
                        rtcr = r.tcr;
                        rst = r.st;
                    }
                    for (int tc = tstart; tc < tend; tc += 32) {
                        const int it = tc + lane;
                        const bool on = it < tend;
                        float tq = 0.f;
                        if (on) {
                            float tv;
                            if (wnt <= kTprof) tv = __ldg(tprof + (size_t)wi.x * kTprof + it);
                            else if (poff >= 0) tv = __ldg(pool.val + poff + it);
                            else tv = unit_bin(it, tbs, rtcr, rst);
                            tq = tv * qn * scale[(cb + it) / kScaleBlock];
                        }
                        int* dst = grid + wi.y * kGridLd + cb + it;
                        for (int g = 0; g < ng; ++g) {
                            if (on) atomicAdd(dst, __float2int_rn(vc[g] * tq));
                            dst += kGridLd;
                        }
                    }
                }
            }
        }
        __syncwarp();
    }
    __syncthreads();
    // write the tile's G rows, four columns per thread: grid column c is plane
    // column tick_lo + c - col0 (zero at or past the window's ncols)
    const int qc0 = tick_lo - P.col0;
    constexpr int kQuads = kTile / 4;
    for (int k = tid; k < G * kQuads; k += kRasterThreads) {
        const int g = k / kQuads, c = (k - g * kQuads) * 4;
        const int4 cell = *reinterpret_cast<const int4*>(grid + g * kGridLd + c);
        const float is = iscale[c / kScaleBlock];  // the four columns share one 64-tick block
        float* dst = Q + P.qoff + ((size_t)g * P.nin + row) * P.N + qc0 + c;
        const int q0 = qc0 + c;
        const float v[4] = {(float)cell.x * is, (float)cell.y * is, (float)cell.z * is, (float)cell.w * is};
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (q0 + u >= 0 && q0 + u < P.N) dst[u] = q0 + u < P.ncols ? v[u] : 0.f;
    }
}

__global__ void __launch_bounds__(kRasterThreads, 5) k_raster_wires(const PatchRec* __restrict__ rec,
                                                                 const float* __restrict__ tprof,
                                                                 const int* __restrict__ wire_cnt,
                                                                 const int* __restrict__ wire_off,
                                                                 const Visit* __restrict__ visits, long long vcap,
                                                                 const unsigned long long* __restrict__ key_bound,
                                                                 GridSet gs, float* __restrict__ Q, TprofPool pool,
                                                                 const unsigned char* __restrict__ wide_key)
{
    extern __shared__ int smem_i[];
    __shared__ float scale[kTileBlocks], iscale[kTileBlocks];
    int ip = 0;
    while (ip + 1 < gs.nplanes && (int)blockIdx.x >= gs.p[ip + 1].row_base) ++ip;
    const GridPlane& P = gs.p[ip];
    const int rel = blockIdx.x - P.row_base;
    const int row = rel / P.ntile;
    const int ktile = P.ktile0 + (rel - row * P.ntile);  // absolute tick tile
    raster_tile(P, row, ktile, 0, gs.ntiles_abs, rec, tprof, pool, wide_key, wire_cnt, wire_off, visits, vcap,
                key_bound, Q, smem_i, scale, iscale);
}

void launch_raster_wires(const PatchRec* rec, const float* tprof, const TprofPool& pool, const unsigned char* wide_key,
                         const int* wire_cnt,
                         const int* wire_off, const Visit* visits, long long vcap,
                         const unsigned long long* key_bound, const GridSet& gs, float* Q, cudaStream_t s)
{
    if (gs.nrows_total <= 0) return;
    size_t smem = 0;
    for (int i = 0; i < gs.nplanes; ++i) smem = std::max(smem, raster_smem_bytes(gs.p[i].G));
    cudaFuncSetAttribute((const void*)k_raster_wires, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_raster_wires<<<gs.nrows_total, kRasterThreads, smem, s>>>(rec, tprof, wire_cnt, wire_off, visits, vcap,
                                                                    key_bound, gs, Q, pool, wide_key);
}

// ---------------------------------------------------------------------------
// Fluctuated patches (GaussianDiffusion::set_sampling with an IRandom,
// gen/src/GaussianDiffusion.cxx:184-213): every cell (k, tau) of a patch is
// redrawn as N ~ Binomial((int)|Q|, p_k t_tau / (sum p * sum t)) and the
// patch is rescaled by Q / sum N; a patch whose draws are all zero adds
// nothing.  The draws are counter-based: k_fluc_sums draws every cell to get
// sum N, and the fluctuated raster draws the same cells again.  The unit bin
// integrals that set each cell's probability come from one non-inlined
// function with explicitly rounded operations, so both passes see the same
// probabilities bit for bit and therefore the same draws.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int event_of_depo(const EventTable& et, int i)
{
    int lo = 0, hi = et.nev - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (et.dep0[mid] <= i) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// The draw of cell (k, tau) of depo i_ev (index within its event) on plane ip.
__device__ __forceinline__ int cell_draw(const FlucParams& fp, int ident, int i_ev, int ip, int cell, int nq,
                                         float relval)
{
    Philox g;
    g.init(fp.key0, fp.key1 + 0x9E3779B9u * (unsigned)ident, (unsigned)i_ev, (unsigned)ip, (unsigned)cell);
    return binomial(nq, (double)relval, g);
}

constexpr int kFlucWarps = 4;
constexpr int kFlucTab = 1024;  // patches hold at most kMaxPatchT ticks and kMaxPatchP bins

// One warp per (plane, depo): the sum of the cell draws.
__global__ void __launch_bounds__(kFlucWarps * 32) k_fluc_sums(const PatchRec* __restrict__ rec, EventTable evt,
                                                               PlaneSet ps, float tbs, FlucParams fp,
                                                               const double* __restrict__ fq,
                                                               FlucRec* __restrict__ fluc)
{
    __shared__ float s_p[kFlucWarps][kFlucTab], s_t[kFlucWarps][kFlucTab];
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n = evt.dep0[evt.nev];
    const long long gw = (long long)blockIdx.x * kFlucWarps + wib;
    if (gw >= (long long)n * ps.nplanes) return;  // whole warps only; no block barrier follows
    const int ip = (int)(gw / n), i = (int)(gw - (long long)ip * n);
    const PatchRec r = rec[(size_t)ip * n + i];
    FlucRec out{0, 0.f, 0.f, 0};
    if (r.np > 0 && r.nt > 0) {
        const float pbs = (float)ps.p[ip].imp_bs;
        const int np = r.np, nt = r.nt;
        for (int k = lane; k < np; k += 32) s_p[wib][k] = unit_bin(k, pbs, r.pcr, r.sp);
        for (int t = lane; t < nt; t += 32) s_t[wib][t] = unit_bin(t, tbs, r.tcr, r.st);
        __syncwarp();
        const float invS = patch_inv_norm(r, pbs, tbs);
        const double Q = fq[(size_t)ip * n + i];
        const int nq = (int)fabs(Q);
        const int ev = event_of_depo(evt, i);
        const int ident = fluc_ident(fp, ev), i_ev = i - evt.dep0[ev];
        long long sum = 0;
        for (int c = lane; c < np * nt; c += 32) {
            const int k = c / nt, t = c - k * nt;
            const float relval = __fmul_rn(__fmul_rn(s_p[wib][k], s_t[wib][t]), invS);
            sum += cell_draw(fp, ident, i_ev, ip, c, nq, relval);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        out.nq = nq;
        out.invS = invS;
        out.scale = sum > 0 ? (float)(Q / (double)sum) : 0.f;
    }
    if (lane == 0) fluc[(size_t)ip * n + i] = out;
}

void launch_fluc_sums(const PatchRec* rec, const EventTable& et, const PlaneSet& ps, float tbs, const FlucParams& fp,
                      const double* fq, FlucRec* fluc, cudaStream_t s)
{
    const long long warps = (long long)et.dep0[et.nev] * ps.nplanes;
    if (warps <= 0) return;
    const long long blocks = (warps + kFlucWarps - 1) / kFlucWarps;
    k_fluc_sums<<<(unsigned)blocks, kFlucWarps * 32, 0, s>>>(rec, et, ps, tbs, fp, fq, fluc);
}

// Fluctuated raster of one (charge row, tick tile) item: one warp per visit,
// lanes over the visit's ticks in the tile, a loop over the patch bins of the
// row's wire; cell charges N * Q / sum N split between the two impact groups
// of the bin by its linear weight (BinnedDiffusion_transform.cxx:296-367).
// Accumulation in 64-bit fixed point (2^-16 electron), so the grid does not
// depend on the order of the adds.
constexpr int kFlucRasterThreads = 256;
constexpr float kFlucFix = 65536.0f;

size_t raster_fluc_smem_bytes(int G) { return sizeof(long long) * (size_t)G * kTileLd; }

__device__ __forceinline__ void raster_tile_fluc(const GridPlane& P, int ip, int row, int ktile, int key_base,
                                                 int ntiles_abs, const EventTable& evt, const FlucParams& fp,
                                                 const PatchRec* __restrict__ rec, const FlucRec* __restrict__ fluc,
                                                 const int* __restrict__ wire_cnt, const int* __restrict__ wire_off,
                                                 const Visit* __restrict__ visits, long long vcap,
                                                 float* __restrict__ Q, long long* grid)
{
    __syncthreads();  // the previous item of a persistent block is done with the grid
    __shared__ float s_p[kFlucRasterThreads / 32][16], s_w[kFlucRasterThreads / 32][16];
    __shared__ float s_tv[kFlucRasterThreads / 32][kTile];  // unit time bins of the current visit
    const int w = P.start_ch + row;
    const int G = P.G, nimp = P.nimp;
    const int tick_lo = ktile * kTile;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int nwarps = blockDim.x >> 5;
    int cnt = 0;
    const Visit* list = nullptr;
    if (w >= 0 && w < P.nwires && ktile >= 0 && ktile < ntiles_abs) {
        const int key = key_base + (P.wire_base + w) * ntiles_abs + ktile;
        const int off = wire_off[key];
        cnt = off < 0 ? 0 : (int)min((long long)wire_cnt[key], max(0ll, vcap - off));
        list = visits + max(off, 0);
    }
    for (int k = tid; k < G * kTileLd; k += blockDim.x) grid[k] = 0;
    __syncthreads();
    const float pbs = P.pbs, tbs = P.tbs, inv_pbs = 1.0f / pbs;
    const int wlo = w * nimp;
    for (int e = wid; e < cnt; e += nwarps) {
        const int d = list[e];
        const FlucRec fr = fluc[P.recoff + d];
        const PatchRec r = rec[P.recoff + d];
        const int rnp = r.np, rnt = r.nt;
        const int l_lo = max(r.poff, wlo) - wlo, l_hi = min(r.poff + rnp, wlo + nimp) - wlo;
        if (fr.scale == 0.f || l_hi <= l_lo) continue;  // warp-uniform
        const int nb = l_hi - l_lo;
        const int k0 = wlo + l_lo - r.poff;  // first patch bin on this wire
        if (lane < nb) {
            const int k = k0 + lane;
            const float p = unit_bin(k, pbs, r.pcr, r.sp);
            float wt;
            if (r.sp > 0.f) {
                const float isg = __frcp_rn(r.sp);
                const float x1 = (float)k * pbs - r.pcr, x2 = (float)(k + 1) * pbs - r.pcr;
                const float g1 = __expf(-0.5f * (x1 * isg) * (x1 * isg)), g2 = __expf(-0.5f * (x2 * isg) * (x2 * isg));
                const float c0 = r.sp * inv_pbs * 0.39894228040143268f;
                wt = p > 0.f ? fmaf(c0 * (g2 - g1), __frcp_rn(p), x2 * inv_pbs) : 0.f;
            }
            else wt = (pbs - r.pcr) * inv_pbs;
            s_p[wid][lane] = p;
            s_w[wid][lane] = wt;
        }
        __syncwarp();
        const int ev = event_of_depo(evt, d);
        const int ident = fluc_ident(fp, ev), i_ev = d - evt.dep0[ev];
        const int cb = r.toff - tick_lo;
        const int tstart = max(0, -cb), tend = min(rnt, kTile - cb);
        const int ntt = tend - tstart;
        if (ntt <= 0) continue;  // warp-uniform
        for (int t = lane; t < ntt; t += 32) s_tv[wid][t] = unit_bin(tstart + t, tbs, r.tcr, r.st);
        __syncwarp();
        // cells (bin b, tick t) of the visit in this tile, spread over the lanes
        for (int cell = lane; cell < nb * ntt; cell += 32) {
            const int b = cell / ntt, tt = cell - b * ntt;
            const int t = tstart + tt;
            const int k = k0 + b;
            const float relval = __fmul_rn(__fmul_rn(s_p[wid][b], s_tv[wid][tt]), fr.invS);
            const int N = cell_draw(fp, ident, i_ev, ip, k * rnt + t, fr.nq, relval);
            if (N) {
                const float c = (float)N * fr.scale;
                const float a = c * s_w[wid][b];
                long long* dst = grid + (size_t)(l_lo + b) * kTileLd + cb + t;
                atomicAdd(reinterpret_cast<unsigned long long*>(dst), (unsigned long long)__float2ll_rn(a * kFlucFix));
                atomicAdd(reinterpret_cast<unsigned long long*>(dst + kTileLd),
                          (unsigned long long)__float2ll_rn((c - a) * kFlucFix));
            }
        }
        __syncwarp();
    }
    __syncthreads();
    const int qc0 = tick_lo - P.col0;
    for (int k = tid; k < G * kTile; k += blockDim.x) {
        const int g = k / kTile, c = k - g * kTile;
        const int qc = qc0 + c;
        if (qc < 0 || qc >= P.N) continue;
        float val = 0.f;
        if (tick_lo + c - P.col0 < P.ncols) val = (float)((double)grid[g * kTileLd + c] * (1.0 / 65536.0));
        Q[P.qoff + ((size_t)g * P.nin + row) * P.N + qc] = val;
    }
}

__global__ void __launch_bounds__(kFlucRasterThreads) k_raster_fluc(const PatchRec* __restrict__ rec,
                                                                    const FlucRec* __restrict__ fluc, FlucParams fp,
                                                                    EventTable evt,
                                                                    const int* __restrict__ wire_cnt,
                                                                    const int* __restrict__ wire_off,
                                                                    const Visit* __restrict__ visits, long long vcap,
                                                                    GridSet gs, float* __restrict__ Q)
{
    extern __shared__ long long grid64[];
    int ip = 0;
    while (ip + 1 < gs.nplanes && (int)blockIdx.x >= gs.p[ip + 1].row_base) ++ip;
    const GridPlane& P = gs.p[ip];
    const int rel = blockIdx.x - P.row_base;
    const int row = rel / P.ntile;
    const int ktile = P.ktile0 + (rel - row * P.ntile);
    raster_tile_fluc(P, ip, row, ktile, 0, gs.ntiles_abs, evt, fp, rec, fluc, wire_cnt, wire_off, visits, vcap, Q,
                     grid64);
}

void launch_raster_fluc(const PatchRec* rec, const FlucRec* fluc, const FlucParams& fp, const EventTable& evt,
                        const int* wire_cnt, const int* wire_off, const Visit* visits, long long vcap,
                        const GridSet& gs, float* Q, cudaStream_t s)
{
    if (gs.nrows_total <= 0) return;
    size_t smem = 0;
    for (int i = 0; i < gs.nplanes; ++i) smem = std::max(smem, raster_fluc_smem_bytes(gs.p[i].G));
    cudaFuncSetAttribute((const void*)k_raster_fluc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_raster_fluc<<<gs.nrows_total, kFlucRasterThreads, smem, s>>>(rec, fluc, fp, evt, wire_cnt, wire_off, visits,
                                                                     vcap, gs, Q);
}

// Independent Binomial(n, p) draws: out[i] from the stream of key (seed,
// ident) and counter (i, kRngSampleTag, 0) -- IRandom::binomial in bulk.
__global__ void k_binomial_samples(unsigned int key0, unsigned int key1, int n, double p, long long count,
                                   int* __restrict__ out)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (long long)gridDim.x * blockDim.x) {
        Philox g;
        g.init(key0, key1, (unsigned)(i & 0xffffffffll), kRngSampleTag, (unsigned)(i >> 32));
        out[i] = binomial(n, p, g);
    }
}

void launch_binomial_samples(unsigned long long seed, int ident, int n, double p, long long count, int* out,
                             cudaStream_t s)
{
    if (count <= 0) return;
    const unsigned key0 = (unsigned)(seed & 0xffffffffull);
    const unsigned key1 = (unsigned)(seed >> 32) + 0x9E3779B9u * (unsigned)ident;
    const long long blocks = std::min<long long>((count + 255) / 256, 148LL * 32);
    k_binomial_samples<<<(unsigned)blocks, 256, 0, s>>>(key0, key1, n, p, count, out);
}

// ---------------------------------------------------------------------------
// Real FFT of rows (forward), packed output.  One row per block.
// ---------------------------------------------------------------------------
// One row: x (in_len real values, zero padded to 2M) -> o (M packed bins).
// Called by all threads of the block; sm holds 2M complex values.
__device__ __forceinline__ void rfft_row(const float* x, int in_len, float2* o, const FftDesc& d, float2* sm)
{
    __syncthreads();  // the previous row of a persistent block is done with sm
    float2* a = sm;
    float2* b = sm + d.M;
    const int M = d.M, tid = threadIdx.x, nth = blockDim.x;
    if (in_len >= 2 * M && ((reinterpret_cast<uintptr_t>(x) & 7) == 0)) {
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
    for (int k = tid; k < M; k += nth) o[k] = r2c_bin(Z, k, M, d.twh);
}

__global__ void k_rfft_rows(const float* in, long in_ld, int in_len, float2* out, long out_ld, int nrows, FftDesc d)
{
    extern __shared__ float2 sm[];
    const int row = blockIdx.x;
    if (row >= nrows) return;
    rfft_row(in + (size_t)row * in_ld, in_len, out + (size_t)row * out_ld, d, sm);
}

// Two complex rows of M bins in dynamic shared memory; raise the opt-in limit
// when they exceed the default 48 KB.
static void allow_smem(const void* f, size_t bytes)
{
    if (bytes > 48 * 1024) cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// ---------------------------------------------------------------------------
// Many rows: a persistent block per SM slot loops over rows, with
//  * the first stage (radix 8, no twiddles) run from registers: each thread
//    loads the eight inputs of its butterfly straight from global memory,
//    and loads them for its next row while the later stages of the current
//    row run in shared memory (the row loads never stall the transform);
//  * the twiddle factors of every later stage and the real-packing twiddles
//    copied into shared memory once per block (stage s holds w^(r k) for
//    r = 1..R-1, k < Ns at [(r-1) Ns + k]: M - 1 values over all stages).
// Needs M % 16 == 0 (radix 8 first; swizzled stage buffers), aligned float2
// rows, and M / 8 <= 2 * threads.
// ---------------------------------------------------------------------------
namespace fftk {
// SIGN -1 forward, +1 inverse; tws holds the stage's twiddles of that sign
template <int R, int SIGN, bool SWI, bool SWO>
__device__ __forceinline__ void stage_smtw(const float2* __restrict__ src, float2* __restrict__ dst, int M, int Ns,
                                           const float2* __restrict__ tws, int tid, int nth)
{
    const int nR = M / R;
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
#pragma unroll
            for (int r = 1; r < R; ++r) v[r] = cmul(v[r], tws[(r - 1) * Ns + k]);
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

template <int R, int SIGN = -1>
__device__ __forceinline__ void stage_smtw_any(const float2* __restrict__ src, float2* __restrict__ dst, int M,
                                               int Ns, const float2* __restrict__ tws, int tid, int nth, bool swi,
                                               bool swo)
{
    if (swi) {
        if (swo) stage_smtw<R, SIGN, true, true>(src, dst, M, Ns, tws, tid, nth);
        else stage_smtw<R, SIGN, true, false>(src, dst, M, Ns, tws, tid, nth);
    }
    else {
        if (swo) stage_smtw<R, SIGN, false, true>(src, dst, M, Ns, tws, tid, nth);
        else stage_smtw<R, SIGN, false, false>(src, dst, M, Ns, tws, tid, nth);
    }
}

// Stages 1 .. nst-1 of a transform whose first stage (radix 8) wrote src,
// swizzled when more stages follow; returns the buffer with the result in
// natural order.  All threads of the block call it.
template <int SIGN>
__device__ __forceinline__ float2* stages_after_first(float2* src, float2* dst, const FftDesc& d,
                                                      const float2* __restrict__ tws, int tid, int nth)
{
    const int M = d.M;
    int Ns = 8, off = 0;
    bool swi = d.nst > 1;  // the first stage's writes have stride 8
    for (int s = 1; s < d.nst; ++s) {
        const int R = d.radix[s];
        const bool swo = s + 1 < d.nst && Ns < 16;  // strided writes only while Ns < 16
        switch (R) {
            case 2: stage_smtw_any<2, SIGN>(src, dst, M, Ns, tws + off, tid, nth, swi, swo); break;
            case 3: stage_smtw_any<3, SIGN>(src, dst, M, Ns, tws + off, tid, nth, swi, swo); break;
            case 4: stage_smtw_any<4, SIGN>(src, dst, M, Ns, tws + off, tid, nth, swi, swo); break;
            case 5: stage_smtw_any<5, SIGN>(src, dst, M, Ns, tws + off, tid, nth, swi, swo); break;
            case 7: stage_smtw_any<7, SIGN>(src, dst, M, Ns, tws + off, tid, nth, swi, swo); break;
            default: stage_smtw_any<8, SIGN>(src, dst, M, Ns, tws + off, tid, nth, swi, swo); break;
        }
        __syncthreads();
        off += (R - 1) * Ns;
        Ns *= R;
        swi = swo;
        float2* t = src;
        src = dst;
        dst = t;
    }
    return src;
}

// The twiddles of stages 1 .. nst-1 (conjugated for SIGN +1) and the
// real-packing twiddles into shared memory, once per block.
template <int SIGN>
__device__ __forceinline__ void load_stage_twiddles(const FftDesc& d, float2* tws, float2* twh, int tid, int nth)
{
    const int M = d.M;
    int Ns = d.radix[0], off = 0;
    for (int s = 1; s < d.nst; ++s) {
        const int R = d.radix[s], step = M / (Ns * R), n = (R - 1) * Ns;
        for (int e = tid; e < n; e += nth) {
            const int r = e / Ns + 1, k = e - (r - 1) * Ns;
            float2 w = __ldg(d.tw + k * r * step);
            if (SIGN > 0) w.y = -w.y;
            tws[off + e] = w;
        }
        off += n;
        Ns *= R;
    }
    for (int k = tid; k < M; k += nth) twh[k] = __ldg(d.twh + k);
}
}  // namespace fftk

// IT: first-stage butterflies per thread (M / 8 <= IT * 256)
template <int IT>
__global__ void __launch_bounds__(256) k_rfft_rows_pf(const float* __restrict__ in, long in_ld, int in_len,
                                                      float2* __restrict__ out, long out_ld, int nrows, FftDesc d)
{
    extern __shared__ float2 sm[];
    const int M = d.M, tid = threadIdx.x, nth = blockDim.x;
    float2* a = sm;
    float2* b = sm + M;
    float2* tws = sm + 2 * M;
    float2* twh = sm + 3 * M;
    fftk::load_stage_twiddles<-1>(d, tws, twh, tid, nth);
    const int nR = M / 8;
    float2 v[IT][8];
    auto fetch = [&](int row) {
        const float* x = in + (size_t)row * in_ld;
        const float2* x2 = reinterpret_cast<const float2*>(x);
#pragma unroll
        for (int it = 0; it < IT; ++it) {
            const int j = tid + it * nth;
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int m = j + q * nR, k = 2 * m;
                float2 val = make_float2(0.f, 0.f);
                if (j < nR) {
                    if (k + 1 < in_len) val = __ldcs(x2 + m);  // streamed once: evict first
                    else if (k < in_len) val.x = x[k];
                }
                v[it][q] = val;
            }
        }
    };
    int row = blockIdx.x;
    if (row < nrows) fetch(row);
    __syncthreads();  // twiddle tables
    const bool more = d.nst > 1;
    while (row < nrows) {
#pragma unroll
        for (int it = 0; it < IT; ++it) {
            const int j = tid + it * nth;
            if (j < nR) {
                fftk::bfly8<-1>(v[it]);
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const int i = j * 8 + q;
                    a[more ? fftk::swz(i) : i] = v[it][q];
                }
            }
        }
        __syncthreads();
        const int next = row + gridDim.x;
        if (next < nrows) fetch(next);
        float2* src = fftk::stages_after_first<-1>(a, b, d, tws, tid, nth);
        float2* o = out + (size_t)row * out_ld;
        for (int k = tid; k < M; k += nth) {
            const float2 zk = src[k];
            float2 res;
            if (k == 0) res = make_float2(zk.x + zk.y, zk.x - zk.y);
            else {
                const float2 zm = cconj(src[M - k]);
                const float2 E = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y + zm.y));
                const float2 D = make_float2(0.5f * (zk.x - zm.x), 0.5f * (zk.y - zm.y));
                res = cadd(E, cmul(twh[k], make_float2(D.y, -D.x)));
            }
            o[k] = res;
        }
        __syncthreads();  // src is the next row's stage-1 output buffer or its stage scratch
        row = next;
    }
}

template <int IT>
static int rfft_pf_blocks(size_t smem)
{
    int dev = 0, nsm = 0, per = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_rfft_rows_pf<IT>, 256, smem) != cudaSuccess) return 0;
    return per * nsm;
}

template <int IT>
static bool launch_rfft_pf(const float* in, long in_ld, int in_len, float2* out, long out_ld, int nrows,
                           const FftDesc& d, cudaStream_t s)
{
    const size_t smem = 4 * (size_t)d.M * sizeof(float2);
    allow_smem((const void*)k_rfft_rows_pf<IT>, smem);
    const int grid = std::min(nrows, rfft_pf_blocks<IT>(smem));
    if (grid <= 0 || nrows < 2 * grid) return false;  // under two rows per block: the per-row kernel
    k_rfft_rows_pf<IT><<<grid, 256, smem, s>>>(in, in_ld, in_len, out, out_ld, nrows, d);
    return true;
}

void launch_rfft_rows(const float* in, long in_ld, int in_len, float2* out, long out_ld, int nrows, const FftDesc& d,
                      cudaStream_t s)
{
    if (nrows <= 0) return;
    const bool aligned = ((reinterpret_cast<uintptr_t>(in) & 7) == 0) && (in_ld % 2 == 0);
    if (aligned && d.M % 16 == 0 && d.nst >= 2 && d.radix[0] == 8 && 4 * (size_t)d.M * sizeof(float2) <= 128 * 1024) {
        if (d.M / 8 <= 256 && launch_rfft_pf<1>(in, in_ld, in_len, out, out_ld, nrows, d, s)) return;
        if (d.M / 8 > 256 && d.M / 8 <= 512 && launch_rfft_pf<2>(in, in_ld, in_len, out, out_ld, nrows, d, s)) return;
    }
    allow_smem((const void*)k_rfft_rows, 2 * d.M * sizeof(float2));
    const int nth = d.M >= 2048 ? 512 : 256;
    k_rfft_rows<<<nrows, nth, 2 * d.M * sizeof(float2), s>>>(in, in_ld, in_len, out, out_ld, nrows, d);
}

// ---------------------------------------------------------------------------
// Inverse real FFT of rows + frame write (ImpactTransform.cxx:303-347).
// Row r of Vh is wire wire0 + r; ticks are tick0 + column.
// ---------------------------------------------------------------------------
// One row: v (M packed bins) -> real values written to f[tick0 + c] for
// c < ncols, 0 <= tick0 + c < nticks.  Called by all threads of the block.
__device__ __forceinline__ void irfft_row(const float2* __restrict__ v, const FftDesc& d, float* __restrict__ f,
                                          int tick0, int ncols, int nticks, float2* sm)
{
    __syncthreads();  // the previous row of a persistent block is done with sm
    float2* a = sm;
    float2* b = sm + d.M;
    const int M = d.M, tid = threadIdx.x, nth = blockDim.x;
    for (int k = tid; k < M; k += nth) b[k] = v[k];
    __syncthreads();
    for (int k = tid; k < M; k += nth) a[k] = c2r_bin(b, k, M, d.twh);
    __syncthreads();
    float2* z = fft_c2c<+1>(a, b, d, tid, nth);
    const float sc = 1.0f / (float)M;
    for (int m = tid; m < M; m += nth) {
        const float2 zz = z[m];
        const int c0 = 2 * m;
        const int t0 = tick0 + c0;
        if (c0 < ncols && t0 >= 0 && t0 < nticks) f[t0] = zz.x * sc;
        if (c0 + 1 < ncols && t0 + 1 >= 0 && t0 + 1 < nticks) f[t0 + 1] = zz.y * sc;
    }
}

__global__ void k_irfft_rows(const float2* __restrict__ Vh, int nrows, FftDesc d, int wire0, int wlo, int whi,
                             int tick0, int ncols, int nticks, float* __restrict__ frame)
{
    extern __shared__ float2 sm[];
    const int row = blockIdx.x;
    const int W = wire0 + row;
    if (row >= nrows || W < wlo || W >= whi) return;
    irfft_row(Vh + (size_t)row * d.M, d, frame + (size_t)W * nticks, tick0, ncols, nticks, sm);
}

// Many rows: persistent blocks (as k_rfft_rows_pf) over the rows that are
// frame wires, each thread holding its share of the next row's packed
// spectrum in registers while the current row is transformed; the complex
// pre-processing of the real inverse is fused into the first (radix-8)
// stage; twiddles in shared memory.  IT: spectrum values per thread
// (M <= 256 IT).
template <int IT>
__global__ void __launch_bounds__(256) k_irfft_rows_pf(const float2* __restrict__ Vh, int r0, int r1, FftDesc d,
                                                       int wire0, int tick0, int ncols, int nticks,
                                                       float* __restrict__ frame)
{
    extern __shared__ float2 sm[];
    const int M = d.M, tid = threadIdx.x, nth = blockDim.x;
    float2* a = sm;
    float2* b = sm + M;
    float2* tws = sm + 2 * M;
    float2* twh = sm + 3 * M;
    fftk::load_stage_twiddles<+1>(d, tws, twh, tid, nth);
    float2 pv[IT];
    auto fetch = [&](int row) {
        const float2* v = Vh + (size_t)row * M;
#pragma unroll
        for (int it = 0; it < IT; ++it) {
            const int k = tid + it * nth;
            pv[it] = k < M ? __ldcs(v + k) : make_float2(0.f, 0.f);
        }
    };
    int row = r0 + blockIdx.x;
    if (row < r1) fetch(row);
    __syncthreads();  // twiddle tables
    const bool more = d.nst > 1;
    const int nR = M / 8;
    const float sc = 1.0f / (float)M;
    while (row < r1) {
#pragma unroll
        for (int it = 0; it < IT; ++it) {
            const int k = tid + it * nth;
            if (k < M) b[k] = pv[it];
        }
        __syncthreads();
        const int next = row + gridDim.x;
        if (next < r1) fetch(next);
        // first stage (radix 8, no twiddles) on the pre-processed bins
        for (int j = tid; j < nR; j += nth) {
            float2 v[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int k = j + q * nR;
                const float2 xk = b[k];
                if (k == 0) {
                    v[q] = make_float2(0.5f * (xk.x + xk.y), 0.5f * (xk.x - xk.y));
                }
                else {
                    const float2 xm = cconj(b[M - k]);
                    const float2 E = make_float2(0.5f * (xk.x + xm.x), 0.5f * (xk.y + xm.y));
                    const float2 D = make_float2(0.5f * (xk.x - xm.x), 0.5f * (xk.y - xm.y));
                    const float2 O = cmulc(D, twh[k]);
                    v[q] = make_float2(E.x - O.y, E.y + O.x);
                }
            }
            fftk::bfly8<+1>(v);
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int i = j * 8 + q;
                a[more ? fftk::swz(i) : i] = v[q];
            }
        }
        __syncthreads();  // b is read by the first stage and written by the second
        const float2* z = fftk::stages_after_first<+1>(a, b, d, tws, tid, nth);
        float* f = frame + (size_t)(wire0 + row) * nticks;
        for (int m = tid; m < M; m += nth) {
            const float2 zz = z[m];
            const int c0 = 2 * m;
            const int t0 = tick0 + c0;
            if (c0 < ncols && t0 >= 0 && t0 < nticks) f[t0] = zz.x * sc;
            if (c0 + 1 < ncols && t0 + 1 >= 0 && t0 + 1 < nticks) f[t0 + 1] = zz.y * sc;
        }
        __syncthreads();  // z is the next row's spectrum or first-stage buffer
        row = next;
    }
}

template <int IT>
static bool launch_irfft_pf(const float2* Vh, int r0, int r1, const FftDesc& d, int wire0, int tick0, int ncols,
                            int nticks, float* frame, cudaStream_t s)
{
    const size_t smem = 4 * (size_t)d.M * sizeof(float2);
    allow_smem((const void*)k_irfft_rows_pf<IT>, smem);
    int dev = 0, nsm = 0, per = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return false;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_irfft_rows_pf<IT>, 256, smem) != cudaSuccess) return false;
    const int grid = std::min(r1 - r0, per * nsm);
    if (grid <= 0 || r1 - r0 < 2 * grid) return false;  // under two rows per block: one block per row
    k_irfft_rows_pf<IT><<<grid, 256, smem, s>>>(Vh, r0, r1, d, wire0, tick0, ncols, nticks, frame);
    return true;
}

void launch_irfft_rows(const float2* Vh, int nrows, const FftDesc& d, int wire0, int wlo, int whi, int tick0,
                       int ncols, int nticks, float* frame, cudaStream_t s)
{
    if (nrows <= 0) return;
    if (d.M % 16 == 0 && d.nst >= 2 && d.radix[0] == 8 && 4 * (size_t)d.M * sizeof(float2) <= 128 * 1024) {
        // the rows that are frame wires: wire0 + r in [wlo, whi)
        const int r0 = std::max(0, wlo - wire0), r1 = std::min(nrows, whi - wire0);
        if (r1 <= r0) return;
        if (d.M <= 1024 && launch_irfft_pf<4>(Vh, r0, r1, d, wire0, tick0, ncols, nticks, frame, s)) return;
        if (d.M > 1024 && d.M <= 2048 && launch_irfft_pf<8>(Vh, r0, r1, d, wire0, tick0, ncols, nticks, frame, s))
            return;
    }
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
// Bin 0 (packed DC/Nyquist) is multiplied component-wise.
// ---------------------------------------------------------------------------
constexpr int kConvRB = 8;
constexpr int kConvRG = 8;
constexpr int kConvRows = kConvRB * kConvRG;

// One tile of the wire convolution: frequencies fblk*32 .. +31, output rows
// oblk*64 .. +63.  Called by all threads of a (32, kConvRG) block.
// PAIR: groups g and G-1-g share one response up to a mirror in wire
// (R_{G-1-g}[j] = R_g[-j], the symmetrised impact map of
// gen/src/PlaneImpactResponse.cxx:256-268), so for each tap the two
// mirrored inputs are added before one complex multiply.
template <int PAD, bool PAIR>
__device__ __forceinline__ void wire_conv_tile(const float2* __restrict__ Qh, const float2* __restrict__ Rh,
                                               float2* __restrict__ Vh, int G, int nin, int nout, int M, int fblk,
                                               int oblk, float2* conv_smem)
{
    constexpr int SROWS = kConvRows + 2 * PAD;
    constexpr int NT = 2 * PAD + 1;
    float2 (*Qs)[32] = reinterpret_cast<float2 (*)[32]>(conv_smem);
    float2 (*Qs2)[32] = reinterpret_cast<float2 (*)[32]>(conv_smem + SROWS * 32);
    float2 (*Rs)[32] = reinterpret_cast<float2 (*)[32]>(conv_smem + (PAIR ? 2 : 1) * SROWS * 32);
    const int lane = threadIdx.x, rg = threadIdx.y;
    const int f = fblk * 32 + lane;
    const int o0 = oblk * kConvRows;
    const bool fok = f < M;
    const bool dc = f == 0;
    float2 acc[kConvRB];
#pragma unroll
    for (int r = 0; r < kConvRB; ++r) acc[r] = make_float2(0.f, 0.f);
    const int rb0 = rg * kConvRB;
    const int ng = PAIR ? (G + 1) / 2 : G;
    for (int gi = 0; gi < ng; ++gi) {
        const int g = gi;
        const int g2 = G - 1 - gi;
        const bool pair = PAIR && g2 != g;
        __syncthreads();
        for (int s = rg; s < SROWS; s += kConvRG) {
            const int i = o0 - 2 * PAD + s;
            const bool ok = fok && i >= 0 && i < nin;
            Qs[s][lane] = ok ? Qh[((size_t)g * nin + i) * M + f] : make_float2(0.f, 0.f);
            if (PAIR) Qs2[s][lane] = (ok && pair) ? Qh[((size_t)g2 * nin + i) * M + f] : make_float2(0.f, 0.f);
        }
        for (int jj = rg; jj < NT; jj += kConvRG)
            Rs[jj][lane] = fok ? Rh[((size_t)g * NT + jj) * M + f] : make_float2(0.f, 0.f);
        __syncthreads();
        if (fok) {
            float2 win[kConvRB], win2[kConvRB];
#pragma unroll
            for (int r = 0; r < kConvRB; ++r) {
                win[r] = Qs[rb0 + r + 2 * PAD][lane];       // input row o - PAD - j at j = -PAD
                if (PAIR) win2[r] = Qs2[rb0 + r][lane];     // input row o - PAD + j at j = -PAD
            }
#pragma unroll
            for (int jj = 0; jj < NT; ++jj) {
                const float2 rr = Rs[jj][lane];
                // bin 0 packs two real spectra (DC, Nyquist): multiply component-wise there
                const float rc = dc ? 0.f : rr.y;
                const float ry = dc ? rr.y : rr.x;
#pragma unroll
                for (int r = 0; r < kConvRB; ++r) {
                    float2 q = win[r];
                    if (PAIR) q = make_float2(q.x + win2[r].x, q.y + win2[r].y);
                    acc[r].x = fmaf(rr.x, q.x, fmaf(-rc, q.y, acc[r].x));
                    acc[r].y = fmaf(ry, q.y, fmaf(rc, q.x, acc[r].y));
                }
                if (jj < NT - 1) {
#pragma unroll
                    for (int r = kConvRB - 1; r > 0; --r) win[r] = win[r - 1];
                    win[0] = Qs[rb0 + 2 * PAD - jj - 1][lane];
                    if (PAIR) {
#pragma unroll
                        for (int r = 0; r < kConvRB - 1; ++r) win2[r] = win2[r + 1];
                        win2[kConvRB - 1] = Qs2[rb0 + kConvRB + jj][lane];
                    }
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

template <int PAD, bool PAIR>
__global__ void __launch_bounds__(32 * kConvRG) k_wire_conv(const float2* __restrict__ Qh,
                                                             const float2* __restrict__ Rh, float2* __restrict__ Vh,
                                                             int G, int nin, int nout, int M)
{
    extern __shared__ float2 conv_smem[];
    wire_conv_tile<PAD, PAIR>(Qh, Rh, Vh, G, nin, nout, M, blockIdx.x, blockIdx.y, conv_smem);
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
            const float rc = f == 0 ? 0.f : rr.y;
            const float ry = f == 0 ? rr.y : rr.x;
            const int j = jj - PAD;
#pragma unroll
            for (int r = 0; r < kConvRB; ++r) {
                const int i = o0 + rg * kConvRB + r - PAD - j;
                if (i < 0 || i >= nin) continue;
                const float2 q = Qh[((size_t)g * nin + i) * M + f];
                acc[r].x = fmaf(rr.x, q.x, fmaf(-rc, q.y, acc[r].x));
                acc[r].y = fmaf(ry, q.y, fmaf(rc, q.x, acc[r].y));
            }
        }
    }
#pragma unroll
    for (int r = 0; r < kConvRB; ++r) {
        const int o = o0 + rg * kConvRB + r;
        if (o < nout) Vh[(size_t)o * M + f] = acc[r];
    }
}

// ---------------------------------------------------------------------------
// The same convolution with the staging of the next group (pair) overlapped
// with the arithmetic of the current one: 16 frequencies x 16 row groups per
// block (128 output rows), the input rows, mirrored rows and taps of group
// gi + 1 copied by cp.async into the second of two shared-memory buffers
// while group gi is multiplied out of the first.  Needs 16-byte aligned
// spectra and an even M (two frequencies per 16-byte copy).
// ---------------------------------------------------------------------------
constexpr int kConv2F = 16;  // frequencies per block
constexpr int kConv2RG = 16; // row groups per block (kConvRB output rows each)
constexpr int kConv2Rows = kConv2RG * kConvRB;


template <int PAD, bool PAIR>
constexpr size_t conv2_stage_f2()  // float2 values per pipeline stage
{
    return (size_t)kConv2F * ((PAIR ? 2 : 1) * (kConv2Rows + 2 * PAD) + (2 * PAD + 1));
}

template <int PAD, bool PAIR>
__global__ void __launch_bounds__(kConv2F * kConv2RG) k_wire_conv2(const float2* __restrict__ Qh,
                                                                  const float2* __restrict__ Rh,
                                                                  float2* __restrict__ Vh, int G, int nin, int nout,
                                                                  int M)
{
    constexpr int SROWS = kConv2Rows + 2 * PAD;
    constexpr int NT = 2 * PAD + 1;
    constexpr size_t STAGE = conv2_stage_f2<PAD, PAIR>();
    extern __shared__ __align__(16) float2 conv2_smem[];
    const int lane = threadIdx.x, rg = threadIdx.y;
    const int tid = rg * kConv2F + lane;
    const int f0 = blockIdx.x * kConv2F;
    const int f = f0 + lane;
    const int o0 = blockIdx.y * kConv2Rows;
    const bool fok = f < M;
    const bool dc = f == 0;
    const int ng = PAIR ? (G + 1) / 2 : G;
    // copy of group gi into stage buffer st: 8 16-byte pieces per row of 16 frequencies
    auto issue = [&](int gi, int st) {
        float2* base = conv2_smem + (size_t)st * STAGE;
        float2* Qs = base;
        float2* Qs2 = base + SROWS * kConv2F;
        float2* Rs = base + (PAIR ? 2 : 1) * SROWS * kConv2F;
        const int g = gi, g2 = G - 1 - gi;
        const bool pair = PAIR && g2 != g;
        const int fp = f0 + 2 * (tid & 7);           // first frequency of this thread's piece
        const int fbytes = fp < M ? 16 : 0;          // M even: both or neither of fp, fp + 1
        constexpr int kPieces = kConv2F / 2;
        constexpr int nthr = kConv2F * kConv2RG;
        for (int e = tid; e < SROWS * kPieces; e += nthr) {
            const int srow = e / kPieces;
            const int i = o0 - 2 * PAD + srow;
            const bool ok = i >= 0 && i < nin && fbytes;
            const float2* src = ok ? Qh + ((size_t)g * nin + i) * M + fp : Qh;
            cp_async16(Qs + srow * kConv2F + 2 * (e % kPieces), src, ok ? 16 : 0);
            if (PAIR) {
                const bool ok2 = ok && pair;
                const float2* src2 = ok2 ? Qh + ((size_t)g2 * nin + i) * M + fp : Qh;
                cp_async16(Qs2 + srow * kConv2F + 2 * (e % kPieces), src2, ok2 ? 16 : 0);
            }
        }
        for (int e = tid; e < NT * kPieces; e += nthr) {
            const int jj = e / kPieces;
            const float2* src = fbytes ? Rh + ((size_t)g * NT + jj) * M + fp : Rh;
            cp_async16(Rs + jj * kConv2F + 2 * (e % kPieces), src, fbytes);
        }
        cp_async_commit();
    };
    float2 acc[kConvRB];
#pragma unroll
    for (int r = 0; r < kConvRB; ++r) acc[r] = make_float2(0.f, 0.f);
    const int rb0 = rg * kConvRB;
    issue(0, 0);
    for (int gi = 0; gi < ng; ++gi) {
        if (gi + 1 < ng) {
            issue(gi + 1, (gi + 1) & 1);
            cp_async_wait<1>();
        }
        else
            cp_async_wait<0>();
        __syncthreads();
        const float2* base = conv2_smem + (size_t)(gi & 1) * STAGE;
        const float2* Qs = base;
        const float2* Qs2 = base + SROWS * kConv2F;
        const float2* Rs = base + (PAIR ? 2 : 1) * SROWS * kConv2F;
        float2 win[kConvRB], win2[kConvRB];
#pragma unroll
        for (int r = 0; r < kConvRB; ++r) {
            win[r] = Qs[(rb0 + r + 2 * PAD) * kConv2F + lane];  // input row o - PAD - j at j = -PAD
            if (PAIR) win2[r] = Qs2[(rb0 + r) * kConv2F + lane];  // input row o - PAD + j at j = -PAD
        }
#pragma unroll
        for (int jj = 0; jj < NT; ++jj) {
            const float2 rr = Rs[jj * kConv2F + lane];
            // bin 0 packs two real spectra (DC, Nyquist): multiply component-wise there
            const float rc = dc ? 0.f : rr.y;
            const float ry = dc ? rr.y : rr.x;
#pragma unroll
            for (int r = 0; r < kConvRB; ++r) {
                float2 q = win[r];
                if (PAIR) q = make_float2(q.x + win2[r].x, q.y + win2[r].y);
                acc[r].x = fmaf(rr.x, q.x, fmaf(-rc, q.y, acc[r].x));
                acc[r].y = fmaf(ry, q.y, fmaf(rc, q.x, acc[r].y));
            }
            if (jj < NT - 1) {
#pragma unroll
                for (int r = kConvRB - 1; r > 0; --r) win[r] = win[r - 1];
                win[0] = Qs[(rb0 + 2 * PAD - jj - 1) * kConv2F + lane];
                if (PAIR) {
#pragma unroll
                    for (int r = 0; r < kConvRB - 1; ++r) win2[r] = win2[r + 1];
                    win2[kConvRB - 1] = Qs2[(rb0 + kConvRB + jj) * kConv2F + lane];
                }
            }
        }
        __syncthreads();  // buffer gi & 1 is refilled with group gi + 2 next
    }
    if (fok) {
#pragma unroll
        for (int r = 0; r < kConvRB; ++r) {
            const int o = o0 + rb0 + r;
            if (o < nout) Vh[(size_t)o * M + f] = acc[r];
        }
    }
}

void launch_wire_conv(const float2* Qh, const float2* Rh, float2* Vh, int ngroups, int npad, int nrows_in,
                      int nrows_out, int M, bool pair, cudaStream_t s)
{
    if (nrows_out <= 0) return;
    const bool al16 = ((reinterpret_cast<uintptr_t>(Qh) | reinterpret_cast<uintptr_t>(Rh)) & 15) == 0 && M % 2 == 0;
    if (al16 && (npad == 21 || npad == 10)) {
        dim3 grid2((M + kConv2F - 1) / kConv2F, (nrows_out + kConv2Rows - 1) / kConv2Rows);
        dim3 block2(kConv2F, kConv2RG);
#define WCT_CONV2(P, B)                                                                                       \
    do {                                                                                                      \
        const size_t sm = 2 * conv2_stage_f2<P, B>() * sizeof(float2);                                       \
        cudaFuncSetAttribute((const void*)k_wire_conv2<P, B>, cudaFuncAttributeMaxDynamicSharedMemorySize,   \
                             (int)sm);                                                                        \
        k_wire_conv2<P, B><<<grid2, block2, sm, s>>>(Qh, Rh, Vh, ngroups, nrows_in, nrows_out, M);            \
        return;                                                                                               \
    } while (0)
        if (npad == 10 && pair) WCT_CONV2(10, true);
        if (npad == 10) WCT_CONV2(10, false);
        if (npad == 21 && pair) WCT_CONV2(21, true);
        WCT_CONV2(21, false);
#undef WCT_CONV2
    }
    launch_wire_conv_tiles(Qh, Rh, Vh, ngroups, npad, nrows_in, nrows_out, M, pair, s);
}

void launch_wire_conv_tiles(const float2* Qh, const float2* Rh, float2* Vh, int ngroups, int npad, int nrows_in,
                            int nrows_out, int M, bool pair, cudaStream_t s)
{
    if (nrows_out <= 0) return;
    dim3 grid((M + 31) / 32, (nrows_out + kConvRows - 1) / kConvRows);
    dim3 block(32, kConvRG);
    auto smem = [](int pad, bool pr) {
        return sizeof(float2) * 32 * ((size_t)(pr ? 2 : 1) * (kConvRows + 2 * pad) + (2 * pad + 1));
    };
#define WCT_CONV(P, B)                                                                                        \
    do {                                                                                                      \
        const size_t sm = smem(P, B);                                                                         \
        cudaFuncSetAttribute((const void*)k_wire_conv<P, B>, cudaFuncAttributeMaxDynamicSharedMemorySize,    \
                             (int)sm);                                                                        \
        k_wire_conv<P, B><<<grid, block, sm, s>>>(Qh, Rh, Vh, ngroups, nrows_in, nrows_out, M);               \
    } while (0)
    if (npad == 10 && pair) WCT_CONV(10, true);
    else if (npad == 10) WCT_CONV(10, false);
    else if (npad == 21 && pair) WCT_CONV(21, true);
    else if (npad == 21) WCT_CONV(21, false);
#undef WCT_CONV
    else k_wire_conv_any<<<grid, block, 0, s>>>(Qh, Rh, Vh, ngroups, npad, nrows_in, nrows_out, M);
}

// ---------------------------------------------------------------------------
// Trace edges (Waveform::edge, util/src/Waveform.cxx:136-153) of frame rows
// [r0, r0 + nrows) over ticks [t0, t1): out[r] = (first non-zero tick, last
// non-zero tick + 1) relative to t0, or (0, 0) for a row without one.  One
// warp per row.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_row_edges(const float* __restrict__ frame, int ld, int r0, int nrows,
                                                   int t0, int t1, int2* __restrict__ out)
{
    const int r = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (r >= nrows) return;  // whole warps
    const float* row = frame + (size_t)(r0 + r) * ld;
    int lo = INT_MAX, hi = -1;
    for (int t = t0 + lane; t < t1; t += 32)
        if (row[t] != 0.0f) {  // -0.0 counts as zero, as the reference's test
            lo = min(lo, t);
            hi = t;
        }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if (lane == 0) out[r] = hi < 0 ? make_int2(0, 0) : make_int2(lo - t0, hi + 1 - t0);
}

void launch_row_edges(const float* frame, int ld, int r0, int nrows, int t0, int t1, int2* out, cudaStream_t s)
{
    if (nrows <= 0) return;
    k_row_edges<<<(nrows + 7) / 8, 256, 0, s>>>(frame, ld, r0, nrows, t0, t1, out);
}

// ---------------------------------------------------------------------------
// PlaneImpactResponse::build_responses on the device
// (gen/src/PlaneImpactResponse.cxx:89-269), in the reference's single
// precision.  k_pir_bin: each path's field response on the tick grid
// (:185-218): sample r at Binning::center(r) = tstart + (r + 1/2) rawbs falls
// in tick bin (size_t)(time / tick) and adds current * period to that bin, a
// float (Waveform::realseq_t: every add rounded to float); rows of n complex
// values with zero imaginary parts.  One thread per path (the samples of a
// path in order, as the reference adds them).
// ---------------------------------------------------------------------------
__global__ void k_pir_bin(const double* __restrict__ current, int npaths, int nsamples, double tstart, double rawbs,
                          double period, double tick, int n, float2* __restrict__ Z)
{
    const int ip = blockIdx.x * blockDim.x + threadIdx.x;
    if (ip >= npaths) return;
    float2* z = Z + (size_t)ip * n;
    for (int k = 0; k < n; ++k) z[k] = make_float2(0.f, 0.f);
    const double* cur = current + (size_t)ip * nsamples;
    long long bin = -1;
    float acc = 0.f;
    for (int r = 0; r < nsamples; ++r) {
        const double time = __dadd_rn(tstart, __dmul_rn(__dadd_rn((double)r, 0.5), rawbs));
        const long long b = __double2ll_rz(__ddiv_rn(time, tick));
        if (b != bin) {  // a new bin: store the finished one, start from what the new one holds
            if (bin >= 0 && bin < n) z[bin].x = acc;
            bin = b;
            acc = (bin >= 0 && bin < n) ? z[bin].x : 0.f;
        }
        acc = (float)__dadd_rn((double)acc, __dmul_rn(cur[r], period));
    }
    if (bin >= 0 && bin < n) z[bin].x = acc;
}

// The product of nrows spectra of length n, bin by bin in row order, into
// out (the reference's short_spec[bin] *= spec[bin] over its short responses,
// starting from 1).
__global__ void k_spec_chain(const float2* __restrict__ S, int nrows, int n, float2* __restrict__ out)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    float2 a = S[k];
    for (int r = 1; r < nrows; ++r) a = cmul(a, S[(size_t)r * n + k]);
    out[k] = a;
}

// Real parts of the first min(n, ncols) values of each complex row of length
// n into float rows of ncols (zero beyond n): inv_c2r and its resize.
__global__ void k_real_rows(const float2* __restrict__ Z, int nrows, int n, float* __restrict__ out, int ncols)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x, r = blockIdx.y;
    if (c >= ncols || r >= nrows) return;
    out[(size_t)r * ncols + c] = c < n ? Z[(size_t)r * n + c].x : 0.f;
}

void launch_pir_bin(const double* current, int npaths, int nsamples, double tstart, double rawbs, double period,
                    double tick, int n, float2* Z, cudaStream_t s)
{
    if (npaths <= 0) return;
    k_pir_bin<<<(npaths + 63) / 64, 64, 0, s>>>(current, npaths, nsamples, tstart, rawbs, period, tick, n, Z);
}

void launch_spec_chain(const float2* S, int nrows, int n, float2* out, cudaStream_t s)
{
    if (nrows <= 0 || n <= 0) return;
    k_spec_chain<<<(n + 255) / 256, 256, 0, s>>>(S, nrows, n, out);
}

void launch_real_rows(const float2* Z, int nrows, int n, float* out, int ncols, cudaStream_t s)
{
    if (nrows <= 0 || ncols <= 0) return;
    k_real_rows<<<dim3((ncols + 255) / 256, nrows), 256, 0, s>>>(Z, nrows, n, out, ncols);
}

// ---------------------------------------------------------------------------
// Batched row convolution helpers (DftTools::convolve, aux/src/DftTools.cxx:145-168).
// ---------------------------------------------------------------------------
// X[row][k] *= R[k] on packed real spectra (bin 0 component-wise).
__global__ void k_spec_mul(float2* __restrict__ X, long ldx, int nrows, int M, const float2* __restrict__ R)
{
    const int row = blockIdx.y;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < M; k += gridDim.x * blockDim.x) {
        const float2 r = R[k];
        float2 x = X[(size_t)row * ldx + k];
        x = k == 0 ? make_float2(x.x * r.x, x.y * r.y) : cmul(x, r);
        X[(size_t)row * ldx + k] = x;
    }
}

void launch_spec_mul(float2* X, long ldx, int nrows, int M, const float2* R, cudaStream_t s)
{
    if (nrows <= 0) return;
    dim3 grid((M + 255) / 256, nrows);
    k_spec_mul<<<grid, 256, 0, s>>>(X, ldx, nrows, M, R);
}

// exp(-2 pi i m / M) and exp(-2 pi i m / (2M)) in double, stored as float.
__global__ void k_twiddles(float2* __restrict__ tw, float2* __restrict__ twh, int M)
{
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < M; m += gridDim.x * blockDim.x) {
        double sa, ca, sb, cb;
        sincospi(-2.0 * (double)m / (double)M, &sa, &ca);
        sincospi(-(double)m / (double)M, &sb, &cb);
        tw[m] = make_float2((float)ca, (float)sa);
        twh[m] = make_float2((float)cb, (float)sb);
    }
}

void launch_twiddles(float2* tw, float2* twh, int M, cudaStream_t s)
{
    k_twiddles<<<(M + 255) / 256, 256, 0, s>>>(tw, twh, M);
}

// ===========================================================================
// Batched events: a device-planned pipeline with no host round trip, so a
// whole batch is one captured CUDA graph.  After the prep/scan/fill kernels
// (the event-table forms of the single-event ones), k_plan_batch computes
// every (event, plane) window on the device -- ImpactTransform's window
// arithmetic (gen/src/ImpactTransform.cxx:83-115) with the reference's FFT
// length tables -- picks the time-FFT length class, places the event's grids
// in fixed event slots, and writes the work-item prefixes that the persistent
// raster, time-FFT, wire-convolution and inverse kernels walk.
// ===========================================================================
}  // namespace wctb200

#include "fft_lengths.h"

namespace wctb200 {

__constant__ int c_fbl_any[] = {WCT_FFT_LENGTHS_ANY};
__constant__ int c_fbl_even[] = {WCT_FFT_LENGTHS_EVEN};
__constant__ int c_fbl_odd[] = {WCT_FFT_LENGTHS_ODD};

template <int N>
__device__ __forceinline__ int fbl_pick(const int (&t)[N], int n)
{
    if (n <= t[N - 1])
        for (int i = 0; i < N; ++i)
            if (t[i] >= n) return t[i];
    return n;
}

// fft_best_length (util/src/FFTBestLength.cxx:12-59)
__device__ int fft_best_length_dev(int n, bool keep_odd_even)
{
    if (!keep_odd_even) return fbl_pick(c_fbl_any, n);
    return (n % 2 == 0) ? fbl_pick(c_fbl_even, n) : fbl_pick(c_fbl_odd, n);
}

// The window of one (event, plane) from its reduced depo extents: the same
// arithmetic, in the same double operations, as the host path.
__device__ void window_dev(const BatchStatic& bs, int ip, const WindowDev& w, EvPlane& o)
{
    const BatchPlaneStatic& pl = bs.pl[ip];
    double pmin = 0, pmax = 0, tmin = 0, tmax = 0;  // gausdesc_range of an empty set
    if (w.nadded > 0) {
        pmin = dkey_inv(w.pmin);
        pmax = dkey_inv(w.pmax);
        tmin = dkey_inv(w.tmin);
        tmax = dkey_inv(w.tmax);
    }
    auto ibin = [&](double v) { return __double2int_rz(__ddiv_rn(__dsub_rn(v, pl.imp_min), pl.imp_bs)); };
    auto tbin = [&](double v) { return __double2int_rz(__ddiv_rn(__dsub_rn(v, bs.start_time), bs.tbs)); };
    const int i0 = max(ibin(pmin), 0), i1 = min(ibin(pmax) + 1, pl.imp_nbins);
    const int t0 = max(tbin(tmin), 0), t1 = min(tbin(tmax) + 1, bs.nticks);
    const int G = pl.G;
    int start_ch = (int)floor(__ddiv_rn((double)i0, (double)(G - 1))) - 1;
    int end_ch = (int)ceil(__ddiv_rn((double)i1, (double)(G - 1))) + 2;
    if ((end_ch - start_ch) % 2 == 1) end_ch += 1;
    int start_tick = t0 - 1;
    int end_tick = t1 + 2;
    if ((end_tick - start_tick) % 2 == 1) end_tick += 1;
    const int ntw = fft_best_length_dev(end_ch - start_ch + 2 * pl.npad, true);
    const int npad_wire = (ntw - end_ch + start_ch) / 2;
    const int ntt = fft_best_length_dev(end_tick - start_tick + pl.waveform_pad, false);
    const int npad_time = ntt - end_tick + start_tick;
    o.start_ch = start_ch;
    o.end_ch = end_ch;
    o.start_tick = start_tick;
    o.end_tick = end_tick;
    o.m_start_ch = start_ch - npad_wire;
    o.m_end_ch = end_ch + npad_wire;
    o.m_start_tick = start_tick;
    o.m_end_tick = end_tick + npad_time;
    o.nw_ref = end_ch - start_ch + 2 * npad_wire;
    o.nt_ref = o.m_end_tick - o.m_start_tick;
    o.ndepos_added = w.nadded;
    o.outside_time = w.out_time;
    o.outside_pitch = w.out_pitch;
}

__device__ __forceinline__ int fdiv_floor(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

// One block of 256 threads: windows and work counts per (event, plane), then
// the prefixes (thread 0; at most kMaxBatch * kMaxPlanes entries).
__global__ void __launch_bounds__(256) k_plan_batch(BatchPlan* __restrict__ plan, BatchStatic bs, int nev,
                                                    const WindowDev* __restrict__ win,
                                                    long long vcap)
{
    __shared__ int s_status;
    __shared__ int c_raster[kMaxBatch * kMaxPlanes], c_rows[kMaxBatch * kMaxPlanes],
        c_orows[kMaxBatch * kMaxPlanes], c_conv[kMaxBatch * kMaxPlanes];
    const int np = bs.np, ne = nev * np;
    if (threadIdx.x == 0) s_status = 0;
    __syncthreads();
    for (int k = threadIdx.x; k < ne; k += blockDim.x) {
        const int e = k / np, ip = k - e * np;
        const WindowDev& w = win[k];
        EvPlane o{};
        window_dev(bs, ip, w, o);
        const BatchPlaneStatic& pl = bs.pl[ip];
        int st = 0;
        if (w.oversize) st |= kBatchOversize;
        if (w.bigcharge) st |= kBatchBigCharge;
        o.nin = w.nadded > 0 ? o.end_ch - o.start_ch : 0;
        o.nout = o.nin ? o.nin + 2 * pl.npad : 0;
        o.ncols = o.end_tick - o.start_tick;
        int cls = -1;
        for (int c = 0; c < bs.ncls; ++c)
            if (bs.cls_N[c] >= o.nt_ref) {
                cls = c;
                break;
            }
        if (cls < 0 || o.nin > pl.nin_max) {
            if (o.nin) st |= kBatchNoClass;
            o.nin = o.nout = 0;
            cls = 0;
        }
        o.cls = cls;
        o.N = bs.cls_N[cls];
        o.M = o.N / 2;
        o.ktile0 = fdiv_floor(o.start_tick, kTile);
        o.ntile = fdiv_floor(o.start_tick + o.N - 1, kTile) - o.ktile0 + 1;
        o.qoff = (long long)e * bs.qslot_total + pl.qslot;
        o.voff = (long long)e * bs.vslot_total + pl.vslot;
        plan->ep[k] = o;
        c_raster[k] = o.nin * o.ntile;
        c_rows[k] = pl.G * o.nin;
        c_orows[k] = o.nout;
        c_conv[k] = o.nin ? ((o.M + 31) / 32) * ((o.nout + kConvRows - 1) / kConvRows) : 0;
        if (st) atomicOr(&s_status, st);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int a = 0, b = 0, c = 0;
        for (int k = 0; k < ne; ++k) {
            plan->pre_raster[k] = a;
            plan->pre_rows[k] = b;
            plan->pre_orows[k] = c;
            a += c_raster[k];
            b += c_rows[k];
            c += c_orows[k];
        }
        plan->pre_raster[ne] = a;
        plan->pre_rows[ne] = b;
        plan->pre_orows[ne] = c;
        for (int ip = 0; ip < np; ++ip) {
            int t = 0;
            for (int e = 0; e < nev; ++e) {
                plan->pre_conv[ip][e] = t;
                t += c_conv[e * np + ip];
            }
            plan->pre_conv[ip][nev] = t;
        }
        unsigned long long tv = 0;  // visits of the pass, 64-bit (the list offsets are int)
        for (int e = 0; e < nev; ++e) tv += win[(size_t)e * np].nvisits;
        plan->total_visits = (long long)tv;
        plan->nev = nev;
        plan->np = np;
        plan->status = s_status | (tv > (unsigned long long)vcap ? kBatchVisitOverflow : 0) |
                       (tv >= 0x7fffffffull ? kBatchTooBig : 0);
        for (int k = 0; k < 3 + kMaxPlanes; ++k) plan->next[k] = 0;
    }
}

void launch_plan_batch(BatchPlan* plan, const BatchStatic& bs, int nev, const WindowDev* win, long long vcap,
                       cudaStream_t s)
{
    k_plan_batch<<<1, 256, 0, s>>>(plan, bs, nev, win, vcap);
}

// Next work item of a persistent block (all threads get the same value):
// blocks take items from a shared counter, so a block that drew a heavy item
// does not hold back the rest.
__device__ __forceinline__ int next_item(int* counter, int* s_item)
{
    if (threadIdx.x == 0 && threadIdx.y == 0) *s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int item = *s_item;
    __syncthreads();  // every thread has read it before the next draw overwrites it
    return item;
}

// Index of the (event, plane) entry whose item range holds `item`: the last
// k in [0, n) with pre[k] <= item (entries with no items are skipped).
__device__ __forceinline__ int find_entry(const int* __restrict__ pre, int n, int item)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pre[mid] <= item) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <bool FLUC>
__global__ void __launch_bounds__(kRasterThreads, FLUC ? 1 : 5) k_raster_batch(const BatchPlan* __restrict__ plan, BatchStatic bs,
                                                                 PlaneSet ps, const PatchRec* __restrict__ rec,
                                                                 long long recstride,
                                                                 const float* __restrict__ tprof, TprofPool pool,
                                                                 const unsigned char* __restrict__ wide_key,
                                                                 const int* __restrict__ wire_cnt,
                                                                 const int* __restrict__ wire_off,
                                                                 const Visit* __restrict__ visits, long long vcap,
                                                                 const unsigned long long* __restrict__ key_bound,
                                                                 float* __restrict__ Q, EventTable evt, FlucParams fp,
                                                                 const FlucRec* __restrict__ fluc)
{
    extern __shared__ int smem_i[];
    __shared__ float scale[kTileBlocks], iscale[kTileBlocks];
    if (plan->status & kBatchSkip) return;
    __shared__ int s_item;
    const int ne = plan->nev * plan->np;
    const int total = plan->pre_raster[ne];
    int* ctr = const_cast<int*>(&plan->next[0]);
    for (int item = next_item(ctr, &s_item); item < total; item = next_item(ctr, &s_item)) {
        const int k = find_entry(plan->pre_raster, ne, item);
        const int e = k / plan->np, ip = k - e * plan->np;
        const EvPlane& E = plan->ep[k];
        GridPlane P;
        P.nimp = ps.p[ip].nimp;
        P.G = bs.pl[ip].G;
        P.nwires = ps.p[ip].nwires;
        P.wire_base = ps.p[ip].wire_base;
        P.start_ch = E.start_ch;
        P.nin = E.nin;
        P.col0 = E.start_tick;
        P.ncols = E.ncols;
        P.N = E.N;
        P.tbs = (float)bs.tbs;
        P.pbs = (float)ps.p[ip].imp_bs;
        P.qoff = E.qoff;
        P.recoff = (long long)ip * recstride;
        P.row_base = 0;
        P.ktile0 = E.ktile0;
        P.ntile = E.ntile;
        const int rel = item - plan->pre_raster[k];
        const int row = rel / E.ntile;
        if constexpr (FLUC)
            raster_tile_fluc(P, ip, row, E.ktile0 + (rel - row * E.ntile), e * bs.nkeys, bs.ntiles, evt, fp, rec,
                             fluc, wire_cnt, wire_off, visits, vcap, Q, reinterpret_cast<long long*>(smem_i));
        else
            raster_tile(P, row, E.ktile0 + (rel - row * E.ntile), e * bs.nkeys, bs.ntiles, rec, tprof, pool,
                        wide_key, wire_cnt, wire_off, visits, vcap, key_bound, Q, smem_i, scale, iscale);
    }
}

void launch_raster_batch(const BatchPlan* plan, const BatchStatic& bs, const PlaneSet& ps, const PatchRec* rec,
                         long long recstride, const float* tprof, const TprofPool& pool,
                         const unsigned char* wide_key, const int* wire_cnt, const int* wire_off,
                         const Visit* visits, long long vcap, const unsigned long long* key_bound, float* Q,
                         int nblocks, int maxG, const EventTable& evt, const FlucParams& fp, const FlucRec* fluc,
                         cudaStream_t s)
{
    const size_t smem = std::max(raster_smem_bytes(maxG), raster_fluc_smem_bytes(maxG));
    if (fp.on_patch)
        k_raster_batch<true><<<nblocks, kRasterThreads, smem, s>>>(plan, bs, ps, rec, recstride, tprof, pool, wide_key,
                                                                    wire_cnt,
                                                                    wire_off, visits, vcap, key_bound, Q, evt, fp,
                                                                    fluc);
    else
        k_raster_batch<false><<<nblocks, kRasterThreads, smem, s>>>(plan, bs, ps, rec, recstride, tprof, pool,
                                                                     wide_key, wire_cnt,
                                                                     wire_off, visits, vcap, key_bound, Q, evt, fp,
                                                                     fluc);
}

// Time FFT of every charge-grid row of the pass, in place (rows of N reals
// become M packed bins), whatever their length class.
__global__ void k_rfft_batch(const BatchPlan* __restrict__ plan, const FftDesc* __restrict__ descs,
                             float* __restrict__ Q)
{
    extern __shared__ float2 sm[];
    if (plan->status & kBatchSkip) return;
    __shared__ int s_item;
    const int ne = plan->nev * plan->np;
    const int total = plan->pre_rows[ne];
    int* ctr = const_cast<int*>(&plan->next[1]);
    for (int item = next_item(ctr, &s_item); item < total; item = next_item(ctr, &s_item)) {
        const int k = find_entry(plan->pre_rows, ne, item);
        const EvPlane& E = plan->ep[k];
        const FftDesc d = descs[E.cls];
        float* x = Q + E.qoff + (size_t)(item - plan->pre_rows[k]) * E.N;
        rfft_row(x, E.N, reinterpret_cast<float2*>(x), d, sm);
    }
}

void launch_rfft_batch(const BatchPlan* plan, const FftDesc* descs, float* Q, int nblocks, int nthreads, int maxM,
                       cudaStream_t s)
{
    const size_t smem = 2 * (size_t)maxM * sizeof(float2);
    k_rfft_batch<<<nblocks, nthreads, smem, s>>>(plan, descs, Q);
}

// Wire convolution with a run-time pad, one tile (generic response widths).
__device__ __forceinline__ void wire_conv_tile_any(const float2* __restrict__ Qh, const float2* __restrict__ Rh,
                                                   float2* __restrict__ Vh, int G, int PAD, int nin, int nout, int M,
                                                   int fblk, int oblk)
{
    const int lane = threadIdx.x, rg = threadIdx.y;
    const int f = fblk * 32 + lane;
    const int o0 = oblk * kConvRows;
    if (f >= M) return;
    float2 acc[kConvRB];
#pragma unroll
    for (int r = 0; r < kConvRB; ++r) acc[r] = make_float2(0.f, 0.f);
    for (int g = 0; g < G; ++g) {
        const float2* Rg = Rh + (size_t)g * (2 * PAD + 1) * M + f;
        for (int jj = 0; jj <= 2 * PAD; ++jj) {
            const float2 rr = Rg[(size_t)jj * M];
            const float rc = f == 0 ? 0.f : rr.y;
            const float ry = f == 0 ? rr.y : rr.x;
            const int j = jj - PAD;
#pragma unroll
            for (int r = 0; r < kConvRB; ++r) {
                const int i = o0 + rg * kConvRB + r - PAD - j;
                if (i < 0 || i >= nin) continue;
                const float2 q = Qh[((size_t)g * nin + i) * M + f];
                acc[r].x = fmaf(rr.x, q.x, fmaf(-rc, q.y, acc[r].x));
                acc[r].y = fmaf(ry, q.y, fmaf(rc, q.x, acc[r].y));
            }
        }
    }
#pragma unroll
    for (int r = 0; r < kConvRB; ++r) {
        const int o = o0 + rg * kConvRB + r;
        if (o < nout) Vh[(size_t)o * M + f] = acc[r];
    }
}

// PAD < 0: run-time pad (bs.pl[ip].npad) without shared-memory staging.
// Items of planes ip0 .. ip1-1 in order; within a plane, events in order.
template <int PAD, bool PAIR>
__global__ void __launch_bounds__(32 * kConvRG) k_conv_batch(const BatchPlan* __restrict__ plan, BatchStatic bs,
                                                             int ip0, int ip1, const float2* const* __restrict__ spec,
                                                             const float* __restrict__ Q, float2* __restrict__ V)
{
    extern __shared__ float2 conv_smem[];
    __shared__ int s_item;
    if (plan->status & kBatchSkip) return;
    const int nev = plan->nev, np = plan->np;
    int total = 0;
    for (int ip = ip0; ip < ip1; ++ip) total += plan->pre_conv[ip][nev];
    int* ctr = const_cast<int*>(&plan->next[3 + ip0]);
    for (int item = next_item(ctr, &s_item); item < total; item = next_item(ctr, &s_item)) {
        int ip = ip0, rel = item;
        while (rel >= plan->pre_conv[ip][nev]) {
            rel -= plan->pre_conv[ip][nev];
            ++ip;
        }
        const int* pre = plan->pre_conv[ip];
        const int e = find_entry(pre, nev, rel);
        const EvPlane& E = plan->ep[e * np + ip];
        rel -= pre[e];
        const int nfb = (E.M + 31) / 32;
        const int oblk = rel / nfb, fblk = rel - oblk * nfb;
        const float2* Qh = reinterpret_cast<const float2*>(Q + E.qoff);
        const float2* R = spec[(size_t)ip * bs.ncls + E.cls];
        if constexpr (PAD >= 0)
            wire_conv_tile<PAD, PAIR>(Qh, R, V + E.voff, bs.pl[ip].G, E.nin, E.nout, E.M, fblk, oblk, conv_smem);
        else
            wire_conv_tile_any(Qh, R, V + E.voff, bs.pl[ip].G, bs.pl[ip].npad, E.nin, E.nout, E.M, fblk, oblk);
    }
}

size_t conv_smem_bytes(int npad, bool pair)
{
    if (npad != 10 && npad != 21) return 0;
    return sizeof(float2) * 32 * ((size_t)(pair ? 2 : 1) * (kConvRows + 2 * npad) + (2 * npad + 1));
}

void launch_conv_batch(const BatchPlan* plan, const BatchStatic& bs, int ip0, int ip1, bool pair,
                       const float2* const* spec, const float* Q, float2* V, int nblocks, cudaStream_t s)
{
    const int npad = bs.pl[ip0].npad;
    dim3 block(32, kConvRG);
    const size_t sm = conv_smem_bytes(npad, pair);
#define WCT_CONVB(P, B) k_conv_batch<P, B><<<nblocks, block, sm, s>>>(plan, bs, ip0, ip1, spec, Q, V)
    if (npad == 10 && pair) WCT_CONVB(10, true);
    else if (npad == 10) WCT_CONVB(10, false);
    else if (npad == 21 && pair) WCT_CONVB(21, true);
    else if (npad == 21) WCT_CONVB(21, false);
#undef WCT_CONVB
    else k_conv_batch<-1, false><<<nblocks, block, 0, s>>>(plan, bs, ip0, ip1, spec, Q, V);
}

// Inverse time FFT of every V row of the pass and the frame write of its event.
__global__ void k_irfft_batch(const BatchPlan* __restrict__ plan, BatchStatic bs, const FftDesc* __restrict__ descs,
                              const float2* __restrict__ V, float* __restrict__ frames, long long frame_stride)
{
    extern __shared__ float2 sm[];
    if (plan->status & kBatchSkip) return;
    __shared__ int s_item;
    const int ne = plan->nev * plan->np;
    const int total = plan->pre_orows[ne];
    int* ctr = const_cast<int*>(&plan->next[2]);
    for (int item = next_item(ctr, &s_item); item < total; item = next_item(ctr, &s_item)) {
        const int k = find_entry(plan->pre_orows, ne, item);
        const int e = k / plan->np, ip = k - e * plan->np;
        const EvPlane& E = plan->ep[k];
        const BatchPlaneStatic& pl = bs.pl[ip];
        const int o = item - plan->pre_orows[k];
        const int W = E.start_ch - pl.npad + o;
        const int wlo = max(0, E.m_start_ch), whi = min(pl.nwires, E.m_end_ch);
        if (W < wlo || W >= whi) continue;  // uniform over the block
        const FftDesc d = descs[E.cls];
        irfft_row(V + E.voff + (size_t)o * E.M, d, frames + (size_t)e * frame_stride + (size_t)(pl.row0 + W) * bs.nticks,
                  E.start_tick, min(E.N, E.nt_ref), bs.nticks, sm);
    }
}

void launch_irfft_batch(const BatchPlan* plan, const BatchStatic& bs, const FftDesc* descs, const float2* V,
                        float* frames, long long frame_stride, int nblocks, int nthreads, int maxM, cudaStream_t s)
{
    const size_t smem = 2 * (size_t)maxM * sizeof(float2);
    k_irfft_batch<<<nblocks, nthreads, smem, s>>>(plan, bs, descs, V, frames, frame_stride);
}

// Shared-memory opt-ins of the batched kernels, set before a graph capture
// (the launchers themselves only enqueue).
void batch_kernel_attributes(int maxG, int maxM)
{
    const int sr = (int)std::max(raster_smem_bytes(maxG), raster_fluc_smem_bytes(maxG));
    const int sf = (int)(2 * (size_t)maxM * sizeof(float2));
    cudaFuncSetAttribute((const void*)k_raster_batch<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sr);
    cudaFuncSetAttribute((const void*)k_raster_batch<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sr);
    cudaFuncSetAttribute((const void*)k_rfft_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, sf);
    cudaFuncSetAttribute((const void*)k_irfft_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, sf);
    cudaFuncSetAttribute((const void*)k_conv_batch<10, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)conv_smem_bytes(10, true));
    cudaFuncSetAttribute((const void*)k_conv_batch<10, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)conv_smem_bytes(10, false));
    cudaFuncSetAttribute((const void*)k_conv_batch<21, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)conv_smem_bytes(21, true));
    cudaFuncSetAttribute((const void*)k_conv_batch<21, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)conv_smem_bytes(21, false));
}

}  // namespace wctb200
