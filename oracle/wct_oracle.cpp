// ============================================================================
// TEST INFRASTRUCTURE ONLY -- NOT PART OF THE PRODUCT.
//
// CPU restatement of the Wire-Cell Toolkit signal-simulation hot path
// (Gen::DepoTransform chain), used as
//   * the parity oracle of the GPU path (tests/ and __graft_entry__.smoke()),
//   * the timed CPU baseline of bench.py (cpu_baseline, --impl reference).
// The product library never links, loads or calls this file.
//
// It is instantiated twice:
//   * real_t = float  : step-for-step FP32 restatement of the reference
//                       (FP32 patches, FP32 FFTs, FP64 drift/erf/weights),
//   * real_t = double : the same algorithm with every FP32 step in FP64
//                       (the "FP64 oracle").
// Every function cites the reference file:line it restates (paths relative to
// the wire-cell-toolkit source tree).
//
// Pins: Binning, GausDesc (distance, binint, weight), Pimpos and the trace
// edges equal the reference's own code compiled from its source tree
// (oracle/_ref; tests/golden/binning_ref.json and ref_funcs.json;
// tests/test_oracle.py and tests/test_ref_funcs.py); the FFT length tables
// equal the reference's text (tests/golden/fft_lengths_ref.json).
// No reference test pins whole frames.
//
// Deliberate differences from the reference, all without numerical effect
// beyond double round-off:
//   * the reference iterates its GaussianDiffusion std::set in heap-pointer
//     order (BinnedDiffusion_transform.cxx:279); this restatement iterates in
//     input order, which only changes the order of double additions;
//   * FFTs are this file's own mixed-radix Stockham transforms instead of
//     FFTW (aux/src/FftwDFT.cxx); they follow the same IDFT conventions
//     (forward unnormalised, inverse 1/n, iface/inc/WireCellIface/IDFT.h:10-80).
// ============================================================================

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <random>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

namespace orc {

// ---------------------------------------------------------------------------
// fft_best_length -- util/src/FFTBestLength.cxx:12-59 (same size tables).
// ---------------------------------------------------------------------------
static const size_t kSizesAny[] = {
    33,   35,   40,   42,   44,   56,   64,   66,   70,   77,   80,   96,   98,   100,  112,  121,  128,
    140,  143,  160,  168,  169,  200,  224,  256,  280,  320,  400,  448,  512,  560,  640,  686,  768,
    800,  847,  896,  1024, 1120, 1280, 1331, 1372, 1400, 1536, 1600, 1792, 2048, 2560, 2662, 2744, 3200,
    3584, 4096, 4116, 4480, 4802, 5120, 5324, 5376, 5544, 5600, 5632, 5929, 6174, 6272, 6292, 6655, 7168,
    7840, 8192, 8232, 8960, 9317, 10240, 10648, 11979, 14336, 15972, 16384};
static const size_t kSizesEven[] = {
    40,   42,   44,   56,   64,   66,   70,   72,   80,   96,   98,   100,  112,  120,  128,  140,  160,
    168,  200,  224,  256,  280,  320,  400,  448,  512,  560,  640,  686,  768,  800,  896,  1024, 1120,
    1280, 1372, 1400, 1536, 1600, 1792, 2048, 2560, 2662, 2744, 3200, 3584, 4096, 4116, 4480, 4802, 5120,
    5324, 5376, 5544, 5600, 5632, 6174, 6272, 6292, 6468, 7168, 7840, 8192, 8232, 8960, 10240, 10648, 11200,
    11858, 11880, 14336, 15972, 16384};
static const size_t kSizesOdd[] = {
    33,   35,   39,   49,   55,   63,   65,   77,   81,   91,   99,   121,  143,  169,  175,  187,  225,
    231,  245,  275,  297,  343,  363,  375,  385,  405,  441,  455,  495,  539,  605,  637,  693,  735,
    847,  875,  891,  945,  1001, 1089, 1331, 1573, 1859, 1875, 2197, 2299, 2431, 2541, 2625, 2695, 3025,
    3267, 3993, 4095, 4125, 4719, 4725, 5005, 5145, 5445, 5929, 6655, 7007, 7623, 7865, 9317, 9801, 11979,
    14157, 14175, 15379, 16335};

template <size_t N>
static size_t first_at_least(const size_t (&tab)[N], size_t n)
{
    if (n <= tab[N - 1]) {
        for (size_t i = 0; i < N; ++i)
            if (tab[i] >= n) return tab[i];
    }
    return n;
}

size_t fft_best_length(size_t n, bool keep_odd_even)
{
    if (!keep_odd_even) return first_at_least(kSizesAny, n);
    if (n % 2 == 0) return first_at_least(kSizesEven, n);
    return first_at_least(kSizesOdd, n);
}

// ---------------------------------------------------------------------------
// Binning -- util/inc/WireCellUtil/Binning.h:25-103.
// ---------------------------------------------------------------------------
struct Binning {
    int nbins{0};
    double minv{0}, maxv{0}, binsize{0};
    Binning() = default;
    Binning(int n, double lo, double hi) : nbins(n), minv(lo), maxv(hi), binsize((hi - lo) / n) {}
    int bin(double v) const { return int((v - minv) / binsize); }           // Binning.h:75
    double center(int i) const { return minv + (i + 0.5) * binsize; }        // Binning.h:79
    double edge(int i) const { return minv + i * binsize; }                  // Binning.h:88
    std::pair<int, int> sample_bin_range(double lo, double hi) const         // Binning.h:99-102
    {
        return {std::max(bin(lo), 0), std::min(bin(hi) + 1, nbins)};
    }
};

// ---------------------------------------------------------------------------
// Minimal 3-vector with the operation order of util/inc/WireCellUtil/D3Vector.h.
// ---------------------------------------------------------------------------
struct V3 {
    double x{0}, y{0}, z{0};
    double dot(const V3& o) const { return x * o.x + y * o.y + z * o.z; }   // D3Vector.h:125-129
    double mag() const { return std::sqrt(x * x + y * y + z * z); }         // D3Vector.h:144
    V3 norm() const                                                         // D3Vector.h:147-154
    {
        double m = mag();
        if (m <= 0) return V3{};
        return V3{x / m, y / m, z / m};
    }
    V3 cross(const V3& r) const                                             // D3Vector.h:157-164
    {
        return V3{y * r.z - z * r.y, z * r.x - x * r.z, x * r.y - y * r.x};
    }
    V3 operator-(const V3& o) const { return V3{x - o.x, y - o.y, z - o.z}; }
};

// ---------------------------------------------------------------------------
// Pimpos -- util/src/Pimpos.cxx:5-68.
// ---------------------------------------------------------------------------
struct Pimpos {
    int nimp{10};
    V3 origin;
    V3 axis[3];
    Binning region, impact;
    Pimpos(int nwires, double minp, double maxp, V3 wire, V3 pitch, V3 org, int nbins)
        : nimp(nbins), origin(org)
    {
        axis[1] = wire.norm();
        axis[2] = pitch.norm();
        axis[0] = axis[1].cross(axis[2]);
        const int nimpstot = nwires * nbins;
        const double regionsize = (maxp - minp) / (nwires - 1);
        const double pmin = minp - 0.5 * regionsize;
        const double pmax = maxp + 0.5 * regionsize;
        region = Binning(nwires, pmin, pmax);
        impact = Binning(nimpstot, pmin, pmax);
    }
    double distance(const V3& pt) const { return axis[2].dot(pt - origin); }  // Pimpos.cxx:58
    int wire_impact(int w) const { return (0.5 + w) * nimp; }                 // Pimpos.cxx:41
    std::pair<int, int> wire_impacts(int w) const                             // Pimpos.cxx:43-47
    {
        const int wi = wire_impact(w);
        return {wi - nimp / 2, wi + nimp / 2};
    }
};

// ---------------------------------------------------------------------------
// FFT: mixed-radix Stockham autosort, IDFT conventions
// (iface/inc/WireCellIface/IDFT.h:10-80: forward unnormalised, inverse 1/n).
// ---------------------------------------------------------------------------
template <typename T>
struct FFTPlan {
    int n{0};
    std::vector<int> radix;
    std::vector<std::complex<T>> tw;  // exp(-2 pi i m / n), m in [0, n)
};

template <typename T>
static const FFTPlan<T>& fft_plan(int n)
{
    static std::mutex mtx;
    static std::map<int, std::unique_ptr<FFTPlan<T>>> cache;
    std::lock_guard<std::mutex> lk(mtx);
    auto it = cache.find(n);
    if (it != cache.end()) return *it->second;
    auto p = std::make_unique<FFTPlan<T>>();
    p->n = n;
    int m = n;
    while (m % 4 == 0) { p->radix.push_back(4); m /= 4; }
    while (m % 2 == 0) { p->radix.push_back(2); m /= 2; }
    for (int f = 3; m > 1; f += 2) {
        while (m % f == 0) { p->radix.push_back(f); m /= f; }
    }
    p->tw.resize(n);
    for (int k = 0; k < n; ++k) {
        long double a = -2.0L * 3.14159265358979323846264338327950288L * (long double)k / (long double)n;
        p->tw[k] = std::complex<T>((T)std::cos(a), (T)std::sin(a));
    }
    auto& ref = *p;
    cache[n] = std::move(p);
    return ref;
}

// In-place 1-D DFT of length n (sign -1 forward, +1 backward, unnormalised).
template <typename T>
static void fft_1d(std::complex<T>* data, int n, int sign, std::complex<T>* work)
{
    if (n <= 1) return;
    const FFTPlan<T>& P = fft_plan<T>(n);
    using C = std::complex<T>;
    C* src = data;
    C* dst = work;
    int Ns = 1;
    C v[64];
    C y[64];
    for (int R : P.radix) {
        const int nR = n / R;
        const int twstep = n / (Ns * R);
        for (int j = 0; j < nR; ++j) {
            const int k = j % Ns;
            for (int r = 0; r < R; ++r) {
                C a = src[j + r * nR];
                if (r && k) {
                    C w = P.tw[(size_t)((long long)k * r * twstep % n)];
                    if (sign > 0) w = std::conj(w);
                    a *= w;
                }
                v[r] = a;
            }
            if (R == 2) {
                y[0] = v[0] + v[1];
                y[1] = v[0] - v[1];
            }
            else if (R == 4) {
                C a0 = v[0] + v[2], a1 = v[0] - v[2];
                C b0 = v[1] + v[3], b1 = v[1] - v[3];
                C jb1 = (sign < 0) ? C(b1.imag(), -b1.real()) : C(-b1.imag(), b1.real());
                y[0] = a0 + b0;
                y[2] = a0 - b0;
                y[1] = a1 + jb1;
                y[3] = a1 - jb1;
            }
            else {
                const int rstep = n / R;
                for (int a = 0; a < R; ++a) {
                    C s = 0;
                    for (int b = 0; b < R; ++b) {
                        C w = P.tw[(size_t)(((a * b) % R) * rstep)];
                        if (sign > 0) w = std::conj(w);
                        s += v[b] * w;
                    }
                    y[a] = s;
                }
            }
            const int idxD = (j / Ns) * Ns * R + k;
            for (int r = 0; r < R; ++r) dst[idxD + r * Ns] = y[r];
        }
        std::swap(src, dst);
        Ns *= R;
    }
    if (src != data) std::copy(src, src + n, data);
}

// Optional external transform in place of fft_1d: a [nrows][ncols] complex
// array (float or double per fp64) transformed along axis (1: each row, 0:
// each column), sign -1 forward / +1 backward, unnormalised.  The timed CPU
// baseline sets it to libtorch-CPU's MKL transforms (oracle/torch_fft.cpp),
// the reference's TorchDFT backend (pytorch/src/DFT.cxx:80-123); parity runs
// leave it unset.
typedef void (*ExtFft)(void* a, int nrows, int ncols, int axis, int sign, int fp64);
static std::atomic<ExtFft> g_ext_fft{nullptr};

template <typename T>
struct Dft {
    using C = std::complex<T>;
    static bool ext(C* a, int nrows, int ncols, int axis, int sign)
    {
        ExtFft f = g_ext_fft.load();
        if (!f) return false;
        f(a, nrows, ncols, axis, sign, sizeof(T) == sizeof(double) ? 1 : 0);
        return true;
    }
    // aux/src/FftwDFT.cxx:88-115 (1d)
    static void fwd1d(C* x, int n)
    {
        if (ext(x, 1, n, 1, -1)) return;
        std::vector<C> w(n);
        fft_1d<T>(x, n, -1, w.data());
    }
    static void inv1d(C* x, int n)
    {
        if (!ext(x, 1, n, 1, +1)) {
            std::vector<C> w(n);
            fft_1d<T>(x, n, +1, w.data());
        }
        for (int i = 0; i < n; ++i) x[i] /= (T)n;
    }
    // Row-major [nrows][ncols]; axis=1 transforms each row, axis=0 each column
    // (aux/src/FftwDFT.cxx:119-176, 1b methods).
    static void do1b(C* a, int nrows, int ncols, int axis, int sign, bool norm)
    {
        if (ext(a, nrows, ncols, axis, sign)) {
            if (norm) {
                const T n = (T)(axis == 1 ? ncols : nrows);
                for (size_t k = 0; k < (size_t)nrows * ncols; ++k) a[k] /= n;
            }
            return;
        }
        if (axis == 1) {
            std::vector<C> w(ncols);
            for (int r = 0; r < nrows; ++r) {
                fft_1d<T>(a + (size_t)r * ncols, ncols, sign, w.data());
                if (norm)
                    for (int c = 0; c < ncols; ++c) a[(size_t)r * ncols + c] /= (T)ncols;
            }
        }
        else {
            std::vector<C> col(nrows), w(nrows);
            for (int c = 0; c < ncols; ++c) {
                for (int r = 0; r < nrows; ++r) col[r] = a[(size_t)r * ncols + c];
                fft_1d<T>(col.data(), nrows, sign, w.data());
                for (int r = 0; r < nrows; ++r) a[(size_t)r * ncols + c] = norm ? col[r] / (T)nrows : col[r];
            }
        }
    }
    static void fwd1b(C* a, int nr, int nc, int axis) { do1b(a, nr, nc, axis, -1, false); }
    static void inv1b(C* a, int nr, int nc, int axis) { do1b(a, nr, nc, axis, +1, true); }
    // aux/src/FftwDFT.cxx:179-217 (2d)
    static void fwd2d(C* a, int nr, int nc)
    {
        do1b(a, nr, nc, 1, -1, false);
        do1b(a, nr, nc, 0, -1, false);
    }
};

// util/inc/WireCellUtil/Spectrum.h:56-89 (hermitian_mirror) +
// aux/src/DftTools.cxx:39-50 (inv_c2r).
template <typename T>
static std::vector<T> inv_c2r(const std::vector<std::complex<T>>& spec)
{
    using C = std::complex<T>;
    const size_t len = spec.size();
    std::vector<C> sym(len);
    const size_t half = len / 2 + 1;
    std::copy(spec.begin(), spec.begin() + std::min(half, len), sym.begin());
    sym[0] = C(std::real(sym[0]), 0);
    const size_t mid = len / 2;
    if (len % 2) {
        for (size_t i = 1; i <= mid; ++i) sym[len - i] = sym[i];
    }
    else {
        sym[mid] = C(std::real(sym[mid]), 0);
        for (size_t i = 1; i < mid; ++i) sym[len - i] = sym[i];
    }
    for (size_t i = mid + 1; i < len; ++i) sym[i] = std::conj(sym[i]);
    Dft<T>::inv1d(sym.data(), (int)len);
    std::vector<T> out(len);
    for (size_t i = 0; i < len; ++i) out[i] = std::real(sym[i]);
    return out;
}

// aux/src/DftTools.cxx:24-30 (fwd_r2c, full complex length)
template <typename T>
static std::vector<std::complex<T>> fwd_r2c(const std::vector<T>& v)
{
    std::vector<std::complex<T>> c(v.size());
    for (size_t i = 0; i < v.size(); ++i) c[i] = std::complex<T>(v[i], 0);
    Dft<T>::fwd1d(c.data(), (int)c.size());
    return c;
}

// Stage clock of the timed CPU baseline: seconds since an arbitrary origin.
static double now_s()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
// Stages timed by orc_run (seconds, summed over planes).
enum { kStDrift = 0, kStRaster, kStRespPrep, kStFftConv, kStExtract, kStPir, kNStages };

// ---------------------------------------------------------------------------
// Depos. Layout of one depo: t, q, x, y, z, extent_long, extent_tran.
// ---------------------------------------------------------------------------
struct Depo {
    double t, q, x, y, z, el, et;
    int index;  // position in the caller's input array
};

// ---------------------------------------------------------------------------
// Drifter::insert -- gen/src/Drifter.cxx:127-196,
// Xregion tests gen/src/Drifter.cxx:53-60.
// ---------------------------------------------------------------------------
struct XRegion {
    double anode, response, cathode;
    bool inside_response(double x) const { return (anode < x and x < response) or (response < x and x < anode); }
    bool inside_bulk(double x) const { return (response < x and x < cathode) or (cathode < x and x < response); }
};

struct DriftParams {
    double DL, DT, lifetime, speed, toffset;
    std::vector<XRegion> xregions;
    std::mt19937* rng{nullptr};  // Drifter "fluctuate": binomial absorption (Drifter.cxx:177-185)
};

static bool drift_one(const DriftParams& dp, const Depo& in, Depo& out)
{
    const double Qi = in.q;
    if (Qi == 0.0) return false;
    double respx = 0, direction = 0.0;
    const XRegion* xr = nullptr;
    for (auto& r : dp.xregions)
        if (r.inside_response(in.x)) { xr = &r; break; }
    if (xr) { respx = xr->response; direction = -1.0; }
    else {
        for (auto& r : dp.xregions)
            if (r.inside_bulk(in.x)) { xr = &r; break; }
        if (xr) { respx = xr->response; direction = 1.0; }
    }
    if (!xr) return false;
    const double dt = std::abs((respx - in.x) / dp.speed);
    double dL = in.el, dT = in.et;
    double Qf = Qi;
    if (direction > 0) {
        const double absorbprob = 1 - exp(-dt / dp.lifetime);
        double dQ = Qi * absorbprob;
        if (dp.rng) {
            const double sign = Qi < 0 ? -1.0 : 1.0;
            std::binomial_distribution<int> bin((int)std::abs(Qi), absorbprob);
            dQ = sign * bin(*dp.rng);
        }
        Qf = Qi - dQ;
        dL = sqrt(2.0 * dp.DL * dt + dL * dL);
        dT = sqrt(2.0 * dp.DT * dt + dT * dT);
    }
    out = in;
    out.t = in.t + direction * dt + dp.toffset;
    out.x = respx;
    out.q = Qf;
    out.el = dL;
    out.et = dT;
    return true;
}

// Drifter::flush -- time-ordered output (gen/src/Drifter.cxx:198-209).
static std::vector<Depo> drift_all(const DriftParams& dp, const std::vector<Depo>& in)
{
    std::vector<Depo> out;
    out.reserve(in.size());
    for (auto& d : in) {
        Depo o;
        if (drift_one(dp, d, o)) out.push_back(o);
    }
    std::stable_sort(out.begin(), out.end(), [](const Depo& a, const Depo& b) { return a.t < b.t; });
    return out;
}

// BoundingBox::inside -- util/src/BoundingBox.cxx:37-56.
static bool bb_inside(const double* lo, const double* hi, const Depo& d)
{
    const double p[3] = {d.x, d.y, d.z};
    for (int i = 0; i < 3; ++i) {
        const double b1 = lo[i], b2 = hi[i];
        if (b1 < b2) {
            if (p[i] < b1 or p[i] > b2) return false;
            continue;
        }
        if (b2 < b1) {
            if (p[i] < b2 or p[i] > b1) return false;
            continue;
        }
    }
    return true;
}

// ---------------------------------------------------------------------------
// GausDesc -- gen/inc/WireCellGen/GaussianDiffusion.h:20-63 and
// gen/src/GaussianDiffusion.cxx:30-92.
// ---------------------------------------------------------------------------
struct GausDesc {
    double center, sigma;
    double distance(double x) const
    {
        double ret = 0.0;
        if (!sigma) ret = x - center;
        else ret = (x - center) / sigma;
        return ret;
    }
    std::pair<double, double> sigma_range(double nsigma) const
    {
        return {center - sigma * nsigma, center + sigma * nsigma};
    }
    std::vector<double> binint(double start, double step, int nbins) const
    {
        std::vector<double> bins;
        if (!sigma) {
            bins.assign(1, 1.0);
        }
        else {
            bins.assign(nbins, 0.0);
            std::vector<double> erfs(nbins + 1, 0.0);
            const double sqrt2 = sqrt(2.0);
            for (int ind = 0; ind <= nbins; ++ind) {
                double x = (start + step * ind - center) / (sqrt2 * sigma);
                erfs[ind] = 0.5 * std::erf(x);
            }
            for (int ib = 0; ib < nbins; ++ib) bins[ib] = erfs[ib + 1] - erfs[ib];
        }
        return bins;
    }
    std::vector<double> weight(double start, double step, int nbins, const std::vector<double>& pvec) const
    {
        std::vector<double> wt;
        if (!sigma) {
            wt.assign(1, (start + step - center) / step);
        }
        else {
            wt.assign(nbins, 0.0);
            const double pi = 4.0 * atan(1);
            double x2 = start;
            double x1 = 0;
            double gaus2 = exp(-0.5 * (start - center) / sigma * (start - center) / sigma);
            double gaus1 = 0;
            for (int ind = 0; ind < nbins; ind++) {
                x1 = x2;
                x2 = x1 + step;
                double rel = (x2 - center) / sigma;
                gaus1 = gaus2;
                gaus2 = exp(-0.5 * rel * rel);
                wt[ind] = -1.0 * sigma / (x1 - x2) * (gaus2 - gaus1) / sqrt(2.0 * pi) / pvec[ind] +
                          (center - x2) / (x1 - x2);
            }
        }
        return wt;
    }
};

// One sampled diffusion patch (GaussianDiffusion, gen/src/GaussianDiffusion.cxx:116-229).
template <typename T>
struct Patch {
    int toffset{-1}, poffset{-1};
    int nt{0}, np{0};
    std::vector<T> val;        // [np][nt]
    std::vector<double> qw;    // np linear weights
};

template <typename T>
static void set_sampling(const Depo& depo, const GausDesc& td, const GausDesc& pd, const Binning& tb,
                         const Binning& pb, double nsigma, Patch<T>& out, std::mt19937* fluctuate = nullptr)
{
    out.toffset = out.poffset = -1;
    out.nt = out.np = 0;
    out.val.clear();
    out.qw.clear();
    auto tr = td.sigma_range(nsigma);
    auto tbr = tb.sample_bin_range(tr.first, tr.second);
    const int ntss = std::max(tbr.second - tbr.first, 0);
    out.toffset = tbr.first;
    auto tvec = td.binint(tb.edge(out.toffset), tb.binsize, ntss);
    if (!ntss || tbr.second <= tbr.first) { out.nt = out.np = 0; return; }

    auto pr = pd.sigma_range(nsigma);
    auto pbr = pb.sample_bin_range(pr.first, pr.second);
    const int npss = std::max(pbr.second - pbr.first, 0);
    out.poffset = pbr.first;
    auto pvec = pd.binint(pb.edge(out.poffset), pb.binsize, npss);
    if (!npss || pbr.second <= pbr.first) { out.nt = out.np = 0; return; }

    out.qw = pd.weight(pb.edge(out.poffset), pb.binsize, npss, pvec);  // weightstrat 2 (linear)
    out.nt = ntss;
    out.np = npss;
    out.val.assign((size_t)npss * ntss, (T)0);
    double raw_sum = 0.0;
    for (int ip = 0; ip < npss; ++ip) {
        for (int it = 0; it < ntss; ++it) {
            const double v = pvec[ip] * tvec[it];
            raw_sum += v;
            out.val[(size_t)ip * ntss + it] = (T)v;
        }
    }
    const double depo_charge = depo.q;
    const T scale = (T)(depo_charge / raw_sum);  // Eigen float array *= double scalar
    for (auto& v : out.val) v *= scale;
    // GaussianDiffusion.cxx:184-213: every cell redrawn as Binomial(|Q|, cell / Q),
    // the patch rescaled to the depo charge; a patch whose draws are all zero is
    // not kept (the depo adds nothing)
    if (fluctuate) {
        const double charge_sign = depo_charge < 0 ? -1 : 1;
        double fluc_sum = 0;
        for (auto& v : out.val) {
            const double relval = (double)v / depo_charge;
            double number;
            if (relval >= 1.0) number = (int)std::abs(depo_charge);
            else {
                std::binomial_distribution<int> bin((int)std::abs(depo_charge), relval);
                number = bin(*fluctuate);
            }
            number *= charge_sign;
            fluc_sum += number;
            v = (T)number;
        }
        if (fluc_sum == 0) {
            out.val.assign(out.val.size(), (T)0);
            return;
        }
        const T f = (T)(depo_charge / fluc_sum);
        for (auto& v : out.val) v *= f;
    }
}

// ---------------------------------------------------------------------------
// PlaneImpactResponse -- gen/src/PlaneImpactResponse.cxx:89-320.
// ---------------------------------------------------------------------------
template <typename T>
struct ImpactResp {
    std::vector<std::complex<T>> spectrum;
    std::vector<T> waveform;
    int waveform_pad{0};
};

template <typename T>
struct PIR {
    std::vector<ImpactResp<T>> ir;
    std::vector<std::vector<int>> bywire;
    double half_extent{0}, pitch{0}, impact{0};
    // long_aux_waveform / long_aux_waveform_pad of every path (PlaneImpactResponse.cxx:121-150,252)
    std::vector<T> long_wf;
    int long_pad{0};
    int nwires() const { return (int)bywire.size(); }
    int nimp_per_wire() const { return (int)bywire[0].size(); }

    // PlaneImpactResponse.cxx:278-292
    std::pair<int, int> closest_wire_impact(double relpitch) const
    {
        const int center_wire = nwires() / 2;
        const int relwire = int(round(relpitch / pitch));
        const int wire_index = center_wire + relwire;
        const double remainder_pitch = relpitch - relwire * pitch;
        const int impact_index = int(round(remainder_pitch / impact)) + nimp_per_wire() / 2;
        return {wire_index, impact_index};
    }
    // PlaneImpactResponse.cxx:294-320; returns -1 where the reference throws.
    int closest(double relpitch) const
    {
        if (relpitch < -half_extent || relpitch > half_extent) return -1;
        auto wi = closest_wire_impact(relpitch);
        if (wi.first < 0 || wi.first >= (int)bywire.size()) return -1;
        const auto& region = bywire[wi.first];
        if (wi.second < 0 || wi.second >= (int)region.size()) return -1;
        int irind = region[wi.second];
        if (irind < 0 || irind > (int)ir.size()) return -1;
        return irind;
    }
};

struct FRPlane {
    int npaths, nsamp;
    const double* pitchpos;  // [npaths]
    const double* current;   // [npaths][nsamp]
    double pitch;            // PlaneResponse::pitch
};

// PlaneImpactResponse::build_responses, gen/src/PlaneImpactResponse.cxx:89-269,
// long responses included (:121-150): the product of their spectra at
// fft_best_length(nbins), back in time.
template <typename T>
static void build_pir(const FRPlane& fr, double tstart, double period, const std::vector<std::vector<double>>& shorts,
                      double overall_short_padding, double tick, int nbins, PIR<T>& pir,
                      const std::vector<std::vector<double>>& longs = {}, double long_padding = 0.0)
{
    pir.long_wf.clear();
    pir.long_pad = 0;
    if (!longs.empty()) {
        const size_t n_long = fft_best_length((size_t)nbins, false);
        std::vector<std::complex<T>> long_spec(n_long, std::complex<T>(1.0, 0.0));
        for (auto& lw : longs) {
            std::vector<T> wave(lw.begin(), lw.end());
            wave.resize(n_long, 0);
            auto spec = fwd_r2c<T>(wave);
            for (size_t i = 0; i < n_long; ++i) long_spec[i] *= spec[i];
        }
        pir.long_wf = inv_c2r<T>(long_spec);
        pir.long_pad = (int)(long_padding / tick);
    }
    using C = std::complex<T>;
    const size_t n_short = fft_best_length((size_t)(overall_short_padding / tick), false);
    std::vector<C> short_spec(n_short, C(1.0, 0.0));
    for (auto& sw : shorts) {
        std::vector<T> wave(sw.begin(), sw.end());
        wave.resize(n_short, 0);
        auto spec = fwd_r2c<T>(wave);
        for (size_t i = 0; i < n_short; ++i) short_spec[i] *= spec[i];
    }
    const int npaths = fr.npaths;
    const int n_per = 6;
    const int n_wires = npaths / n_per;
    const int n_wires_half = n_wires / 2;
    pir.impact = std::abs(fr.pitchpos[1] - fr.pitchpos[0]);
    pir.half_extent = std::max(std::abs(fr.pitchpos[0]), std::abs(fr.pitchpos[npaths - 1]));
    pir.pitch = 2.0 * std::abs(fr.pitchpos[n_per - 1] - fr.pitchpos[0]);

    const int rawresp_size = fr.nsamp;
    Binning rawbins(rawresp_size, tstart, tstart + rawresp_size * period);
    const double oopsilon = 1e-15 * fr.pitch;
    std::map<int, std::vector<int>> wire_to_ind;
    const int waveform_pad = (int)(overall_short_padding / tick);
    pir.ir.clear();
    for (int ipath = 0; ipath < npaths; ++ipath) {
        const int wirenum = int(ceil((fr.pitchpos[ipath] - oopsilon) / fr.pitch));
        wire_to_ind[wirenum].push_back(ipath);
        std::vector<T> wave(n_short, 0.0);
        for (int rind = 0; rind < rawresp_size; ++rind) {
            const double time = rawbins.center(rind);
            const size_t bin = time / tick;
            if (bin >= n_short) throw std::runtime_error("out of bounds field response");
            const double induced_charge = fr.current[(size_t)ipath * fr.nsamp + rind] * period;
            wave[bin] += induced_charge;
        }
        auto spec = fwd_r2c<T>(wave);
        if (!shorts.empty())
            for (size_t f = 0; f < n_short; ++f) spec[f] *= short_spec[f];
        std::vector<T> wf = inv_c2r<T>(spec);
        wf.resize(nbins, 0);
        ImpactResp<T> r;
        r.spectrum = fwd_r2c<T>(wf);
        r.waveform = wf;
        r.waveform_pad = waveform_pad;
        pir.ir.push_back(std::move(r));
    }
    pir.bywire.clear();
    for (int irel = -n_wires_half; irel <= n_wires_half; ++irel) {
        auto direct = wire_to_ind[irel];
        auto other = wire_to_ind[-irel];
        std::vector<int> idx(direct.begin(), direct.end());
        if (!other.empty())
            for (auto it = other.rbegin() + 1; it != other.rend(); ++it) idx.push_back(*it);
        pir.bywire.push_back(idx);
    }
}

// ---------------------------------------------------------------------------
// BinnedDiffusion_transform -- gen/src/BinnedDiffusion_transform.cxx.
// ---------------------------------------------------------------------------
// PlaneImpactResponse is a configured component: the reference builds it
// once (PlaneImpactResponse::configure -> build_responses) and every event
// reuses it.  The oracle keeps the built responses keyed by every input of
// the build, so repeated runs of one configuration (the timed baseline) do
// not rebuild them per event.
template <typename T>
static std::shared_ptr<const PIR<T>> cached_pir(const FRPlane& fr, double tstart, double period,
                                                const std::vector<std::vector<double>>& shorts,
                                                double overall_short_padding, double tick, int nbins,
                                                const std::vector<std::vector<double>>& longs, double long_padding)
{
    std::string key;
    auto put = [&](const void* p, size_t n) { key.append(reinterpret_cast<const char*>(p), n); };
    const double sc[6] = {tstart, period, overall_short_padding, tick, long_padding, fr.pitch};
    const int ic[3] = {fr.npaths, fr.nsamp, nbins};
    const ExtFft backend = g_ext_fft.load();  // the build's transforms are part of the key
    put(&backend, sizeof backend);
    put(sc, sizeof sc);
    put(ic, sizeof ic);
    put(fr.pitchpos, sizeof(double) * fr.npaths);
    put(fr.current, sizeof(double) * fr.npaths * (size_t)fr.nsamp);
    for (auto& v : shorts) { const size_t n = v.size(); put(&n, sizeof n); put(v.data(), sizeof(double) * n); }
    for (auto& v : longs) { const size_t n = v.size(); put(&n, sizeof n); put(v.data(), sizeof(double) * n); }
    static std::mutex mtx;
    static std::map<std::string, std::shared_ptr<const PIR<T>>> cache;
    {
        std::lock_guard<std::mutex> lk(mtx);
        auto it = cache.find(key);
        if (it != cache.end()) return it->second;
    }
    auto pir = std::make_shared<PIR<T>>();
    build_pir<T>(fr, tstart, period, shorts, overall_short_padding, tick, nbins, *pir, longs, long_padding);
    std::lock_guard<std::mutex> lk(mtx);
    if (cache.size() >= 32) cache.clear();
    cache[key] = pir;
    return pir;
}

struct Diff {
    Depo depo;
    GausDesc td, pd;
};

struct PlaneRecord {  // per (plane, input depo) bookkeeping for bit-exact checks
    int added{0}, toffset{-1}, poffset{-1}, nt{0}, np{0};
};

template <typename T>
struct BinnedDiffusion {
    const Pimpos& pimpos;
    Binning tbins;
    double nsigma;
    std::vector<Diff> diffs;
    int outside_time{0}, outside_pitch{0};
    std::mt19937* fluctuate{nullptr};
    BinnedDiffusion(const Pimpos& p, const Binning& tb, double ns) : pimpos(p), tbins(tb), nsigma(ns) {}

    // BinnedDiffusion_transform.cxx:37-92
    bool add(const Depo& depo, double sigma_time, double sigma_pitch)
    {
        const double center_time = depo.t;
        const double center_pitch = pimpos.distance(V3{depo.x, depo.y, depo.z});
        GausDesc td{center_time, sigma_time};
        {
            double nmin = td.distance(tbins.minv);
            double nmax = td.distance(tbins.maxv);
            double eff = sigma_time > 0 ? nsigma : 0;
            if (nmin > eff || nmax < -eff) { ++outside_time; return false; }
        }
        const Binning& ib = pimpos.impact;
        GausDesc pd{center_pitch, sigma_pitch};
        {
            double nmin = pd.distance(ib.minv);
            double nmax = pd.distance(ib.maxv);
            double eff = sigma_pitch > 0 ? nsigma : 0;
            if (nmin > eff || nmax < -eff) { ++outside_pitch; return false; }
        }
        diffs.push_back(Diff{depo, td, pd});
        return true;
    }

    // BinnedDiffusion_transform.cxx:227-391
    void get_charge_vec(std::vector<std::vector<std::tuple<int, int, double>>>& vvc, const std::vector<int>& vec_impact,
                        std::vector<PlaneRecord>* rec)
    {
        const Binning& ib = pimpos.impact;
        std::map<int, int> map_redimp_vec;
        std::vector<std::unordered_map<long int, int>> vmpp(vec_impact.size());
        for (size_t i = 0; i != vec_impact.size(); i++) map_redimp_vec[vec_impact[i]] = int(i);
        const Binning& rb = pimpos.region;
        std::map<int, int> map_imp_ch, map_imp_redimp;
        for (int w = 0; w != rb.nbins; w++) {
            int wimp = pimpos.wire_impact(w);
            auto rr = pimpos.wire_impacts(w);
            for (int imp = rr.first; imp != rr.second; imp++) {
                map_imp_ch[imp] = w;
                map_imp_redimp[imp] = imp - wimp;
            }
        }
        const int min_imp = 0, max_imp = ib.nbins;
        int counter = 0;
        Patch<T> patch;
        for (auto& d : diffs) {
            set_sampling<T>(d.depo, d.td, d.pd, tbins, ib, nsigma, patch, fluctuate);
            counter++;
            if (rec) {
                auto& r = (*rec)[d.depo.index];
                r.toffset = patch.toffset;
                r.poffset = patch.poffset;
                r.nt = patch.nt;
                r.np = patch.np;
            }
            const int np = patch.np, nt = patch.nt;
            for (int pbin = 0; pbin != np; pbin++) {
                int abs_pbin = pbin + patch.poffset;
                if (abs_pbin < min_imp || abs_pbin >= max_imp) continue;
                double weight = patch.qw[pbin];
                const int channel = map_imp_ch[abs_pbin];
                const int redimp = map_imp_redimp[abs_pbin];
                const int a0 = map_redimp_vec[redimp];
                const int a1 = map_redimp_vec[redimp + 1];
                auto& m0 = vmpp.at(a0);
                auto& m1 = vmpp.at(a1);
                auto& v0 = vvc.at(a0);
                auto& v1 = vvc.at(a1);
                for (int tbin = 0; tbin != nt; tbin++) {
                    int abs_tbin = tbin + patch.toffset;
                    double charge = patch.val[(size_t)pbin * nt + tbin];
                    long int key = channel * 100000 + abs_tbin;
                    auto it = m0.find(key);
                    if (it == m0.end()) {
                        m0[key] = v0.size();
                        v0.emplace_back(channel, abs_tbin, charge * weight);
                    }
                    else {
                        std::get<2>(v0.at(it->second)) += charge * weight;
                    }
                    auto it1 = m1.find(key);
                    if (it1 == m1.end()) {
                        m1[key] = v1.size();
                        v1.emplace_back(channel, abs_tbin, charge * (1 - weight));
                    }
                    else {
                        std::get<2>(v1.at(it1->second)) += charge * (1 - weight);
                    }
                }
            }
            if (counter % 5000 == 0)
                for (auto& m : vmpp) m.clear();
        }
    }

    // BinnedDiffusion_transform.cxx:416-464
    std::pair<double, double> range(bool pitch) const
    {
        int ncount = -1;
        double vmin = 0, vmax = 0;
        for (auto& d : diffs) {
            ++ncount;
            const GausDesc& g = pitch ? d.pd : d.td;
            const double lo = g.center - g.sigma * nsigma;
            const double hi = g.center + g.sigma * nsigma;
            if (!ncount) { vmin = lo; vmax = hi; continue; }
            vmin = std::min(vmin, lo);
            vmax = std::max(vmax, hi);
        }
        return {vmin, vmax};
    }
    std::pair<int, int> impact_bin_range() const
    {
        auto mm = range(true);
        const Binning& ib = pimpos.impact;
        return {std::max(ib.bin(mm.first), 0), std::min(ib.bin(mm.second) + 1, ib.nbins)};
    }
    std::pair<int, int> time_bin_range() const
    {
        auto mm = range(false);
        return {std::max(tbins.bin(mm.first), 0), std::min(tbins.bin(mm.second) + 1, tbins.nbins)};
    }
};

// ---------------------------------------------------------------------------
// ImpactTransform -- gen/src/ImpactTransform.cxx:19-347.
// ---------------------------------------------------------------------------
struct Window {
    int start_ch, end_ch, start_tick, end_tick, nw, nt;
};

template <typename T>
struct ImpactTransform {
    using C = std::complex<T>;
    Window win{};
    std::vector<T> decon;  // [nw][nt]

    // Time-domain response reduced to nt samples, then r2c (ImpactTransform.cxx:158-168).
    static std::vector<C> reduced_spectrum(const ImpactResp<T>& r, int nt)
    {
        std::vector<T> t = inv_c2r<T>(r.spectrum);
        std::vector<T> red(nt, 0);
        for (int i = 0; i < nt; ++i) {
            if (i >= (int)t.size()) break;
            red[i] = t[i];
        }
        return fwd_r2c<T>(red);
    }

    const PIR<T>* m_pir{nullptr};
    mutable int long_n{0};
    mutable std::vector<C> long_spec;  // spectrum of the long waveform at long_n

    // st: optional stage clocks (kNStages seconds, added to)
    ImpactTransform(const PIR<T>& pir, BinnedDiffusion<T>& bd, std::vector<PlaneRecord>* rec, double* st = nullptr)
        : m_pir(&pir)
    {
        double t_mark = now_s();
        auto lap = [&](int k) {
            const double t = now_s();
            if (st) st[k] += t - t_mark;
            t_mark = t;
        };
        const int G = std::round(pir.pitch / pir.impact) + 1;
        const int npad = std::round((pir.nwires() - 1) / 2.);
        std::vector<int> vec_impact;
        std::vector<std::map<int, int>> vmr;  // group -> {wire offset -> ir index}
        for (int i = 0; i != G; i++) {
            double rel;
            if (i != G - 1) rel = -pir.pitch / 2. + pir.impact * i + 1e-9;
            else rel = -pir.pitch / 2. + pir.impact * i - 1e-9;
            vec_impact.push_back(std::round(rel / pir.impact));
            std::map<int, int> mr;
            for (int j = 0; j != pir.nwires(); j++) {
                int k = pir.closest(rel - (j - npad) * pir.pitch);
                if (k < 0) continue;
                mr[j - npad] = k;
            }
            vmr.push_back(mr);
        }
        std::vector<std::vector<std::tuple<int, int, double>>> vvc(G);
        lap(kStRespPrep);
        bd.get_charge_vec(vvc, vec_impact, rec);
        lap(kStRaster);

        auto ir = bd.impact_bin_range();
        auto tr = bd.time_bin_range();
        int start_ch = std::floor(ir.first * 1.0 / (G - 1)) - 1;
        int end_ch = std::ceil(ir.second * 1.0 / (G - 1)) + 2;
        if ((end_ch - start_ch) % 2 == 1) end_ch += 1;
        int start_tick = tr.first - 1;
        int end_tick = tr.second + 2;
        if ((end_tick - start_tick) % 2 == 1) end_tick += 1;
        const size_t ntotal_wires = fft_best_length(end_ch - start_ch + 2 * npad, true);
        int npad_wire = (ntotal_wires - end_ch + start_ch) / 2;
        win.start_ch = start_ch - npad_wire;
        win.end_ch = end_ch + npad_wire;
        int npad_time = pir.ir[pir.closest(0)].waveform_pad;
        const size_t ntotal_ticks = fft_best_length(end_tick - start_tick + npad_time, false);
        npad_time = ntotal_ticks - end_tick + start_tick;
        win.start_tick = start_tick;
        win.end_tick = end_tick + npad_time;
        const int NW = end_ch - start_ch + 2 * npad_wire;
        const int NT = win.end_tick - win.start_tick;
        win.nw = NW;
        win.nt = NT;
        std::vector<C> acc((size_t)NW * NT, C(0, 0));
        auto at = [&](std::vector<C>& a, int r, int c) -> C& { return a[(size_t)r * NT + c]; };

        auto build_resp = [&](int i) {
            std::vector<C> resp((size_t)NW * NT, C(0, 0));
            auto& mr = vmr.at(i);
            auto row = [&](int rr, int woff) {
                auto rs = reduced_spectrum(pir.ir.at(mr.at(woff)), NT);
                for (int c = 0; c < NT; ++c) resp[(size_t)rr * NT + c] = rs[c];
            };
            row(0, 0);
            for (int irow = 0; irow != npad; irow++) {
                row(irow + 1, irow + 1);
                row(end_ch - start_ch - 1 - irow + 2 * npad_wire, -irow - 1);
            }
            Dft<T>::fwd1b(resp.data(), NW, NT, 0);
            return resp;
        };

        const int num_double = (G - 1) / 2;
        for (int i = 0; i != num_double; i++) {
            std::vector<C> c((size_t)NW * NT, C(0, 0));
            for (auto& e : vvc.at(i))
                at(c, std::get<0>(e) + npad_wire - start_ch, std::get<1>(e) - win.start_tick) += (T)std::get<2>(e);
            vvc.at(i).clear();
            int ii = num_double * 2 - i;
            for (auto& e : vvc.at(ii))
                at(c, end_ch + npad_wire - 1 - std::get<0>(e), std::get<1>(e) - win.start_tick) +=
                    C(0, (T)std::get<2>(e));
            vvc.at(ii).clear();
            Dft<T>::fwd2d(c.data(), NW, NT);
            lap(kStFftConv);
            auto resp = build_resp(i);
            lap(kStRespPrep);
            for (size_t k = 0; k < c.size(); ++k) c[k] *= resp[k];
            Dft<T>::inv1b(c.data(), NW, NT, 0);
            for (size_t k = 0; k < c.size(); ++k) acc[k] += c[k];
        }
        {
            int i = num_double;
            std::vector<T> dtw((size_t)NW * NT, 0);
            for (auto& e : vvc.at(i)) {
                T& v = dtw[(size_t)(std::get<0>(e) + npad_wire - start_ch) * NT + (std::get<1>(e) - win.start_tick)];
                v = (T)(v + std::get<2>(e));
            }
            vvc.at(i).clear();
            std::vector<C> d((size_t)NW * NT);
            for (size_t k = 0; k < d.size(); ++k) d[k] = C(dtw[k], 0);
            Dft<T>::fwd1b(d.data(), NW, NT, 1);
            Dft<T>::fwd1b(d.data(), NW, NT, 0);
            lap(kStFftConv);
            auto resp = build_resp(i);
            lap(kStRespPrep);
            for (size_t k = 0; k < d.size(); ++k) d[k] *= resp[k];
            Dft<T>::inv1b(d.data(), NW, NT, 0);
            for (size_t k = 0; k < d.size(); ++k) acc[k] += d[k];
        }
        Dft<T>::inv1b(acc.data(), NW, NT, 1);
        decon.assign((size_t)NW * NT, 0);
        for (int r = 0; r < NW; ++r)
            for (int c2 = 0; c2 < NT; ++c2)
                decon[(size_t)r * NT + c2] = std::real(acc[(size_t)r * NT + c2]) +
                                             std::imag(acc[(size_t)(NW - 1 - r) * NT + c2]);
        lap(kStFftConv);
    }

    // ImpactTransform::waveform, ImpactTransform.cxx:312-347, with the
    // long-range step (:327-343) when the PIR has a long response.
    void waveform(int iwire, int nsamples, T* out) const
    {
        std::fill(out, out + nsamples, (T)0);
        if (iwire < win.start_ch || iwire >= win.end_ch) return;
        for (int i = 0; i != nsamples; i++)
            if (i >= win.start_tick && i < win.end_tick)
                out[i] = decon[(size_t)(iwire - win.start_ch) * win.nt + (i - win.start_tick)];
        if (m_pir && !m_pir->long_wf.empty()) {
            const int nlength = (int)fft_best_length((size_t)nsamples + m_pir->long_pad, false);
            if (long_n != nlength) {
                std::vector<T> lr(m_pir->long_wf.begin(), m_pir->long_wf.end());
                lr.resize(nlength, 0);
                long_spec = fwd_r2c<T>(lr);
                long_n = nlength;
            }
            std::vector<T> wf(out, out + nsamples);
            wf.resize(nlength, 0);
            auto spec = fwd_r2c<T>(wf);
            for (int i = 0; i < nlength; ++i) spec[i] *= long_spec[i];
            wf = inv_c2r<T>(spec);
            for (int i = 0; i < nsamples; ++i) out[i] = wf[i];
        }
    }
};

}  // namespace orc

// ============================================================================
// C interface for the Python test harness (ctypes).
// ============================================================================
extern "C" {

struct OrcPlane {
    int nwires;
    int nimp;
    double pitchmin, pitchmax;
    double wire[3], pitch[3], origin[3];
    // field response of this plane (Response::Schema::PlaneResponse)
    int npaths, nfr;
    const double* pitchpos;  // [npaths]
    const double* current;   // [npaths][nfr]
    double fr_pitch;
};

struct OrcJob {
    // DepoTransform configuration (gen/src/DepoTransform.cxx:76-153)
    double start_time, readout_time, tick, drift_speed, nsigma;
    // Drifter configuration (gen/src/Drifter.cxx:94-123); drift=0 means the depos are already drifted.
    int drift;
    double DL, DT, lifetime, drifter_speed, toffset;
    int nxregions;
    const double* xregions;  // [n][3] anode, response, cathode
    // face sensitive volume (two corners); have_bb=0 means no cut
    int have_bb;
    double bb_lo[3], bb_hi[3];
    // PlaneImpactResponse configuration (gen/src/PlaneImpactResponse.cxx:35-87)
    double fr_tstart, fr_period;
    int nshort;
    const int* short_len;
    const double* short_wave;  // concatenated
    double overall_short_padding;
    int pir_nticks;
    int nplanes;
    const OrcPlane* planes;
    int ndepos;
    const double* depos;  // [n][7] t, q, x, y, z, extent_long, extent_tran
    int fp64;
    int nthreads;
    // fluctuation (reference distribution): DepoTransform "fluctuate" and the
    // Drifter's, drawn with std::mt19937 and std::binomial_distribution as
    // gen/src/Random.cxx does; seed of the streams (one per plane, one for the drift)
    int fluctuate;
    int drift_fluctuate;
    unsigned long long seed;
    // PlaneImpactResponse "long_responses" (concatenated) and "long_padding"
    int nlong;
    const int* long_len;
    const double* long_wave;
    double long_padding;
    // optional: seconds per stage of orc_run (kNStages: drift + sensitive cut,
    // rasterise + scatter, response prep, FFT convolution, extraction, PIR
    // build), summed over planes; null: not timed
    double* stage_s;
    // several anode faces (DepoTransform.cxx:169-213 loops over
    // IAnodePlane::faces()): nfaces > 0 gives each face's sensitive box
    // (face_bb [nfaces][lo xyz, hi xyz], face_have_bb 0: no cut) and each
    // plane's face (plane_face [nplanes], planes of a face consecutive);
    // nfaces = 0: one face with the box above
    int nfaces;
    const double* face_bb;
    const int* face_have_bb;
    const int* plane_face;
    // modify_depo (gen/inc/WireCellGen/DepoTransform.h:33-35, called before
    // BinnedDiffusion_transform::add at DepoTransform.cxx:182) as a charge
    // scale: depo i brings charge * charge_scale[i][plane] to the plane
    // ([ndepos][nplanes]); null: unmodified
    const double* charge_scale;
};

// The external transform of the timed CPU baseline (null: the oracle's own).
void orc_set_fft_backend(orc::ExtFft f) { orc::g_ext_fft.store(f); }

static std::vector<std::vector<double>> job_longs(const OrcJob* job)
{
    std::vector<std::vector<double>> longs;
    size_t off = 0;
    for (int s = 0; s < job->nlong; ++s) {
        longs.emplace_back(job->long_wave + off, job->long_wave + off + job->long_len[s]);
        off += job->long_len[s];
    }
    return longs;
}

struct OrcPlaneOut {
    int start_ch, end_ch, start_tick, end_tick, nw, nt;
    int ndepos_added, outside_time, outside_pitch;
};

int orc_fft_best_length(long n, int keep) { return (int)orc::fft_best_length((size_t)n, keep != 0); }

// Binomial draws of the reference's generator (gen/src/Random.cxx:55-58 with
// the "twister" engine): std::binomial_distribution<int> over std::mt19937.
void orc_binomial_samples(unsigned long long seed, int n, double p, long count, int* out)
{
    std::mt19937 g((std::uint32_t)seed);
    for (long i = 0; i < count; ++i) {
        std::binomial_distribution<int> bin(n, p);
        out[i] = bin(g);
    }
}

int orc_binning_bin(int nbins, double lo, double hi, double v) { return orc::Binning(nbins, lo, hi).bin(v); }

void orc_sample_bin_range(int nbins, double lo, double hi, double a, double b, int* out)
{
    auto r = orc::Binning(nbins, lo, hi).sample_bin_range(a, b);
    out[0] = r.first;
    out[1] = r.second;
}

// 1-D complex transforms for tests: data is interleaved re,im.
void orc_fft_f32(float* data, int n, int inverse)
{
    auto* c = reinterpret_cast<std::complex<float>*>(data);
    if (inverse) orc::Dft<float>::inv1d(c, n);
    else orc::Dft<float>::fwd1d(c, n);
}
void orc_fft_f64(double* data, int n, int inverse)
{
    auto* c = reinterpret_cast<std::complex<double>*>(data);
    if (inverse) orc::Dft<double>::inv1d(c, n);
    else orc::Dft<double>::fwd1d(c, n);
}

// One GaussianDiffusion::set_sampling for tests. out_i: toffset, poffset, nt, np.
// patch receives np*nt values (caller provides capacity cap), weights np values.
int orc_set_sampling(double t, double q, double pitch_center, double sigma_t, double sigma_p, int ntbins, double tmin,
                     double tmax, int nibins, double imin, double imax, double nsigma, int fp64, int cap,
                     double* patch, double* weights, int* out_i)
{
    orc::Depo d{t, q, 0, 0, 0, 0, 0, 0};
    orc::GausDesc td{t, sigma_t}, pd{pitch_center, sigma_p};
    orc::Binning tb(ntbins, tmin, tmax), pb(nibins, imin, imax);
    auto emit = [&](auto& P) {
        out_i[0] = P.toffset;
        out_i[1] = P.poffset;
        out_i[2] = P.nt;
        out_i[3] = P.np;
        if ((long)P.nt * P.np > cap) return -1;
        for (size_t i = 0; i < P.val.size(); ++i) patch[i] = P.val[i];
        for (int i = 0; i < P.np; ++i) weights[i] = P.qw[i];
        return 0;
    };
    if (fp64) {
        orc::Patch<double> P;
        orc::set_sampling<double>(d, td, pd, tb, pb, nsigma, P);
        return emit(P);
    }
    orc::Patch<float> P;
    orc::set_sampling<float>(d, td, pd, tb, pb, nsigma, P);
    return emit(P);
}

// Drifter::insert + flush for tests: returns the number of output depos
// (time ordered); out has room for n*8 doubles (7 fields + input index).
int orc_drift(const OrcJob* job, double* out)
{
    orc::DriftParams dp{job->DL, job->DT, job->lifetime, job->drifter_speed, job->toffset, {}};
    for (int i = 0; i < job->nxregions; ++i)
        dp.xregions.push_back({job->xregions[3 * i], job->xregions[3 * i + 1], job->xregions[3 * i + 2]});
    std::vector<orc::Depo> in;
    for (int i = 0; i < job->ndepos; ++i) {
        const double* p = job->depos + 7 * (size_t)i;
        in.push_back({p[0], p[1], p[2], p[3], p[4], p[5], p[6], i});
    }
    auto o = orc::drift_all(dp, in);
    for (size_t i = 0; i < o.size(); ++i) {
        double* q = out + 8 * i;
        q[0] = o[i].t; q[1] = o[i].q; q[2] = o[i].x; q[3] = o[i].y; q[4] = o[i].z;
        q[5] = o[i].el; q[6] = o[i].et; q[7] = o[i].index;
    }
    return (int)o.size();
}

// PIR build for tests: fills waveforms [npaths][pir_nticks] (as double),
// bywire [nwires][nimp] indices; returns nwires*1000+nimp, or -1 on error.
int orc_pir_build(const OrcJob* job, int iplane, double* waveforms, int* bywire, double* pitch_impact_extent)
{
    auto run = [&](auto tag) -> int {
        using T = decltype(tag);
        const OrcPlane& pl = job->planes[iplane];
        std::vector<std::vector<double>> shorts;
        size_t off = 0;
        for (int s = 0; s < job->nshort; ++s) {
            shorts.emplace_back(job->short_wave + off, job->short_wave + off + job->short_len[s]);
            off += job->short_len[s];
        }
        orc::FRPlane fr{pl.npaths, pl.nfr, pl.pitchpos, pl.current, pl.fr_pitch};
        orc::PIR<T> pir;
        orc::build_pir<T>(fr, job->fr_tstart, job->fr_period, shorts, job->overall_short_padding, job->tick,
                          job->pir_nticks, pir, job_longs(job), job->long_padding);
        for (size_t p = 0; p < pir.ir.size(); ++p)
            for (int k = 0; k < job->pir_nticks; ++k)
                waveforms[p * job->pir_nticks + k] = pir.ir[p].waveform[k];
        const int nw = pir.nwires(), ni = pir.nimp_per_wire();
        for (int w = 0; w < nw; ++w)
            for (int k = 0; k < ni; ++k)
                bywire[w * ni + k] = k < (int)pir.bywire[w].size() ? pir.bywire[w][k] : -1;
        pitch_impact_extent[0] = pir.pitch;
        pitch_impact_extent[1] = pir.impact;
        pitch_impact_extent[2] = pir.half_extent;
        return nw * 1000 + ni;
    };
    try {
        return job->fp64 ? run(double{}) : run(float{});
    }
    catch (...) {
        return -1;
    }
}

// The whole DepoTransform::operator() (gen/src/DepoTransform.cxx:155-224) for
// one face: optional drift, sensitive cut, then per plane BinnedDiffusion +
// ImpactTransform + waveform extraction.
//   frame : [sum_p nwires_p][nticks] dense waveforms (float or double per fp64)
//   pout  : per-plane window and counters
//   rec   : optional [nplanes][ndepos][5] ints (added, toffset, poffset, nt, np)
//           indexed by the depo's position in the input array
// Returns 0 on success.
int orc_run(const OrcJob* job, void* frame, OrcPlaneOut* pout, int* rec)
{
    try {
        std::mutex st_mtx;
        double t_drift = orc::now_s();
        std::vector<orc::Depo> depos;
        for (int i = 0; i < job->ndepos; ++i) {
            const double* p = job->depos + 7 * (size_t)i;
            depos.push_back({p[0], p[1], p[2], p[3], p[4], p[5], p[6], i});
        }
        if (job->drift) {
            orc::DriftParams dp{job->DL, job->DT, job->lifetime, job->drifter_speed, job->toffset, {}};
            for (int i = 0; i < job->nxregions; ++i)
                dp.xregions.push_back({job->xregions[3 * i], job->xregions[3 * i + 1], job->xregions[3 * i + 2]});
            std::mt19937 drng((std::uint32_t)(job->seed * 2654435761ull + 977));
            if (job->drift_fluctuate) dp.rng = &drng;
            depos = orc::drift_all(dp, depos);  // keeps each depo's input index
        }
        // each face's sensitive volume: DepoTools.cxx:110-123
        const int nfaces = job->nfaces > 0 ? job->nfaces : 1;
        std::vector<std::vector<orc::Depo>> faces(nfaces);
        for (int f = 0; f < nfaces; ++f) {
            const bool have = job->nfaces > 0 ? job->face_have_bb[f] != 0 : job->have_bb != 0;
            const double* lo = job->nfaces > 0 ? job->face_bb + 6 * f : job->bb_lo;
            const double* hi = job->nfaces > 0 ? job->face_bb + 6 * f + 3 : job->bb_hi;
            for (auto& d : depos)
                if (!have || orc::bb_inside(lo, hi, d)) faces[f].push_back(d);
        }
        for (int ip = 0; ip < job->nplanes; ++ip)
            if (job->nfaces > 0 && (job->plane_face[ip] < 0 || job->plane_face[ip] >= nfaces)) return -1;
        if (job->stage_s) job->stage_s[orc::kStDrift] += orc::now_s() - t_drift;

        const int nticks = (int)(job->readout_time / job->tick);
        std::vector<std::vector<double>> shorts;
        size_t off = 0;
        for (int s = 0; s < job->nshort; ++s) {
            shorts.emplace_back(job->short_wave + off, job->short_wave + off + job->short_len[s]);
            off += job->short_len[s];
        }
        std::vector<size_t> row0(job->nplanes + 1, 0);
        for (int p = 0; p < job->nplanes; ++p) row0[p + 1] = row0[p] + job->planes[p].nwires;
        const size_t ndep_rec = (size_t)job->ndepos;

        const std::vector<std::vector<double>> longs = job_longs(job);
        auto do_plane = [&](int ip, auto tag) {
            using T = decltype(tag);
            const OrcPlane& pl = job->planes[ip];
            orc::Pimpos pim(pl.nwires, pl.pitchmin, pl.pitchmax, orc::V3{pl.wire[0], pl.wire[1], pl.wire[2]},
                            orc::V3{pl.pitch[0], pl.pitch[1], pl.pitch[2]},
                            orc::V3{pl.origin[0], pl.origin[1], pl.origin[2]}, pl.nimp);
            double st[orc::kNStages] = {0, 0, 0, 0, 0, 0};
            double t0 = orc::now_s();
            orc::FRPlane fr{pl.npaths, pl.nfr, pl.pitchpos, pl.current, pl.fr_pitch};
            const auto pir_ptr = orc::cached_pir<T>(fr, job->fr_tstart, job->fr_period, shorts,
                                                    job->overall_short_padding, job->tick, job->pir_nticks, longs,
                                                    job->long_padding);
            const orc::PIR<T>& pir = *pir_ptr;
            st[orc::kStPir] += orc::now_s() - t0;
            t0 = orc::now_s();
            orc::Binning tbins(job->readout_time / job->tick, job->start_time, job->start_time + job->readout_time);
            orc::BinnedDiffusion<T> bd(pim, tbins, job->nsigma);
            std::mt19937 prng((std::uint32_t)(job->seed * 2654435761ull + 31 * (unsigned long long)ip + 1));
            if (job->fluctuate) bd.fluctuate = &prng;
            std::vector<orc::PlaneRecord> precs(ndep_rec);
            const std::vector<orc::Depo>& face = faces[job->nfaces > 0 ? job->plane_face[ip] : 0];
            for (const auto& d0 : face) {
                orc::Depo d = d0;
                if (job->charge_scale) d.q = d.q * job->charge_scale[(size_t)d.index * job->nplanes + ip];
                bool ok = bd.add(d, d.el / job->drift_speed, d.et);
                precs[d.index].added = ok ? 1 : 0;
            }
            st[orc::kStRaster] += orc::now_s() - t0;
            orc::ImpactTransform<T> it(pir, bd, &precs, st);
            OrcPlaneOut& po = pout[ip];
            po.start_ch = it.win.start_ch;
            po.end_ch = it.win.end_ch;
            po.start_tick = it.win.start_tick;
            po.end_tick = it.win.end_tick;
            po.nw = it.win.nw;
            po.nt = it.win.nt;
            po.ndepos_added = (int)bd.diffs.size();
            po.outside_time = bd.outside_time;
            po.outside_pitch = bd.outside_pitch;
            T* fr_out = reinterpret_cast<T*>(frame) + row0[ip] * (size_t)nticks;
            t0 = orc::now_s();
            for (int w = 0; w < pl.nwires; ++w) it.waveform(w, nticks, fr_out + (size_t)w * nticks);
            st[orc::kStExtract] += orc::now_s() - t0;
            if (job->stage_s) {
                std::lock_guard<std::mutex> lk(st_mtx);
                for (int k = 0; k < orc::kNStages; ++k) job->stage_s[k] += st[k];
            }
            if (rec) {
                for (size_t k = 0; k < ndep_rec; ++k) {
                    int* r = rec + ((size_t)ip * ndep_rec + k) * 5;
                    r[0] = precs[k].added;
                    r[1] = precs[k].toffset;
                    r[2] = precs[k].poffset;
                    r[3] = precs[k].nt;
                    r[4] = precs[k].np;
                }
            }
        };
        std::atomic<int> err{0};
        auto worker = [&](int ip) {
            try {
                if (job->fp64) do_plane(ip, double{});
                else do_plane(ip, float{});
            }
            catch (...) {
                err = 1;
            }
        };
        const int nth = std::max(1, std::min(job->nthreads, job->nplanes));
        if (nth == 1) {
            for (int ip = 0; ip < job->nplanes; ++ip) worker(ip);
        }
        else {
            std::vector<std::thread> th;
            std::atomic<int> next{0};
            for (int t = 0; t < nth; ++t)
                th.emplace_back([&]() {
                    for (int ip = next++; ip < job->nplanes; ip = next++) worker(ip);
                });
            for (auto& t : th) t.join();
        }
        return err ? -2 : 0;
    }
    catch (...) {
        return -1;
    }
}

// Waveform::edge (util/src/Waveform.cxx:136-153) over a float row.
// DepoFluxSplat (gen/src/DepoFluxSplat.cxx:81-135 configuration,
// :247-390 operator()): for each depo in the face (DepoTools sensitive
// cut here) and each plane in order, a GaussianDiffusion with time
// t + response_plane / drift_speed, time sigma extent_long (smeared by
// smear_long ticks) / speed and pitch sigma extent_tran (smeared by
// smear_tran wire pitches), sampled on the window's tick binning and the
// plane's wire (region) binning; a depo whose time span misses the window
// skips the plane, one whose pitch span misses the wire plane skips the
// remaining planes (the reference's `break`).  |patch| is added at
// tick (int)(toffset + time_offset / tick) + k.  Dense accumulation in
// double; frame [sum of nwires][nbins], nbins = (int)(window_duration / tick).
struct OrcSplat {
    double tick, window_start, window_duration, nsigma, drift_speed, response_plane;
    double time_offsets[3], smear_long[3], smear_tran[3];
};

}  // extern "C"

// The splat with its cells summed in A: double (as the device sums them) or
// float in depo order (as the reference's dense accumulator sums its float
// trace charges).
template <typename A>
static int splat_impl(const OrcJob* job, const OrcSplat* sp, A* frame)
{
    try {
        const int nbins = (int)(sp->window_duration / sp->tick);
        orc::Binning tb(nbins, sp->window_start, sp->window_start + nbins * sp->tick);
        std::vector<size_t> row0(job->nplanes + 1, 0);
        for (int p = 0; p < job->nplanes; ++p) row0[p + 1] = row0[p] + job->planes[p].nwires;
        std::fill(frame, frame + row0[job->nplanes] * (size_t)nbins, (A)0);
        for (int i = 0; i < job->ndepos; ++i) {
            const double* q = job->depos + 7 * (size_t)i;
            orc::Depo d{q[0], q[1], q[2], q[3], q[4], q[5], q[6], i};
            if (job->have_bb && !orc::bb_inside(job->bb_lo, job->bb_hi, d)) continue;
            const double nominal = d.t + sp->response_plane / sp->drift_speed;
            for (int ip = 0; ip < job->nplanes && ip < 3; ++ip) {
                const OrcPlane& pl = job->planes[ip];
                double sigma_L = d.el;
                if (sp->smear_long[ip] > 0) {
                    const double extra = sp->smear_long[ip] * tb.binsize * sp->drift_speed;
                    sigma_L = std::sqrt(sigma_L * sigma_L + extra * extra);
                }
                orc::GausDesc td{nominal, sigma_L / sp->drift_speed};
                const double eff_t = d.el > 0 ? sp->nsigma : 0;
                if (td.distance(tb.minv) > eff_t || td.distance(tb.maxv) < -eff_t) continue;
                orc::Pimpos pim(pl.nwires, pl.pitchmin, pl.pitchmax, orc::V3{pl.wire[0], pl.wire[1], pl.wire[2]},
                                orc::V3{pl.pitch[0], pl.pitch[1], pl.pitch[2]},
                                orc::V3{pl.origin[0], pl.origin[1], pl.origin[2]}, pl.nimp);
                const orc::Binning& wb = pim.region;
                double sigma_T = d.et;
                if (sp->smear_tran[ip] > 0) {
                    const double extra = sp->smear_tran[ip] * wb.binsize;
                    sigma_T = std::sqrt(sigma_T * sigma_T + extra * extra);
                }
                orc::GausDesc pd{pim.distance(orc::V3{d.x, d.y, d.z}), sigma_T};
                const double eff_p = d.et > 0 ? sp->nsigma : 0;
                if (pd.distance(wb.minv) > eff_p || pd.distance(wb.maxv) < -eff_p) break;
                orc::Patch<float> patch;
                orc::set_sampling(d, td, pd, tb, wb, sp->nsigma, patch);
                if (!patch.np || !patch.nt) continue;
                const int tstart = (int)(patch.toffset + sp->time_offsets[ip] / sp->tick);
                for (int a = 0; a < patch.np; ++a) {
                    const int pbin = patch.poffset + a;
                    if (pbin < 0 || pbin >= pl.nwires) continue;
                    for (int k = 0; k < patch.nt; ++k) {
                        const int tick = tstart + k;
                        if (tick < 0 || tick >= nbins) continue;
                        frame[(row0[ip] + pbin) * (size_t)nbins + tick] +=
                            (A)std::abs(patch.val[(size_t)a * patch.nt + k]);
                    }
                }
            }
        }
        return 0;
    }
    catch (...) {
        return -1;
    }
}

extern "C" {

int orc_splat(const OrcJob* job, const OrcSplat* sp, double* frame) { return splat_impl(job, sp, frame); }
int orc_splat_float(const OrcJob* job, const OrcSplat* sp, float* frame) { return splat_impl(job, sp, frame); }

void orc_edge(const float* wave, int size, int* out)
{
    int imin = size, imax = size;
    for (int ind = 0; ind < size; ++ind) {
        if (wave[ind] != 0.0f) {
            if (imin == size) imin = ind;
            if (imin < size) imax = ind + 1;
        }
    }
    out[0] = imin;
    out[1] = imax;
}

// GausDesc::binint / weight / distance of the restatement, for the pins
// against the reference-compiled functions.  Return the result length; out
// holds max(nbins, 1) values.
int orc_gd_binint(double center, double sigma, double start, double step, int nbins, double* out)
{
    auto v = orc::GausDesc{center, sigma}.binint(start, step, nbins);
    for (size_t i = 0; i < v.size(); ++i) out[i] = v[i];
    return (int)v.size();
}
int orc_gd_weight(double center, double sigma, double start, double step, int nbins, const double* pvec,
                  double* out)
{
    std::vector<double> p(pvec, pvec + nbins);
    auto v = orc::GausDesc{center, sigma}.weight(start, step, nbins, p);
    for (size_t i = 0; i < v.size(); ++i) out[i] = v[i];
    return (int)v.size();
}
double orc_gd_distance(double center, double sigma, double x) { return orc::GausDesc{center, sigma}.distance(x); }

// The restatement's Pimpos, laid out as the reference harness's ref_pimpos:
// out = {region nbins, min, max, impact nbins, min, max, axis0..2}; dist [n]
// = pitch coordinate of pts [n][3].
void orc_pimpos(int nwires, double minp, double maxp, const double* wire, const double* pitch, const double* origin,
                int nbins, int n, const double* pts, double* out, double* dist)
{
    orc::Pimpos p(nwires, minp, maxp, orc::V3{wire[0], wire[1], wire[2]}, orc::V3{pitch[0], pitch[1], pitch[2]},
                  orc::V3{origin[0], origin[1], origin[2]}, nbins);
    const double head[6] = {(double)p.region.nbins, p.region.minv, p.region.maxv,
                            (double)p.impact.nbins, p.impact.minv, p.impact.maxv};
    for (int k = 0; k < 6; ++k) out[k] = head[k];
    for (int a = 0; a < 3; ++a) {
        out[6 + 3 * a] = p.axis[a].x;
        out[7 + 3 * a] = p.axis[a].y;
        out[8 + 3 * a] = p.axis[a].z;
    }
    for (int j = 0; j < n; ++j) dist[j] = p.distance(orc::V3{pts[3 * j], pts[3 * j + 1], pts[3 * j + 2]});
}

// Drifter::insert of one depo, fluctuation off (the restatement's drift_one):
// xr [nxr][3] (anode, response, cathode), depo and out (t, q, x, y, z,
// extent_long, extent_tran).  Returns 1 and the drifted depo when kept, else 0.
int orc_drift_one(const double* xr, int nxr, double DL, double DT, double lifetime, double speed, double toffset,
                  const double* depo, double* out)
{
    orc::DriftParams dp{DL, DT, lifetime, speed, toffset, {}};
    for (int k = 0; k < nxr; ++k) dp.xregions.push_back({xr[3 * k], xr[3 * k + 1], xr[3 * k + 2]});
    orc::Depo in{depo[0], depo[1], depo[2], depo[3], depo[4], depo[5], depo[6], 0}, o{};
    if (!orc::drift_one(dp, in, o)) return 0;
    const double v[7] = {o.t, o.q, o.x, o.y, o.z, o.el, o.et};
    for (int k = 0; k < 7; ++k) out[k] = v[k];
    return 1;
}

// BinnedDiffusion_transform::add of one depo (the restatement's
// BinnedDiffusion::add) on a plane given by its Pimpos arguments and the
// readout binning; counters[0..1] get outside_time and outside_pitch.
int orc_bdt_add(int nwires, double minp, double maxp, const double* wire, const double* pitch, const double* origin,
                int nimp, int ntbins, double tmin, double tmax, double nsigma, const double* depo, double sigma_time,
                double sigma_pitch, int* counters)
{
    orc::Pimpos pim(nwires, minp, maxp, orc::V3{wire[0], wire[1], wire[2]}, orc::V3{pitch[0], pitch[1], pitch[2]},
                    orc::V3{origin[0], origin[1], origin[2]}, nimp);
    orc::Binning tb(ntbins, tmin, tmax);
    orc::BinnedDiffusion<double> bd(pim, tb, nsigma);
    orc::Depo d{depo[0], depo[1], depo[2], depo[3], depo[4], depo[5], depo[6], 0};
    const bool ok = bd.add(d, sigma_time, sigma_pitch);
    counters[0] = bd.outside_time;
    counters[1] = bd.outside_pitch;
    return ok ? 1 : 0;
}

}  // extern "C"
