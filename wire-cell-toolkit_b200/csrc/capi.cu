// Host side of the DepoTransform component and the C ABI (include/wctb200.h).
//
// DepoTransformCore mirrors Gen::DepoTransform (gen/src/DepoTransform.cxx):
// configure() takes the same JSON keys, forward() is operator(), and the
// per-plane window arithmetic is ImpactTransform's (gen/src/ImpactTransform.cxx:83-115).

#include <cuda_runtime.h>

#include <algorithm>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/wctb200.h"
#include "json.hpp"
#include "kernels.cuh"
#include "pir.hpp"

namespace wctb200 {

static thread_local char g_last_error[512];

static int fail(int code, const char* msg)
{
    std::strncpy(g_last_error, msg, sizeof(g_last_error) - 1);
    g_last_error[sizeof(g_last_error) - 1] = '\0';
    return code;
}
static int fail(int code, const std::string& msg) { return fail(code, msg.c_str()); }

#define CUDA_TRY(expr)                                                                                   \
    do {                                                                                                 \
        cudaError_t _e = (expr);                                                                         \
        if (_e != cudaSuccess)                                                                           \
            return fail(WCT_ERR_CUDA, std::string(#expr ": ") + cudaGetErrorString(_e));                \
    } while (0)

// ---------------------------------------------------------------------------
// Device buffer that only grows.
// ---------------------------------------------------------------------------
struct DevBuf {
    void* p{nullptr};
    size_t n{0};
    ~DevBuf() { release(); }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    cudaError_t ensure(size_t bytes)
    {
        if (bytes <= n) return cudaSuccess;
        release();
        size_t b = std::max<size_t>(bytes, 256);
        cudaError_t e = cudaMalloc(&p, b);
        if (e == cudaSuccess) n = b;
        return e;
    }
    template <typename T>
    T* as() const { return reinterpret_cast<T*>(p); }
};

// ---------------------------------------------------------------------------
// FFT plans: radices and twiddle tables per complex length M.
// ---------------------------------------------------------------------------
struct FftPlanDev {
    FftDesc desc{};
    DevBuf tw, twh;
};

// Radix schedule for M (no heap use); false if M has a prime factor above 7
// or needs more than kFftMaxStages stages.
static bool fft_radices(int M, int* r, int& nst)
{
    nst = 0;
    if (M < 1) return false;
    int m = M;
    auto push = [&](int f) {
        if (nst >= kFftMaxStages) return false;
        r[nst++] = f;
        m /= f;
        return true;
    };
    while (m % 8 == 0) if (!push(8)) return false;
    if (m % 4 == 0 && !push(4)) return false;
    if (m % 2 == 0 && !push(2)) return false;
    for (int f : {7, 5, 3})
        while (m % f == 0) if (!push(f)) return false;
    return m == 1;
}
static bool fft_supported(int M)
{
    int r[kFftMaxStages], n = 0;
    return fft_radices(M, r, n);
}

// Smallest N >= n, N a multiple of 4, whose half has only the factors 2, 3, 5, 7
// (the reference's own length whenever it qualifies).
static int gpu_fft_length(int n)
{
    int N = (n + 3) & ~3;
    while (!fft_supported(N / 2)) N += 4;
    return N;
}

static int make_plan(int M, FftPlanDev& p)
{
    int nst = 0;
    if (!fft_radices(M, p.desc.radix, nst)) return fail(WCT_ERR_SIZE, "FFT length has a prime factor above 7");
    p.desc.M = M;
    p.desc.nst = nst;
    std::vector<float2> tw(M), twh(M);
    const double twopi = 6.283185307179586476925286766559;
    for (int m = 0; m < M; ++m) {
        const double a = -twopi * (double)m / (double)M;
        tw[m] = make_float2((float)std::cos(a), (float)std::sin(a));
        const double b = -twopi * (double)m / (2.0 * (double)M);
        twh[m] = make_float2((float)std::cos(b), (float)std::sin(b));
    }
    CUDA_TRY(p.tw.ensure(sizeof(float2) * M));
    CUDA_TRY(p.twh.ensure(sizeof(float2) * M));
    CUDA_TRY(cudaMemcpy(p.tw.p, tw.data(), sizeof(float2) * M, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(p.twh.p, twh.data(), sizeof(float2) * M, cudaMemcpyHostToDevice));
    p.desc.tw = p.tw.as<float2>();
    p.desc.twh = p.twh.as<float2>();
    return WCT_OK;
}

// ---------------------------------------------------------------------------
// Component state.
// ---------------------------------------------------------------------------
struct PlaneState {
    int face{0}, index{0};
    wct_plane_desc desc{};
    std::vector<int> channels;
    PlaneDev dev{};
    // response table
    bool have_resp{false};
    int G{0}, npad{0}, nresp{0}, ldr{0}, waveform_pad{0};
    bool mirror{false};    // table[G-1-g][-j] == table[g][j] exactly: pair groups in the convolution
    double pitch{0}, impact{0};
    DevBuf d_table;        // [G][2npad+1][ldr] floats
    int spec_N{0};
    DevBuf d_spec;         // [G][2npad+1][M] packed spectra for spec_N
    // long-range response (ImpactTransform::waveform, gen/src/ImpactTransform.cxx:327-343); empty: none
    std::vector<float> long_wf;
    int long_pad{0};
    int long_nfft{0};
    DevBuf d_long_spec;    // [long_nfft] spectrum of long_wf cut or zero padded to long_nfft
    int row0{0};           // frame row offset
};

struct FaceState {
    bool have_bb{false};
    double lo[3]{}, hi[3]{};
    std::vector<int> planes;
};

struct Core {
    // configuration (gen/src/DepoTransform.cxx:63-72 defaults)
    double start_time{0.0};
    double readout_time{5.0e6};
    double tick{500.0};
    double drift_speed{1.0e-3};
    double nsigma{3.0};
    bool fluctuate{false};
    bool drift_fluctuate{false};
    unsigned long long seed{0};  // key of the counter-based random streams
    int frame_count{0};
    int device{0};
    bool have_drifter{false};
    DriftDev drifter{};
    std::vector<FaceState> faces;
    std::vector<std::unique_ptr<PlaneState>> planes;
    cudaStream_t own_stream{nullptr};
    cudaStream_t copy_stream{nullptr};  // frame downloads of the host API, overlapped with later planes
    cudaStream_t plane_streams[kMaxPlanes]{};  // each plane's FFT / convolution / inverse chain
    int plane_stream(int ip, cudaStream_t& out)
    {
        if (!plane_streams[ip]) {
            cudaError_t e = cudaStreamCreateWithFlags(&plane_streams[ip], cudaStreamNonBlocking);
            if (e != cudaSuccess) return fail(WCT_ERR_CUDA, std::string("plane stream: ") + cudaGetErrorString(e));
        }
        out = plane_streams[ip];
        return WCT_OK;
    }
    std::map<int, std::unique_ptr<FftPlanDev>> plans;
    // workspace
    DevBuf d_rec, d_win, d_Q, d_V, d_depos, d_frame, d_wcnt, d_woff, d_wcur, d_wlist, d_tprof, d_kbound;
    DevBuf d_long_z, d_glong;  // long-range step: packed row spectra; adjoint's frame-gradient rows
    DevBuf d_splat;            // DepoFluxSplat accumulator (doubles)
    DevBuf d_gframe, d_gdep, d_gglob;  // adjoint host entry point
    DevBuf d_fq, d_fluc;               // fluctuation: drifted charges, per (plane, depo) draw sums
    DevBuf d_pool, d_pool_off, d_pool_used;  // time profiles of long patches
    DevBuf d_wide;                           // per visit key: holds a long patch
    // modify_depo charge scale ([depo][plane], wct_dt_set_charge_scale); used
    // by calls whose depo count is qscale_n
    DevBuf d_qscale;
    size_t qscale_n{0};
    int qscale_planes{0};
    bool have_qscale{false};
    const double* qscale() const { return have_qscale ? d_qscale.as<double>() : nullptr; }
    int config_gen{0};                 // bumped by every change of planes or responses
    std::unique_ptr<struct BatchState> batch;
    WindowDev* h_win{nullptr};
    size_t last_n{0};
    DevBuf d_edges;             // trace edges of the frame rows (wct_dt_forward_traces)
    int2* h_edges{nullptr};
    size_t h_edges_n{0};
    // stage profiling
    static constexpr int kStages = 10;
    bool profiling{false};
    double stage_ms[kStages]{};
    long stage_launches[kStages]{};
    long total_launches{0};
    struct Pending {
        int stage;
        cudaEvent_t a, b;
    };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> event_pool;
    cudaEvent_t take_event()
    {
        if (!event_pool.empty()) {
            cudaEvent_t e = event_pool.back();
            event_pool.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        return e;
    }
    // Open a timed stage on stream s; close() records its end.
    struct StageTimer {
        Core* c;
        int stage;
        cudaStream_t s;
        cudaEvent_t a{nullptr};
        StageTimer(Core* c_, int st, cudaStream_t s_) : c(c_), stage(st), s(s_)
        {
            if (c->profiling) {
                a = c->take_event();
                cudaEventRecord(a, s);
            }
        }
        void close(int launches)
        {
            c->total_launches += launches;
            c->stage_launches[stage] += launches;
            if (a) {
                cudaEvent_t b = c->take_event();
                cudaEventRecord(b, s);
                c->pending.push_back({stage, a, b});
                a = nullptr;
            }
        }
    };
    void harvest()
    {
        for (auto& p : pending) {
            cudaEventSynchronize(p.b);
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) stage_ms[p.stage] += ms;
            event_pool.push_back(p.a);
            event_pool.push_back(p.b);
        }
        pending.clear();
    }
    size_t h_win_n{0};
    std::mutex mtx;

    int nticks() const { return (int)(readout_time / tick); }
    int nrows() const
    {
        int n = 0;
        for (auto& p : planes) n += p->desc.nwires;
        return n;
    }
    ~Core();
    void destroy()
    {
        harvest();
        for (auto e : event_pool) cudaEventDestroy(e);
        if (h_win) cudaFreeHost(h_win);
        if (h_edges) cudaFreeHost(h_edges);
        if (own_stream) cudaStreamDestroy(own_stream);
        if (copy_stream) cudaStreamDestroy(copy_stream);
        for (auto& pst : plane_streams)
            if (pst) cudaStreamDestroy(pst);
    }

    int plan_for(int M, FftDesc& d)
    {
        auto it = plans.find(M);
        if (it == plans.end()) {
            auto p = std::make_unique<FftPlanDev>();
            int rc = make_plan(M, *p);
            if (rc) return rc;
            it = plans.emplace(M, std::move(p)).first;
        }
        d = it->second->desc;
        return WCT_OK;
    }
};

static int configure(Core& c, const std::string& js)
{
    json::Value cfg;
    try {
        cfg = json::parse(js.empty() ? std::string("{}") : js);
    }
    catch (std::exception& e) {
        return fail(WCT_ERR_CONFIG, e.what());
    }
    c.nsigma = cfg["nsigma"].as_number(c.nsigma);
    c.fluctuate = cfg["fluctuate"].as_bool(false);
    // integer keys: in range before the conversion (an out-of-range conversion is undefined)
    const double seed = cfg["seed"].as_number(0.0);
    const double first = cfg["first_frame_number"].as_number(c.frame_count);
    const double device = cfg["device"].as_number(0.0);
    if (!(seed >= 0.0 && seed < 18446744073709551616.0))
        return fail(WCT_ERR_CONFIG, "seed must be a non-negative 64-bit integer");
    if (!(first >= -2147483648.0 && first <= 2147483647.0))
        return fail(WCT_ERR_CONFIG, "first_frame_number out of the int range");
    if (!(device >= 0.0 && device <= 1024.0)) return fail(WCT_ERR_CONFIG, "device must be a CUDA device ordinal");
    c.seed = (unsigned long long)seed;
    c.readout_time = cfg["readout_time"].as_number(c.readout_time);
    c.tick = cfg["tick"].as_number(c.tick);
    c.start_time = cfg["start_time"].as_number(c.start_time);
    c.drift_speed = cfg["drift_speed"].as_number(c.drift_speed);
    c.frame_count = (int)first;
    c.device = (int)device;
    if (cfg.has("pirs")) {
        const auto& p = cfg["pirs"];
        if (p.kind != json::Value::Array || p.arr.empty())
            return fail(WCT_ERR_CONFIG, "must configure with some plane impact response components");
    }
    if (c.tick <= 0 || c.readout_time <= 0) return fail(WCT_ERR_CONFIG, "tick and readout_time must be positive");
    if (!(c.readout_time / c.tick >= 1.0 && c.readout_time / c.tick < 2147483647.0))
        return fail(WCT_ERR_CONFIG, "readout_time / tick must give between 1 and 2^31 - 1 ticks");
    if (c.drift_speed <= 0) return fail(WCT_ERR_CONFIG, "illegal drift speed");
    const auto& dr = cfg["drifter"];
    if (dr.kind == json::Value::Object) {
        c.have_drifter = true;
        DriftDev& d = c.drifter;
        d.DL = dr["DL"].as_number(7.2e-7);                  // Drifter.cxx:66-71 defaults
        d.DT = dr["DT"].as_number(12.0e-7);
        d.lifetime = dr["lifetime"].as_number(8.0e6);
        d.speed = dr["drift_speed"].as_number(1.6e-3);
        d.toffset = dr["time_offset"].as_number(0.0);
        c.drift_fluctuate = dr["fluctuate"].as_bool(false);
        const auto& xr = dr["xregions"];
        if (xr.kind != json::Value::Array || xr.arr.empty()) return fail(WCT_ERR_CONFIG, "no xregions given");
        if (xr.arr.size() > 8) return fail(WCT_ERR_CONFIG, "at most 8 xregions");
        d.nxr = (int)xr.arr.size();
        for (int i = 0; i < d.nxr; ++i) {
            const auto& r = xr.arr[i];
            // Drifter::Xregion (gen/src/Drifter.cxx:35-52): a missing anode
            // takes the response plane's x, a missing response the anode's
            const json::Value& ja = r["anode"].is_null() ? r["response"] : r["anode"];
            const json::Value& jr = r["response"].is_null() ? r["anode"] : r["response"];
            d.xr[i][0] = ja.as_number(0.0);
            d.xr[i][1] = jr.as_number(0.0);
            d.xr[i][2] = r["cathode"].as_number(0.0);
        }
        if (d.speed <= 0) return fail(WCT_ERR_CONFIG, "illegal drift speed");
    }
    return WCT_OK;
}

// Per-plane window of ImpactTransform (gen/src/ImpactTransform.cxx:83-115).
struct PlaneWindow {
    int start_ch, end_ch, start_tick, end_tick;  // before padding
    int m_start_ch, m_end_ch, m_start_tick, m_end_tick;
    int nw_ref, nt_ref, nt_gpu;
};

static PlaneWindow window_of(const Core& c, const PlaneState& ps, const WindowDev& w)
{
    PlaneWindow o{};
    double pmin = 0, pmax = 0, tmin = 0, tmax = 0;  // gausdesc_range of an empty set
    if (w.nadded > 0) {
        pmin = dkey_inv(w.pmin);
        pmax = dkey_inv(w.pmax);
        tmin = dkey_inv(w.tmin);
        tmax = dkey_inv(w.tmax);
    }
    const PlaneDev& pl = ps.dev;
    auto ibin = [&](double v) { return int((v - pl.imp_min) / pl.imp_bs); };
    const double tbs = (c.start_time + c.readout_time - c.start_time) / (int)(c.readout_time / c.tick);
    auto tbin = [&](double v) { return int((v - c.start_time) / tbs); };
    const int nt = c.nticks();
    const int i0 = std::max(ibin(pmin), 0), i1 = std::min(ibin(pmax) + 1, pl.imp_nbins);
    const int t0 = std::max(tbin(tmin), 0), t1 = std::min(tbin(tmax) + 1, nt);
    const int G = ps.G;
    int start_ch = std::floor(i0 * 1.0 / (G - 1)) - 1;
    int end_ch = std::ceil(i1 * 1.0 / (G - 1)) + 2;
    if ((end_ch - start_ch) % 2 == 1) end_ch += 1;
    int start_tick = t0 - 1;
    int end_tick = t1 + 2;
    if ((end_tick - start_tick) % 2 == 1) end_tick += 1;
    const size_t ntw = fft_best_length(end_ch - start_ch + 2 * ps.npad, true);
    const int npad_wire = (ntw - end_ch + start_ch) / 2;
    o.start_ch = start_ch;
    o.end_ch = end_ch;
    o.start_tick = start_tick;
    o.end_tick = end_tick;
    o.m_start_ch = start_ch - npad_wire;
    o.m_end_ch = end_ch + npad_wire;
    const size_t ntt = fft_best_length(end_tick - start_tick + ps.waveform_pad, false);
    const int npad_time = ntt - end_tick + start_tick;
    o.m_start_tick = start_tick;
    o.m_end_tick = end_tick + npad_time;
    o.nw_ref = end_ch - start_ch + 2 * npad_wire;
    o.nt_ref = o.m_end_tick - o.m_start_tick;
    o.nt_gpu = gpu_fft_length(o.nt_ref);
    return o;
}

static int ensure_spectra(Core& c, PlaneState& ps, int N)
{
    if (ps.spec_N == N) return WCT_OK;
    FftDesc d;
    int rc = c.plan_for(N / 2, d);
    if (rc) return rc;
    const int rows = ps.G * (2 * ps.npad + 1);
    CUDA_TRY(ps.d_spec.ensure(sizeof(float2) * (size_t)rows * (N / 2)));
    launch_rfft_rows(ps.d_table.as<float>(), ps.ldr, std::min(ps.nresp, N), ps.d_spec.as<float2>(), N / 2, rows, d,
                     c.own_stream);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(c.own_stream));
    ps.spec_N = N;
    return WCT_OK;
}

__global__ void k_win_init(WindowDev* w, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    w[i].pmin = ~0ull;
    w[i].tmin = ~0ull;
    w[i].pmax = 0ull;
    w[i].tmax = 0ull;
    w[i].nadded = w[i].out_time = w[i].out_pitch = w[i].oversize = w[i].bigcharge = 0;
    w[i].wide_ticks = w[i].nvisits = 0;
}

// Drift, patch records, per-plane windows and charge-grid layout of one event:
// the part of the forward that the adjoint recomputes (patches are never
// stored between the two).
struct EventPlan {
    int n{0}, np{0}, nticks{0};
    int nkeys{0};
    EventTable et{};
    FlucParams fp{};
    TimeDev tb{};
    PlaneSet pset{};
    GridSet gset{};
    std::vector<PlaneWindow> pw;
    std::vector<size_t> voff;  // per plane: its wire-convolution rows in d_V (complex values)
    int total_visits{0};
};

// Random-stream parameters of one call (fluct = false: the mean model, as the adjoint needs).
static FlucParams fluc_params(const Core& c, bool fluct, int ident0, const int* ident_base)
{
    FlucParams fp{};
    fp.on_patch = fluct && c.fluctuate ? 1 : 0;
    fp.on_drift = fluct && c.drift_fluctuate && c.have_drifter ? 1 : 0;
    fp.key0 = (unsigned)(c.seed & 0xffffffffull);
    fp.key1 = (unsigned)(c.seed >> 32);
    fp.ident0 = ident0;
    fp.ident_base = ident_base;
    return fp;
}

// h_depos (optional): the depos in host memory, uploaded into d_depos here
// in chunks on the copy stream, each chunk's prep blocks launched as soon as
// it has arrived.
static int prepare_event(Core& c, const double* d_depos, size_t ndepos, cudaStream_t s, EventPlan& ev,
                         bool fluct = true, const double* h_depos = nullptr)
{
    if (c.planes.empty()) return fail(WCT_ERR_STATE, "no planes configured");
    if ((int)c.planes.size() > kMaxPlanes) return fail(WCT_ERR_CONFIG, "too many planes for one component");
    for (auto& p : c.planes)
        if (!p->have_resp) return fail(WCT_ERR_STATE, "a plane has no response");
    if (ndepos > (size_t)0x7fffffff) return fail(WCT_ERR_SIZE, "too many depos");
    if (c.have_qscale && (ndepos != c.qscale_n || c.qscale_planes != (int)c.planes.size()))
        return fail(WCT_ERR_ARG, "the charge scale was set for another depo count or plane set");
    CUDA_TRY(cudaSetDevice(c.device));
    const int n = (int)ndepos;
    const int np = (int)c.planes.size();
    const int nticks = c.nticks();
    ev.n = n;
    ev.np = np;
    ev.nticks = nticks;
    TimeDev& tb = ev.tb;
    tb.nbins = nticks;
    tb.tmin = c.start_time;
    tb.tmax = c.start_time + c.readout_time;
    tb.bs = (tb.tmax - tb.tmin) / tb.nbins;

    PlaneSet& pset = ev.pset;
    pset = PlaneSet{};
    pset.nplanes = np;
    int nwt = 0;
    for (int ip = 0; ip < np; ++ip) {
        pset.p[ip] = c.planes[ip]->dev;
        pset.p[ip].wire_base = nwt;
        nwt += c.planes[ip]->desc.nwires;
    }
    pset.nwires_total = nwt;
    pset.ntiles = (nticks + kTile - 1) / kTile;
    const int nkeys = nwt * pset.ntiles;
    ev.nkeys = nkeys;

    CUDA_TRY(c.d_rec.ensure(sizeof(PatchRec) * (size_t)np * std::max(n, 1)));
    CUDA_TRY(c.d_tprof.ensure(sizeof(float) * kTprof * (size_t)std::max(n, 1)));
    CUDA_TRY(c.d_win.ensure(sizeof(WindowDev) * np));
    CUDA_TRY(c.d_wcnt.ensure(sizeof(int) * (nkeys + 1)));
    CUDA_TRY(c.d_woff.ensure(sizeof(int) * (nkeys + 1)));
    CUDA_TRY(c.d_wcur.ensure(sizeof(int) * (nkeys + 1 + (nkeys + 1023) / 1024)));  // + scan block sums
    if (c.h_win_n < (size_t)np) {
        if (c.h_win) cudaFreeHost(c.h_win);
        CUDA_TRY(cudaMallocHost(&c.h_win, sizeof(WindowDev) * np + sizeof(int)));
        c.h_win_n = np;
    }
    int* h_total = reinterpret_cast<int*>(c.h_win + np);

    Core::StageTimer t_prep(&c, 0, s);
    CUDA_TRY(cudaMemsetAsync(c.d_wcnt.p, 0, sizeof(int) * (nkeys + 1), s));
    CUDA_TRY(c.d_kbound.ensure(sizeof(unsigned long long) * (size_t)nkeys * kTileBlocks));
    CUDA_TRY(c.d_wide.ensure((size_t)nkeys));
    CUDA_TRY(cudaMemsetAsync(c.d_wide.p, 0, (size_t)nkeys, s));
    CUDA_TRY(cudaMemsetAsync(c.d_kbound.p, 0, sizeof(unsigned long long) * (size_t)nkeys * kTileBlocks, s));
    k_win_init<<<1, 64, 0, s>>>(c.d_win.as<WindowDev>(), np);
    EventTable& et = ev.et;
    et.nev = 1;
    et.dep0[0] = 0;
    et.dep0[1] = n;
    et.blk0[0] = 0;
    et.blk0[1] = (n + 255) / 256;
    ev.fp = fluc_params(c, fluct, c.frame_count, nullptr);
    if (ev.fp.on_patch) {
        CUDA_TRY(c.d_fq.ensure(sizeof(double) * (size_t)np * std::max(n, 1)));
        CUDA_TRY(c.d_fluc.ensure(sizeof(FlucRec) * (size_t)np * std::max(n, 1)));
    }
    auto prep = [&](int b0, int b1) {
        launch_prep_all(d_depos, et, nkeys, c.drifter, c.have_drifter ? 1 : 0, pset, tb, c.drift_speed, c.nsigma,
                        c.d_rec.as<PatchRec>(), c.d_win.as<WindowDev>(), c.d_wcnt.as<int>(), c.d_tprof.as<float>(),
                        c.d_kbound.as<unsigned long long>(), ev.fp, ev.fp.on_patch ? c.d_fq.as<double>() : nullptr,
                        c.d_wide.as<unsigned char>(), s, b0, b1, c.qscale());
    };
    if (h_depos && n > 0) {
        // 4 chunks (whole 256-depo blocks): upload k + 1 runs while the prep of chunk k does
        const int nb = et.blk0[1], per = (nb + 3) / 4;
        std::vector<cudaEvent_t> up;
        int rc = WCT_OK;
        for (int b0 = 0; b0 < nb && rc == WCT_OK; b0 += per) {
            const int b1 = std::min(nb, b0 + per);
            const size_t d0 = (size_t)b0 * 256, d1 = std::min((size_t)b1 * 256, (size_t)n);
            cudaEvent_t e = c.take_event();
            up.push_back(e);
            cudaError_t ce = cudaMemcpyAsync(const_cast<double*>(d_depos) + 7 * d0, h_depos + 7 * d0,
                                             sizeof(double) * 7 * (d1 - d0), cudaMemcpyHostToDevice, c.copy_stream);
            if (ce == cudaSuccess) ce = cudaEventRecord(e, c.copy_stream);
            if (ce == cudaSuccess) ce = cudaStreamWaitEvent(s, e, 0);
            if (ce != cudaSuccess) rc = fail(WCT_ERR_CUDA, std::string("depo upload: ") + cudaGetErrorString(ce));
            else prep(b0, b1);
        }
        for (auto e : up) c.event_pool.push_back(e);  // reusable once s has passed its wait
        if (rc) return rc;
    }
    else
        prep(0, -1);
    launch_scan(c.d_wcnt.as<int>(), nkeys, c.d_woff.as<int>(), c.d_wcur.as<int>(), s);
    t_prep.close(4 + (n > 0 ? 1 : 0));
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(c.h_win, c.d_win.p, sizeof(WindowDev) * np, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaMemcpyAsync(h_total, c.d_woff.as<int>() + nkeys, sizeof(int), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    for (int ip = 0; ip < np; ++ip)
        if (c.h_win[ip].oversize) return fail(WCT_ERR_SIZE, "a diffusion patch exceeds 1024 ticks or 1024 impact bins");
    for (int ip = 0; ip < np; ++ip)
        if (c.h_win[ip].bigcharge) return fail(WCT_ERR_SIZE, "a depo charge exceeds 5e11 electrons");
    if (c.h_win[0].nvisits >= 0x7fffffffull)
        return fail(WCT_ERR_SIZE, "an event holds 2^31 or more patch visits (wire x 256-tick tile); split it");
    ev.total_visits = *h_total;

    std::vector<PlaneWindow>& pw = ev.pw;
    pw.assign(np, PlaneWindow{});
    GridSet& gset = ev.gset;
    gset = GridSet{};
    gset.nplanes = np;
    gset.ntiles_abs = pset.ntiles;
    size_t qfloats = 0, vcomplex = 0, smem = 0;
    int rows = 0;
    ev.voff.assign(np, 0);
    for (int ip = 0; ip < np; ++ip) {
        PlaneState& ps = *c.planes[ip];
        pw[ip] = window_of(c, ps, c.h_win[ip]);
        const PlaneWindow& w = pw[ip];
        GridPlane& g = gset.p[ip];
        g.nimp = ps.dev.nimp;
        g.G = ps.G;
        g.nwires = ps.desc.nwires;
        g.wire_base = pset.p[ip].wire_base;
        g.start_ch = w.start_ch;
        g.nin = c.h_win[ip].nadded > 0 ? w.end_ch - w.start_ch : 0;
        g.col0 = w.start_tick;
        g.ncols = w.end_tick - w.start_tick;
        g.N = w.nt_gpu;
        g.tbs = (float)tb.bs;
        g.pbs = (float)ps.dev.imp_bs;
        g.qoff = (long long)qfloats;
        g.recoff = (long long)ip * n;
        g.row_base = rows;
        // absolute tick tiles covering grid columns [0, N) (ticks col0 .. col0+N-1), floor division
        auto fdiv = [](int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); };
        g.ktile0 = fdiv(g.col0, kTile);
        g.ntile = fdiv(g.col0 + g.N - 1, kTile) - g.ktile0 + 1;
        rows += g.nin * g.ntile;
        qfloats += (size_t)ps.G * g.nin * g.N;
        ev.voff[ip] = vcomplex;  // each plane its own rows: the planes' chains may run at once
        if (g.nin) vcomplex += (size_t)(g.nin + 2 * ps.npad) * (g.N / 2);
        if (g.nin) {
            smem = std::max(smem, raster_smem_bytes(g.G));
            int rc = ensure_spectra(c, ps, g.N);
            if (rc) return rc;
        }
    }
    gset.nrows_total = rows;
    if (smem > 227 * 1024) return fail(WCT_ERR_SIZE, "event time window too long for the shared-memory charge grid");
    if (qfloats >= (size_t)1 << 40) return fail(WCT_ERR_SIZE, "charge grid too large");
    CUDA_TRY(c.d_Q.ensure(sizeof(float) * std::max<size_t>(qfloats, 1)));
    CUDA_TRY(c.d_V.ensure(sizeof(float2) * std::max<size_t>(vcomplex, 1)));
    return WCT_OK;
}

static int dft_rows(const float2* in, long ld_in, float2* out, long ld_out, int nrows, int n, int sign,
                    cudaStream_t s);

// The long-range step of ImpactTransform::waveform
// (gen/src/ImpactTransform.cxx:327-343) on nrows frame rows of nticks
// samples (row stride ld): each row, zero padded to nfft =
// fft_best_length(nticks + long_pad), is circularly convolved with the long
// waveform cut or zero padded to nfft, and cut back to nticks.  Rows go two
// per complex transform (the kernel is real); any nfft of the reference's
// tables (7-smooth directly, others through Bluestein).  transpose: the
// adjoint (correlation, conjugate spectrum).
static int long_conv_rows(Core& c, PlaneState& ps, float* rows, long ld, int nrows, int nticks, bool transpose,
                          cudaStream_t s)
{
    if (ps.long_wf.empty() || nrows <= 0 || nticks <= 0) return WCT_OK;
    const int nfft = (int)fft_best_length((size_t)nticks + (size_t)ps.long_pad, false);
    if (ps.long_nfft != nfft) {
        std::vector<float2> lw(nfft, make_float2(0.f, 0.f));
        for (int k = 0; k < nfft && k < (int)ps.long_wf.size(); ++k) lw[k].x = ps.long_wf[k];
        CUDA_TRY(ps.d_long_spec.ensure(sizeof(float2) * nfft));
        CUDA_TRY(cudaMemcpyAsync(ps.d_long_spec.p, lw.data(), sizeof(float2) * nfft, cudaMemcpyHostToDevice, s));
        int rc = dft_rows(ps.d_long_spec.as<float2>(), nfft, ps.d_long_spec.as<float2>(), nfft, 1, nfft, -1, s);
        if (rc) return rc;
        CUDA_TRY(cudaStreamSynchronize(s));  // lw goes out of scope
        ps.long_nfft = nfft;
    }
    const int nz = (nrows + 1) / 2;
    CUDA_TRY(c.d_long_z.ensure(sizeof(float2) * (size_t)nz * nfft));
    float2* Z = c.d_long_z.as<float2>();
    launch_pack_rows(rows, ld, nrows, nticks, Z, nfft, s);
    int rc = dft_rows(Z, nfft, Z, nfft, nz, nfft, -1, s);
    if (rc) return rc;
    launch_cmul_rows(Z, nfft, nz, ps.d_long_spec.as<float2>(), transpose, s);
    rc = dft_rows(Z, nfft, Z, nfft, nz, nfft, +1, s);
    if (rc) return rc;
    launch_unpack_rows(Z, nfft, rows, ld, nrows, nticks, s);
    CUDA_TRY(cudaGetLastError());
    return WCT_OK;
}

// The part of a plane's frame rows that the forward writes (plane rows
// [rlo, rhi), ticks [tlo, thi)); the rest of the plane stays zero.
struct FrameRegion {
    int rlo{0}, rhi{0}, tlo{0}, thi{0};
};

// plane_done (optional, one event per plane): recorded once the plane's
// frame rows are final (on the plane's stream), so a caller can download them while later planes run;
// zeroed (optional): recorded once the frame is cleared; regions (optional):
// each plane's written block, so the zero rest can go first.
//
// after_plane (optional): called once a plane's frame work is enqueued, with
// the plane, its written block and the stream that work is on, to enqueue
// work that reads the plane's rows (a non-zero return aborts the call with
// that status).
//
// fork_planes: after the raster, each plane's time FFT, wire convolution and
// inverse run on a stream of their own (forked from s, joined back into s at
// the end), so the planes' kernels fill one another's last waves (the
// device-buffer call).  The host-buffer calls keep the planes one after
// another on s instead: each plane's rows then go back while the next planes
// are transformed, which hides more copy time than the overlap of the planes
// saves.  With stage profiling on, or a plane with a long-range response
// (one shared workspace), the planes always run one after another.
static int forward_device(Core& c, const double* d_depos, size_t ndepos, float* d_frame, wct_plane_window* wins,
                          int* frame_ident, cudaStream_t s, cudaEvent_t* plane_done = nullptr,
                          cudaEvent_t zeroed = nullptr, std::vector<FrameRegion>* regions = nullptr,
                          const double* h_depos = nullptr,
                          const std::function<int(int, const FrameRegion&, cudaStream_t)>& after_plane = nullptr,
                          bool fork_planes = false)
{
    EventPlan ev;
    int prc = prepare_event(c, d_depos, ndepos, s, ev, true, h_depos);
    if (prc) return prc;
    const int n = ev.n, np = ev.np, nticks = ev.nticks, total_visits = ev.total_visits, rows = ev.gset.nrows_total;
    const PlaneSet& pset = ev.pset;
    const GridSet& gset = ev.gset;
    const std::vector<PlaneWindow>& pw = ev.pw;
    CUDA_TRY(c.d_wlist.ensure(sizeof(Visit) * std::max(total_visits, 1)));
    CUDA_TRY(cudaMemsetAsync(d_frame, 0, sizeof(float) * (size_t)c.nrows() * nticks, s));
    if (zeroed) CUDA_TRY(cudaEventRecord(zeroed, s));
    if (regions) regions->assign(np, FrameRegion{});

    // time profiles of the long patches: exactly the room counted by the prep kernel
    // (int offsets: beyond 2^31 - 2 ticks the rest is computed in the raster)
    const long long wide = (long long)std::min<unsigned long long>(c.h_win[0].wide_ticks, 0x7ffffffeull);
    CUDA_TRY(c.d_pool.ensure(sizeof(float) * (size_t)std::max<long long>(wide, 1)));
    CUDA_TRY(c.d_pool_off.ensure(sizeof(int) * (size_t)std::max(n, 1)));
    CUDA_TRY(c.d_pool_used.ensure(sizeof(unsigned long long)));
    CUDA_TRY(cudaMemsetAsync(c.d_pool_used.p, 0, sizeof(unsigned long long), s));
    const TprofPool pool{c.d_pool.as<float>(), c.d_pool_off.as<int>(), c.d_pool_used.as<unsigned long long>(),
                         wide};

    Core::StageTimer t_r(&c, 1, s);
    launch_fill(c.d_rec.as<PatchRec>(), ev.et, ev.nkeys, pset, c.d_wcur.as<int>(), c.d_wlist.as<Visit>(),
                (long long)std::max(total_visits, 1), s);
    if (!ev.fp.on_patch && wide > 0)
        launch_tprof_pool(c.d_rec.as<PatchRec>(), ev.et, np, (float)ev.tb.bs, pool, nullptr, s);
    if (ev.fp.on_patch) {
        launch_fluc_sums(c.d_rec.as<PatchRec>(), ev.et, pset, (float)ev.tb.bs, ev.fp, c.d_fq.as<double>(),
                         c.d_fluc.as<FlucRec>(), s);
        launch_raster_fluc(c.d_rec.as<PatchRec>(), c.d_fluc.as<FlucRec>(), ev.fp, ev.et, c.d_wcnt.as<int>(),
                           c.d_woff.as<int>(), c.d_wlist.as<Visit>(), (long long)std::max(total_visits, 1), gset,
                           c.d_Q.as<float>(), s);
    }
    else
        launch_raster_wires(c.d_rec.as<PatchRec>(), c.d_tprof.as<float>(), pool, c.d_wide.as<unsigned char>(),
                            c.d_wcnt.as<int>(),
                            c.d_woff.as<int>(), c.d_wlist.as<Visit>(), (long long)std::max(total_visits, 1),
                            c.d_kbound.as<unsigned long long>(), gset, c.d_Q.as<float>(), s);
    t_r.close((n > 0 ? 1 : 0) + (ev.fp.on_patch && n > 0 ? 1 : 0) + (!ev.fp.on_patch && wide > 0 ? 1 : 0) +
              (rows > 0 ? 1 : 0));
    CUDA_TRY(cudaGetLastError());

    // the planes' chains: on streams of their own unless profiling or a long-range step needs s alone
    bool fork = fork_planes && !c.profiling && np > 1;
    for (int ip = 0; ip < np; ++ip)
        if (!c.planes[ip]->long_wf.empty()) fork = false;
    cudaEvent_t rastered = nullptr;
    if (fork) {
        rastered = c.take_event();
        CUDA_TRY(cudaEventRecord(rastered, s));
    }
    std::vector<cudaEvent_t> joined;
    int rc_planes = WCT_OK;
    for (int ip = 0; ip < np && rc_planes == WCT_OK; ++ip) {
        PlaneState& ps = *c.planes[ip];
        const PlaneWindow& w = pw[ip];
        const GridPlane& g = gset.p[ip];
        if (wins) {
            wct_plane_window& o = wins[ip];
            o.face = ps.face;
            o.plane = ps.index;
            o.start_ch = w.m_start_ch;
            o.end_ch = w.m_end_ch;
            o.start_tick = w.m_start_tick;
            o.end_tick = w.m_end_tick;
            o.nw_fft = w.nw_ref;
            o.nt_fft = w.nt_ref;
            o.nt_gpu = w.nt_gpu;
            o.charge_rows = w.end_ch - w.start_ch;
            o.npad = ps.npad;
            o.ndepos_added = c.h_win[ip].nadded;
            o.outside_time = c.h_win[ip].out_time;
            o.outside_pitch = c.h_win[ip].out_pitch;
        }
        cudaStream_t ps_s = s;
        if (fork && g.nin > 0) {
            int rc = c.plane_stream(ip, ps_s);
            if (rc) {
                rc_planes = rc;
                break;
            }
            CUDA_TRY(cudaStreamWaitEvent(ps_s, rastered, 0));
        }
        auto plane_chain = [&]() -> int {
            FrameRegion r;
            if (g.nin > 0) {  // else: no charge, the plane's frame rows stay zero
                const int nin = g.nin;
                const int nout = nin + 2 * ps.npad;
                const int N = g.N, M = N / 2;
                FftDesc d;
                int rc = c.plan_for(M, d);
                if (rc) return rc;
                float* Q = c.d_Q.as<float>() + g.qoff;
                float2* V = c.d_V.as<float2>() + ev.voff[ip];
                Core::StageTimer t_f(&c, 2, ps_s);
                launch_rfft_rows(Q, N, N, reinterpret_cast<float2*>(Q), M, ps.G * nin, d, ps_s);
                t_f.close(1);
                Core::StageTimer t_c(&c, 3, ps_s);
                launch_wire_conv(reinterpret_cast<const float2*>(Q), ps.d_spec.as<float2>(), V, ps.G, ps.npad, nin,
                                 nout, M, ps.mirror, ps_s);
                t_c.close(1);
                const int wlo = std::max(0, w.m_start_ch), whi = std::min(ps.desc.nwires, w.m_end_ch);
                Core::StageTimer t_i(&c, 4, ps_s);
                launch_irfft_rows(V, nout, d, w.start_ch - ps.npad, wlo, whi, w.start_tick, std::min(N, w.nt_ref),
                                  nticks, d_frame + (size_t)ps.row0 * nticks, ps_s);
                if (!ps.long_wf.empty() && whi > wlo) {
                    rc = long_conv_rows(c, ps, d_frame + ((size_t)ps.row0 + wlo) * nticks, nticks, whi - wlo, nticks,
                                        false, ps_s);
                    if (rc) return rc;
                }
                if (whi > wlo) {  // what the inverse (and the long-range step) wrote
                    r.rlo = wlo;
                    r.rhi = whi;
                    r.tlo = ps.long_wf.empty() ? std::max(0, w.start_tick) : 0;
                    r.thi = ps.long_wf.empty() ? std::min(nticks, w.start_tick + std::min(N, w.nt_ref)) : nticks;
                    if (r.thi < r.tlo) r.thi = r.tlo;
                }
                t_i.close(ps.long_wf.empty() || whi <= wlo ? 1 : 6);
                CUDA_TRY(cudaGetLastError());
            }
            if (regions) (*regions)[ip] = r;
            if (after_plane) {
                const int arc = after_plane(ip, r, ps_s);
                if (arc) return arc;
            }
            if (plane_done) CUDA_TRY(cudaEventRecord(plane_done[ip], ps_s));
            return WCT_OK;
        };
        rc_planes = plane_chain();
        if (ps_s != s) {  // join back into s (also after an error, so nothing is left behind)
            cudaEvent_t e = c.take_event();
            joined.push_back(e);
            cudaError_t ce = cudaEventRecord(e, ps_s);
            if (ce == cudaSuccess) ce = cudaStreamWaitEvent(s, e, 0);
            if (ce != cudaSuccess && rc_planes == WCT_OK)
                rc_planes = fail(WCT_ERR_CUDA, std::string("plane join: ") + cudaGetErrorString(ce));
        }
    }
    if (rastered) c.event_pool.push_back(rastered);  // reusable: s and the plane streams have enqueued their waits
    for (auto e : joined) c.event_pool.push_back(e);
    if (rc_planes) return rc_planes;
    if (frame_ident) *frame_ident = c.frame_count;
    ++c.frame_count;
    c.last_n = ndepos;
    return WCT_OK;
}

// ---------------------------------------------------------------------------
// Adjoint: dL/d(depos) and dL/d(DL, DT, lifetime) from dL/d(frame).
// Patch records and windows are recomputed (prepare_event), then per plane
// the frame gradient is correlated with the responses (the transpose of the
// FFT convolution) into dL/dQ, which the gather kernel reduces per depo.
// ---------------------------------------------------------------------------
static int adjoint_device(Core& c, const double* d_depos, size_t ndepos, const float* d_gframe, double* d_gdep,
                          double* d_gglob, cudaStream_t s)
{
    EventPlan ev;
    int prc = prepare_event(c, d_depos, ndepos, s, ev, false);  // the mean model
    if (prc) return prc;
    const int n = ev.n, np = ev.np, nticks = ev.nticks;
    if (n) CUDA_TRY(cudaMemsetAsync(d_gdep, 0, sizeof(double) * 7 * (size_t)n, s));
    if (d_gglob) CUDA_TRY(cudaMemsetAsync(d_gglob, 0, sizeof(double) * 3, s));
    CUDA_TRY(c.d_gglob.ensure(sizeof(double) * 3));
    double* gg = d_gglob ? d_gglob : c.d_gglob.as<double>();
    if (!d_gglob) CUDA_TRY(cudaMemsetAsync(gg, 0, sizeof(double) * 3, s));
    AdjSet as{};
    as.nplanes = np;
    for (int ip = 0; ip < np; ++ip) {
        PlaneState& ps = *c.planes[ip];
        const PlaneWindow& w = ev.pw[ip];
        const GridPlane& g = ev.gset.p[ip];
        AdjPlane& a = as.p[ip];
        a.nimp = g.nimp;
        a.nin = g.nin;
        a.N = g.N;
        a.start_ch = g.start_ch;
        a.col0 = g.col0;
        a.qoff = g.qoff;
        a.pbs = g.pbs;
        a.tbs = g.tbs;
        a.ax = ps.dev.ax;
        a.ay = ps.dev.ay;
        a.az = ps.dev.az;
        if (g.nin == 0) continue;
        const int nin = g.nin, nout = nin + 2 * ps.npad, N = g.N, M = N / 2;
        FftDesc d;
        int rc = c.plan_for(M, d);
        if (rc) return rc;
        float* Gr = c.d_V.as<float>();  // [nout][N] real, then [nout][M] spectra in place
        const int wlo = std::max(0, w.m_start_ch), whi = std::min(ps.desc.nwires, w.m_end_ch);
        Core::StageTimer t_f(&c, 6, s);
        const float* gplane = d_gframe + (size_t)ps.row0 * nticks;
        if (!ps.long_wf.empty() && whi > wlo) {
            // the long-range step's transpose on a copy of the window rows (same row indices)
            CUDA_TRY(c.d_glong.ensure(sizeof(float) * (size_t)whi * nticks));
            float* gl = c.d_glong.as<float>();
            CUDA_TRY(cudaMemcpyAsync(gl + (size_t)wlo * nticks, gplane + (size_t)wlo * nticks,
                                     sizeof(float) * (size_t)(whi - wlo) * nticks, cudaMemcpyDeviceToDevice, s));
            rc = long_conv_rows(c, ps, gl + (size_t)wlo * nticks, nticks, whi - wlo, nticks, true, s);
            if (rc) return rc;
            gplane = gl;
        }
        launch_grad_rows(gplane, nticks, w.start_ch - ps.npad, wlo, whi, w.start_tick, std::min(N, w.nt_ref), nout,
                         N, Gr, s);
        launch_rfft_rows(Gr, N, N, reinterpret_cast<float2*>(Gr), M, nout, d, s);
        t_f.close(2);
        float* dQ = c.d_Q.as<float>() + g.qoff;
        Core::StageTimer t_c(&c, 7, s);
        launch_wire_conv_adj(reinterpret_cast<const float2*>(Gr), ps.d_spec.as<float2>(),
                             reinterpret_cast<float2*>(dQ), ps.G, ps.npad, nin, nout, M, s);
        t_c.close(1);
        Core::StageTimer t_i(&c, 8, s);
        launch_irfft_rows(reinterpret_cast<const float2*>(dQ), ps.G * nin, d, 0, 0, ps.G * nin, 0, N, N, dQ, s);
        t_i.close(1);
        CUDA_TRY(cudaGetLastError());
    }
    Core::StageTimer t_g(&c, 9, s);
    launch_adj_gather(d_depos, n, c.drifter, c.have_drifter ? 1 : 0, ev.pset, as, c.drift_speed,
                      c.d_rec.as<PatchRec>(), c.d_Q.as<float>(), d_gdep, gg, s, c.qscale());
    t_g.close(n ? (c.have_drifter ? 2 : 1) : 0);
    CUDA_TRY(cudaGetLastError());
    return WCT_OK;
}

// ---------------------------------------------------------------------------
// Stand-alone operations: per-device FFT plans.
// ---------------------------------------------------------------------------
static std::mutex g_ops_mtx;
static std::map<std::pair<int, int>, std::unique_ptr<FftPlanDev>> g_plans;  // (device, M)

static int device_plan(int M, FftDesc& d)
{
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_ops_mtx);
    auto key = std::make_pair(dev, M);
    auto it = g_plans.find(key);
    if (it == g_plans.end()) {
        auto p = std::make_unique<FftPlanDev>();
        int rc = make_plan(M, *p);
        if (rc) return rc;
        it = g_plans.emplace(key, std::move(p)).first;
    }
    d = it->second->desc;
    return WCT_OK;
}

// Checks shared by the row-convolution entry points; picks the FFT length.
static int convolve_args(const float* in, long ld_in, int nrows, int n_in, const float* resp, int n_resp, int& nfft,
                         float* out, long ld_out, int n_out)
{
    if (!in || !resp || !out || nrows < 0 || n_in < 0 || n_resp <= 0 || n_out < 0 || ld_in < n_in ||
        ld_out < n_out)
        return fail(WCT_ERR_ARG, "convolve rows: bad arguments");
    if (nfft == 0) nfft = gpu_fft_length(std::max(4, n_in + n_resp - 1));
    if (nfft <= 0 || nfft % 4 || !fft_supported(nfft / 2))
        return fail(WCT_ERR_SIZE, "convolve rows: unsupported FFT length");
    if (n_out > nfft) return fail(WCT_ERR_ARG, "convolve rows: n_out exceeds the FFT length");
    return WCT_OK;
}

// The convolution itself on caller-provided scratch: X [nrows][M] and R [M].
static int convolve_on(const float* in, long ld_in, int nrows, int n_in, const float* resp, int n_resp, int nfft,
                       float* out, long ld_out, int n_out, const FftDesc& d, float2* X, float2* R, cudaStream_t s)
{
    const int M = nfft / 2;
    launch_rfft_rows(resp, n_resp, std::min(n_resp, nfft), R, M, 1, d, s);
    launch_rfft_rows(in, ld_in, std::min(n_in, nfft), X, M, nrows, d, s);
    launch_spec_mul(X, M, nrows, M, R, s);
    launch_irfft_rows(X, nrows, d, 0, 0, nrows, 0, n_out, (int)ld_out, out, s);
    CUDA_TRY(cudaGetLastError());
    return WCT_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free row convolution: all scratch (twiddle tables, the response
// spectrum and the row spectra) lives in this fixed device array, reserved on
// every GPU that loads the library for as long as the process runs.  Every
// call overwrites the parts it uses, so nothing needs clearing, and calls that
// overlap on a GPU (other streams or host threads) race on it.
// ---------------------------------------------------------------------------
constexpr size_t kNoAllocComplex = (size_t)4 << 20;  // 4 Mi complex floats = 32 MiB per GPU
static __device__ __align__(256) float2 g_noalloc_scratch[kNoAllocComplex];
constexpr int kNoAllocMaxDevices = 64;
static std::mutex g_noalloc_mtx;
static float2* g_noalloc_addr[kNoAllocMaxDevices] = {};

// Device address of the scratch array on the current device, looked up once
// per device (cudaGetSymbolAddress with that device current) and kept for the
// life of the process: a cudaDeviceReset of that device would leave it stale,
// and the header rules out calls after one.
static int noalloc_scratch(float2** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(WCT_ERR_CUDA, cudaGetErrorString(e));
    if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(WCT_ERR_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_noalloc_mtx);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return fail(WCT_ERR_CUDA, cudaGetErrorString(e));
        g_noalloc_addr[dev] = static_cast<float2*>(p);
    }
    *out = g_noalloc_addr[dev];
    return WCT_OK;
}

// ---------------------------------------------------------------------------
// Batched events.  The whole batch -- every pass of up to `slots` events
// through prep, scan, device planning, fill and the persistent raster,
// time-FFT, wire-convolution and inverse kernels -- is captured once as a
// CUDA graph and replayed while the batch shape, buffers and drift
// parameters stay the same.  Time FFTs use a fixed ladder of lengths (about
// 10% apart) so that the response spectra of every length are ready before
// the graph runs.
// ---------------------------------------------------------------------------
struct BatchState {
    int gen{-1};  // Core::config_gen of the setup
    BatchStatic bs{};
    std::vector<std::unique_ptr<FftPlanDev>> cls_plans;
    DevBuf d_descs;
    std::vector<std::unique_ptr<DevBuf>> spec;  // [plane * ncls + cls]
    DevBuf d_spec_tab;                          // const float2* [plane][ncls]
    int maxM{0}, maxG{0}, nsm{148};
    DevBuf d_Q, d_V, d_rec, d_tprof, d_win, d_wcnt, d_woff, d_wcur, d_kbound, d_wlist, d_plans;
    DevBuf d_fq, d_fluc, d_ident;  // fluctuation: drifted charges, draw sums, first frame ident of the call
    DevBuf d_pool, d_pool_off, d_pool_used;  // time profiles of long patches
    DevBuf d_wide;                           // per key: holds a long patch
    long long pool_cap{0};
    int* h_ident{nullptr};         // pinned source of d_ident
    long long vcap{0};
    BatchPlan* h_plans{nullptr};
    size_t h_plans_n{0};
    BatchTune tune{16, 6, 256, 4, 4};  // autotuned on a 64-event full-APA batch
    // the instantiated graph and what it was captured for
    cudaGraphExec_t exec{nullptr};
    const void* g_depos{nullptr};
    void* g_frames{nullptr};
    std::vector<long long> g_offsets;
    BatchTune g_tune{};
    long long g_vcap{0};
    cudaStream_t g_stream{nullptr};
    DriftDev g_drift{};
    int g_fluc[2]{0, 0};
    unsigned long long g_seed{0};
    long long g_pool_cap{0};
    std::vector<void*> g_bufs;
    void drop_graph()
    {
        if (exec) cudaGraphExecDestroy(exec);
        exec = nullptr;
    }
    ~BatchState()
    {
        drop_graph();
        if (h_plans) cudaFreeHost(h_plans);
        if (h_ident) cudaFreeHost(h_ident);
    }
};

Core::~Core()
{
    batch.reset();
    destroy();
}

static int batch_setup(Core& c)
{
    if (!c.batch) c.batch = std::make_unique<BatchState>();
    BatchState& b = *c.batch;
    if (b.gen == c.config_gen) return WCT_OK;
    b.drop_graph();
    const int np = (int)c.planes.size();
    BatchStatic& bs = b.bs;
    bs = BatchStatic{};
    bs.np = np;
    bs.nticks = c.nticks();
    bs.ntiles = (bs.nticks + kTile - 1) / kTile;
    int nwt = 0, minpad = 1 << 30;
    size_t nneed = 0;
    for (auto& ps : c.planes) {
        nwt += ps->desc.nwires;
        minpad = std::min(minpad, ps->waveform_pad);
        // longest reference time window: end_tick - start_tick <= nticks + 4
        nneed = std::max(nneed, fft_best_length((size_t)bs.nticks + 4 + ps->waveform_pad, false));
    }
    bs.nkeys = nwt * bs.ntiles;
    bs.start_time = c.start_time;
    bs.tbs = (c.start_time + c.readout_time - c.start_time) / (int)(c.readout_time / c.tick);
    // ladder of time-FFT lengths from the shortest possible window up
    std::vector<int> cls;
    const int nfirst = gpu_fft_length(std::max(64, (int)fft_best_length((size_t)4 + std::max(minpad, 0), false)));
    for (double ratio = 1.1;; ratio *= 1.05) {
        cls.clear();
        int N = nfirst;
        for (;;) {
            cls.push_back(N);
            if ((size_t)N >= nneed) break;
            N = gpu_fft_length(std::max((int)std::ceil(N * ratio), N + 4));
        }
        if ((int)cls.size() <= kMaxClasses) break;
    }
    bs.ncls = (int)cls.size();
    for (int k = 0; k < bs.ncls; ++k) bs.cls_N[k] = cls[k];
    b.maxM = cls.back() / 2;
    b.cls_plans.clear();
    std::vector<FftDesc> descs;
    for (int N : cls) {
        auto pl = std::make_unique<FftPlanDev>();
        int rc = make_plan(N / 2, *pl);
        if (rc) return rc;
        descs.push_back(pl->desc);
        b.cls_plans.push_back(std::move(pl));
    }
    CUDA_TRY(b.d_descs.ensure(sizeof(FftDesc) * descs.size()));
    CUDA_TRY(cudaMemcpy(b.d_descs.p, descs.data(), sizeof(FftDesc) * descs.size(), cudaMemcpyHostToDevice));
    long long q = 0, v = 0;
    b.maxG = 0;
    b.spec.clear();
    std::vector<const float2*> tab((size_t)np * bs.ncls);
    for (int ip = 0; ip < np; ++ip) {
        PlaneState& ps = *c.planes[ip];
        BatchPlaneStatic& pl = bs.pl[ip];
        pl.G = ps.G;
        pl.npad = ps.npad;
        pl.waveform_pad = ps.waveform_pad;
        pl.nwires = ps.desc.nwires;
        pl.imp_nbins = ps.dev.imp_nbins;
        pl.row0 = ps.row0;
        pl.nin_max = ps.desc.nwires + 4;  // end_ch - start_ch of any window
        pl.imp_min = ps.dev.imp_min;
        pl.imp_bs = ps.dev.imp_bs;
        pl.qslot = q;
        pl.vslot = v;
        q += (long long)ps.G * pl.nin_max * cls.back();
        v += (long long)(pl.nin_max + 2 * ps.npad) * b.maxM;
        b.maxG = std::max(b.maxG, ps.G);
        const int rows = ps.G * (2 * ps.npad + 1);
        for (int k = 0; k < bs.ncls; ++k) {
            const int N = cls[k];
            auto sp = std::make_unique<DevBuf>();
            CUDA_TRY(sp->ensure(sizeof(float2) * (size_t)rows * (N / 2)));
            launch_rfft_rows(ps.d_table.as<float>(), ps.ldr, std::min(ps.nresp, N), sp->as<float2>(), N / 2, rows,
                             b.cls_plans[k]->desc, c.own_stream);
            CUDA_TRY(cudaGetLastError());
            tab[(size_t)ip * bs.ncls + k] = sp->as<float2>();
            b.spec.push_back(std::move(sp));
        }
    }
    bs.qslot_total = q;
    bs.vslot_total = v;
    CUDA_TRY(b.d_spec_tab.ensure(sizeof(const float2*) * tab.size()));
    CUDA_TRY(cudaMemcpyAsync(b.d_spec_tab.p, tab.data(), sizeof(const float2*) * tab.size(), cudaMemcpyHostToDevice,
                             c.own_stream));
    CUDA_TRY(cudaStreamSynchronize(c.own_stream));
    CUDA_TRY(cudaDeviceGetAttribute(&b.nsm, cudaDevAttrMultiProcessorCount, c.device));
    batch_kernel_attributes(b.maxG, b.maxM);
    CUDA_TRY(cudaGetLastError());
    b.gen = c.config_gen;
    return WCT_OK;
}

// Device bytes of one event slot (charge grids, V rows, per-event keys).
constexpr long long kMaxPassDepos = 16LL << 20;  // depos per pass of the batched path

static size_t batch_slot_bytes(const BatchState& b)
{
    const BatchStatic& bs = b.bs;
    return sizeof(float) * (size_t)bs.qslot_total + sizeof(float2) * (size_t)bs.vslot_total +
           (sizeof(int) * 3 + sizeof(unsigned long long) * kTileBlocks) * (size_t)bs.nkeys;
}

static int batch_slots(Core& c, int nev)
{
    BatchState& b = *c.batch;
    int K = std::max(1, std::min({b.tune.slots, kMaxBatch, nev}));
    size_t fre = 0, tot = 0;
    if (cudaMemGetInfo(&fre, &tot) == cudaSuccess) {
        // keep the arenas within about half of what is free (plus what they hold already)
        const size_t held = b.d_Q.n + b.d_V.n;
        const size_t budget = (fre + held) / 2;
        const size_t per = std::max<size_t>(batch_slot_bytes(b), 1);
        K = std::max(1, std::min<int>(K, (int)(budget / per)));
    }
    return K;
}

static int forward_batch_device(Core& c, const double* d_depos, const long long* offsets, int nev, float* d_frames,
                                wct_plane_window* wins, int* first_ident, cudaStream_t s)
{
    if (c.planes.empty()) return fail(WCT_ERR_STATE, "no planes configured");
    if ((int)c.planes.size() > kMaxPlanes) return fail(WCT_ERR_CONFIG, "too many planes for one component");
    for (auto& p : c.planes)
        if (!p->have_resp) return fail(WCT_ERR_STATE, "a plane has no response");
    if (nev < 0 || !offsets || (nev > 0 && !d_frames)) return fail(WCT_ERR_ARG, "forward batch: bad arguments");
    if (offsets[0] != 0) return fail(WCT_ERR_ARG, "forward batch: offsets[0] must be 0");
    for (int e = 0; e < nev; ++e)
        if (offsets[e + 1] < offsets[e]) return fail(WCT_ERR_ARG, "forward batch: offsets must not decrease");
    if (nev > 0 && offsets[nev] > 0 && !d_depos) return fail(WCT_ERR_ARG, "forward batch: null depos");
    if (c.have_qscale && ((size_t)offsets[nev] != c.qscale_n || c.qscale_planes != (int)c.planes.size()))
        return fail(WCT_ERR_ARG, "the charge scale was set for another depo count or plane set");
    if (first_ident) *first_ident = c.frame_count;
    if (nev == 0) return WCT_OK;
    CUDA_TRY(cudaSetDevice(c.device));
    int rc = batch_setup(c);
    if (rc) return rc;
    BatchState& b = *c.batch;
    const BatchStatic& bs = b.bs;
    const int np = bs.np;
    int K = batch_slots(c, nev);
    int nch = 1;
    long long maxdep = 1;
    // events per pass: K, fewer while a pass would hold more than kMaxPassDepos
    // depos (bounded work arrays; their visit lists keep int offsets)
    auto layout = [&]() {
        for (;;) {
            nch = (nev + K - 1) / K;
            maxdep = 1;
            for (int c0 = 0; c0 < nev; c0 += K)
                maxdep = std::max(maxdep, offsets[std::min(nev, c0 + K)] - offsets[c0]);
            if (K == 1 || maxdep <= kMaxPassDepos) return;
            K = std::max(1, K / 2);
        }
    };
    layout();
    if (maxdep > 0x7fffff00LL) return fail(WCT_ERR_SIZE, "forward batch: too many depos in one event");
    const long long fstride = (long long)c.nrows() * bs.nticks;
    const long long est = 6LL * np * maxdep + 4096;
    if (b.vcap < est) b.vcap = est;
    PlaneSet pset{};
    pset.nplanes = np;
    {
        int nwt = 0;
        for (int ip = 0; ip < np; ++ip) {
            pset.p[ip] = c.planes[ip]->dev;
            pset.p[ip].wire_base = nwt;
            nwt += c.planes[ip]->desc.nwires;
        }
        pset.nwires_total = nwt;
        pset.ntiles = bs.ntiles;
    }
    TimeDev tb;
    tb.nbins = bs.nticks;
    tb.tmin = c.start_time;
    tb.tmax = c.start_time + c.readout_time;
    tb.bs = (tb.tmax - tb.tmin) / tb.nbins;
    for (int attempt = 0; attempt < 8; ++attempt) {
        const long long nkeysK = (long long)K * bs.nkeys;
        std::vector<void*> before = {b.d_Q.p, b.d_V.p, b.d_rec.p, b.d_tprof.p, b.d_win.p, b.d_wcnt.p, b.d_woff.p,
                                     b.d_wcur.p, b.d_kbound.p, b.d_wlist.p, b.d_plans.p, b.d_fq.p, b.d_fluc.p,
                                     b.d_ident.p, b.d_pool.p, b.d_pool_off.p, b.d_pool_used.p, b.d_wide.p,
                                     const_cast<double*>(c.qscale())};
        CUDA_TRY(b.d_Q.ensure(sizeof(float) * (size_t)bs.qslot_total * K));
        CUDA_TRY(b.d_V.ensure(sizeof(float2) * (size_t)bs.vslot_total * K));
        CUDA_TRY(b.d_rec.ensure(sizeof(PatchRec) * (size_t)np * maxdep));
        CUDA_TRY(b.d_tprof.ensure(sizeof(float) * kTprof * (size_t)maxdep));
        CUDA_TRY(b.d_win.ensure(sizeof(WindowDev) * (size_t)K * np));
        CUDA_TRY(b.d_wcnt.ensure(sizeof(int) * (size_t)(nkeysK + 1)));
        CUDA_TRY(b.d_woff.ensure(sizeof(int) * (size_t)(nkeysK + 1)));
        CUDA_TRY(b.d_wcur.ensure(sizeof(int) * (size_t)(nkeysK + 1 + (nkeysK + 1023) / 1024)));
        CUDA_TRY(b.d_kbound.ensure(sizeof(unsigned long long) * (size_t)nkeysK * kTileBlocks));
        CUDA_TRY(b.d_wide.ensure((size_t)nkeysK));
        CUDA_TRY(b.d_wlist.ensure(sizeof(Visit) * (size_t)b.vcap));
        CUDA_TRY(b.d_plans.ensure(sizeof(BatchPlan) * (size_t)nch));
        CUDA_TRY(b.d_ident.ensure(sizeof(int)));
        if (b.pool_cap < 32 * maxdep) b.pool_cap = 32 * maxdep;
        b.pool_cap = std::min<long long>(b.pool_cap, 0x7ffffffeLL);  // int offsets
        CUDA_TRY(b.d_pool.ensure(sizeof(float) * (size_t)b.pool_cap));
        CUDA_TRY(b.d_pool_off.ensure(sizeof(int) * (size_t)maxdep));
        CUDA_TRY(b.d_pool_used.ensure(sizeof(unsigned long long)));
        if (c.fluctuate) {
            CUDA_TRY(b.d_fq.ensure(sizeof(double) * (size_t)np * maxdep));
            CUDA_TRY(b.d_fluc.ensure(sizeof(FlucRec) * (size_t)np * maxdep));
        }
        if (!b.h_ident) CUDA_TRY(cudaMallocHost(&b.h_ident, sizeof(int)));
        std::vector<void*> after = {b.d_Q.p, b.d_V.p, b.d_rec.p, b.d_tprof.p, b.d_win.p, b.d_wcnt.p, b.d_woff.p,
                                    b.d_wcur.p, b.d_kbound.p, b.d_wlist.p, b.d_plans.p, b.d_fq.p, b.d_fluc.p,
                                    b.d_ident.p, b.d_pool.p, b.d_pool_off.p, b.d_pool_used.p, b.d_wide.p,
                                    const_cast<double*>(c.qscale())};
        if (b.h_plans_n < (size_t)nch) {
            if (b.h_plans) cudaFreeHost(b.h_plans);
            b.h_plans = nullptr;
            CUDA_TRY(cudaMallocHost(&b.h_plans, sizeof(BatchPlan) * (size_t)nch));
            b.h_plans_n = nch;
        }
        const bool same = b.exec && before == after && after == b.g_bufs && b.g_depos == d_depos &&
                          b.g_frames == d_frames && b.g_stream == s && b.g_vcap == b.vcap &&
                          std::memcmp(&b.g_tune, &b.tune, sizeof(BatchTune)) == 0 &&
                          std::memcmp(&b.g_drift, &c.drifter, sizeof(DriftDev)) == 0 &&
                          b.g_fluc[0] == (int)c.fluctuate && b.g_fluc[1] == (int)c.drift_fluctuate &&
                          b.g_seed == c.seed && b.g_pool_cap == b.pool_cap &&
                          b.g_offsets.size() == (size_t)nev + 1 &&
                          std::equal(b.g_offsets.begin(), b.g_offsets.end(), offsets);
        if (!same) {
            b.drop_graph();
            cudaGraph_t graph = nullptr;
            CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            BatchPlan* plans = b.d_plans.as<BatchPlan>();
            const int nb_r = std::max(1, b.nsm * b.tune.raster_per_sm);
            const int nb_f = std::max(1, b.nsm * b.tune.fft_per_sm);
            const int nb_c = std::max(1, b.nsm * b.tune.conv_per_sm);
            for (int ch = 0; ch < nch; ++ch) {
                const int c0 = ch * K, c1 = std::min(nev, c0 + K), ne = c1 - c0;
                EventTable et{};
                et.nev = ne;
                int blk = 0;
                for (int j = 0; j <= ne; ++j) {
                    et.dep0[j] = (int)(offsets[c0 + j] - offsets[c0]);
                    et.blk0[j] = blk;
                    if (j < ne) blk += (int)((offsets[c0 + j + 1] - offsets[c0 + j] + 255) / 256);
                }
                const long long nk = (long long)ne * bs.nkeys;
                const double* dep = d_depos ? d_depos + 7 * offsets[c0] : nullptr;
                cudaMemsetAsync(b.d_wcnt.p, 0, sizeof(int) * (size_t)(nk + 1), s);
                cudaMemsetAsync(b.d_kbound.p, 0, sizeof(unsigned long long) * (size_t)nk * kTileBlocks, s);
                cudaMemsetAsync(b.d_wide.p, 0, (size_t)nk, s);
                k_win_init<<<(ne * np + 63) / 64, 64, 0, s>>>(b.d_win.as<WindowDev>(), ne * np);
                // random streams keyed by the frame ident of each event: base (a device
                // value written before every launch of the graph) + c0 + event
                const FlucParams fp = fluc_params(c, true, c0, b.d_ident.as<int>());
                launch_prep_all(dep, et, bs.nkeys, c.drifter, c.have_drifter ? 1 : 0, pset, tb, c.drift_speed,
                                c.nsigma, b.d_rec.as<PatchRec>(), b.d_win.as<WindowDev>(), b.d_wcnt.as<int>(),
                                b.d_tprof.as<float>(), b.d_kbound.as<unsigned long long>(), fp,
                                fp.on_patch ? b.d_fq.as<double>() : nullptr, b.d_wide.as<unsigned char>(), s, 0, -1,
                                c.qscale() ? c.qscale() + (size_t)offsets[c0] * np : nullptr);
                launch_scan(b.d_wcnt.as<int>(), (int)nk, b.d_woff.as<int>(), b.d_wcur.as<int>(), s);
                launch_plan_batch(plans + ch, bs, ne, b.d_win.as<WindowDev>(), b.vcap, s);
                launch_fill(b.d_rec.as<PatchRec>(), et, bs.nkeys, pset, b.d_wcur.as<int>(), b.d_wlist.as<Visit>(),
                            b.vcap, s);
                cudaMemsetAsync(d_frames + c0 * fstride, 0, sizeof(float) * (size_t)(ne * fstride), s);
                const TprofPool pool{b.d_pool.as<float>(), b.d_pool_off.as<int>(),
                                     b.d_pool_used.as<unsigned long long>(), b.pool_cap};
                if (fp.on_patch)
                    launch_fluc_sums(b.d_rec.as<PatchRec>(), et, pset, (float)tb.bs, fp, b.d_fq.as<double>(),
                                     b.d_fluc.as<FlucRec>(), s);
                else {
                    cudaMemsetAsync(b.d_pool_used.p, 0, sizeof(unsigned long long), s);
                    launch_tprof_pool(b.d_rec.as<PatchRec>(), et, np, (float)tb.bs, pool, &plans[ch].status, s);
                }
                launch_raster_batch(plans + ch, bs, pset, b.d_rec.as<PatchRec>(), et.dep0[ne], b.d_tprof.as<float>(),
                                    pool, b.d_wide.as<unsigned char>(), b.d_wcnt.as<int>(), b.d_woff.as<int>(), b.d_wlist.as<Visit>(), b.vcap,
                                    b.d_kbound.as<unsigned long long>(), b.d_Q.as<float>(), nb_r, b.maxG, et, fp,
                                    b.d_fluc.as<FlucRec>(), s);
                launch_rfft_batch(plans + ch, b.d_descs.as<FftDesc>(), b.d_Q.as<float>(), nb_f, b.tune.fft_threads,
                                  b.maxM, s);
                // one launch per run of planes that share the pad and the group pairing
                // (the launches use one work counter, so they must not overlap: same stream)
                for (int ip0 = 0; ip0 < np;) {
                    int ip1 = ip0 + 1;
                    while (ip1 < np && c.planes[ip1]->npad == c.planes[ip0]->npad &&
                           c.planes[ip1]->mirror == c.planes[ip0]->mirror)
                        ++ip1;
                    launch_conv_batch(plans + ch, bs, ip0, ip1, c.planes[ip0]->mirror,
                                      b.d_spec_tab.as<const float2*>(), b.d_Q.as<float>(), b.d_V.as<float2>(), nb_c, s);
                    ip0 = ip1;
                }
                launch_irfft_batch(plans + ch, bs, b.d_descs.as<FftDesc>(), b.d_V.as<float2>(), d_frames + c0 * fstride,
                                   fstride, nb_f, b.tune.fft_threads, b.maxM, s);
            }
            cudaError_t ce = cudaStreamEndCapture(s, &graph);
            if (ce != cudaSuccess) {
                if (graph) cudaGraphDestroy(graph);
                return fail(WCT_ERR_CUDA, std::string("forward batch: graph capture: ") + cudaGetErrorString(ce));
            }
            ce = cudaGraphInstantiate(&b.exec, graph, 0);
            cudaGraphDestroy(graph);
            if (ce != cudaSuccess) {
                b.exec = nullptr;
                return fail(WCT_ERR_CUDA, std::string("forward batch: graph instantiate: ") + cudaGetErrorString(ce));
            }
            b.g_bufs = after;
            b.g_depos = d_depos;
            b.g_frames = d_frames;
            b.g_stream = s;
            b.g_vcap = b.vcap;
            b.g_tune = b.tune;
            b.g_drift = c.drifter;
            b.g_fluc[0] = (int)c.fluctuate;
            b.g_fluc[1] = (int)c.drift_fluctuate;
            b.g_seed = c.seed;
            b.g_pool_cap = b.pool_cap;
            b.g_offsets.assign(offsets, offsets + nev + 1);
        }
        *b.h_ident = c.frame_count;
        CUDA_TRY(cudaMemcpyAsync(b.d_ident.p, b.h_ident, sizeof(int), cudaMemcpyHostToDevice, s));
        CUDA_TRY(cudaGraphLaunch(b.exec, s));
        // statuses (and windows when asked for) of every pass
        const size_t head = offsetof(BatchPlan, pre_raster);
        for (int ch = 0; ch < nch; ++ch) {
            const size_t bytes = wins ? sizeof(BatchPlan) : head;
            CUDA_TRY(cudaMemcpyAsync(b.h_plans + ch, b.d_plans.as<BatchPlan>() + ch, bytes, cudaMemcpyDeviceToHost, s));
        }
        CUDA_TRY(cudaStreamSynchronize(s));
        int st = 0;
        long long need = 0;
        for (int ch = 0; ch < nch; ++ch) {
            st |= b.h_plans[ch].status;
            need = std::max<long long>(need, b.h_plans[ch].total_visits);
        }
        if (st & kBatchPoolShort) b.pool_cap *= 2;  // frames are right; the next call gets more room
        if (st & kBatchTooBig) {  // 2^31 visits in a pass: fewer events per pass
            if (K == 1) return fail(WCT_ERR_SIZE, "an event holds 2^31 or more patch visits; split it");
            K = std::max(1, K / 2);
            layout();
            b.drop_graph();
            continue;
        }
        if (st & kBatchVisitOverflow) {
            b.vcap = need + need / 4 + 4096;  // grow the visit list and run again
            continue;
        }
        if (st & kBatchOversize) return fail(WCT_ERR_SIZE, "a diffusion patch exceeds 1024 ticks or 1024 impact bins");
        if (st & kBatchBigCharge) return fail(WCT_ERR_SIZE, "a depo charge exceeds 5e11 electrons");
        if (st & kBatchNoClass) return fail(WCT_ERR_SIZE, "forward batch: a window exceeds the time-FFT ladder");
        // long-range step on every plane with one (rows outside an event's window are zero and stay zero)
        for (int ip = 0; ip < np; ++ip) {
            PlaneState& ps = *c.planes[ip];
            if (ps.long_wf.empty()) continue;
            const int nticks = c.nticks();
            for (int e = 0; e < nev; ++e) {
                int rc2 = long_conv_rows(c, ps, d_frames + (size_t)e * c.nrows() * nticks + (size_t)ps.row0 * nticks,
                                         nticks, ps.desc.nwires, nticks, false, s);
                if (rc2) return rc2;
            }
        }
        if (wins) {
            for (int e = 0; e < nev; ++e) {
                const BatchPlan& P = b.h_plans[e / K];
                for (int ip = 0; ip < np; ++ip) {
                    const EvPlane& E = P.ep[(e % K) * np + ip];
                    const PlaneState& ps = *c.planes[ip];
                    wct_plane_window& o = wins[(size_t)e * np + ip];
                    o.face = ps.face;
                    o.plane = ps.index;
                    o.start_ch = E.m_start_ch;
                    o.end_ch = E.m_end_ch;
                    o.start_tick = E.m_start_tick;
                    o.end_tick = E.m_end_tick;
                    o.nw_fft = E.nw_ref;
                    o.nt_fft = E.nt_ref;
                    o.nt_gpu = E.N;
                    o.charge_rows = E.end_ch - E.start_ch;
                    o.npad = ps.npad;
                    o.ndepos_added = E.ndepos_added;
                    o.outside_time = E.outside_time;
                    o.outside_pitch = E.outside_pitch;
                }
            }
        }
        c.frame_count += nev;
        return WCT_OK;
    }
    return fail(WCT_ERR_SIZE, "forward batch: visit lists kept overflowing");
}

// Coordinate search over the launch shapes of the batched path on the
// caller's batch: each candidate is captured, run once, then timed over three
// graph replays (CUDA events on the stream); the fastest is kept.

// A time in milliseconds as a JSON number, 4 decimals, independent of the
// process locale (printf's %f follows LC_NUMERIC, which a host framework may
// set to a decimal comma).
static std::string json_ms(double ms)
{
    if (!std::isfinite(ms)) return "null";
    char buf[64];
    const auto r = std::to_chars(buf, buf + sizeof buf, ms, std::chars_format::fixed, 4);
    return std::string(buf, r.ptr);
}

static int autotune_batch(Core& c, const double* d_depos, const long long* offsets, int nev, float* d_frames,
                          cudaStream_t s, std::string& report)
{
    if (nev <= 0) return fail(WCT_ERR_ARG, "autotune: empty batch");
    int rc = batch_setup(c);
    if (rc) return rc;
    BatchState& b = *c.batch;
    cudaEvent_t e0, e1;
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    auto measure = [&](float& ms) -> int {
        int r = forward_batch_device(c, d_depos, offsets, nev, d_frames, nullptr, nullptr, s);
        if (r) return r;
        float best = 1e30f;
        for (int k = 0; k < 3; ++k) {
            cudaEventRecord(e0, s);
            r = forward_batch_device(c, d_depos, offsets, nev, d_frames, nullptr, nullptr, s);
            if (r) return r;
            cudaEventRecord(e1, s);
            cudaEventSynchronize(e1);
            float t = 0.f;
            cudaEventElapsedTime(&t, e0, e1);
            best = std::min(best, t);
        }
        ms = best;
        return WCT_OK;
    };
    std::string rows;
    auto note = [&](const BatchTune& t, float ms) {
        char buf[200];
        std::snprintf(buf, sizeof buf,
                      "%s{\"slots\": %d, \"raster_per_sm\": %d, \"fft_threads\": %d, \"fft_per_sm\": %d, "
                      "\"conv_per_sm\": %d, \"ms\": %s}",
                      rows.empty() ? "" : ", ", t.slots, t.raster_per_sm, t.fft_threads, t.fft_per_sm, t.conv_per_sm,
                      json_ms(ms).c_str());
        rows += buf;
    };
    BatchTune best = b.tune;
    float best_ms = 0.f;
    rc = measure(best_ms);
    if (rc) return rc;
    note(best, best_ms);
    const std::vector<std::vector<int>> cand = {
        {4, 8, 16, 32, 64}, {2, 3, 4, 6}, {256, 512}, {2, 3, 4}, {2, 3, 4}};
    for (int par = 0; par < 5; ++par) {
        for (int v : cand[par]) {
            BatchTune t = best;
            int* f[5] = {&t.slots, &t.raster_per_sm, &t.fft_threads, &t.fft_per_sm, &t.conv_per_sm};
            if (*f[par] == v) continue;
            if (par == 0 && v > std::max(nev, 4)) continue;
            *f[par] = v;
            b.tune = t;
            float ms = 0.f;
            rc = measure(ms);
            if (rc) {
                b.tune = best;
                cudaEventDestroy(e0);
                cudaEventDestroy(e1);
                return rc;
            }
            note(t, ms);
            if (ms < best_ms) {
                best_ms = ms;
                best = t;
            }
        }
    }
    b.tune = best;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    char buf[200];
    std::snprintf(buf, sizeof buf,
                  "{\"best\": {\"slots\": %d, \"raster_per_sm\": %d, \"fft_threads\": %d, \"fft_per_sm\": %d, "
                  "\"conv_per_sm\": %d, \"ms\": %s}, \"tried\": [",
                  best.slots, best.raster_per_sm, best.fft_threads, best.fft_per_sm, best.conv_per_sm,
                  json_ms(best_ms).c_str());
    report = std::string(buf) + rows + "]}";
    return WCT_OK;
}

// ---------------------------------------------------------------------------
// GPU IDFT (iface/inc/WireCellIface/IDFT.h; the cuFftDFT plugin that
// cuda/test/test_idft_cufftdft.bats expects): complex single-precision
// transforms, forward unnormalised, inverse with 1/n, C (row-major) order,
// in place allowed.  Lengths whose prime factors are at most 7 use the
// shared-memory FFT directly; any other length goes through Bluestein's
// chirp-z transform with a 7-smooth FFT length >= 2n - 1.  Column transforms
// (axis 0 of the 1b methods, the second pass of the 2d methods) are row
// transforms between two transposes.  Host-pointer calls copy through the
// current device on the per-thread default stream and return when done, so
// several threads may call at once.
// ---------------------------------------------------------------------------
constexpr int kDftMaxFft = 14336;  // longest shared-memory FFT: two buffers of 14336 complex = 224 KB

static bool dft_smooth(long long n)
{
    if (n < 1) return false;
    for (int p : {2, 3, 5, 7})
        while (n % p == 0) n /= p;
    return n == 1;
}

static int dft_bluestein_length(int n)
{
    for (long long P = 2LL * n - 1; P < (1LL << 30); ++P)
        if (dft_smooth(P)) return (int)P;
    return 0;
}

// Four-step split of a 7-smooth N > kDftMaxFft: N = N1 * N2, both <= kDftMaxFft,
// N1 the largest such divisor not above sqrt(N).
static bool four_step_split(int N, int& N1, int& N2)
{
    for (int d = (int)std::sqrt((double)N) + 1; d >= 1; --d) {
        if (N % d || d > kDftMaxFft || N / d > kDftMaxFft || (long long)d * d > N) continue;
        N1 = d;
        N2 = N / d;
        return true;
    }
    return false;
}

// Stream-ordered scratch freed when it goes out of scope.
struct AsyncBuf {
    void* p{nullptr};
    cudaStream_t s{nullptr};
    ~AsyncBuf()
    {
        if (p) cudaFreeAsync(p, s);
    }
};

struct BluesteinDev {
    int N{0}, P{0};
    DevBuf chirp, bhat;
};
static std::mutex g_blue_mtx;
static std::map<std::pair<int, int>, std::unique_ptr<BluesteinDev>> g_bluestein;  // (device, N)

static int dft_rows(const float2* in, long ld_in, float2* out, long ld_out, int nrows, int n, int sign,
                    cudaStream_t s);

// Chirp c_n = exp(-pi i n^2 / N) (phase from n^2 mod 2N, exact in integers)
// and the spectrum of the chirp filter, built once per device and length.
static int bluestein_plan(int N, int& P, const float2*& chirp, const float2*& bhat)
{
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    P = dft_bluestein_length(N);
    if (!P) return fail(WCT_ERR_SIZE, "DFT length " + std::to_string(N) + " too long");
    std::lock_guard<std::mutex> lk(g_blue_mtx);
    auto key = std::make_pair(dev, N);
    auto it = g_bluestein.find(key);
    if (it == g_bluestein.end()) {
        auto b = std::make_unique<BluesteinDev>();
        b->N = N;
        b->P = P;
        std::vector<float2> c(N);
        const double pi = 3.14159265358979323846;
        for (int n = 0; n < N; ++n) {
            const long long q = ((long long)n * n) % (2LL * N);
            const double ph = pi * (double)q / (double)N;
            c[n] = make_float2((float)std::cos(ph), (float)-std::sin(ph));
        }
        CUDA_TRY(b->chirp.ensure(sizeof(float2) * N));
        CUDA_TRY(b->bhat.ensure(sizeof(float2) * P));
        cudaStream_t st = cudaStreamPerThread;
        CUDA_TRY(cudaMemcpyAsync(b->chirp.p, c.data(), sizeof(float2) * N, cudaMemcpyHostToDevice, st));
        launch_bluestein_b(b->chirp.as<float2>(), b->bhat.as<float2>(), N, P, st);
        int rc = dft_rows(b->bhat.as<float2>(), P, b->bhat.as<float2>(), P, 1, P, -1, st);
        if (rc) return rc;
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaStreamSynchronize(st));
        it = g_bluestein.emplace(key, std::move(b)).first;
    }
    chirp = it->second->chirp.as<float2>();
    bhat = it->second->bhat.as<float2>();
    return WCT_OK;
}

// Four-step FFT of contiguous rows of a 7-smooth length N = N1 * N2: column
// transforms of the N1 x N2 view (transpose, rows of N1), twiddles, rows of
// N2, transpose back.  Inverse scales by 1/N (1/N1 * 1/N2).
static int four_step_rows(const float2* in, float2* out, int nrows, int N, int sign, cudaStream_t s)
{
    int N1 = 0, N2 = 0;
    if (!four_step_split(N, N1, N2)) return fail(WCT_ERR_SIZE, "DFT length " + std::to_string(N) + " too long");
    const int chunk = std::max(1, std::min(65535, (int)std::min<long long>(nrows, (1LL << 28) / N)));
    AsyncBuf w;
    w.s = s;
    CUDA_TRY(cudaMallocAsync(&w.p, sizeof(float2) * (size_t)chunk * N, s));
    float2* W = static_cast<float2*>(w.p);
    for (int r0 = 0; r0 < nrows; r0 += chunk) {
        const int nb = std::min(chunk, nrows - r0);
        const float2* src = in + (size_t)r0 * N;
        float2* dst = out + (size_t)r0 * N;
        launch_transpose_c(src, W, N1, N2, s, nb);                       // [N2][N1]
        int rc = dft_rows(W, N1, W, N1, nb * N2, N1, sign, s);          // along n1
        if (rc) return rc;
        launch_twiddle4(W, (long long)nb * N, N1, N2, sign, s);
        launch_transpose_c(W, dst, N2, N1, s, nb);                      // [N1][N2]
        rc = dft_rows(dst, N2, dst, N2, nb * N1, N2, sign, s);          // along n2
        if (rc) return rc;
        launch_transpose_c(dst, W, N1, N2, s, nb);                      // X[k2 * N1 + k1]
        CUDA_TRY(cudaMemcpyAsync(dst, W, sizeof(float2) * (size_t)nb * N, cudaMemcpyDeviceToDevice, s));
    }
    CUDA_TRY(cudaGetLastError());
    return WCT_OK;
}

// nrows transforms of length n along rows (row strides ld_in, ld_out; the
// four-step and long Bluestein paths take contiguous rows).
static int dft_rows(const float2* in, long ld_in, float2* out, long ld_out, int nrows, int n, int sign, cudaStream_t s)
{
    if (nrows <= 0 || n <= 0) return WCT_OK;
    const float scale = sign > 0 ? 1.0f / (float)n : 1.0f;
    if (dft_smooth(n) && n <= kDftMaxFft) {
        FftDesc d;
        int rc = device_plan(n, d);
        if (rc) return rc;
        launch_c2c_rows(in, ld_in, out, ld_out, nrows, d, sign, scale, s);
    }
    else if (dft_smooth(n)) {
        if (ld_in != n || ld_out != n) return fail(WCT_ERR_ARG, "DFT: long rows must be contiguous");
        return four_step_rows(in, out, nrows, n, sign, s);
    }
    else {
        int P = 0;
        const float2 *chirp = nullptr, *bhat = nullptr;
        int rc = bluestein_plan(n, P, chirp, bhat);
        if (rc) return rc;
        if (P <= kDftMaxFft) {
            FftDesc dP;
            rc = device_plan(P, dP);
            if (rc) return rc;
            launch_bluestein_rows(in, ld_in, out, ld_out, nrows, n, dP, chirp, bhat, sign, scale, s);
        }
        else {  // through global memory, the length-P transforms by four steps
            const int chunk = std::max(1, std::min(nrows, (int)std::min<long long>(65535, (1LL << 28) / P)));
            AsyncBuf z;
            z.s = s;
            CUDA_TRY(cudaMallocAsync(&z.p, sizeof(float2) * (size_t)chunk * P, s));
            float2* Z = static_cast<float2*>(z.p);
            for (int r0 = 0; r0 < nrows; r0 += chunk) {
                const int nb = std::min(chunk, nrows - r0);
                launch_blue_pre(in + (size_t)r0 * ld_in, ld_in, Z, nb, n, P, chirp, sign > 0, s);
                rc = dft_rows(Z, P, Z, P, nb, P, -1, s);
                if (rc) return rc;
                launch_cmul_rows(Z, P, nb, bhat, false, s);
                rc = dft_rows(Z, P, Z, P, nb, P, +1, s);  // carries 1/P
                if (rc) return rc;
                launch_blue_post(Z, P, out + (size_t)r0 * ld_out, ld_out, nb, n, chirp, sign > 0, scale, s);
            }
        }
    }
    CUDA_TRY(cudaGetLastError());
    return WCT_OK;
}

static int dft_check(const void* in, const void* out, int nrows, int ncols)
{
    if (!in || !out || nrows < 0 || ncols < 0) return fail(WCT_ERR_ARG, "DFT: null array or negative size");
    if ((long long)nrows * ncols > (1LL << 30)) return fail(WCT_ERR_SIZE, "DFT: array too large");
    return WCT_OK;
}

// Transposes tile the matrix with a grid of 32 x 32 blocks (at most 65535 tiles per side).
static int dft_check_transpose(int nrows, int ncols)
{
    if (nrows > 65535 * 32 || ncols > 65535 * 32) return fail(WCT_ERR_SIZE, "DFT: a side longer than 2097120");
    return WCT_OK;
}

// Transforms along axis 1 (rows) or 0 (columns) of a row-major nrows x ncols array.
static int dft_1b_dev(const float2* in, float2* out, int nrows, int ncols, int axis, int sign, cudaStream_t s)
{
    if (axis != 0 && axis != 1) return fail(WCT_ERR_ARG, "DFT: axis must be 0 or 1");
    if (nrows == 0 || ncols == 0) return WCT_OK;
    if (axis == 1) return dft_rows(in, ncols, out, ncols, nrows, ncols, sign, s);
    int rc0 = dft_check_transpose(nrows, ncols);
    if (rc0) return rc0;
    AsyncBuf t;
    t.s = s;
    CUDA_TRY(cudaMallocAsync(&t.p, sizeof(float2) * (size_t)nrows * ncols, s));
    float2* tp = static_cast<float2*>(t.p);
    launch_transpose_c(in, tp, nrows, ncols, s);
    int rc = dft_rows(tp, nrows, tp, nrows, ncols, nrows, sign, s);
    if (rc) return rc;
    launch_transpose_c(tp, out, ncols, nrows, s);
    CUDA_TRY(cudaGetLastError());
    return WCT_OK;
}

static int dft_2d_dev(const float2* in, float2* out, int nrows, int ncols, int sign, cudaStream_t s)
{
    int rc = dft_1b_dev(in, out, nrows, ncols, 1, sign, s);
    if (rc) return rc;
    return dft_1b_dev(out, out, nrows, ncols, 0, sign, s);
}

static int dft_transpose_dev(const float* in, float* out, int nrows, int ncols, bool cplx, cudaStream_t s)
{
    if (nrows == 0 || ncols == 0) return WCT_OK;
    int rc0 = dft_check_transpose(nrows, ncols);
    if (rc0) return rc0;
    const size_t bytes = (cplx ? sizeof(float2) : sizeof(float)) * (size_t)nrows * ncols;
    AsyncBuf t;
    t.s = s;
    void* dst = out;
    if (in == out) {  // through scratch
        CUDA_TRY(cudaMallocAsync(&t.p, bytes, s));
        dst = t.p;
    }
    if (cplx)
        launch_transpose_c(reinterpret_cast<const float2*>(in), static_cast<float2*>(dst), nrows, ncols, s);
    else
        launch_transpose_r(in, static_cast<float*>(dst), nrows, ncols, s);
    CUDA_TRY(cudaGetLastError());
    if (dst != out) CUDA_TRY(cudaMemcpyAsync(out, dst, bytes, cudaMemcpyDeviceToDevice, s));
    return WCT_OK;
}

// Host arrays: copy in, transform on the current device, copy out.
// kind 0: 1b (axis), 1: 2d, 2: transpose (cplx).
static int dft_host(const float* in, float* out, int nrows, int ncols, int kind, int axis, int sign, bool cplx)
{
    int rc = dft_check(in, out, nrows, ncols);
    if (rc) return rc;
    if (nrows == 0 || ncols == 0) return WCT_OK;
    cudaStream_t s = cudaStreamPerThread;
    const size_t bytes = (cplx ? sizeof(float2) : sizeof(float)) * (size_t)nrows * ncols;
    {
        AsyncBuf d;
        d.s = s;
        CUDA_TRY(cudaMallocAsync(&d.p, bytes, s));
        CUDA_TRY(cudaMemcpyAsync(d.p, in, bytes, cudaMemcpyHostToDevice, s));
        float2* dp = static_cast<float2*>(d.p);
        if (kind == 0) rc = dft_1b_dev(dp, dp, nrows, ncols, axis, sign, s);
        else if (kind == 1) rc = dft_2d_dev(dp, dp, nrows, ncols, sign, s);
        else rc = dft_transpose_dev(static_cast<float*>(d.p), static_cast<float*>(d.p), nrows, ncols, cplx, s);
        if (rc) return rc;
        CUDA_TRY(cudaMemcpyAsync(out, d.p, bytes, cudaMemcpyDeviceToHost, s));
    }
    CUDA_TRY(cudaStreamSynchronize(s));
    return WCT_OK;
}

}  // namespace wctb200

using namespace wctb200;

struct wct_depotransform {
    Core core;
};
struct wct_pir {
    Pir pir;
};

extern "C" {

const char* wct_version(void) { return "wctb200 0.1 (sm_100a)"; }
const char* wct_last_error(void) { return g_last_error; }

int wct_pir_create(const wct_fr_plane* fr, int nshort, const int* short_len, const double* short_wave,
                   double overall_short_padding, double tick, int nticks, wct_pir** out)
{
    if (!fr || !out || !fr->pitchpos || !fr->current || fr->npaths <= 0 || fr->nsamples <= 0 || nticks <= 0 ||
        tick <= 0 || nshort < 0 || (nshort && (!short_len || !short_wave)))
        return fail(WCT_ERR_ARG, "wct_pir_create: bad arguments");
    for (int i = 0; i < nshort; ++i)
        if (short_len[i] < 0) return fail(WCT_ERR_ARG, "wct_pir_create: negative short response length");
    try {
        std::vector<std::vector<double>> shorts;
        size_t off = 0;
        for (int i = 0; i < nshort; ++i) {
            shorts.emplace_back(short_wave + off, short_wave + off + short_len[i]);
            off += short_len[i];
        }
        auto p = std::make_unique<wct_pir>();
        p->pir = build_pir(fr->npaths, fr->nsamples, fr->pitchpos, fr->current, fr->pitch, fr->tstart, fr->period,
                           shorts, overall_short_padding, tick, nticks);
        *out = p.release();
        return WCT_OK;
    }
    catch (std::exception& e) {
        return fail(WCT_ERR_CONFIG, e.what());
    }
}

// The spectrum product of nw real responses (concatenated in wave, lengths
// len; each cut or zero padded to n), and optionally its real inverse: the
// reference's "short_spec" / "long_spec" chain (PlaneImpactResponse.cxx:96-146)
// in single precision on the current device.  spec receives the product
// spectrum [n]; real (optional, host) the real inverse [n].
static int response_chain_device(int nw, const int* len, const double* wave, int n, DevBuf& spec, float* real,
                                 cudaStream_t s)
{
    std::vector<float2> rows((size_t)nw * n, make_float2(0.f, 0.f));
    size_t off = 0;
    for (int i = 0; i < nw; ++i) {
        for (int k = 0; k < n && k < len[i]; ++k) rows[(size_t)i * n + k].x = (float)wave[off + k];
        off += len[i];
    }
    DevBuf d_rows, d_out;
    CUDA_TRY(d_rows.ensure(sizeof(float2) * rows.size()));
    CUDA_TRY(spec.ensure(sizeof(float2) * (size_t)n));
    CUDA_TRY(cudaMemcpyAsync(d_rows.p, rows.data(), sizeof(float2) * rows.size(), cudaMemcpyHostToDevice, s));
    int rc = dft_rows(d_rows.as<float2>(), n, d_rows.as<float2>(), n, nw, n, -1, s);
    if (rc) return rc;
    launch_spec_chain(d_rows.as<float2>(), nw, n, spec.as<float2>(), s);
    if (real) {
        CUDA_TRY(d_out.ensure(sizeof(float) * (size_t)n));
        rc = dft_rows(spec.as<float2>(), n, d_rows.as<float2>(), n, 1, n, +1, s);
        if (rc) return rc;
        launch_real_rows(d_rows.as<float2>(), 1, n, d_out.as<float>(), n, s);
        CUDA_TRY(cudaMemcpyAsync(real, d_out.p, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost, s));
    }
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(s));  // rows, d_rows and d_out go out of scope
    return WCT_OK;
}

int wct_pir_create_device(const wct_fr_plane* fr, int nshort, const int* short_len, const double* short_wave,
                          double overall_short_padding, double tick, int nticks, wct_pir** out)
{
    if (!fr || !out || !fr->pitchpos || !fr->current || fr->npaths <= 0 || fr->nsamples <= 0 || nticks <= 0 ||
        tick <= 0 || nshort < 0 || (nshort && (!short_len || !short_wave)))
        return fail(WCT_ERR_ARG, "wct_pir_create_device: bad arguments");
    for (int i = 0; i < nshort; ++i)
        if (short_len[i] < 0) return fail(WCT_ERR_ARG, "wct_pir_create_device: negative short response length");
    std::unique_ptr<wct_pir> p;
    try {
        p = std::make_unique<wct_pir>();
        p->pir = build_pir_layout(fr->npaths, fr->nsamples, fr->pitchpos, fr->pitch, fr->tstart, fr->period,
                                  overall_short_padding, tick, nticks);
    }
    catch (std::exception& e) {
        return fail(WCT_ERR_CONFIG, e.what());
    }
    Pir& pir = p->pir;
    const int n = pir.n_short, np = fr->npaths;
    cudaStream_t s = cudaStreamPerThread;
    DevBuf d_short, d_cur, d_Z, d_wf;
    // short responses: the product of their spectra (PlaneImpactResponse.cxx:96-121)
    if (nshort) {
        int rc = response_chain_device(nshort, short_len, short_wave, n, d_short, nullptr, s);
        if (rc) return rc;
    }
    // each path: tick-binned charge, spectrum x short spectrum, real inverse, cut to nticks (:185-240)
    CUDA_TRY(d_cur.ensure(sizeof(double) * (size_t)np * fr->nsamples));
    CUDA_TRY(d_Z.ensure(sizeof(float2) * (size_t)np * n));
    CUDA_TRY(d_wf.ensure(sizeof(float) * (size_t)np * nticks));
    CUDA_TRY(cudaMemcpyAsync(d_cur.p, fr->current, sizeof(double) * (size_t)np * fr->nsamples,
                             cudaMemcpyHostToDevice, s));
    const double rawbs = (fr->tstart + fr->nsamples * fr->period - fr->tstart) / fr->nsamples;  // Binning
    launch_pir_bin(d_cur.as<double>(), np, fr->nsamples, fr->tstart, rawbs, fr->period, tick, n, d_Z.as<float2>(), s);
    if (nshort) {
        int rc = dft_rows(d_Z.as<float2>(), n, d_Z.as<float2>(), n, np, n, -1, s);
        if (rc) return rc;
        launch_cmul_rows(d_Z.as<float2>(), n, np, d_short.as<float2>(), false, s);
        rc = dft_rows(d_Z.as<float2>(), n, d_Z.as<float2>(), n, np, n, +1, s);
        if (rc) return rc;
    }
    launch_real_rows(d_Z.as<float2>(), np, n, d_wf.as<float>(), nticks, s);
    std::vector<float> wf((size_t)np * nticks);
    CUDA_TRY(cudaMemcpyAsync(wf.data(), d_wf.p, sizeof(float) * wf.size(), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(s));
    for (int ip = 0; ip < np; ++ip)
        pir.waveform[ip].assign(wf.begin() + (size_t)ip * nticks, wf.begin() + (size_t)(ip + 1) * nticks);
    *out = p.release();
    return WCT_OK;
}

int wct_pir_set_long_responses_device(wct_pir* p, int nlong, const int* long_len, const double* long_wave,
                                      double long_padding)
{
    if (!p || nlong < 0 || (nlong && (!long_len || !long_wave)) || long_padding < 0)
        return fail(WCT_ERR_ARG, "wct_pir_set_long_responses_device: bad arguments");
    for (int i = 0; i < nlong; ++i)
        if (long_len[i] < 0) return fail(WCT_ERR_ARG, "wct_pir_set_long_responses_device: negative length");
    Pir& pir = p->pir;
    pir.long_wf.clear();
    pir.long_pad = 0;
    if (nlong == 0) return WCT_OK;
    const int n = (int)fft_best_length((size_t)pir.nticks, false);
    std::vector<float> wf(n);
    DevBuf spec;
    int rc = response_chain_device(nlong, long_len, long_wave, n, spec, wf.data(), cudaStreamPerThread);
    if (rc) return rc;
    pir.long_wf.assign(wf.begin(), wf.end());
    pir.long_pad = (int)(long_padding / pir.tick);
    return WCT_OK;
}

int wct_pir_set_long_responses(wct_pir* p, int nlong, const int* long_len, const double* long_wave,
                               double long_padding)
{
    if (!p || nlong < 0 || (nlong && (!long_len || !long_wave)) || long_padding < 0)
        return fail(WCT_ERR_ARG, "wct_pir_set_long_responses: bad arguments");
    for (int i = 0; i < nlong; ++i)
        if (long_len[i] < 0) return fail(WCT_ERR_ARG, "wct_pir_set_long_responses: negative length");
    try {
        std::vector<std::vector<double>> longs;
        size_t off = 0;
        for (int i = 0; i < nlong; ++i) {
            longs.emplace_back(long_wave + off, long_wave + off + long_len[i]);
            off += long_len[i];
        }
        set_long_responses(p->pir, longs, long_padding);
        return WCT_OK;
    }
    catch (std::exception& e) {
        return fail(WCT_ERR_CONFIG, e.what());
    }
}

int wct_pir_long_info(const wct_pir* p, int* nsamples, int* pad)
{
    if (!p) return fail(WCT_ERR_ARG, "wct_pir_long_info: null pir");
    if (nsamples) *nsamples = (int)p->pir.long_wf.size();
    if (pad) *pad = p->pir.long_pad;
    return WCT_OK;
}

int wct_pir_long_waveform(const wct_pir* p, float* out)
{
    if (!p || (!out && !p->pir.long_wf.empty())) return fail(WCT_ERR_ARG, "wct_pir_long_waveform: bad arguments");
    std::copy(p->pir.long_wf.begin(), p->pir.long_wf.end(), out);
    return WCT_OK;
}

long wct_fft_best_length(long n, int keep_odd_even)
{
    if (n < 0) return 0;
    return (long)fft_best_length((size_t)n, keep_odd_even != 0);
}

int wct_pir_closest(const wct_pir* p, double relpitch, int* path)
{
    if (!p || !path) return fail(WCT_ERR_ARG, "wct_pir_closest: bad arguments");
    int k = p->pir.closest(relpitch);
    if (k < 0) return fail(WCT_ERR_RESPONSE, "relative pitch outside PIR extent");
    *path = k;
    return WCT_OK;
}

int wct_pir_info(const wct_pir* p, double* pitch, double* impact, double* half_extent, int* nwires,
                 int* nimp_per_wire, int* npaths, int* nticks, int* waveform_pad)
{
    if (!p) return fail(WCT_ERR_ARG, "wct_pir_info: null pir");
    if (pitch) *pitch = p->pir.pitch;
    if (impact) *impact = p->pir.impact;
    if (half_extent) *half_extent = p->pir.half_extent;
    if (nwires) *nwires = p->pir.nwires();
    if (nimp_per_wire) *nimp_per_wire = p->pir.nimp_per_wire();
    if (npaths) *npaths = (int)p->pir.waveform.size();
    if (nticks) *nticks = p->pir.nticks;
    if (waveform_pad) *waveform_pad = p->pir.waveform_pad;
    return WCT_OK;
}

int wct_pir_waveform(const wct_pir* p, int path, float* out)
{
    if (!p || !out || path < 0 || path >= (int)p->pir.waveform.size())
        return fail(WCT_ERR_ARG, "wct_pir_waveform: bad arguments");
    std::copy(p->pir.waveform[path].begin(), p->pir.waveform[path].end(), out);
    return WCT_OK;
}

int wct_pir_destroy(wct_pir* p)
{
    delete p;
    return WCT_OK;
}

int wct_convolve_rows_device(const float* in, long ld_in, int nrows, int n_in, const float* resp, int n_resp,
                             int nfft, float* out, long ld_out, int n_out, void* stream)
{
    int rc = convolve_args(in, ld_in, nrows, n_in, resp, n_resp, nfft, out, ld_out, n_out);
    if (rc) return rc;
    if (nrows == 0 || n_out == 0) return WCT_OK;
    FftDesc d;
    rc = device_plan(nfft / 2, d);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const int M = nfft / 2;
    float2* scratch = nullptr;
    CUDA_TRY(cudaMallocAsync(&scratch, sizeof(float2) * (size_t)M * (nrows + 1), s));
    rc = convolve_on(in, ld_in, nrows, n_in, resp, n_resp, nfft, out, ld_out, n_out, d, scratch + M, scratch, s);
    cudaError_t e = cudaFreeAsync(scratch, s);
    if (rc) return rc;
    if (e != cudaSuccess) return fail(WCT_ERR_CUDA, cudaGetErrorString(e));
    return WCT_OK;
}

int wct_convolve_rows_device_noalloc(const float* in, long ld_in, int nrows, int n_in, const float* resp,
                                     int n_resp, int nfft, float* out, long ld_out, int n_out, void* stream)
{
    int rc = convolve_args(in, ld_in, nrows, n_in, resp, n_resp, nfft, out, ld_out, n_out);
    if (rc) return rc;
    const size_t M = (size_t)nfft / 2;
    if ((3 + (size_t)nrows) * M > kNoAllocComplex)
        return fail(WCT_ERR_SIZE,
                    "convolve rows (no allocation): (nrows + 3) * nfft / 2 exceeds the fixed scratch of 4194304 "
                    "complex values (32 MiB)");
    if (nrows == 0 || n_out == 0) return WCT_OK;
    float2* base = nullptr;
    rc = noalloc_scratch(&base);
    if (rc) return rc;
    FftDesc d{};
    if (!fft_radices((int)M, d.radix, d.nst)) return fail(WCT_ERR_SIZE, "convolve rows: unsupported FFT length");
    d.M = (int)M;
    float2* tw = base;
    float2* twh = base + M;
    d.tw = tw;
    d.twh = twh;
    cudaStream_t s = (cudaStream_t)stream;
    launch_twiddles(tw, twh, (int)M, s);
    return convolve_on(in, ld_in, nrows, n_in, resp, n_resp, nfft, out, ld_out, n_out, d, base + 3 * M, base + 2 * M,
                       s);
}

int wct_dt_create(const char* json_config, wct_depotransform** out)
{
    if (!out) return fail(WCT_ERR_ARG, "wct_dt_create: null out");
    auto* h = new wct_depotransform;
    int rc = configure(h->core, json_config ? std::string(json_config) : std::string());
    if (rc) {
        delete h;
        return rc;
    }
    cudaError_t e = cudaSetDevice(h->core.device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->core.own_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->core.copy_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete h;
        return fail(WCT_ERR_CUDA, std::string("wct_dt_create: ") + cudaGetErrorString(e));
    }
    *out = h;
    return WCT_OK;
}

int wct_dt_default_configuration(char* buf, size_t len)
{
    const char* js =
        "{\"nsigma\": 3.0, \"fluctuate\": false, \"start_time\": 0.0, \"readout_time\": 5000000.0, "
        "\"tick\": 500.0, \"drift_speed\": 0.001, \"first_frame_number\": 0, \"anode\": \"\", \"rng\": \"\", "
        "\"pirs\": [], \"dft\": \"FftwDFT\"}";
    if (!buf || len <= strlen(js)) return fail(WCT_ERR_ARG, "buffer too small");
    strcpy(buf, js);
    return WCT_OK;
}

int wct_dt_add_face(wct_depotransform* h, const double* lo, const double* hi, int* face)
{
    if (!h) return fail(WCT_ERR_ARG, "null component");
    std::lock_guard<std::mutex> lk(h->core.mtx);
    FaceState f;
    if (lo && hi) {
        f.have_bb = true;
        for (int i = 0; i < 3; ++i) {
            f.lo[i] = lo[i];
            f.hi[i] = hi[i];
        }
    }
    h->core.faces.push_back(f);
    if (face) *face = (int)h->core.faces.size() - 1;
    return WCT_OK;
}

int wct_dt_add_plane(wct_depotransform* h, int face, const wct_plane_desc* d, int* plane)
{
    if (!h || !d) return fail(WCT_ERR_ARG, "wct_dt_add_plane: bad arguments");
    std::lock_guard<std::mutex> lk(h->core.mtx);
    if (face < 0 || face >= (int)h->core.faces.size()) return fail(WCT_ERR_ARG, "wct_dt_add_plane: bad face");
    if (d->nwires < 2 || d->nimpacts < 2 || (d->nimpacts % 2))
        return fail(WCT_ERR_CONFIG, "need >= 2 wires and an even number of impacts per wire");
    if (!(d->pitchmax > d->pitchmin)) return fail(WCT_ERR_CONFIG, "pitchmax must exceed pitchmin");
    Core& c = h->core;
    ++c.config_gen;
    auto ps = std::make_unique<PlaneState>();
    ps->face = face;
    ps->index = (int)c.faces[face].planes.size();
    ps->desc = *d;
    if (d->channels) ps->channels.assign(d->channels, d->channels + d->nwires);
    else {
        ps->channels.resize(d->nwires);
        for (int i = 0; i < d->nwires; ++i) ps->channels[i] = i;
    }
    ps->desc.channels = nullptr;
    // Pimpos (util/src/Pimpos.cxx:5-33) with D3Vector::norm (D3Vector.h:147-154)
    const double* p = d->pitch;
    const double m = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
    if (!(m > 0)) return fail(WCT_ERR_CONFIG, "zero pitch direction");
    PlaneDev& pd = ps->dev;
    pd.ax = p[0] / m;
    pd.ay = p[1] / m;
    pd.az = p[2] / m;
    pd.ox = d->origin[0];
    pd.oy = d->origin[1];
    pd.oz = d->origin[2];
    pd.nwires = d->nwires;
    pd.nimp = d->nimpacts;
    const double regionsize = (d->pitchmax - d->pitchmin) / (d->nwires - 1);
    pd.imp_min = d->pitchmin - 0.5 * regionsize;
    pd.imp_max = d->pitchmax + 0.5 * regionsize;
    pd.imp_nbins = d->nwires * d->nimpacts;
    pd.imp_bs = (pd.imp_max - pd.imp_min) / pd.imp_nbins;
    const FaceState& f = c.faces[face];
    pd.have_bb = f.have_bb ? 1 : 0;
    for (int i = 0; i < 3; ++i) {
        pd.bb_lo[i] = f.lo[i];
        pd.bb_hi[i] = f.hi[i];
    }
    ps->row0 = c.nrows();
    c.faces[face].planes.push_back((int)c.planes.size());
    c.planes.push_back(std::move(ps));
    if (plane) *plane = c.faces[face].planes.size() - 1;
    return WCT_OK;
}

static PlaneState* find_plane(wct_depotransform* h, int face, int plane)
{
    if (!h || face < 0 || face >= (int)h->core.faces.size()) return nullptr;
    auto& f = h->core.faces[face];
    if (plane < 0 || plane >= (int)f.planes.size()) return nullptr;
    return h->core.planes[f.planes[plane]].get();
}

int wct_dt_set_response_table(wct_depotransform* h, int face, int plane, int ngroups, int npad, int nsamples,
                              double pitch, double impact, int waveform_pad, const float* table)
{
    if (!h) return fail(WCT_ERR_ARG, "wct_dt_set_response_table: null component");
    std::lock_guard<std::mutex> lk(h->core.mtx);
    PlaneState* ps = find_plane(h, face, plane);
    if (!ps || !table || ngroups < 3 || npad < 0 || nsamples <= 0)
        return fail(WCT_ERR_ARG, "wct_dt_set_response_table: bad arguments");
    if (ngroups - 1 != ps->desc.nimpacts)
        return fail(WCT_ERR_CONFIG, "response impact groups do not match the plane's impact binning");
    if (ngroups > 12) return fail(WCT_ERR_CONFIG, "at most 12 impact groups (11 impact positions per wire) supported");
    CUDA_TRY(cudaSetDevice(h->core.device));
    ps->G = ngroups;
    ps->npad = npad;
    ps->nresp = nsamples;
    ps->ldr = nsamples + (nsamples & 1);
    ps->pitch = pitch;
    ps->impact = impact;
    ps->waveform_pad = waveform_pad;
    const size_t rows = (size_t)ngroups * (2 * npad + 1);
    std::vector<float> t(rows * ps->ldr, 0.0f);
    for (size_t r = 0; r < rows; ++r) std::copy(table + r * nsamples, table + (r + 1) * nsamples, t.data() + r * ps->ldr);
    CUDA_TRY(ps->d_table.ensure(sizeof(float) * t.size()));
    CUDA_TRY(cudaMemcpy(ps->d_table.p, t.data(), sizeof(float) * t.size(), cudaMemcpyHostToDevice));
    // mirror symmetry of the impact groups (gen/src/PlaneImpactResponse.cxx:256-268)
    bool mirror = true;
    const int J = 2 * npad + 1;
    for (int g = 0; g < ngroups && mirror; ++g) {
        if (2 * g == ngroups - 1) continue;  // the centre group is convolved on its own
        for (int j = 0; j < J && mirror; ++j) {
            const float* a = table + ((size_t)g * J + j) * nsamples;
            const float* b = table + ((size_t)(ngroups - 1 - g) * J + (J - 1 - j)) * nsamples;
            if (std::memcmp(a, b, sizeof(float) * nsamples) != 0) mirror = false;
        }
    }
    ps->mirror = mirror;
    ps->spec_N = 0;
    ps->have_resp = true;
    ++h->core.config_gen;
    return WCT_OK;
}

int wct_dt_set_response_pir(wct_depotransform* h, int face, int plane, const wct_pir* p)
{
    bool have_plane = false;
    if (h) {
        std::lock_guard<std::mutex> lk(h->core.mtx);
        have_plane = find_plane(h, face, plane) != nullptr;
    }
    if (!have_plane || !p) return fail(WCT_ERR_ARG, "wct_dt_set_response_pir: bad arguments");
    const Pir& pir = p->pir;
    // ImpactTransform.cxx:28-74
    const int G = std::round(pir.pitch / pir.impact) + 1;
    const int npad = std::round((pir.nwires() - 1) / 2.);
    const int ns = std::max(1, std::min(pir.nticks, pir.n_short));
    std::vector<float> table((size_t)G * (2 * npad + 1) * ns, 0.0f);
    for (int i = 0; i < G; ++i) {
        double rel;
        if (i != G - 1) rel = -pir.pitch / 2. + pir.impact * i + 1e-9;
        else rel = -pir.pitch / 2. + pir.impact * i - 1e-9;
        for (int j = 0; j < pir.nwires(); ++j) {
            const int k = pir.closest(rel - (j - npad) * pir.pitch);
            if (k < 0) return fail(WCT_ERR_RESPONSE, "ImpactTransform response lookup outside the PIR extent");
            std::copy(pir.waveform[k].begin(), pir.waveform[k].begin() + ns,
                      table.begin() + ((size_t)i * (2 * npad + 1) + j) * ns);
        }
    }
    int rc = wct_dt_set_response_table(h, face, plane, G, npad, ns, pir.pitch, pir.impact, pir.waveform_pad,
                                        table.data());
    if (rc) return rc;
    return wct_dt_set_long_response(h, face, plane, (int)pir.long_wf.size(), pir.long_wf.data(), pir.long_pad);
}

int wct_dt_set_long_response(wct_depotransform* h, int face, int plane, int nsamples, const float* wave, int pad)
{
    if (!h) return fail(WCT_ERR_ARG, "wct_dt_set_long_response: null component");
    std::lock_guard<std::mutex> lk(h->core.mtx);
    PlaneState* ps = find_plane(h, face, plane);
    if (!ps || nsamples < 0 || (nsamples && !wave) || pad < 0)
        return fail(WCT_ERR_ARG, "wct_dt_set_long_response: bad arguments");
    ps->long_wf.assign(wave, wave + nsamples);
    ps->long_pad = pad;
    ps->long_nfft = 0;  // spectrum rebuilt at the next use
    return WCT_OK;
}

int wct_dt_frame_shape(const wct_depotransform* h, int* nrows, int* nticks)
{
    if (!h) return fail(WCT_ERR_ARG, "null component");
    if (nrows) *nrows = h->core.nrows();
    if (nticks) *nticks = h->core.nticks();
    return WCT_OK;
}

int wct_dt_set_charge_scale(wct_depotransform* h, const double* scale, size_t ndepos, int on_device)
{
    if (!h) return fail(WCT_ERR_ARG, "null component");
    std::lock_guard<std::mutex> lk(h->core.mtx);
    Core& c = h->core;
    if (!scale) {
        c.have_qscale = false;
        c.qscale_n = 0;
        c.qscale_planes = 0;
        return WCT_OK;
    }
    const int np = (int)c.planes.size();
    if (np == 0) return fail(WCT_ERR_STATE, "wct_dt_set_charge_scale: no planes configured");
    if (ndepos == 0 || ndepos > (size_t)0x7fffffff)
        return fail(WCT_ERR_ARG, "wct_dt_set_charge_scale: depo count out of range");
    CUDA_TRY(cudaSetDevice(c.device));
    const size_t bytes = sizeof(double) * ndepos * (size_t)np;
    CUDA_TRY(c.d_qscale.ensure(bytes));
    // ordered after the work already queued on the component's stream, which
    // may still read the previous scale
    CUDA_TRY(cudaMemcpyAsync(c.d_qscale.p, scale, bytes,
                             on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, c.own_stream));
    CUDA_TRY(cudaStreamSynchronize(c.own_stream));
    c.have_qscale = true;
    c.qscale_n = ndepos;
    c.qscale_planes = np;
    return WCT_OK;
}

int wct_dt_forward_device(wct_depotransform* h, const double* d_depos, size_t ndepos, float* d_frame,
                          wct_plane_window* windows, int* frame_ident, void* stream)
{
    if (!h || !d_frame || (ndepos && !d_depos)) return fail(WCT_ERR_ARG, "wct_dt_forward_device: bad arguments");
    std::lock_guard<std::mutex> lk(h->core.mtx);
    cudaStream_t s = stream ? (cudaStream_t)stream : h->core.own_stream;
    return forward_device(h->core, d_depos, ndepos, d_frame, windows, frame_ident, s, nullptr, nullptr, nullptr,
                          nullptr, nullptr, true);
}

int wct_dt_forward(wct_depotransform* h, const double* depos, size_t ndepos, float* frame, wct_plane_window* windows,
                   int* frame_ident)
{
    if (!h || !frame || (ndepos && !depos)) return fail(WCT_ERR_ARG, "wct_dt_forward: bad arguments");
    std::lock_guard<std::mutex> lk(h->core.mtx);
    Core& c = h->core;
    CUDA_TRY(cudaSetDevice(c.device));
    cudaStream_t s = c.own_stream;
    const size_t fbytes = sizeof(float) * (size_t)c.nrows() * c.nticks();
    CUDA_TRY(c.d_depos.ensure(sizeof(double) * 7 * std::max<size_t>(ndepos, 1)));
    CUDA_TRY(c.d_frame.ensure(fbytes));
    // the depos go up in chunks on the copy stream, each chunk's prep starting as it arrives
    // each plane's rows go back as soon as they are final (copy stream), while
    // the next planes are still transformed
    // the frame goes back on the copy stream in two parts: first the zero
    // rest of every plane (as soon as the frame is cleared, while the
    // kernels run), then each plane's written block once the plane is final
    const int np = (int)c.planes.size();
    std::vector<cudaEvent_t> done(np);
    for (auto& ev : done) ev = c.take_event();
    cudaEvent_t zeroed = c.take_event();
    std::vector<FrameRegion> reg;
    int rc = forward_device(c, c.d_depos.as<double>(), ndepos, c.d_frame.as<float>(), windows, frame_ident, s,
                            done.data(), zeroed, &reg, ndepos ? depos : nullptr);
    if (rc == WCT_OK) {
        const int nt = c.nticks();
        const float* df = c.d_frame.as<float>();
        const size_t rowb = sizeof(float) * (size_t)nt;
        auto rows = [&](int r0, int r1) {  // whole rows [r0, r1) of the frame
            if (r1 <= r0) return cudaSuccess;
            return cudaMemcpyAsync(frame + (size_t)r0 * nt, df + (size_t)r0 * nt, rowb * (r1 - r0),
                                   cudaMemcpyDeviceToHost, c.copy_stream);
        };
        auto block = [&](int r0, int r1, int t0, int t1) {  // rows [r0, r1), ticks [t0, t1)
            if (r1 <= r0 || t1 <= t0) return cudaSuccess;
            return cudaMemcpy2DAsync(frame + (size_t)r0 * nt + t0, rowb, df + (size_t)r0 * nt + t0, rowb,
                                     sizeof(float) * (size_t)(t1 - t0), r1 - r0, cudaMemcpyDeviceToHost,
                                     c.copy_stream);
        };
        cudaError_t e = cudaStreamWaitEvent(c.copy_stream, zeroed, 0);
        for (int ip = 0; ip < np && e == cudaSuccess; ++ip) {
            const PlaneState& ps = *c.planes[ip];
            const int base = ps.row0, nw = ps.desc.nwires;
            const FrameRegion& r = reg[ip];
            if (r.rhi <= r.rlo) {
                e = rows(base, base + nw);
                continue;
            }
            e = rows(base, base + r.rlo);
            if (e == cudaSuccess) e = rows(base + r.rhi, base + nw);
            if (e == cudaSuccess) e = block(base + r.rlo, base + r.rhi, 0, r.tlo);
            if (e == cudaSuccess) e = block(base + r.rlo, base + r.rhi, r.thi, nt);
        }
        for (int ip = 0; ip < np && e == cudaSuccess; ++ip) {
            const FrameRegion& r = reg[ip];
            if (r.rhi <= r.rlo) continue;
            const int base = c.planes[ip]->row0;
            e = cudaStreamWaitEvent(c.copy_stream, done[ip], 0);
            if (e == cudaSuccess) e = block(base + r.rlo, base + r.rhi, r.tlo, r.thi);
        }
        if (e != cudaSuccess)
            rc = fail(WCT_ERR_CUDA, std::string("wct_dt_forward: frame download: ") + cudaGetErrorString(e));
    }
    cudaError_t e1 = cudaStreamSynchronize(c.copy_stream);
    cudaError_t e2 = cudaStreamSynchronize(s);
    for (auto& ev : done) c.event_pool.push_back(ev);
    c.event_pool.push_back(zeroed);
    if (rc) return rc;
    if (e1 != cudaSuccess || e2 != cudaSuccess)
        return fail(WCT_ERR_CUDA, std::string("wct_dt_forward: ") + cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
    (void)fbytes;
    return WCT_OK;
}

int wct_dt_adjoint_device(wct_depotransform* h, const double* d_depos, size_t ndepos, const float* d_grad_frame,
                          double* d_grad_depos, double* d_grad_drift, void* stream)
{
    if (!h || !d_grad_frame || (ndepos && (!d_depos || !d_grad_depos)))
        return fail(WCT_ERR_ARG, "wct_dt_adjoint_device: bad arguments");
    std::lock_guard<std::mutex> lk(h->core.mtx);
    cudaStream_t s = stream ? (cudaStream_t)stream : h->core.own_stream;
    return adjoint_device(h->core, d_depos, ndepos, d_grad_frame, d_grad_depos, d_grad_drift, s);
}

int wct_dt_adjoint(wct_depotransform* h, const double* depos, size_t ndepos, const float* grad_frame,
                   double* grad_depos, double* grad_drift)
{
    if (!h || !grad_frame || (ndepos && (!depos || !grad_depos)))
        return fail(WCT_ERR_ARG, "wct_dt_adjoint: bad arguments");
    std::lock_guard<std::mutex> lk(h->core.mtx);
    Core& c = h->core;
    CUDA_TRY(cudaSetDevice(c.device));
    cudaStream_t s = c.own_stream;
    const size_t fbytes = sizeof(float) * (size_t)c.nrows() * c.nticks();
    const size_t dbytes = sizeof(double) * 7 * std::max<size_t>(ndepos, 1);
    CUDA_TRY(c.d_depos.ensure(dbytes));
    CUDA_TRY(c.d_gdep.ensure(dbytes));
    CUDA_TRY(c.d_gframe.ensure(fbytes));
    CUDA_TRY(c.d_gglob.ensure(sizeof(double) * 3));
    if (ndepos)
        CUDA_TRY(cudaMemcpyAsync(c.d_depos.p, depos, sizeof(double) * 7 * ndepos, cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaMemcpyAsync(c.d_gframe.p, grad_frame, fbytes, cudaMemcpyHostToDevice, s));
    int rc = adjoint_device(c, c.d_depos.as<double>(), ndepos, c.d_gframe.as<float>(), c.d_gdep.as<double>(),
                            c.d_gglob.as<double>(), s);
    if (rc) return rc;
    if (ndepos)
        CUDA_TRY(cudaMemcpyAsync(grad_depos, c.d_gdep.p, sizeof(double) * 7 * ndepos, cudaMemcpyDeviceToHost, s));
    double gg[3];
    CUDA_TRY(cudaMemcpyAsync(gg, c.d_gglob.p, sizeof gg, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    if (grad_drift) std::memcpy(grad_drift, gg, sizeof gg);
    return WCT_OK;
}

int wct_dt_set_drift_params(wct_depotransform* h, double DL, double DT, double lifetime)
{
    if (!h) return fail(WCT_ERR_ARG, "null component");
    std::lock_guard<std::mutex> lk(h->core.mtx);
    Core& c = h->core;
    if (!c.have_drifter) return fail(WCT_ERR_STATE, "no drifter configured");
    if (!(DL >= 0) || !(DT >= 0) || !(lifetime > 0))
        return fail(WCT_ERR_ARG, "DL and DT must be non-negative and lifetime positive");
    c.drifter.DL = DL;
    c.drifter.DT = DT;
    c.drifter.lifetime = lifetime;
    return WCT_OK;
}

int wct_dt_get_drift_params(const wct_depotransform* h, double* DL, double* DT, double* lifetime)
{
    if (!h) return fail(WCT_ERR_ARG, "null component");
    const Core& c = h->core;
    if (!c.have_drifter) return fail(WCT_ERR_STATE, "no drifter configured");
    if (DL) *DL = c.drifter.DL;
    if (DT) *DT = c.drifter.DT;
    if (lifetime) *lifetime = c.drifter.lifetime;
    return WCT_OK;
}

// Graphs cannot be captured on the legacy or per-thread default stream: run
// on the component's own stream, ordered after and before the caller's.
static int on_capturable_stream(Core& c, cudaStream_t s, const std::function<int(cudaStream_t)>& f)
{
    if (s != nullptr && s != cudaStreamLegacy && s != cudaStreamPerThread) return f(s);
    CUDA_TRY(cudaSetDevice(c.device));
    cudaEvent_t a = c.take_event(), b = c.take_event();
    CUDA_TRY(cudaEventRecord(a, s));
    CUDA_TRY(cudaStreamWaitEvent(c.own_stream, a, 0));
    const int rc = f(c.own_stream);
    cudaEventRecord(b, c.own_stream);
    cudaStreamWaitEvent(s, b, 0);
    c.event_pool.push_back(a);
    c.event_pool.push_back(b);
    return rc;
}

int wct_dt_forward_batch_device(wct_depotransform* h, const double* d_depos, const long long* offsets, int nevents,
                                float* d_frames, wct_plane_window* windows, int* first_ident, void* stream)
{
    if (!h) return fail(WCT_ERR_ARG, "null component");
    std::lock_guard<std::mutex> lk(h->core.mtx);
    cudaStream_t s = stream ? (cudaStream_t)stream : h->core.own_stream;
    return on_capturable_stream(h->core, s, [&](cudaStream_t r) {
        return forward_batch_device(h->core, d_depos, offsets, nevents, d_frames, windows, first_ident, r);
    });
}

int wct_dt_forward_batch(wct_depotransform* h, const double* depos, const long long* offsets, int nevents,
                         float* frames, wct_plane_window* windows, int* first_ident)
{
    if (!h || !offsets || nevents < 0 || (nevents > 0 && !frames)) return fail(WCT_ERR_ARG, "wct_dt_forward_batch: bad arguments");
    if (nevents == 0) return WCT_OK;
    std::lock_guard<std::mutex> lk(h->core.mtx);
    Core& c = h->core;
    CUDA_TRY(cudaSetDevice(c.device));
    cudaStream_t s = c.own_stream;
    const long long ndep = offsets[nevents];
    if (ndep < 0 || (ndep > 0 && !depos)) return fail(WCT_ERR_ARG, "wct_dt_forward_batch: bad depos");
    const size_t fbytes = sizeof(float) * (size_t)c.nrows() * c.nticks() * (size_t)nevents;
    CUDA_TRY(c.d_depos.ensure(sizeof(double) * 7 * std::max<long long>(ndep, 1)));
    CUDA_TRY(c.d_frame.ensure(fbytes));
    if (ndep)
        CUDA_TRY(cudaMemcpyAsync(c.d_depos.p, depos, sizeof(double) * 7 * (size_t)ndep, cudaMemcpyHostToDevice, s));
    int rc = forward_batch_device(c, c.d_depos.as<double>(), offsets, nevents, c.d_frame.as<float>(), windows,
                                  first_ident, s);
    if (rc) return rc;
    CUDA_TRY(cudaMemcpyAsync(frames, c.d_frame.p, fbytes, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    return WCT_OK;
}

int wct_dt_autotune_batch(wct_depotransform* h, const double* d_depos, const long long* offsets, int nevents,
                          float* d_frames, void* stream, char* report, size_t len)
{
    if (!h) return fail(WCT_ERR_ARG, "null component");
    std::lock_guard<std::mutex> lk(h->core.mtx);
    cudaStream_t s = stream ? (cudaStream_t)stream : h->core.own_stream;
    std::string rep;
    int rc = on_capturable_stream(h->core, s, [&](cudaStream_t r) {
        return autotune_batch(h->core, d_depos, offsets, nevents, d_frames, r, rep);
    });
    if (rc) return rc;
    if (report && len) {
        std::strncpy(report, rep.c_str(), len - 1);
        report[len - 1] = '\0';
        if (rep.size() >= len) return fail(WCT_ERR_SIZE, "autotune report truncated");
    }
    return WCT_OK;
}

int wct_dt_batch_tune(wct_depotransform* h, int* params, int set)
{
    if (!h || !params) return fail(WCT_ERR_ARG, "wct_dt_batch_tune: bad arguments");
    std::lock_guard<std::mutex> lk(h->core.mtx);
    Core& c = h->core;
    if (!c.batch) c.batch = std::make_unique<BatchState>();
    BatchTune& t = c.batch->tune;
    if (set) {
        if (params[0] < 1 || params[0] > kMaxBatch || params[1] < 1 || params[1] > 64 ||
            (params[2] != 128 && params[2] != 256 && params[2] != 512 && params[2] != 1024) || params[3] < 1 ||
            params[3] > 64 || params[4] < 1 || params[4] > 64)
            return fail(WCT_ERR_ARG, "wct_dt_batch_tune: value out of range");
        t = BatchTune{params[0], params[1], params[2], params[3], params[4]};
    }
    else {
        params[0] = t.slots;
        params[1] = t.raster_per_sm;
        params[2] = t.fft_threads;
        params[3] = t.fft_per_sm;
        params[4] = t.conv_per_sm;
    }
    return WCT_OK;
}

int wct_random_binomial_device(unsigned long long seed, int ident, int n, double p, long count, int* d_out,
                               void* stream)
{
    if (n < 0 || count < 0 || (count > 0 && !d_out) || !(p >= 0.0 && p <= 1.0))
        return fail(WCT_ERR_ARG, "wct_random_binomial_device: bad arguments");
    launch_binomial_samples(seed, ident, n, p, count, d_out, (cudaStream_t)stream);
    CUDA_TRY(cudaGetLastError());
    return WCT_OK;
}

int wct_dt_eos(wct_depotransform* h)
{
    if (!h) return fail(WCT_ERR_ARG, "null component");
    return WCT_EOS;
}

int wct_dt_forward_traces(wct_depotransform* h, const double* depos, size_t ndepos, float* charge, size_t capacity,
                          int* channel, int* tbin, int* length, long* offset, int* ntraces, size_t* nsamples,
                          wct_plane_window* windows, int* frame_ident)
{
    if (!h || (ndepos && !depos) || !channel || !tbin || !length || !offset || !ntraces)
        return fail(WCT_ERR_ARG, "wct_dt_forward_traces: bad arguments");
    std::lock_guard<std::mutex> lk(h->core.mtx);
    Core& c = h->core;
    CUDA_TRY(cudaSetDevice(c.device));
    cudaStream_t s = c.own_stream;
    const int np = (int)c.planes.size(), nt = c.nticks();
    CUDA_TRY(c.d_depos.ensure(sizeof(double) * 7 * std::max<size_t>(ndepos, 1)));
    CUDA_TRY(c.d_frame.ensure(sizeof(float) * (size_t)c.nrows() * nt));
    CUDA_TRY(c.d_edges.ensure(sizeof(int2) * (size_t)std::max(c.nrows(), 1)));
    if (c.h_edges_n < (size_t)c.nrows()) {
        if (c.h_edges) cudaFreeHost(c.h_edges);
        c.h_edges = nullptr;
        CUDA_TRY(cudaMallocHost(&c.h_edges, sizeof(int2) * (size_t)std::max(c.nrows(), 1)));
        c.h_edges_n = c.nrows();
    }
    std::vector<cudaEvent_t> done(np);
    for (auto& ev : done) ev = c.take_event();
    // each plane's block (window rows x window ticks; the frame is zero
    // outside it) and the edges of its rows go back on the copy stream as
    // soon as the plane is final, while later planes are transformed
    std::vector<FrameRegion> reg(np);
    std::vector<size_t> boff(np + 1, 0);
    const float* df = c.d_frame.as<float>();
    int2* de = c.d_edges.as<int2>();
    auto after = [&](int ip, const FrameRegion& r, cudaStream_t ps_s) -> int {
        reg[ip] = r;
        const size_t w = (size_t)std::max(0, r.thi - r.tlo);
        const size_t blk = r.rhi > r.rlo ? (size_t)(r.rhi - r.rlo) * w : 0;
        boff[ip + 1] = boff[ip] + blk;
        if (blk == 0) return WCT_OK;
        if (boff[ip + 1] > capacity)
            return fail(WCT_ERR_SIZE, "wct_dt_forward_traces: the charge buffer holds fewer samples than the windows");
        if (!charge) return fail(WCT_ERR_ARG, "wct_dt_forward_traces: null charge buffer");
        const int base = c.planes[ip]->row0;
        launch_row_edges(df, nt, base + r.rlo, r.rhi - r.rlo, r.tlo, r.thi, de + base + r.rlo, ps_s);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaEventRecord(done[ip], ps_s);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(c.copy_stream, done[ip], 0);
        if (e == cudaSuccess)
            e = cudaMemcpy2DAsync(charge + boff[ip], sizeof(float) * w, df + (size_t)(base + r.rlo) * nt + r.tlo,
                                  sizeof(float) * (size_t)nt, sizeof(float) * w, r.rhi - r.rlo, cudaMemcpyDeviceToHost,
                                  c.copy_stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(c.h_edges + base + r.rlo, de + base + r.rlo, sizeof(int2) * (r.rhi - r.rlo),
                                cudaMemcpyDeviceToHost, c.copy_stream);
        if (e != cudaSuccess)
            return fail(WCT_ERR_CUDA, std::string("wct_dt_forward_traces: download: ") + cudaGetErrorString(e));
        return WCT_OK;
    };
    int rc = forward_device(c, c.d_depos.as<double>(), ndepos, c.d_frame.as<float>(), windows, frame_ident, s,
                            nullptr, nullptr, nullptr, ndepos ? depos : nullptr, after);
    cudaError_t e1 = cudaStreamSynchronize(c.copy_stream);
    cudaError_t e2 = cudaStreamSynchronize(s);
    for (auto& ev : done) c.event_pool.push_back(ev);
    if (rc) return rc;
    if (e1 != cudaSuccess || e2 != cudaSuccess)
        return fail(WCT_ERR_CUDA,
                    std::string("wct_dt_forward_traces: ") + cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
    // traces in frame row order (DepoTransform.cxx:193-208)
    int k = 0;
    for (int ip = 0; ip < np; ++ip) {
        const FrameRegion& r = reg[ip];
        if (boff[ip + 1] == boff[ip]) continue;
        const PlaneState& ps = *c.planes[ip];
        const size_t w = (size_t)(r.thi - r.tlo);
        for (int row = r.rlo; row < r.rhi; ++row) {
            const int2 ed = c.h_edges[ps.row0 + row];
            if (ed.y <= ed.x) continue;
            channel[k] = ps.channels[row];
            tbin[k] = r.tlo + ed.x;
            length[k] = ed.y - ed.x;
            offset[k] = (long)(boff[ip] + (size_t)(row - r.rlo) * w + ed.x);
            ++k;
        }
    }
    *ntraces = k;
    if (nsamples) *nsamples = boff[np];
    return WCT_OK;
}

int wct_dt_traces(const wct_depotransform* h, const float* frame, int* channel, int* tbin, int* length, long* offset,
                  int* ntraces)
{
    if (!h || !frame || !channel || !tbin || !length || !offset || !ntraces)
        return fail(WCT_ERR_ARG, "wct_dt_traces: bad arguments");
    const Core& c = h->core;
    const int nt = c.nticks();
    int k = 0;
    for (auto& ps : c.planes) {
        for (int w = 0; w < ps->desc.nwires; ++w) {
            const float* row = frame + (size_t)(ps->row0 + w) * nt;
            int imin = nt, imax = nt;  // Waveform::edge
            for (int i = 0; i < nt; ++i) {
                if (row[i] != 0.0f) {
                    if (imin == nt) imin = i;
                    imax = i + 1;
                }
            }
            if (imin == nt) continue;
            channel[k] = ps->channels[w];
            tbin[k] = imin;
            length[k] = imax - imin;
            offset[k] = (long)(ps->row0 + w) * nt + imin;
            ++k;
        }
    }
    *ntraces = k;
    return WCT_OK;
}

int wct_dt_patch_records(const wct_depotransform* h, int face, int plane, int* out, size_t n)
{
    PlaneState* ps = find_plane(const_cast<wct_depotransform*>(h), face, plane);
    if (!ps || !out) return fail(WCT_ERR_ARG, "wct_dt_patch_records: bad arguments");
    const Core& c = h->core;
    if (n != c.last_n) return fail(WCT_ERR_STATE, "depo count differs from the last forward call");
    if (n == 0) return WCT_OK;
    int ip = 0;
    for (; ip < (int)c.planes.size(); ++ip)
        if (c.planes[ip].get() == ps) break;
    std::vector<PatchRec> rec(n);
    CUDA_TRY(cudaSetDevice(c.device));
    CUDA_TRY(cudaMemcpy(rec.data(), c.d_rec.as<PatchRec>() + (size_t)ip * n, sizeof(PatchRec) * n,
                        cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < n; ++i) {
        out[4 * i + 0] = rec[i].toff;
        out[4 * i + 1] = rec[i].poff;
        out[4 * i + 2] = rec[i].nt;
        out[4 * i + 3] = rec[i].np;
    }
    return WCT_OK;
}

int wct_dt_set_profiling(wct_depotransform* h, int on)
{
    if (!h) return fail(WCT_ERR_ARG, "null component");
    std::lock_guard<std::mutex> lk(h->core.mtx);
    h->core.profiling = on != 0;
    return WCT_OK;
}

int wct_dt_stage_times(wct_depotransform* h, double* ms, long* launches, int nstages, long* total_launches, int reset)
{
    if (!h) return fail(WCT_ERR_ARG, "null component");
    std::lock_guard<std::mutex> lk(h->core.mtx);
    Core& c = h->core;
    CUDA_TRY(cudaSetDevice(c.device));
    c.harvest();
    for (int i = 0; i < nstages && i < Core::kStages; ++i) {
        if (ms) ms[i] = c.stage_ms[i];
        if (launches) launches[i] = c.stage_launches[i];
    }
    if (total_launches) *total_launches = c.total_launches;
    if (reset) {
        for (int i = 0; i < Core::kStages; ++i) {
            c.stage_ms[i] = 0;
            c.stage_launches[i] = 0;
        }
        c.total_launches = 0;
    }
    return WCT_OK;
}

int wct_dt_destroy(wct_depotransform* h)
{
    if (h) {
        cudaSetDevice(h->core.device);
        delete h;
    }
    return WCT_OK;
}

/* ---- GPU IDFT ---- */

int wct_dft_fwd1d(const float* in, float* out, int size) { return dft_host(in, out, 1, size, 0, 1, -1, true); }
int wct_dft_inv1d(const float* in, float* out, int size) { return dft_host(in, out, 1, size, 0, 1, +1, true); }
int wct_dft_fwd1b(const float* in, float* out, int nrows, int ncols, int axis)
{
    return dft_host(in, out, nrows, ncols, 0, axis, -1, true);
}
int wct_dft_inv1b(const float* in, float* out, int nrows, int ncols, int axis)
{
    return dft_host(in, out, nrows, ncols, 0, axis, +1, true);
}
int wct_dft_fwd2d(const float* in, float* out, int nrows, int ncols)
{
    return dft_host(in, out, nrows, ncols, 1, 1, -1, true);
}
int wct_dft_inv2d(const float* in, float* out, int nrows, int ncols)
{
    return dft_host(in, out, nrows, ncols, 1, 1, +1, true);
}
int wct_dft_transpose_real(const float* in, float* out, int nrows, int ncols)
{
    return dft_host(in, out, nrows, ncols, 2, 1, -1, false);
}
int wct_dft_transpose_complex(const float* in, float* out, int nrows, int ncols)
{
    return dft_host(in, out, nrows, ncols, 2, 1, -1, true);
}
int wct_dft_1b_device(const float* in, float* out, int nrows, int ncols, int axis, int inverse, void* stream)
{
    int rc = dft_check(in, out, nrows, ncols);
    if (rc) return rc;
    return dft_1b_dev(reinterpret_cast<const float2*>(in), reinterpret_cast<float2*>(out), nrows, ncols, axis,
                      inverse ? +1 : -1, (cudaStream_t)stream);
}
int wct_dft_2d_device(const float* in, float* out, int nrows, int ncols, int inverse, void* stream)
{
    int rc = dft_check(in, out, nrows, ncols);
    if (rc) return rc;
    if (nrows == 0 || ncols == 0) return WCT_OK;
    return dft_2d_dev(reinterpret_cast<const float2*>(in), reinterpret_cast<float2*>(out), nrows, ncols,
                      inverse ? +1 : -1, (cudaStream_t)stream);
}
int wct_dft_transpose_device(const float* in, float* out, int nrows, int ncols, int is_complex, void* stream)
{
    int rc = dft_check(in, out, nrows, ncols);
    if (rc) return rc;
    return dft_transpose_dev(in, out, nrows, ncols, is_complex != 0, (cudaStream_t)stream);
}

/* ---- Noise ---- */

static int noise_args(const void* frame, int nrows, int ncols, const void* spectra, int nspec, const void* row_spec,
                      const void* row_stream, FftDesc& d)
{
    if (!frame || !spectra || !row_spec || !row_stream || nrows < 0 || ncols < 0 || nspec <= 0)
        return fail(WCT_ERR_ARG, "add noise: bad arguments");
    if (nspec % 2 || nspec / 2 > kDftMaxFft || !dft_smooth(nspec / 2))
        return fail(WCT_ERR_SIZE, "add noise: the spectrum length must be even with a 7-smooth half up to 14336");
    return device_plan(nspec / 2, d);
}

int wct_add_noise_device(float* frame, long ld, int nrows, int ncols, const float* spectra, int nspec,
                         const int* row_spec, const int* row_stream, unsigned long long seed, int ident, int model,
                         void* stream)
{
    FftDesc d;
    int rc = noise_args(frame, nrows, ncols, spectra, nspec, row_spec, row_stream, d);
    if (rc) return rc;
    if (ld < ncols) return fail(WCT_ERR_ARG, "add noise: row stride below the row length");
    const unsigned k0 = (unsigned)(seed & 0xffffffffull);
    const unsigned k1 = (unsigned)(seed >> 32) + 0x9E3779B9u * (unsigned)ident;
    launch_add_noise(frame, ld, nrows, ncols, spectra, nspec, row_spec, row_stream, k0, k1, (unsigned)model, d,
                     (cudaStream_t)stream);
    CUDA_TRY(cudaGetLastError());
    return WCT_OK;
}

int wct_add_noise(float* frame, int nrows, int ncols, const float* spectra, int nspectra, int nspec,
                  const int* row_spec, const int* row_stream, unsigned long long seed, int ident, int model)
{
    FftDesc d;
    int rc = noise_args(frame, nrows, ncols, spectra, nspec, row_spec, row_stream, d);
    if (rc) return rc;
    if (nspectra < 0) return fail(WCT_ERR_ARG, "add noise: bad arguments");
    for (int r = 0; r < nrows; ++r)
        if (row_spec[r] >= nspectra) return fail(WCT_ERR_ARG, "add noise: spectrum index out of range");
    if (!nrows || !ncols) return WCT_OK;
    cudaStream_t s = cudaStreamPerThread;
    const size_t fb = sizeof(float) * (size_t)nrows * ncols;
    const size_t sb = sizeof(float) * (size_t)std::max(nspectra, 1) * nspec;
    {
        AsyncBuf f, sp, rs, rt;
        f.s = sp.s = rs.s = rt.s = s;
        CUDA_TRY(cudaMallocAsync(&f.p, fb, s));
        CUDA_TRY(cudaMallocAsync(&sp.p, sb, s));
        CUDA_TRY(cudaMallocAsync(&rs.p, sizeof(int) * (size_t)nrows, s));
        CUDA_TRY(cudaMallocAsync(&rt.p, sizeof(int) * (size_t)nrows, s));
        CUDA_TRY(cudaMemcpyAsync(f.p, frame, fb, cudaMemcpyHostToDevice, s));
        if (nspectra)
            CUDA_TRY(cudaMemcpyAsync(sp.p, spectra, sizeof(float) * (size_t)nspectra * nspec, cudaMemcpyHostToDevice,
                                     s));
        CUDA_TRY(cudaMemcpyAsync(rs.p, row_spec, sizeof(int) * (size_t)nrows, cudaMemcpyHostToDevice, s));
        CUDA_TRY(cudaMemcpyAsync(rt.p, row_stream, sizeof(int) * (size_t)nrows, cudaMemcpyHostToDevice, s));
        rc = wct_add_noise_device(static_cast<float*>(f.p), ncols, nrows, ncols, static_cast<const float*>(sp.p),
                                  nspec, static_cast<const int*>(rs.p), static_cast<const int*>(rt.p), seed, ident,
                                  model, s);
        if (rc) return rc;
        CUDA_TRY(cudaMemcpyAsync(frame, f.p, fb, cudaMemcpyDeviceToHost, s));
    }
    CUDA_TRY(cudaStreamSynchronize(s));
    return WCT_OK;
}

/* ---- Digitizer ---- */

static int digitize_args(const void* in, int nrows, int ncols, const void* base, double fs_lo, double fs_hi,
                         int resolution, const void* out)
{
    if (!in || !out || !base || nrows < 0 || ncols < 0) return fail(WCT_ERR_ARG, "digitize: bad arguments");
    if (resolution < 1 || resolution > 30) return fail(WCT_ERR_ARG, "digitize: resolution must be 1..30 bits");
    if (!(fs_hi > fs_lo)) return fail(WCT_ERR_ARG, "digitize: fullscale[1] must exceed fullscale[0]");
    return WCT_OK;
}

int wct_digitize_device(const float* frame, long ld_in, int nrows, int ncols, const float* row_baseline, double gain,
                        double fs_lo, double fs_hi, int resolution, int round_adc, float* adc, long ld_out,
                        void* stream)
{
    int rc = digitize_args(frame, nrows, ncols, row_baseline, fs_lo, fs_hi, resolution, adc);
    if (rc) return rc;
    if (ld_in < ncols || ld_out < ncols) return fail(WCT_ERR_ARG, "digitize: row stride below the row length");
    launch_digitize(frame, ld_in, adc, ld_out, nrows, ncols, row_baseline, gain, fs_lo, fs_hi, resolution,
                    round_adc != 0, (cudaStream_t)stream);
    CUDA_TRY(cudaGetLastError());
    return WCT_OK;
}

int wct_digitize(const float* frame, int nrows, int ncols, const float* row_baseline, double gain, double fs_lo,
                 double fs_hi, int resolution, int round_adc, float* adc)
{
    int rc = digitize_args(frame, nrows, ncols, row_baseline, fs_lo, fs_hi, resolution, adc);
    if (rc) return rc;
    if (!nrows || !ncols) return WCT_OK;
    cudaStream_t s = cudaStreamPerThread;
    const size_t bytes = sizeof(float) * (size_t)nrows * ncols;
    {
        AsyncBuf d, b;
        d.s = b.s = s;
        CUDA_TRY(cudaMallocAsync(&d.p, bytes, s));
        CUDA_TRY(cudaMallocAsync(&b.p, sizeof(float) * (size_t)nrows, s));
        CUDA_TRY(cudaMemcpyAsync(d.p, frame, bytes, cudaMemcpyHostToDevice, s));
        CUDA_TRY(cudaMemcpyAsync(b.p, row_baseline, sizeof(float) * (size_t)nrows, cudaMemcpyHostToDevice, s));
        float* dp = static_cast<float*>(d.p);
        launch_digitize(dp, ncols, dp, ncols, nrows, ncols, static_cast<const float*>(b.p), gain, fs_lo, fs_hi,
                        resolution, round_adc != 0, s);
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaMemcpyAsync(adc, d.p, bytes, cudaMemcpyDeviceToHost, s));
    }
    CUDA_TRY(cudaStreamSynchronize(s));
    return WCT_OK;
}

/* ---- DepoFluxSplat ---- */

static int splat_setup(const wct_depotransform* h, const wct_splat_config* cfg, SplatParams& sp, int& nrows)
{
    if (!h || !cfg) return fail(WCT_ERR_ARG, "splat: bad arguments");
    if (!(cfg->tick > 0) || !(cfg->window_duration >= 0) || !(cfg->drift_speed > 0) || !(cfg->nsigma >= 0))
        return fail(WCT_ERR_CONFIG, "splat: tick and drift_speed must be positive, window_duration and nsigma not negative");
    if (cfg->window_duration / cfg->tick >= 2147483647.0) return fail(WCT_ERR_SIZE, "splat: more than 2^31 - 1 ticks");
    sp = SplatParams{};
    const int nbins = (int)(cfg->window_duration / cfg->tick);
    sp.tb.nbins = nbins;
    sp.tb.tmin = cfg->window_start;
    sp.tb.tmax = cfg->window_start + nbins * cfg->tick;
    sp.tb.bs = (sp.tb.tmax - sp.tb.tmin) / nbins;
    sp.nsigma = cfg->nsigma;
    sp.speed = cfg->drift_speed;
    sp.time_shift = cfg->response_plane / cfg->drift_speed;
    for (int k = 0; k < 3; ++k) {
        sp.pl[k].smear_long = cfg->smear_long[k];
        sp.pl[k].smear_tran = cfg->smear_tran[k];
        sp.pl[k].tick_offset = cfg->time_offsets[k] / cfg->tick;
    }
    nrows = h->core.nrows();
    return WCT_OK;
}

int wct_dt_splat_shape(const wct_depotransform* h, const wct_splat_config* cfg, int* nrows, int* nticks)
{
    SplatParams sp;
    int nr = 0;
    int rc = splat_setup(h, cfg, sp, nr);
    if (rc) return rc;
    if (nrows) *nrows = nr;
    if (nticks) *nticks = sp.tb.nbins;
    return WCT_OK;
}

int wct_dt_splat_device(wct_depotransform* h, const wct_splat_config* cfg, const double* d_depos, size_t ndepos,
                        float* d_frame, void* stream)
{
    SplatParams sp;
    int nrows = 0;
    int rc = splat_setup(h, cfg, sp, nrows);
    if (rc) return rc;
    if (!d_frame || (ndepos && !d_depos)) return fail(WCT_ERR_ARG, "splat: bad arguments");
    if (ndepos > (size_t)0x7fffffff) return fail(WCT_ERR_SIZE, "splat: more than 2^31 - 1 depos");
    std::lock_guard<std::mutex> lk(h->core.mtx);
    Core& c = h->core;
    CUDA_TRY(cudaSetDevice(c.device));
    cudaStream_t s = stream ? (cudaStream_t)stream : c.own_stream;
    const long long count = (long long)nrows * sp.tb.nbins;
    if (count <= 0) return WCT_OK;
    CUDA_TRY(c.d_splat.ensure(sizeof(double) * (size_t)count));
    CUDA_TRY(cudaMemsetAsync(c.d_splat.p, 0, sizeof(double) * (size_t)count, s));
    for (const FaceState& f : c.faces) {
        PlaneSet ps{};
        ps.nplanes = std::min((int)f.planes.size(), kMaxPlanes);
        for (int k = 0; k < ps.nplanes; ++k) {
            const PlaneState& pl = *c.planes[f.planes[k]];
            ps.p[k] = pl.dev;
            ps.p[k].wire_base = pl.row0;
            ps.nwires_total += pl.desc.nwires;
        }
        SplatParams fsp = sp;
        for (int k = 3; k < kMaxPlanes; ++k) fsp.pl[k] = SplatPlane{};
        launch_splat_face(d_depos, (int)ndepos, ps, fsp, c.d_splat.as<double>(), s);
    }
    launch_splat_finish(c.d_splat.as<double>(), d_frame, count, s);
    CUDA_TRY(cudaGetLastError());
    return WCT_OK;
}

int wct_dt_splat(wct_depotransform* h, const wct_splat_config* cfg, const double* depos, size_t ndepos, float* frame)
{
    SplatParams sp;
    int nrows = 0;
    int rc = splat_setup(h, cfg, sp, nrows);
    if (rc) return rc;
    if (!frame || (ndepos && !depos)) return fail(WCT_ERR_ARG, "splat: bad arguments");
    const size_t fbytes = sizeof(float) * (size_t)nrows * sp.tb.nbins;
    if (!fbytes) return WCT_OK;
    cudaStream_t s = nullptr;
    {
        std::lock_guard<std::mutex> lk(h->core.mtx);
        CUDA_TRY(cudaSetDevice(h->core.device));
        s = h->core.own_stream;
    }
    AsyncBuf dd, df;
    dd.s = df.s = s;
    if (ndepos) {
        CUDA_TRY(cudaMallocAsync(&dd.p, sizeof(double) * 7 * ndepos, s));
        CUDA_TRY(cudaMemcpyAsync(dd.p, depos, sizeof(double) * 7 * ndepos, cudaMemcpyHostToDevice, s));
    }
    CUDA_TRY(cudaMallocAsync(&df.p, fbytes, s));
    rc = wct_dt_splat_device(h, cfg, static_cast<const double*>(dd.p), ndepos, static_cast<float*>(df.p), s);
    if (rc) return rc;
    CUDA_TRY(cudaMemcpyAsync(frame, df.p, fbytes, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    return WCT_OK;
}

}  // extern "C"
