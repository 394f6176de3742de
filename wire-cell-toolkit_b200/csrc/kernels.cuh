// Device data structures and launcher declarations for the DepoTransform
// forward path.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "fft.cuh"

namespace wctb200 {

constexpr int kMaxPlanes = 8;

// Drifter configuration (gen/src/Drifter.cxx:62-123).
struct DriftDev {
    double DL, DT, lifetime, speed, toffset;
    int nxr;
    double xr[8][3];  // anode, response, cathode
};

// One wire plane: pitch axis / origin of its Pimpos (util/src/Pimpos.cxx:5-33),
// its impact binning, the face's sensitive box (gen/src/AnodePlane.cxx:259-290)
// and the offset of its wires in the event-wide wire arrays.
struct PlaneDev {
    double ax, ay, az;        // unit pitch axis
    double ox, oy, oz;        // Pimpos origin
    int nwires, nimp;
    int imp_nbins;
    double imp_min, imp_max, imp_bs;
    int have_bb;
    double bb_lo[3], bb_hi[3];
    int wire_base;            // first entry of this plane in per-wire arrays
};

struct PlaneSet {
    int nplanes;
    int nwires_total;
    int ntiles;               // tick tiles of the readout: ceil(nticks / kTile)
    PlaneDev p[kMaxPlanes];
};

// Readout time binning (gen/src/DepoTransform.cxx:180).
struct TimeDev {
    int nbins;
    double tmin, tmax, bs;
};

// Per (plane, depo) patch description, written by the prep kernel.
// np == 0 marks a depo that does not contribute to the plane.
struct __align__(16) PatchRec {  // 16-byte aligned: two 128-bit loads per record
    int toff, poff;
    unsigned short nt, np;
    float tcr;   // center_time - edge(toff)
    float pcr;   // center_pitch - edge(poff)
    float st;    // sigma_time
    float sp;    // sigma_pitch
    float qn;    // charge / (sum of unit bin integrals in time * in pitch)
};
static_assert(sizeof(PatchRec) == 32, "PatchRec layout");

// One depo visit of a (wire, tick tile): the depo's index in the launch's
// depo array (its PatchRec, time profile and pool entry are read from there).
typedef int Visit;

// Per-plane window reduction (BinnedDiffusion_transform.cxx:416-464).
struct WindowDev {
    unsigned long long pmin, pmax, tmin, tmax;  // order-preserving double keys
    // (plane 0 entry of an event only) 64-bit totals of the event: ticks of
    // its patches longer than kTprof, and raster visits of all its patches
    unsigned long long wide_ticks, nvisits;
    int nadded, out_time, out_pitch, oversize;
    int bigcharge;  // patches whose raster bound exceeds kMaxVisitBound
};

constexpr int kTprof = 16;        // time profiles up to this many ticks are computed once per depo
constexpr int kTile = 256;        // ticks per charge-grid tile (one raster block per wire x tile)
constexpr int kScaleBlock = 64;   // ticks sharing one fixed-point scale in the raster
constexpr int kTileBlocks = kTile / kScaleBlock;
constexpr int kMaxPatchT = 1024;  // ticks per patch
constexpr int kMaxPatchP = 1024;  // impact bins per patch
// Largest per-visit bound (2 |q| x peak bin fractions, in electrons) of the
// raster's integer bound sums (units of 2^-16 in 64 bits).
constexpr float kMaxVisitBound = 1.0e12f;

// Per-plane parameters of the charge-grid stage of one event.
struct GridPlane {
    int nimp, G;
    int nwires, wire_base;
    int start_ch, nin;        // charge rows: wires start_ch .. start_ch+nin-1
    int col0, ncols;          // charge columns: ticks col0 .. col0+ncols-1
    int N;                    // row length of the grid (time FFT length)
    float tbs, pbs;           // tick and impact bin sizes
    long long qoff;           // offset of this plane's grid [G][nin][N] in floats
    long long recoff;         // offset of this plane's PatchRecs
    int row_base;             // first block of this plane in the raster grid
    int ktile0, ntile;        // absolute tick tiles covering grid columns [0, N)
};

struct GridSet {
    int nplanes;
    int nrows_total;          // raster blocks (wire rows x tiles, all planes)
    int ntiles_abs;           // tick tiles of the readout (visit-list key stride)
    GridPlane p[kMaxPlanes];
};

// Per-plane parameters of the adjoint's gather (adjoint.cu).
struct AdjPlane {
    int nimp, nin, N, start_ch, col0;
    long long qoff;           // offset of the plane's dL/dQ grid [G][nin][N] in floats
    float pbs, tbs;
    double ax, ay, az;        // unit pitch axis
};

struct AdjSet {
    int nplanes;
    AdjPlane p[kMaxPlanes];
};

// Events of one launch of the prep and fill kernels: depo ranges in the
// concatenated depo array and the first 256-thread block of each event
// (blocks never straddle events).  A single event is a table of one.
constexpr int kMaxBatch = 64;
struct EventTable {
    int nev;
    int dep0[kMaxBatch + 1];
    int blk0[kMaxBatch + 1];
};

// ---- batched events: device-planned pipeline ----
constexpr int kMaxClasses = 48;  // time-FFT length classes of the batched path

// Static description of the batched path (a kernel parameter): the window
// arithmetic inputs of every plane and the layout of one event slot in the
// charge-grid (Q, floats) and wire-convolution (V, complex) arenas.
struct BatchPlaneStatic {
    int G, npad, waveform_pad, nwires, imp_nbins, row0, nin_max;
    double imp_min, imp_bs;
    long long qslot;  // offset of the plane's grid within an event slot (floats)
    long long vslot;  // offset of the plane's V rows within an event slot (complex values)
};

struct BatchStatic {
    int np, nticks, nkeys, ntiles;
    double start_time, tbs;   // tick binning of the window arithmetic (ImpactTransform)
    int ncls;
    int cls_N[kMaxClasses];   // ascending time-FFT lengths
    long long qslot_total, vslot_total;
    BatchPlaneStatic pl[kMaxPlanes];
};

// Per (event, plane) plan, written on the device by the planner.
struct EvPlane {
    int start_ch, end_ch, start_tick, end_tick;           // window before padding
    int m_start_ch, m_end_ch, m_start_tick, m_end_tick;   // ImpactTransform's padded window
    int nw_ref, nt_ref;
    int nin, nout, ncols, N, M, cls;
    int ktile0, ntile;
    int ndepos_added, outside_time, outside_pitch;
    long long qoff;  // grid offset in the Q arena (floats)
    long long voff;  // V offset in the V arena (complex values)
};

// One pass of the batched pipeline over up to kMaxBatch events: the plan of
// every (event, plane) and the work-item prefixes of the persistent kernels
// (index e * np + ip, events major).
struct BatchPlan {
    int nev, np;
    int status;        // kBatch* bits
    int pad_;
    long long total_visits;
    int pre_raster[kMaxBatch * kMaxPlanes + 1];
    int pre_rows[kMaxBatch * kMaxPlanes + 1];   // time-FFT rows: G * nin
    int pre_orows[kMaxBatch * kMaxPlanes + 1];  // inverse-FFT rows: nout
    int pre_conv[kMaxPlanes][kMaxBatch + 1];    // wire-convolution tiles of plane ip over events
    int next[3 + kMaxPlanes];                   // work-stealing counters: raster, rfft, irfft, conv from plane ip0
    EvPlane ep[kMaxBatch * kMaxPlanes];
};
constexpr int kBatchVisitOverflow = 1;
constexpr int kBatchOversize = 2;
constexpr int kBatchBigCharge = 4;
constexpr int kBatchNoClass = 8;
constexpr int kBatchPoolShort = 16;  // not an error: some time profiles were computed in the raster
constexpr int kBatchTooBig = 32;     // a pass holds 2^31 or more visits: fewer events per pass
constexpr int kBatchSkip = kBatchVisitOverflow | kBatchTooBig;  // the raster and later stages skip the pass

// Launch shapes of the persistent kernels (chosen by the autotuner).
struct BatchTune {
    int slots;            // events per pass (event slots in the arenas)
    int raster_per_sm;    // persistent raster blocks per SM
    int fft_threads;      // threads per time-FFT row
    int fft_per_sm;       // persistent time-FFT blocks per SM
    int conv_per_sm;      // persistent wire-convolution blocks per SM
};

// ---- fluctuation (counter-based binomial draws, rng.cuh) ----
// Streams: key (key0, key1 + 0x9E3779B9 * ident) with ident the frame ident of
// the event; counter (depo index within its event, plane or drift tag, cell).
struct FlucParams {
    int on_patch;           // DepoTransform "fluctuate": patch cells (GaussianDiffusion.cxx:184-213)
    int on_drift;           // Drifter "fluctuate": absorbed electrons (Drifter.cxx:177-185)
    unsigned int key0, key1;
    int ident0;             // frame ident of the launch's first event, relative to *ident_base
    const int* ident_base;  // device value added to ident0 (lets a replayed graph draw afresh), or null
};

// Per (plane, depo) normalisation of a fluctuated patch.
struct FlucRec {
    int nq;          // (int)|Q|, the binomial trial count of every cell
    float scale;     // Q / (sum of the cell draws), 0 when every draw is 0
    float invS;      // 1 / (sum of unit bin integrals in pitch * in time)
    int pad;
};

// Time profiles of patches longer than kTprof ticks, computed once per depo
// (the raster would otherwise recompute them on every wire it visits).
// off[i] < 0: no room in the pool, the raster computes the values itself
// with the same function, so the frame does not depend on the pool.
struct TprofPool {
    float* val;
    int* off;                  // per depo
    unsigned long long* used;  // allocation counter
    long long cap;             // at most INT_MAX - 1 (offsets are int)
};

// ---- launchers (kernels.cu) ----
void launch_prep_all(const double* depos, const EventTable& et, int nkeys, const DriftDev& dd, int do_drift,
                     const PlaneSet& ps, const TimeDev& tb, double drift_speed, double nsigma, PatchRec* rec,
                     WindowDev* win, int* wire_cnt, float* tprof, unsigned long long* key_bound,
                     const FlucParams& fp, double* fq, unsigned char* wide, cudaStream_t s, int blk_begin = 0,
                     int blk_end = -1,  // blocks [blk_begin, blk_end) of the table (-1: to the end)
                     const double* qscale = nullptr);  // [depo][plane] charge scale of the table's depos, or null
// fq (fluctuation): [plane][depo] charge each plane's patch draws from, written by the prep
void launch_binomial_samples(unsigned long long seed, int ident, int n, double p, long long count, int* out,
                             cudaStream_t s);
void launch_fluc_sums(const PatchRec* rec, const EventTable& et, const PlaneSet& ps, float tbs, const FlucParams& fp,
                      const double* fq, FlucRec* fluc, cudaStream_t s);
void launch_raster_fluc(const PatchRec* rec, const FlucRec* fluc, const FlucParams& fp, const EventTable& evt,
                        const int* wire_cnt, const int* wire_off, const Visit* visits, long long vcap,
                        const GridSet& gs, float* Q, cudaStream_t s);
void launch_scan(const int* wire_cnt, int nwires_total, int* wire_off, int* wire_cur, cudaStream_t s);
void launch_tprof_pool(const PatchRec* rec, const EventTable& et, int nplanes, float tbs, const TprofPool& pool,
                       int* status, cudaStream_t s);
void launch_fill(const PatchRec* rec, const EventTable& et, int nkeys, const PlaneSet& ps, int* wire_cur,
                 Visit* visits, long long cap, cudaStream_t s);
size_t raster_smem_bytes(int G);
void launch_raster_wires(const PatchRec* rec, const float* tprof, const TprofPool& pool, const unsigned char* wide_key,
                         const int* wire_cnt,
                         const int* wire_off, const Visit* visits, long long vcap,
                         const unsigned long long* key_bound, const GridSet& gs, float* Q, cudaStream_t s);
void launch_rfft_rows(const float* in, long in_ld, int in_len, float2* out, long out_ld, int nrows,
                      const FftDesc& d, cudaStream_t s);
void launch_wire_conv(const float2* Qh, const float2* Rh, float2* Vh, int ngroups, int npad, int nrows_in,
                      int nrows_out, int M, bool pair, cudaStream_t s);
// the single-buffered 32-frequency tiles (any alignment; the fallback of launch_wire_conv)
void launch_wire_conv_tiles(const float2* Qh, const float2* Rh, float2* Vh, int ngroups, int npad, int nrows_in,
                            int nrows_out, int M, bool pair, cudaStream_t s);
void launch_irfft_rows(const float2* Vh, int nrows, const FftDesc& d, int wire0, int wlo, int whi, int tick0,
                       int ncols, int nticks, float* frame, cudaStream_t s);

void launch_spec_mul(float2* X, long ldx, int nrows, int M, const float2* R, cudaStream_t s);
// Waveform::edge of frame rows [r0, r0 + nrows) within ticks [t0, t1) (ld: row
// stride): out[r] = (first, last + 1) non-zero tick relative to t0, (0, 0) if none.
void launch_row_edges(const float* frame, int ld, int r0, int nrows, int t0, int t1, int2* out, cudaStream_t s);
// Device PlaneImpactResponse build: field responses binned on the tick grid
// (Z: npaths rows of n complex values), the bin-wise product of nrows spectra,
// and real parts of complex rows (length n) into float rows of ncols.
void launch_pir_bin(const double* current, int npaths, int nsamples, double tstart, double rawbs, double period,
                    double tick, int n, float2* Z, cudaStream_t s);
void launch_spec_chain(const float2* S, int nrows, int n, float2* out, cudaStream_t s);
void launch_real_rows(const float2* Z, int nrows, int n, float* out, int ncols, cudaStream_t s);

// GPU IDFT (dft.cu): complex row transforms (sign -1 forward, +1 inverse,
// result times scale), Bluestein rows for any length N (FFT length dP.M >=
// 2N - 1, chirp c_n = exp(-pi i n^2 / N), bhat = FFT of the chirp filter
// built by launch_bluestein_b), and transposes of row-major matrices.
void launch_c2c_rows(const float2* in, long ld_in, float2* out, long ld_out, int nrows, const FftDesc& d, int sign,
                     float scale, cudaStream_t s);
void launch_bluestein_rows(const float2* in, long ld_in, float2* out, long ld_out, int nrows, int N, const FftDesc& dP,
                           const float2* chirp, const float2* bhat, int sign, float scale, cudaStream_t s);
void launch_bluestein_b(const float2* chirp, float2* b, int N, int P, cudaStream_t s);
// batch: that many nrows x ncols matrices back to back (at most 65535)
void launch_transpose_c(const float2* in, float2* out, int nrows, int ncols, cudaStream_t s, int batch = 1);
// Four-step FFT twiddles on count elements of [b][n2][k1] blocks (N1 x N2 = N):
// times exp(sign 2 pi i n2 k1 / N).
void launch_twiddle4(float2* Z, long long count, int N1, int N2, int sign, cudaStream_t s);
// Bluestein through global memory: chirp-multiplied, zero-padded rows of
// length P, and the chirp-multiplied first N values back (scaled).
void launch_blue_pre(const float2* in, long ld_in, float2* Z, int nrows, int N, int P, const float2* chirp, bool inv,
                     cudaStream_t s);
void launch_blue_post(const float2* Z, int P, float2* out, long ld_out, int nrows, int N, const float2* chirp,
                      bool inv, float scale, cudaStream_t s);
void launch_transpose_r(const float* in, float* out, int nrows, int ncols, cudaStream_t s);
// Real rows packed two per complex row of length nfft (zero padded beyond n),
// the unpacking of the first n values, and a product with one spectrum.
void launch_pack_rows(const float* rows, long ld, int nrows, int n, float2* Z, int nfft, cudaStream_t s);
void launch_unpack_rows(const float2* Z, int nfft, float* rows, long ld, int nrows, int n, cudaStream_t s);
void launch_cmul_rows(float2* Z, int nfft, int nz, const float2* L, bool conj, cudaStream_t s);
// DepoFluxSplat (splat.cu): per plane the smear (ticks, wire pitches) and the
// time offset in ticks; the window binning, nsigma, drift speed and the time
// shift response_plane / drift_speed.
struct SplatPlane {
    double smear_long, smear_tran, tick_offset;
};
struct SplatParams {
    TimeDev tb;
    double nsigma, speed, time_shift;
    SplatPlane pl[kMaxPlanes];
};
// The planes of one face (wire_base = frame row of each plane's first wire)
// added into acc [rows][tb.nbins] doubles (zeroed by the caller); then the
// float frame from acc.
void launch_splat_face(const double* depos, int n, const PlaneSet& ps, const SplatParams& sp, double* acc,
                       cudaStream_t s);
void launch_splat_finish(const double* acc, float* frame, long long count, cudaStream_t s);
// Digitizer::digitize of every sample (one baseline per row, in the frame's units).
void launch_digitize(const float* in, long ld_in, float* out, long ld_out, int nrows, int ncols,
                     const float* row_baseline, double gain, double fs0, double fs1, int resolution, bool rnd,
                     cudaStream_t s);
// Noise waveforms of GeneratorN (aux/src/NoiseTools.cxx) from per-row channel
// spectra (row_spec: spectrum index, -1 none) on random streams row_stream,
// added to the frame rows; d: plan of length nspec / 2.
void launch_add_noise(float* frame, long ld, int nrows, int ncols, const float* spectra, int nspec,
                      const int* row_spec, const int* row_stream, unsigned k0, unsigned k1, unsigned model,
                      const FftDesc& d, cudaStream_t s);
void launch_twiddles(float2* tw, float2* twh, int M, cudaStream_t s);

// ---- batched-path launchers (kernels.cu) ----
void launch_plan_batch(BatchPlan* plan, const BatchStatic& bs, int nev, const WindowDev* win, long long vcap,
                       cudaStream_t s);
void launch_raster_batch(const BatchPlan* plan, const BatchStatic& bs, const PlaneSet& ps, const PatchRec* rec,
                         long long recstride, const float* tprof, const TprofPool& pool,
                         const unsigned char* wide_key, const int* wire_cnt, const int* wire_off,
                         const Visit* visits, long long vcap, const unsigned long long* key_bound, float* Q,
                         int nblocks, int maxG, const EventTable& evt, const FlucParams& fp, const FlucRec* fluc,
                         cudaStream_t s);
void launch_rfft_batch(const BatchPlan* plan, const FftDesc* descs, float* Q, int nblocks, int nthreads, int maxM,
                       cudaStream_t s);
// Wire convolution of planes [ip0, ip1) (all with the same pad and pairing) in one launch.
void launch_conv_batch(const BatchPlan* plan, const BatchStatic& bs, int ip0, int ip1, bool pair,
                       const float2* const* spec, const float* Q, float2* V, int nblocks, cudaStream_t s);
void launch_irfft_batch(const BatchPlan* plan, const BatchStatic& bs, const FftDesc* descs, const float2* V,
                        float* frames, long long frame_stride, int nblocks, int nthreads, int maxM, cudaStream_t s);
size_t conv_smem_bytes(int npad, bool pair);
void batch_kernel_attributes(int maxG, int maxM);

// ---- adjoint launchers (adjoint.cu) ----
void launch_grad_rows(const float* gframe, int nticks, int wire0, int wlo, int whi, int tick0, int ncols, int nrows,
                      int N, float* out, cudaStream_t s);
void launch_wire_conv_adj(const float2* Gh, const float2* Rh, float2* dQh, int G, int npad, int nin, int nout, int M,
                          cudaStream_t s);
void launch_adj_gather(const double* depos, int n, const DriftDev& dd, int do_drift, const PlaneSet& ps,
                       const AdjSet& as, double drift_speed, const PatchRec* rec, const float* dQ, double* grad,
                       double* gglob, cudaStream_t s, const double* qscale = nullptr);

}  // namespace wctb200
