/*
 * wctb200 -- B200-native Wire-Cell DepoTransform (signal simulation hot path)
 *
 * C ABI of libwctb200.so.  Plain pointers and sizes only; every entry point
 * returns an int status (WCT_OK on success) and never throws.  The message of
 * the last failure on the calling thread is available from wct_last_error().
 *
 * Each entry point cites the reference interface it stands in for (paths in
 * the wire-cell-toolkit source tree).  Units are the Wire-Cell system of
 * units (util/inc/WireCellUtil/Units.h): mm = 1, ns = 1, positron charge = 1.
 *
 * Depo layout (IDepo, iface/inc/WireCellIface/IDepo.h:14-51): 7 doubles per
 * depo: time, charge, x, y, z, extent_long, extent_tran.  The transform drops
 * a depo with a NaN or infinite value, as it drops one outside the drift
 * volume (the reference's result is undefined for such a depo).
 *
 * Frame layout: dense float32 rows, one row per wire of every plane (faces in
 * the order added, planes in the order added within a face), nticks columns
 * (readout_time / tick).  Row r of plane p holds ImpactTransform::waveform(r)
 * (gen/src/ImpactTransform.cxx:312-347); traces with the reference's exact-zero
 * trimming are produced by wct_dt_traces().
 */
#ifndef WCTB200_H
#define WCTB200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    WCT_OK = 0,
    WCT_ERR_ARG = 1,      /* bad argument (null pointer, index out of range) */
    WCT_ERR_CONFIG = 2,   /* invalid configuration (DepoTransform::configure would throw) */
    WCT_ERR_CUDA = 3,     /* CUDA runtime failure */
    WCT_ERR_STATE = 4,    /* call out of order (e.g. forward before responses are set) */
    WCT_ERR_RESPONSE = 5, /* response lookup outside the PIR extent (PlaneImpactResponse::closest throws) */
    WCT_ERR_SIZE = 6,     /* a patch or window exceeds a compiled limit */
    WCT_EOS = 7           /* end of stream acknowledged */
};

typedef struct wct_depotransform wct_depotransform; /* one DepoTransform component */
typedef struct wct_pir wct_pir;                     /* one PlaneImpactResponse */

/* Pimpos constructor arguments of one wire plane (util/inc/WireCellUtil/Pimpos.h:35-68)
 * plus the channel ident of each wire (IWire::channel). */
typedef struct {
    int nwires;
    int nimpacts;          /* impact bins per wire region (Pimpos nbins, default 10) */
    double pitchmin;       /* pitch location of wire 0 */
    double pitchmax;       /* pitch location of wire nwires-1 */
    double wire[3];        /* wire direction */
    double pitch[3];       /* pitch direction */
    double origin[3];      /* Pimpos origin */
    const int* channels;   /* nwires channel idents (copied) */
} wct_plane_desc;

/* One plane's field response (Response::Schema::PlaneResponse,
 * util/inc/WireCellUtil/Response.h:28-110). */
typedef struct {
    int npaths;            /* PathResponse count, ordered by increasing pitchpos */
    int nsamples;          /* samples per path current */
    const double* pitchpos;/* [npaths] */
    const double* current; /* [npaths][nsamples] induced current */
    double pitch;          /* PlaneResponse::pitch */
    double tstart;         /* FieldResponse::tstart */
    double period;         /* FieldResponse::period */
} wct_fr_plane;

/* Per-plane window of one forward call: ImpactTransform's m_start_ch,
 * m_end_ch, m_start_tick, m_end_tick (gen/src/ImpactTransform.cxx:90-115)
 * and BinnedDiffusion_transform's counters. */
typedef struct {
    int face, plane;
    int start_ch, end_ch;       /* wire window (may extend past [0, nwires)) */
    int start_tick, end_tick;   /* tick window (may extend past [0, nticks)) */
    int nw_fft, nt_fft;         /* the reference's FFT sizes for this window */
    int nt_gpu;                 /* time FFT length used on the device */
    int charge_rows;            /* wires of the charge grid (window before padding) */
    int npad;                   /* response half width in wires */
    int ndepos_added;           /* depos accepted by BinnedDiffusion_transform::add */
    int outside_time, outside_pitch;
} wct_plane_window;

const char* wct_version(void);
/* Message of the last failing call on this thread (empty if none). */
const char* wct_last_error(void);

/* ---- PlaneImpactResponse (gen/src/PlaneImpactResponse.cxx:56-320) ---- */

/* Build a plane impact response: PlaneImpactResponse::configure + build_responses
 * (gen/src/PlaneImpactResponse.cxx:56-269).  short_wave holds nshort short
 * responses (ColdElecResponse/RCResponse samples, IWaveform::waveform_samples)
 * concatenated, short_len their lengths; nticks is the PIR "nticks". */
int wct_pir_create(const wct_fr_plane* fr, int nshort, const int* short_len, const double* short_wave,
                   double overall_short_padding, double tick, int nticks, wct_pir** out);
/* PlaneImpactResponse::closest (gen/src/PlaneImpactResponse.cxx:294-320): path index
 * of the response closest to relpitch, or WCT_ERR_RESPONSE where the reference throws. */
int wct_pir_closest(const wct_pir* pir, double relpitch, int* path);
/* pitch(), impact(), half extent, nwires(), nimp_per_wire(), path count, nticks, waveform_pad. */
int wct_pir_info(const wct_pir* pir, double* pitch, double* impact, double* half_extent, int* nwires,
                 int* nimp_per_wire, int* npaths, int* nticks, int* waveform_pad);
/* IImpactResponse::waveform() of one path: nticks floats. */
int wct_pir_waveform(const wct_pir* pir, int path, float* out);
/* PlaneImpactResponse "long_responses" and "long_padding"
 * (gen/src/PlaneImpactResponse.cxx:46-47,121-150): the long-range response
 * is the circular convolution, at fft_best_length(nticks), of the nlong
 * waveforms (concatenated in long_wave, lengths long_len; each cut or zero
 * padded to that length); its pad is long_padding / tick ticks
 * (IImpactResponse::long_aux_waveform, long_aux_waveform_pad).  nlong = 0
 * removes it. */
int wct_pir_set_long_responses(wct_pir* pir, int nlong, const int* long_len, const double* long_wave,
                               double long_padding);
/* The same two builds on the current CUDA device, in the reference's single
 * precision: its fwd_r2c / spectrum product / inv_c2r chain
 * (PlaneImpactResponse.cxx:96-146,185-240) through the library's GPU
 * transforms, the field response binned onto ticks with float sums as the
 * reference's realseq_t.  The result is the same host-side wct_pir (the
 * waveforms agree with wct_pir_create's double-precision direct
 * convolution to single-precision rounding); the grouping, symmetry and
 * checks are wct_pir_create's. */
int wct_pir_create_device(const wct_fr_plane* fr, int nshort, const int* short_len, const double* short_wave,
                          double overall_short_padding, double tick, int nticks, wct_pir** out);
int wct_pir_set_long_responses_device(wct_pir* pir, int nlong, const int* long_len, const double* long_wave,
                                      double long_padding);
/* Length (0: no long-range response) and pad of the long-range response, and its samples. */
int wct_pir_long_info(const wct_pir* pir, int* nsamples, int* pad);
int wct_pir_long_waveform(const wct_pir* pir, float* out);
int wct_pir_destroy(wct_pir* pir);

/* fft_best_length (util/src/FFTBestLength.cxx:12-59): the smallest length
 * >= n of the reference's fast-size tables (keep_odd_even: of n's parity),
 * n itself above the tables; 0 for a negative n. */
long wct_fft_best_length(long n, int keep_odd_even);

/* ---- Batched FFT convolution of rows ---- */

/* Circular convolution of each real row with one real response at FFT length
 * nfft: out[r][k] = sum_m in[r][m] * resp[(k - m) mod nfft] for k < n_out,
 * rows and response zero padded to nfft.  nfft = 0 picks the smallest
 * supported length >= n_in + n_resp - 1 (a linear convolution).  This is
 * DftTools::convolve (aux/src/DftTools.cxx:145-168) applied to many rows, and
 * the long-range response step of ImpactTransform::waveform
 * (gen/src/ImpactTransform.cxx:327-343).  Device pointers, enqueued on stream
 * (cudaStream_t, NULL = legacy default stream) of the current device; scratch
 * is taken from the stream-ordered allocator.  Supported nfft: multiples of 4
 * whose half has no prime factor above 7 (WCT_ERR_SIZE otherwise). */
int wct_convolve_rows_device(const float* in, long ld_in, int nrows, int n_in, const float* resp, int n_resp,
                             int nfft, float* out, long ld_out, int n_out, void* stream);

/* The same convolution without any allocation, for callers that may not
 * allocate device memory once they are running: an online trigger or DAQ
 * process whose device-memory budget is fixed at start-up, or a host
 * framework that owns all device memory through its own pool and forbids
 * allocations behind its back (an allocation can fail under fragmentation and
 * can synchronise the device mid-run).  No counterpart in the reference, which
 * has no device path here.  Scratch is a fixed 32 MiB array in the library's
 * device image, held by every GPU that loads the library until the process
 * exits; a call needs (nrows + 3) * nfft / 2 <= 4194304 complex values and
 * returns WCT_ERR_SIZE beyond that.  The first call on a device looks up the
 * array's address (cudaGetSymbolAddress) with that device current and keeps
 * it for the life of the process; make that first call before any stream
 * capture, and make no call on a device after a cudaDeviceReset of it (the
 * kept address would be stale).  All calls share the array and each
 * overwrites what it uses: calls that overlap on the GPU (other streams or
 * threads) race, so serialise them. */
int wct_convolve_rows_device_noalloc(const float* in, long ld_in, int nrows, int n_in, const float* resp,
                                     int n_resp, int nfft, float* out, long ld_out, int n_out, void* stream);

/* ---- GPU IDFT (iface/inc/WireCellIface/IDFT.h) ---- */

/* The IDFT interface on the GPU: the cuFftDFT plugin that
 * cuda/test/test_idft_cufftdft.bats names (the reference has no GPU
 * implementation; FftwDFT, aux/src/FftwDFT.cxx:149-217, and TorchDFT,
 * pytorch/src/DFT.cxx:80-123, are its CPU ones).  Arrays are single
 * precision complex values stored as interleaved (re, im) float pairs in C
 * (row-major) order; in and out may be the same array.  Forward transforms
 * are unnormalised, inverse transforms carry 1/n (1/(nrows*ncols) for 2d).
 * 1b: axis = 1 transforms each of the nrows rows (length ncols), axis = 0
 * each column (length nrows), as numpy.fft.  Any length from 1 up: lengths
 * whose prime factors are at most 7 run in shared memory up to 14336 and as
 * four-step transforms (two passes of shorter ones) above; any other length
 * runs through Bluestein's chirp-z transform on such a length.  Arrays hold
 * at most 2^30 values, and the column transforms and transposes at most
 * 2097120 per side (WCT_ERR_SIZE beyond).  The host-pointer calls (IDFT::fwd1d, inv1d, fwd1b,
 * inv1b, fwd2d, inv2d, transpose) copy through the current device and
 * return when the result is in out; they may be called from several
 * threads at once (IDFT.h: "safe concurrent calls"). */
int wct_dft_fwd1d(const float* in, float* out, int size);
int wct_dft_inv1d(const float* in, float* out, int size);
int wct_dft_fwd1b(const float* in, float* out, int nrows, int ncols, int axis);
int wct_dft_inv1b(const float* in, float* out, int nrows, int ncols, int axis);
int wct_dft_fwd2d(const float* in, float* out, int nrows, int ncols);
int wct_dft_inv2d(const float* in, float* out, int nrows, int ncols);
/* IDFT::transpose: out[c][r] = in[r][c] for an nrows x ncols input, real or
 * complex elements. */
int wct_dft_transpose_real(const float* in, float* out, int nrows, int ncols);
int wct_dft_transpose_complex(const float* in, float* out, int nrows, int ncols);
/* The same on device arrays, enqueued on stream (cudaStream_t, NULL = legacy
 * default stream) of the current device; inverse != 0 selects the inverse.
 * Column transforms and in-place transposes take scratch from the
 * stream-ordered allocator. */
int wct_dft_1b_device(const float* in, float* out, int nrows, int ncols, int axis, int inverse, void* stream);
int wct_dft_2d_device(const float* in, float* out, int nrows, int ncols, int inverse, void* stream);
int wct_dft_transpose_device(const float* in, float* out, int nrows, int ncols, int is_complex, void* stream);

/* ---- DepoFluxSplat (gen/src/DepoFluxSplat.cxx, IDepoFramer) ---- */

/* DepoFluxSplat's configuration keys (gen/src/DepoFluxSplat.cxx:81-128):
 * tick, window_start, window_duration (frame ticks = (int)(duration / tick)),
 * nsigma, drift_speed, response_plane (depo times are shifted by
 * response_plane / drift_speed), time_offsets (per plane, in time), and the
 * extra smearing per plane: smear_long in ticks, smear_tran in wire pitches. */
typedef struct {
    double tick, window_start, window_duration, nsigma, drift_speed, response_plane;
    double time_offsets[3], smear_long[3], smear_tran[3];
} wct_splat_config;

/* The dense truth frame of DepoFluxSplat::operator() (:247-390) for drifted
 * depos ([n][7] t, q, x, y, z, extent_long, extent_tran, as at the response
 * plane) over the component's faces and planes: each depo's erf-integrated
 * Gaussian patch on (wire, tick), |charge| added; frame rows are the
 * component's wires (as the DepoTransform frame), columns the window's ticks;
 * samples that time_offsets move outside the window are dropped (the
 * reference keeps them in its traces).  wct_dt_splat_shape gives the frame
 * shape; the device version takes device depos and frame on stream (NULL:
 * the component's stream). */
int wct_dt_splat_shape(const wct_depotransform* dt, const wct_splat_config* cfg, int* nrows, int* nticks);
int wct_dt_splat_device(wct_depotransform* dt, const wct_splat_config* cfg, const double* depos, size_t ndepos,
                        float* frame, void* stream);
int wct_dt_splat(wct_depotransform* dt, const wct_splat_config* cfg, const double* depos, size_t ndepos, float* frame);

/* ---- Noise (gen/src/AddNoise.cxx, IFrameFilter) ---- */

/* IncoherentAddNoise / CoherentAddNoise (gen/src/AddNoise.cxx:44-160) with
 * the waveform of GeneratorN (aux/src/NoiseTools.cxx: sigma_k = S_k *
 * sqrt(2/3.141592); bins 0 .. N/2 drawn as sigma_k (n_k, n_{k+N/2}), DC and
 * Nyquist by modulus, Hermitian, inverse DFT with 1/N) added to each frame
 * row's first min(N, ncols) samples.  Row r uses spectrum row_spec[r] of
 * spectra [nspectra][nspec] (the model's channel_spectrum or group_spectrum;
 * -1: the row gets no noise) and the random stream row_stream[r]: the
 * channel number for incoherent noise, the group id for coherent noise (so
 * every channel of a group gets the same waveform).  Normals are
 * counter-based (key: seed, ident = frame ident; counter: stream, model,
 * normal index), so a frame's noise is reproducible and independent of the
 * launch; the reference's generator (std::mt19937 with recycled normals) is
 * matched in distribution, not in values.  nspec even with a 7-smooth half
 * up to 14336.  Device version on the current device and stream, the
 * spectrum indices unchecked (each below the number of spectra the caller
 * holds on the device); host version on host arrays (frame updated in place,
 * indices checked against nspectra). */
int wct_add_noise_device(float* frame, long ld, int nrows, int ncols, const float* spectra, int nspec,
                         const int* row_spec, const int* row_stream, unsigned long long seed, int ident, int model,
                         void* stream);
int wct_add_noise(float* frame, int nrows, int ncols, const float* spectra, int nspectra, int nspec,
                  const int* row_spec, const int* row_stream, unsigned long long seed, int ident, int model);

/* ---- Digitizer (gen/src/Digitizer.cxx, IFrameFilter) ---- */

/* Digitizer's per-sample arithmetic (gen/src/Digitizer.cxx:82-141) on a
 * dense frame: voltage = gain * value + row_baseline[row] (the baseline of
 * the row's plane, a float as the reference reads it), then ADC = 0 at or
 * below fs_lo, 2^resolution - 1 at or above fs_hi, otherwise
 * (voltage - fs_lo) / (fs_hi - fs_lo) * (2^resolution - 1), rounded (half
 * away from zero) when round_adc, else floored; in double precision, bit
 * for bit the reference's values.  The reference emits these for the
 * channels and tick range of its input traces; the dense result holds them
 * at the same rows and ticks.  Configuration keys map as resolution,
 * gain, fullscale = [fs_lo, fs_hi], baselines (per plane), round.
 * Device version: frame and adc (may be the same array) and row_baseline on
 * the current device, enqueued on stream; host version: host arrays. */
int wct_digitize_device(const float* frame, long ld_in, int nrows, int ncols, const float* row_baseline, double gain,
                        double fs_lo, double fs_hi, int resolution, int round_adc, float* adc, long ld_out,
                        void* stream);
int wct_digitize(const float* frame, int nrows, int ncols, const float* row_baseline, double gain, double fs_lo,
                 double fs_hi, int resolution, int round_adc, float* adc);

/* ---- DepoTransform (gen/src/DepoTransform.cxx, IDepoFramer) ---- */

/* DepoTransform::configure (gen/src/DepoTransform.cxx:76-113) from JSON with
 * the reference keys: anode, pirs, dft, rng, fluctuate, nsigma, start_time,
 * readout_time, tick, drift_speed, first_frame_number.  Optional extra keys:
 * "drifter" {DL, DT, lifetime, drift_speed, time_offset, fluctuate,
 * xregions:[{anode, response, cathode}]} to drift depos on the device before
 * the transform (Drifter, gen/src/Drifter.cxx:94-123; fluctuate defaults to
 * false here), "device" (CUDA ordinal) and "seed" (key of the random streams
 * that "fluctuate" draws from, in place of the reference's "rng" component).
 * WCT_ERR_CONFIG where DepoTransform::configure throws (empty "pirs"), for
 * malformed JSON, for a non-positive tick, readout_time or drift_speed, a
 * readout of less than one tick, and integer keys out of their range. */
int wct_dt_create(const char* json_config, wct_depotransform** out);
/* The calls below that take a component are serialised on it: configuration
 * calls and forwards from several host threads take turns (as the
 * reference's single-threaded node); separate components run concurrently. */
/* DepoTransform::default_configuration (gen/src/DepoTransform.cxx:114-153) as JSON. */
int wct_dt_default_configuration(char* buf, size_t len);
/* Add an anode face with its sensitive volume (IAnodeFace::sensitive,
 * gen/src/AnodePlane.cxx:259-290); bb_lo == NULL means no volume cut. */
int wct_dt_add_face(wct_depotransform* dt, const double* bb_lo, const double* bb_hi, int* face);
/* Add a wire plane to a face (IAnodeFace::planes order); WCT_ERR_CONFIG
 * unless nwires >= 2, nimpacts even and >= 2, and pitchmax > pitchmin. */
int wct_dt_add_plane(wct_depotransform* dt, int face, const wct_plane_desc* desc, int* plane);
/* Use a PIR for a plane: ImpactTransform's response selection
 * (gen/src/ImpactTransform.cxx:26-74) over pirs[plane]. */
int wct_dt_set_response_pir(wct_depotransform* dt, int face, int plane, const wct_pir* pir);
/* The plane's long-range response (set by wct_dt_set_response_pir from the
 * PIR; nsamples = 0: none): every frame row inside the plane's window is
 * circularly convolved with wave, both zero padded to
 * fft_best_length(nticks + pad), and cut back to nticks
 * (ImpactTransform::waveform, gen/src/ImpactTransform.cxx:327-343); the
 * adjoint applies the transposed step. */
int wct_dt_set_long_response(wct_depotransform* dt, int face, int plane, int nsamples, const float* wave, int pad);
/* Same from a ready table: table[g][j][k] for impact group g < ngroups, wire
 * offset j - npad in [-npad, npad], tick k < nsamples (the closest() waveform
 * for that group and offset). */
int wct_dt_set_response_table(wct_depotransform* dt, int face, int plane, int ngroups, int npad, int nsamples,
                              double pitch, double impact, int waveform_pad, const float* table);
/* Frame geometry: total wire rows and nticks. */
int wct_dt_frame_shape(const wct_depotransform* dt, int* nrows, int* nticks);

/* DepoTransform::modify_depo (gen/inc/WireCellGen/DepoTransform.h:33-35),
 * the per-plane hook a subclass overrides to rescale each depo's charge
 * before BinnedDiffusion_transform::add (gen/src/DepoTransform.cxx:182;
 * dQ/dx calibrations of larwirecell and uboonecode), as data: depo i brings
 * charge * scale[i * nplanes + p] to plane p (p over every plane of every
 * face, in frame order), after the drift and the face's sensitive-volume
 * cut, before the rejection tests, the patch normalisation and the
 * fluctuation draws.  scale has ndepos * nplanes doubles, in host memory
 * (on_device = 0) or device memory of the component's device (on_device !=
 * 0); it is copied, and the copy is complete when the call returns.  It holds
 * for every later forward, batched forward (ndepos = the batch's total, depos
 * concatenated) and adjoint call with exactly ndepos depos and the same
 * planes; other counts return WCT_ERR_ARG.  The adjoint's charge gradient
 * carries the scale.  scale == NULL removes it.  Work already enqueued on
 * other streams must be done with the previous scale before this call
 * overwrites it (synchronise those streams first). */
int wct_dt_set_charge_scale(wct_depotransform* dt, const double* scale, size_t ndepos, int on_device);

/* DepoTransform::operator() (gen/src/DepoTransform.cxx:155-224) on host
 * buffers: depos [ndepos][7] in, dense frame [nrows][nticks] out, one window
 * per plane (may be NULL), frame ident out (may be NULL).  The transfers
 * overlap the kernels: the depos go up in chunks that the first kernel takes
 * as they arrive, each plane's zero rows and ticks come back while the
 * kernels run and its window block once the plane is done; every element of
 * frame is written.  Page-locked host buffers let the copies run alongside
 * the kernels. */
int wct_dt_forward(wct_depotransform* dt, const double* depos, size_t ndepos, float* frame,
                   wct_plane_window* windows, int* frame_ident);
/* DepoTransform::operator() (gen/src/DepoTransform.cxx:155-224) with its
 * output as the reference builds it: the trace list of SimpleFrame
 * (:193-215), one trace per wire with a non-zero sample, trimmed to
 * [first non-zero, last non-zero] by Waveform::edge
 * (util/src/Waveform.cxx:136-153), in frame row order (faces, planes,
 * wires).  Trace k is channel[k], tbin[k], length[k] samples at
 * charge + offset[k]; *ntraces receives the count (channel, tbin, length and
 * offset have room for nrows entries).  Every trace lies inside its plane's
 * window (the frame is zero elsewhere), so only the window blocks cross from
 * the device: charge holds them one after another and needs at most the sum
 * over planes of window rows x window ticks floats (capacity; nrows * nticks
 * always suffices; WCT_ERR_SIZE if it is too small).  The edges are found on
 * the device and each plane's block comes back as soon as the plane is
 * final.  *nsamples (may be NULL) receives the number of charge values
 * written.  windows and frame_ident as wct_dt_forward (may be NULL). */
int wct_dt_forward_traces(wct_depotransform* dt, const double* depos, size_t ndepos, float* charge, size_t capacity,
                          int* channel, int* tbin, int* length, long* offset, int* ntraces, size_t* nsamples,
                          wct_plane_window* windows, int* frame_ident);
/* The same on device buffers, enqueued on stream (cudaStream_t, NULL = the
 * component's own stream).  Returns after the work is enqueued; one small
 * device-to-host read of the window sizes synchronises the stream mid-way. */
int wct_dt_forward_device(wct_depotransform* dt, const double* d_depos, size_t ndepos, float* d_frame,
                          wct_plane_window* windows, int* frame_ident, void* stream);
/* End of stream (DepoTransform.cxx:157-162): acknowledges with WCT_EOS. */
int wct_dt_eos(wct_depotransform* dt);
/* Trace assembly (DepoTransform.cxx:193-208 with Waveform::edge,
 * util/src/Waveform.cxx:136-153) from a host frame: for every wire with a
 * non-zero sample, channel, first tick and length of [first nonzero, last
 * nonzero].  Arrays have room for nrows entries; *ntraces receives the count. */
int wct_dt_traces(const wct_depotransform* dt, const float* frame, int* channel, int* tbin, int* length,
                  long* offset, int* ntraces);
/* Patch placement of every input depo on one plane from the last forward
 * call: out[i] = {toffset, poffset, nt, np} of GaussianDiffusion::set_sampling
 * (gen/src/GaussianDiffusion.cxx:116-149); nt = np = 0 where the depo adds no
 * patch (dropped by the drift, the sensitive volume, BinnedDiffusion_transform::add
 * or an empty sample range).  n must equal the last call's depo count.  The
 * records are read with a blocking copy on the legacy default stream, which
 * does not wait for the component's streams: after wct_dt_forward_device,
 * synchronise its stream first (wct_dt_forward returns complete). */
int wct_dt_patch_records(const wct_depotransform* dt, int face, int plane, int* out, size_t n);
/* Stage profiling (the engine-level timers of pgraph/src/Graph.cxx:118-122,
 * here per device stage): when enabled, every forward call records CUDA
 * events around its stages on the launch stream.  wct_dt_stage_times
 * returns, per stage, the accumulated milliseconds and launch count since the
 * last reset (stages: 0 drift+prep, 1 raster, 2 time FFT, 3 wire convolution,
 * 4 inverse FFT + frame, 5 other; adjoint calls add 6 frame-gradient time FFT,
 * 7 transposed wire convolution, 8 inverse FFT to dL/dQ, 9 per-depo gather),
 * and the total number of kernel launches. */
int wct_dt_set_profiling(wct_depotransform* dt, int on);
int wct_dt_stage_times(wct_depotransform* dt, double* ms, long* launches, int nstages, long* total_launches,
                       int reset);

/* ---- Batched events (no counterpart in the reference, which frames one
 * event per DepoTransform call) ----
 *
 * DepoTransform::operator() over nevents events at once: event e holds depos
 * [offsets[e], offsets[e+1]) of d_depos ([offsets[nevents]][7], device) and
 * its frame is d_frames + e * nrows * nticks (device).  Each frame equals the
 * frame of wct_dt_forward_device for that event within floating-point
 * rounding (time FFT lengths come from a fixed ladder instead of each
 * window's own length).  The windows of all events are planned on the device,
 * so the whole batch runs as one CUDA graph, captured on the first call and
 * replayed while the offsets, buffers, stream, launch shapes and drift
 * parameters stay the same.  windows: [nevents][nplanes] or NULL; frame
 * idents are first_ident .. first_ident + nevents - 1.  Returns after the
 * batch completes.  offsets is a host array of nevents + 1 values with
 * offsets[0] = 0. */
int wct_dt_forward_batch_device(wct_depotransform* dt, const double* d_depos, const long long* offsets, int nevents,
                                float* d_frames, wct_plane_window* windows, int* first_ident, void* stream);
/* The same on host buffers (frames [nevents][nrows][nticks]). */
int wct_dt_forward_batch(wct_depotransform* dt, const double* depos, const long long* offsets, int nevents,
                         float* frames, wct_plane_window* windows, int* first_ident);
/* Launch shapes of the batched path: params[5] = {events per pass, persistent
 * raster blocks per SM, threads per time-FFT row (128..1024, power of 2),
 * time-FFT blocks per SM, wire-convolution blocks per SM}; set != 0 sets them,
 * otherwise they are read. */
int wct_dt_batch_tune(wct_depotransform* dt, int* params, int set);
/* Autotuner: times candidate launch shapes on the given batch (device
 * buffers as for wct_dt_forward_batch_device), keeps the fastest and writes a
 * JSON report of every candidate and its time to report (may be NULL). */
int wct_dt_autotune_batch(wct_depotransform* dt, const double* d_depos, const long long* offsets, int nevents,
                          float* d_frames, void* stream, char* report, size_t len);

/* ---- Random numbers of the fluctuated forward ----
 *
 * With "fluctuate": true (DepoTransform, gen/src/DepoTransform.cxx:82-87) every
 * patch cell is redrawn as Binomial(|Q|, cell fraction) and the patch rescaled
 * to Q (gen/src/GaussianDiffusion.cxx:184-213); with a drifter "fluctuate":
 * true the absorbed electrons are Binomial(|Q|, 1 - exp(-dt / lifetime))
 * (gen/src/Drifter.cxx:177-185).  The draws come from counter-based streams
 * (Philox-4x32-10) keyed by the configuration's "seed" and each event's frame
 * ident, so a call is reproducible and successive frames draw afresh.
 * IRandom::binomial (iface/inc/WireCellIface/IRandom.h) in bulk: count
 * independent Binomial(n, p) draws of the stream (seed, ident) into d_out
 * (device), enqueued on stream (NULL = legacy default stream). */
int wct_random_binomial_device(unsigned long long seed, int ident, int n, double p, long count, int* d_out,
                               void* stream);

/* Reverse-mode derivative of wct_dt_forward (no counterpart in the reference,
 * whose DepoTransform is forward only).  Given grad_frame = dL/d(frame)
 * [nrows][nticks] for the same depos, writes grad_depos[i][k] = dL/d(depos[i][k])
 * for k = t, q, x, y, z, extent_long, extent_tran, and, when grad_drift is not
 * NULL, dL/d(DL, DT, lifetime) of the drifter (zeros without one).  Patch
 * placement is recomputed from the depos, and patch windows, rejections and
 * event windows are held fixed (they are the piecewise-constant part of the
 * forward).  Outputs are overwritten. */
int wct_dt_adjoint(wct_depotransform* dt, const double* depos, size_t ndepos, const float* grad_frame,
                   double* grad_depos, double* grad_drift);
/* The same on device buffers, enqueued on stream (NULL = the component's own
 * stream); grad_drift is a device array of 3 doubles or NULL. */
int wct_dt_adjoint_device(wct_depotransform* dt, const double* d_depos, size_t ndepos, const float* d_grad_frame,
                          double* d_grad_depos, double* d_grad_drift, void* stream);
/* Drifter parameters DL, DT (length^2/time) and electron lifetime of a
 * component configured with a "drifter" (Drifter, gen/src/Drifter.cxx:62-71);
 * WCT_ERR_STATE without one. */
int wct_dt_set_drift_params(wct_depotransform* dt, double DL, double DT, double lifetime);
int wct_dt_get_drift_params(const wct_depotransform* dt, double* DL, double* DT, double* lifetime);
int wct_dt_destroy(wct_depotransform* dt);

#ifdef __cplusplus
}
#endif

#endif /* WCTB200_H */
