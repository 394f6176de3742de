"""wctb200: B200-native Wire-Cell DepoTransform.

Python front end of ``libwctb200.so`` (C ABI in include/wctb200.h).  The
classes mirror the reference components used on the signal-simulation path:

* :class:`PlaneImpactResponse`  Gen::PlaneImpactResponse (gen/src/PlaneImpactResponse.cxx)
* :class:`DepoTransform`        Gen::DepoTransform, an IDepoFramer (gen/src/DepoTransform.cxx)

The compute path is the CUDA library; there is no CPU fallback.  Importing
works without a GPU (the library loads), but every compute call needs one.
"""

import ctypes as C
import json
import os

import numpy as np

from . import _build

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = _build.LIB

WCT_OK, WCT_ERR_ARG, WCT_ERR_CONFIG, WCT_ERR_CUDA, WCT_ERR_STATE, WCT_ERR_RESPONSE, WCT_ERR_SIZE, WCT_EOS = range(8)

_lib = None


class WctError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("wctb200 error %d: %s" % (code, msg))
        self.code = code


class PlaneDesc(C.Structure):
    _fields_ = [
        ("nwires", C.c_int), ("nimpacts", C.c_int),
        ("pitchmin", C.c_double), ("pitchmax", C.c_double),
        ("wire", C.c_double * 3), ("pitch", C.c_double * 3), ("origin", C.c_double * 3),
        ("channels", C.c_void_p),
    ]


class FrPlane(C.Structure):
    _fields_ = [
        ("npaths", C.c_int), ("nsamples", C.c_int),
        ("pitchpos", C.c_void_p), ("current", C.c_void_p),
        ("pitch", C.c_double), ("tstart", C.c_double), ("period", C.c_double),
    ]


class SplatConfig(C.Structure):
    """wct_splat_config: DepoFluxSplat's configuration keys (gen/src/DepoFluxSplat.cxx:81-128)."""
    _fields_ = [(n, C.c_double) for n in ("tick", "window_start", "window_duration", "nsigma", "drift_speed",
                                          "response_plane")] + \
        [("time_offsets", C.c_double * 3), ("smear_long", C.c_double * 3), ("smear_tran", C.c_double * 3)]

    @classmethod
    def make(cls, tick=500.0, window_start=0.0, window_duration=8096 * 500.0, nsigma=3.0, drift_speed=1.6e-3,
             response_plane=100.0, time_offsets=None, smear_long=None, smear_tran=None):
        c = cls(tick, window_start, window_duration, nsigma, drift_speed, response_plane)
        for name, v in (("time_offsets", time_offsets), ("smear_long", smear_long), ("smear_tran", smear_tran)):
            v = v or [0.0, 0.0, 0.0]
            for i in range(3):
                getattr(c, name)[i] = float(v[i])
        return c


class PlaneWindow(C.Structure):
    _fields_ = [(n, C.c_int) for n in (
        "face", "plane", "start_ch", "end_ch", "start_tick", "end_tick", "nw_fft", "nt_fft", "nt_gpu",
        "charge_rows", "npad", "ndepos_added", "outside_time", "outside_pitch")]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


# name -> (restype, argtypes); every function listed here is declared in include/wctb200.h
SIGNATURES = {
    "wct_version": (C.c_char_p, []),
    "wct_last_error": (C.c_char_p, []),
    "wct_pir_create": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_int,
                                 C.POINTER(C.c_void_p)]),
    "wct_pir_closest": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(C.c_int)]),
    "wct_pir_info": (C.c_int, [C.c_void_p] + [C.c_void_p] * 8),
    "wct_pir_waveform": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "wct_pir_destroy": (C.c_int, [C.c_void_p]),
    "wct_pir_create_device": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_int,
                                        C.POINTER(C.c_void_p)]),
    "wct_pir_set_long_responses_device": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_double]),
    "wct_pir_set_long_responses": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_double]),
    "wct_pir_long_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "wct_pir_long_waveform": (C.c_int, [C.c_void_p, C.c_void_p]),
    "wct_convolve_rows_device": (C.c_int, [C.c_void_p, C.c_long, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int,
                                           C.c_void_p, C.c_long, C.c_int, C.c_void_p]),
    "wct_fft_best_length": (C.c_long, [C.c_long, C.c_int]),
    "wct_dt_splat_shape": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "wct_dt_splat_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p]),
    "wct_dt_splat": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]),
    "wct_add_noise_device": (C.c_int, [C.c_void_p, C.c_long, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                       C.c_void_p, C.c_ulonglong, C.c_int, C.c_int, C.c_void_p]),
    "wct_add_noise": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                C.c_ulonglong, C.c_int, C.c_int]),
    "wct_digitize_device": (C.c_int, [C.c_void_p, C.c_long, C.c_int, C.c_int, C.c_void_p, C.c_double, C.c_double,
                                      C.c_double, C.c_int, C.c_int, C.c_void_p, C.c_long, C.c_void_p]),
    "wct_digitize": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_int,
                               C.c_int, C.c_void_p]),
    "wct_dft_fwd1d": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "wct_dft_inv1d": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "wct_dft_fwd1b": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int]),
    "wct_dft_inv1b": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int]),
    "wct_dft_fwd2d": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int]),
    "wct_dft_inv2d": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int]),
    "wct_dft_transpose_real": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int]),
    "wct_dft_transpose_complex": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int]),
    "wct_dft_1b_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]),
    "wct_dft_2d_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p]),
    "wct_dft_transpose_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p]),
    "wct_convolve_rows_device_noalloc": (C.c_int, [C.c_void_p, C.c_long, C.c_int, C.c_int, C.c_void_p, C.c_int,
                                                   C.c_int, C.c_void_p, C.c_long, C.c_int, C.c_void_p]),
    "wct_dt_create": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "wct_dt_default_configuration": (C.c_int, [C.c_char_p, C.c_size_t]),
    "wct_dt_add_face": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_int)]),
    "wct_dt_add_plane": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.POINTER(C.c_int)]),
    "wct_dt_set_response_pir": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    "wct_dt_set_long_response": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int]),
    "wct_dt_set_response_table": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                            C.c_double, C.c_int, C.c_void_p]),
    "wct_dt_frame_shape": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "wct_dt_set_charge_scale": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]),
    "wct_dt_forward_traces": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_int),
                                        C.POINTER(C.c_size_t), C.c_void_p, C.POINTER(C.c_int)]),
    "wct_dt_forward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p, C.POINTER(C.c_int)]),
    "wct_dt_forward_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p,
                                        C.POINTER(C.c_int), C.c_void_p]),
    "wct_dt_eos": (C.c_int, [C.c_void_p]),
    "wct_dt_traces": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                C.POINTER(C.c_int)]),
    "wct_dt_patch_records": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_size_t]),
    "wct_dt_set_profiling": (C.c_int, [C.c_void_p, C.c_int]),
    "wct_dt_stage_times": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_long), C.c_int]),
    "wct_dt_adjoint": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p]),
    "wct_dt_adjoint_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p]),
    "wct_dt_set_drift_params": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double]),
    "wct_dt_get_drift_params": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                          C.POINTER(C.c_double)]),
    "wct_dt_forward_batch_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                              C.POINTER(C.c_int), C.c_void_p]),
    "wct_dt_forward_batch": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                       C.POINTER(C.c_int)]),
    "wct_dt_batch_tune": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "wct_dt_autotune_batch": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                        C.c_char_p, C.c_size_t]),
    "wct_random_binomial_device": (C.c_int, [C.c_ulonglong, C.c_int, C.c_int, C.c_double, C.c_long, C.c_void_p,
                                             C.c_void_p]),
    "wct_dt_destroy": (C.c_int, [C.c_void_p]),
}

STAGES = ("drift+prep", "raster", "time_fft", "wire_conv", "inverse_fft+frame", "other",
          "adj_time_fft", "adj_wire_conv", "adj_inverse_fft", "adj_gather")


def build(force=False):
    return _build.build(force=force)


def lib():
    """Load libwctb200.so (building it first if it is missing or stale)."""
    global _lib
    if _lib is None:
        if _build.stale():
            _build.build()
        _lib = C.CDLL(LIB_PATH)
        for name, (rt, at) in SIGNATURES.items():
            f = getattr(_lib, name)
            f.restype = rt
            f.argtypes = at
    return _lib


CUDA_STREAM_LEGACY = 1  # cudaStreamLegacy


def _dt_stream(stream):
    """Stream argument of the component's device entry points: None selects the
    component's own stream; 0 (the handle of torch's default stream) is passed
    as the legacy default stream, since the C ABI reads NULL as the former."""
    if stream is None:
        return None
    return C.c_void_p(stream if stream else CUDA_STREAM_LEGACY)


def _check(rc):
    if rc != WCT_OK:
        raise WctError(rc, lib().wct_last_error().decode())
    return rc


class PlaneImpactResponse:
    """Gen::PlaneImpactResponse built from a Response::Schema plane, short
    responses and optional long responses with their padding
    (gen/src/PlaneImpactResponse.cxx:56-269); ``device=True`` builds the
    waveforms on the current CUDA device in single precision (the
    reference's FFT chain), else on the host in double precision."""

    def __init__(self, fr, short_responses, overall_short_padding, tick, nticks, long_responses=(),
                 long_padding=1.5e6, device=False):
        L = lib()
        pp = np.ascontiguousarray(fr["pitchpos"], dtype=np.float64)
        cur = np.ascontiguousarray(fr["current"], dtype=np.float64)
        d = FrPlane(pp.shape[0], cur.shape[1], pp.ctypes.data, cur.ctypes.data, fr["pitch"], fr["tstart"],
                    fr["period"])
        shorts = [np.asarray(s, dtype=np.float64) for s in short_responses]
        sl = np.array([len(s) for s in shorts] or [0], dtype=np.int32)
        sw = np.concatenate(shorts) if shorts else np.zeros(1)
        h = C.c_void_p()
        create = L.wct_pir_create_device if device else L.wct_pir_create
        _check(create(C.byref(d), len(shorts), sl.ctypes.data, sw.ctypes.data, overall_short_padding, tick, nticks,
                      C.byref(h)))
        self.h = h
        longs = [np.asarray(w, dtype=np.float64) for w in long_responses]
        if longs:
            ll = np.array([len(w) for w in longs], dtype=np.int32)
            lw = np.concatenate(longs)
            setl = L.wct_pir_set_long_responses_device if device else L.wct_pir_set_long_responses
            _check(setl(h, len(longs), ll.ctypes.data, lw.ctypes.data, long_padding))

    def long_waveform(self):
        """(long-range response samples, pad in ticks); an empty array without one."""
        n, pad = C.c_int(), C.c_int()
        _check(lib().wct_pir_long_info(self.h, C.byref(n), C.byref(pad)))
        out = np.zeros(n.value, dtype=np.float32)
        if n.value:
            _check(lib().wct_pir_long_waveform(self.h, out.ctypes.data))
        return out, pad.value

    def info(self):
        pitch, impact, he = C.c_double(), C.c_double(), C.c_double()
        nw, ni, npth, nt, wp = C.c_int(), C.c_int(), C.c_int(), C.c_int(), C.c_int()
        _check(lib().wct_pir_info(self.h, C.byref(pitch), C.byref(impact), C.byref(he), C.byref(nw), C.byref(ni),
                                  C.byref(npth), C.byref(nt), C.byref(wp)))
        return dict(pitch=pitch.value, impact=impact.value, half_extent=he.value, nwires=nw.value,
                    nimp_per_wire=ni.value, npaths=npth.value, nticks=nt.value, waveform_pad=wp.value)

    def closest(self, relpitch):
        k = C.c_int()
        _check(lib().wct_pir_closest(self.h, relpitch, C.byref(k)))
        return k.value

    def waveform(self, path):
        out = np.zeros(self.info()["nticks"], dtype=np.float32)
        _check(lib().wct_pir_waveform(self.h, path, out.ctypes.data))
        return out

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.wct_pir_destroy(self.h)
            self.h = None


def convolve_rows(d_in, ld_in, nrows, n_in, d_resp, n_resp, d_out, ld_out, n_out, nfft=0, stream=None):
    """Batched FFT convolution of device rows with one response (pointers as ints)."""
    _check(lib().wct_convolve_rows_device(C.c_void_p(d_in), ld_in, nrows, n_in, C.c_void_p(d_resp), n_resp, nfft,
                                          C.c_void_p(d_out), ld_out, n_out, C.c_void_p(stream) if stream else None))


def fft_best_length(n, keep_odd_even=False):
    """util/src/FFTBestLength.cxx: smallest fast FFT length >= n of the reference's tables."""
    return int(lib().wct_fft_best_length(int(n), 1 if keep_odd_even else 0))


def add_noise_device(d_frame, ld, nrows, ncols, d_spectra, nspec, d_row_spec, d_row_stream, seed=0, ident=0, model=0,
                     stream=None):
    """add_noise on device arrays (pointers as ints), enqueued on stream."""
    _check(lib().wct_add_noise_device(C.c_void_p(d_frame), ld, nrows, ncols, C.c_void_p(d_spectra), nspec,
                                      C.c_void_p(d_row_spec), C.c_void_p(d_row_stream), int(seed), int(ident),
                                      int(model), C.c_void_p(stream) if stream else None))


def add_noise(frame, spectra, row_spec, row_stream, seed=0, ident=0, model=0):
    """IncoherentAddNoise / CoherentAddNoise on a host frame [nrows][ncols]
    float32 (updated in place and returned): spectra [nspectra][nspec]
    amplitude spectra, row_spec[r] the spectrum of row r (-1: none),
    row_stream[r] its random stream (channel number, or group id for
    coherent noise)."""
    f = frame if (isinstance(frame, np.ndarray) and frame.dtype == np.float32 and frame.flags.c_contiguous) \
        else np.ascontiguousarray(frame, dtype=np.float32)
    sp = np.ascontiguousarray(spectra, dtype=np.float32)
    rs = np.ascontiguousarray(row_spec, dtype=np.int32)
    rt = np.ascontiguousarray(row_stream, dtype=np.int32)
    _check(lib().wct_add_noise(f.ctypes.data, f.shape[0], f.shape[1], sp.ctypes.data, sp.shape[0], sp.shape[1],
                               rs.ctypes.data, rt.ctypes.data, int(seed), int(ident), int(model)))
    return f


class Digitizer:
    """Gen::Digitizer (gen/src/Digitizer.cxx) on a dense frame: configuration
    keys resolution, gain, fullscale, baselines (per plane), round with the
    reference's defaults; ``rows_per_plane`` gives the frame's row count of
    each plane in order (the DepoTransform frame layout)."""

    VOLT = 1.0e-6  # the toolkit's system of units (WireCellUtil/Units.h)

    def __init__(self, rows_per_plane, resolution=12, gain=1.0, fullscale=(0.0, 2.0 * VOLT), baselines=None,
                 round=False):
        # reference defaults: 12 bits, gain 1, 0 .. 2 V, baselines 900, 900, 200 mV
        self.rows_per_plane = list(rows_per_plane)
        if baselines is None:
            baselines = [0.9 * self.VOLT, 0.9 * self.VOLT, 0.2 * self.VOLT][:len(self.rows_per_plane)]
        self.resolution, self.gain, self.fullscale, self.round = int(resolution), float(gain), fullscale, bool(round)
        self.row_baseline = np.concatenate([np.full(n, b, dtype=np.float32)
                                            for n, b in zip(self.rows_per_plane, baselines)])

    def __call__(self, frame, out=None):
        f = np.ascontiguousarray(frame, dtype=np.float32)
        out = np.empty_like(f) if out is None else out
        _check(lib().wct_digitize(f.ctypes.data, f.shape[0], f.shape[1], self.row_baseline.ctypes.data, self.gain,
                                  self.fullscale[0], self.fullscale[1], self.resolution, int(self.round),
                                  out.ctypes.data))
        return out

    def device(self, d_frame, ld_in, nrows, ncols, d_row_baseline, d_adc, ld_out, stream=None):
        _check(lib().wct_digitize_device(C.c_void_p(d_frame), ld_in, nrows, ncols, C.c_void_p(d_row_baseline),
                                         self.gain, self.fullscale[0], self.fullscale[1], self.resolution,
                                         int(self.round), C.c_void_p(d_adc), ld_out,
                                         C.c_void_p(stream) if stream else None))


class IDFT:
    """The IDFT interface (iface/inc/WireCellIface/IDFT.h) on the GPU, for
    numpy arrays: complex64 in and out (converted if needed), C order, forward
    unnormalised, inverse with 1/n; 1b axis as numpy.fft (1: along rows).
    Each call copies through the current device and returns the result."""

    @staticmethod
    def _c(a):
        return np.ascontiguousarray(a, dtype=np.complex64)

    def _run(self, fn, x, *shape):
        x = self._c(x)
        out = np.empty_like(x)
        _check(fn(x.ctypes.data, out.ctypes.data, *shape))
        return out

    def fwd1d(self, x):
        x = self._c(x).reshape(-1)
        return self._run(lib().wct_dft_fwd1d, x, x.size)

    def inv1d(self, x):
        x = self._c(x).reshape(-1)
        return self._run(lib().wct_dft_inv1d, x, x.size)

    def fwd1b(self, x, axis):
        x = self._c(x)
        return self._run(lib().wct_dft_fwd1b, x, x.shape[0], x.shape[1], int(axis))

    def inv1b(self, x, axis):
        x = self._c(x)
        return self._run(lib().wct_dft_inv1b, x, x.shape[0], x.shape[1], int(axis))

    def fwd2d(self, x):
        x = self._c(x)
        return self._run(lib().wct_dft_fwd2d, x, x.shape[0], x.shape[1])

    def inv2d(self, x):
        x = self._c(x)
        return self._run(lib().wct_dft_inv2d, x, x.shape[0], x.shape[1])

    def transpose(self, x):
        """IDFT::transpose of a 2-D float32 or complex64 array."""
        if np.iscomplexobj(x):
            x = self._c(x)
            out = np.empty((x.shape[1], x.shape[0]), dtype=np.complex64)
            _check(lib().wct_dft_transpose_complex(x.ctypes.data, out.ctypes.data, x.shape[0], x.shape[1]))
        else:
            x = np.ascontiguousarray(x, dtype=np.float32)
            out = np.empty((x.shape[1], x.shape[0]), dtype=np.float32)
            _check(lib().wct_dft_transpose_real(x.ctypes.data, out.ctypes.data, x.shape[0], x.shape[1]))
        return out


def dft_1b_device(d_in, d_out, nrows, ncols, axis, inverse=False, stream=None):
    """IDFT 1b transform of a device complex64 array (pointers as ints)."""
    _check(lib().wct_dft_1b_device(C.c_void_p(d_in), C.c_void_p(d_out), nrows, ncols, int(axis), int(bool(inverse)),
                                   C.c_void_p(stream) if stream else None))


def dft_2d_device(d_in, d_out, nrows, ncols, inverse=False, stream=None):
    """IDFT 2d transform of a device complex64 array (pointers as ints)."""
    _check(lib().wct_dft_2d_device(C.c_void_p(d_in), C.c_void_p(d_out), nrows, ncols, int(bool(inverse)),
                                   C.c_void_p(stream) if stream else None))


def convolve_rows_noalloc(d_in, ld_in, nrows, n_in, d_resp, n_resp, d_out, ld_out, n_out, nfft=0, stream=None):
    """Same as convolve_rows with no device allocation: scratch is the library's
    fixed 32 MiB device array (see wct_convolve_rows_device_noalloc)."""
    _check(lib().wct_convolve_rows_device_noalloc(C.c_void_p(d_in), ld_in, nrows, n_in, C.c_void_p(d_resp), n_resp,
                                                  nfft, C.c_void_p(d_out), ld_out, n_out,
                                                  C.c_void_p(stream) if stream else None))


class DepoTransform:
    """Gen::DepoTransform (IDepoFramer) on the B200.

    ``cfg`` is the reference configuration (gen/src/DepoTransform.cxx:76-153)
    as a dict, optionally with a "drifter" sub-configuration to drift the
    depos on the device first."""

    CONFIG_KEYS = ("anode", "pirs", "dft", "rng", "fluctuate", "nsigma", "start_time", "readout_time", "tick",
                   "drift_speed", "first_frame_number", "drifter", "device", "seed")

    def __init__(self, cfg=None):
        L = lib()
        js = json.dumps(_jsonable({k: v for k, v in (cfg or {}).items() if k in self.CONFIG_KEYS}))
        h = C.c_void_p()
        _check(L.wct_dt_create(js.encode(), C.byref(h)))
        self.h = h
        self._pirs = []
        self.planes = []

    @staticmethod
    def default_configuration():
        buf = C.create_string_buffer(4096)
        _check(lib().wct_dt_default_configuration(buf, 4096))
        return json.loads(buf.value.decode())

    def add_face(self, bb=None):
        f = C.c_int()
        if bb is None:
            _check(lib().wct_dt_add_face(self.h, None, None, C.byref(f)))
        else:
            lo = np.ascontiguousarray(bb[0], dtype=np.float64)
            hi = np.ascontiguousarray(bb[1], dtype=np.float64)
            _check(lib().wct_dt_add_face(self.h, lo.ctypes.data, hi.ctypes.data, C.byref(f)))
        return f.value

    def add_plane(self, face, pl):
        ch = np.ascontiguousarray(pl.get("channels", np.arange(pl["nwires"])), dtype=np.int32)
        d = PlaneDesc(pl["nwires"], pl.get("nimp", 10), pl["pitchmin"], pl["pitchmax"], (C.c_double * 3)(*pl["wire"]),
                      (C.c_double * 3)(*pl["pitch"]), (C.c_double * 3)(*pl["origin"]), ch.ctypes.data)
        p = C.c_int()
        _check(lib().wct_dt_add_plane(self.h, face, C.byref(d), C.byref(p)))
        self.planes.append((face, p.value, pl["nwires"]))
        return p.value

    def set_response_pir(self, face, plane, pir):
        _check(lib().wct_dt_set_response_pir(self.h, face, plane, pir.h))
        self._pirs.append(pir)

    def set_response_table(self, face, plane, table, pitch, impact, waveform_pad):
        t = np.ascontiguousarray(table, dtype=np.float32)
        G, J, K = t.shape
        _check(lib().wct_dt_set_response_table(self.h, face, plane, G, (J - 1) // 2, K, pitch, impact, waveform_pad,
                                               t.ctypes.data))

    def set_charge_scale(self, scale=None, d_scale_ptr=None, ndepos=None):
        """DepoTransform::modify_depo as a per-plane charge scale: depo i
        brings charge * scale[i][p] to plane p (frame order over all faces)
        for the following calls with that many depos.  ``scale``: host array
        [ndepos][nplanes]; or a device pointer ``d_scale_ptr`` with
        ``ndepos``; neither: remove it."""
        if scale is None and d_scale_ptr is None:
            _check(lib().wct_dt_set_charge_scale(self.h, None, 0, 0))
            return
        if d_scale_ptr is not None:
            _check(lib().wct_dt_set_charge_scale(self.h, C.c_void_p(d_scale_ptr), int(ndepos), 1))
            return
        a = np.ascontiguousarray(scale, dtype=np.float64)
        assert a.ndim == 2 and a.shape[1] == len(self.planes), a.shape
        self._qscale = a
        _check(lib().wct_dt_set_charge_scale(self.h, a.ctypes.data, a.shape[0], 0))

    def frame_shape(self):
        r, t = C.c_int(), C.c_int()
        _check(lib().wct_dt_frame_shape(self.h, C.byref(r), C.byref(t)))
        return r.value, t.value

    def __call__(self, depos, out=None):
        """Host-buffer forward: returns (frame [nrows][nticks] float32, windows, ident).
        ``out`` may supply the frame buffer (e.g. pinned host memory)."""
        d = np.ascontiguousarray(depos, dtype=np.float64).reshape(-1, 7)
        nrows, nticks = self.frame_shape()
        if out is not None:
            assert out.shape == (nrows, nticks) and out.dtype == np.float32 and out.flags.c_contiguous
            frame = out
        else:
            frame = np.empty((nrows, nticks), dtype=np.float32)
        wins = (PlaneWindow * len(self.planes))()
        ident = C.c_int()
        _check(lib().wct_dt_forward(self.h, d.ctypes.data if len(d) else None, len(d), frame.ctypes.data,
                                    C.cast(wins, C.c_void_p), C.byref(ident)))
        return frame, [w.as_dict() for w in wins], ident.value

    def forward_traces(self, depos, charge=None, meta=None):
        """Host-buffer forward returning the reference's trace list: (traces,
        windows, ident, nsamples) with traces a list of (channel, tbin, charges
        view) and nsamples the charge values that came back from the device.
        ``charge`` (float32, e.g. pinned) receives the window blocks (default:
        nrows * nticks floats); ``meta`` may supply the four per-trace arrays
        (trace_meta())."""
        nrows, nticks = self.frame_shape()
        if charge is None:
            charge = np.empty(nrows * nticks, dtype=np.float32)
        if meta is None:
            meta = self.trace_meta()
        ch, tb, ln, off = meta
        wins = (PlaneWindow * len(self.planes))()
        k, ns, ident = self.forward_traces_raw(depos, charge, meta, wins)
        flat = charge.reshape(-1)
        traces = [(int(ch[i]), int(tb[i]), flat[off[i]:off[i] + ln[i]]) for i in range(k)]
        return traces, [w.as_dict() for w in wins], ident, ns

    def trace_meta(self):
        """The four per-trace arrays of forward_traces_raw (channel, tbin,
        length, offset), one entry per frame row."""
        nrows, _ = self.frame_shape()
        return (np.empty(nrows, np.int32), np.empty(nrows, np.int32), np.empty(nrows, np.int32),
                np.empty(nrows, np.int64))

    def forward_traces_raw(self, depos, charge, meta, windows=None):
        """wct_dt_forward_traces into caller arrays, as a C adapter calls it:
        returns (ntraces, nsamples, ident); the traces are in meta and charge."""
        d = np.ascontiguousarray(depos, dtype=np.float64).reshape(-1, 7)
        assert charge.dtype == np.float32 and charge.flags.c_contiguous
        ch, tb, ln, off = meta
        k = C.c_int()
        ns = C.c_size_t()
        ident = C.c_int()
        _check(lib().wct_dt_forward_traces(self.h, d.ctypes.data if len(d) else None, len(d), charge.ctypes.data,
                                           charge.size, ch.ctypes.data, tb.ctypes.data, ln.ctypes.data,
                                           off.ctypes.data, C.byref(k), C.byref(ns),
                                           C.cast(windows, C.c_void_p) if windows is not None else None,
                                           C.byref(ident)))
        return k.value, ns.value, ident.value

    def forward_device(self, d_depos_ptr, ndepos, d_frame_ptr, stream=None):
        """Device-buffer forward (pointers as ints, e.g. torch.Tensor.data_ptr())."""
        wins = (PlaneWindow * len(self.planes))()
        ident = C.c_int()
        _check(lib().wct_dt_forward_device(self.h, C.c_void_p(d_depos_ptr), ndepos, C.c_void_p(d_frame_ptr),
                                           C.cast(wins, C.c_void_p), C.byref(ident),
                                           _dt_stream(stream)))
        return [w.as_dict() for w in wins], ident.value

    def adjoint(self, depos, grad_frame):
        """Host-buffer adjoint: (dL/d depos [n][7] float64, dL/d (DL, DT, lifetime) [3]) for the
        frame gradient ``grad_frame`` [nrows][nticks] of the same depos."""
        d = np.ascontiguousarray(depos, dtype=np.float64).reshape(-1, 7)
        g = np.ascontiguousarray(grad_frame, dtype=np.float32)
        nrows, nticks = self.frame_shape()
        assert g.shape == (nrows, nticks)
        gd = np.zeros_like(d)
        gg = np.zeros(3)
        _check(lib().wct_dt_adjoint(self.h, d.ctypes.data if len(d) else None, len(d), g.ctypes.data,
                                    gd.ctypes.data if len(d) else None, gg.ctypes.data))
        return gd, gg

    def adjoint_device(self, d_depos_ptr, ndepos, d_grad_frame_ptr, d_grad_depos_ptr, d_grad_drift_ptr=None,
                       stream=None):
        """Device-buffer adjoint (pointers as ints)."""
        _check(lib().wct_dt_adjoint_device(self.h, C.c_void_p(d_depos_ptr), ndepos, C.c_void_p(d_grad_frame_ptr),
                                           C.c_void_p(d_grad_depos_ptr),
                                           C.c_void_p(d_grad_drift_ptr) if d_grad_drift_ptr else None,
                                           _dt_stream(stream)))

    def splat(self, depos, **cfg):
        """DepoFluxSplat truth frame [nrows][ticks] float32 of drifted depos
        (keys as SplatConfig.make: tick, window_start, window_duration, nsigma,
        drift_speed, response_plane, time_offsets, smear_long, smear_tran)."""
        sc = SplatConfig.make(**cfg)
        nr, nt = C.c_int(), C.c_int()
        _check(lib().wct_dt_splat_shape(self.h, C.byref(sc), C.byref(nr), C.byref(nt)))
        d = np.ascontiguousarray(depos, dtype=np.float64).reshape(-1, 7)
        out = np.zeros((nr.value, nt.value), dtype=np.float32)
        _check(lib().wct_dt_splat(self.h, C.byref(sc), d.ctypes.data if len(d) else None, len(d), out.ctypes.data))
        return out

    def splat_device(self, d_depos_ptr, ndepos, d_frame_ptr, stream=None, **cfg):
        """DepoFluxSplat on device buffers (frame of splat_shape(**cfg))."""
        sc = SplatConfig.make(**cfg)
        _check(lib().wct_dt_splat_device(self.h, C.byref(sc), C.c_void_p(d_depos_ptr), ndepos, C.c_void_p(d_frame_ptr),
                                          C.c_void_p(stream) if stream else None))

    def splat_shape(self, **cfg):
        sc = SplatConfig.make(**cfg)
        nr, nt = C.c_int(), C.c_int()
        _check(lib().wct_dt_splat_shape(self.h, C.byref(sc), C.byref(nr), C.byref(nt)))
        return nr.value, nt.value

    def forward_batch(self, events, out=None):
        """Host-buffer batch: ``events`` is a list of [n_e][7] depo arrays.  Returns
        (frames [nevents][nrows][nticks] float32, windows per event, first ident)."""
        evs = [np.ascontiguousarray(e, dtype=np.float64).reshape(-1, 7) for e in events]
        offsets = np.zeros(len(evs) + 1, dtype=np.int64)
        offsets[1:] = np.cumsum([len(e) for e in evs])
        d = np.concatenate(evs) if offsets[-1] else np.zeros((1, 7))
        nrows, nticks = self.frame_shape()
        if out is None:
            out = np.empty((len(evs), nrows, nticks), dtype=np.float32)
        assert out.shape == (len(evs), nrows, nticks) and out.dtype == np.float32 and out.flags.c_contiguous
        wins = (PlaneWindow * max(1, len(evs) * len(self.planes)))()
        ident = C.c_int()
        _check(lib().wct_dt_forward_batch(self.h, d.ctypes.data, offsets.ctypes.data, len(evs), out.ctypes.data,
                                          C.cast(wins, C.c_void_p), C.byref(ident)))
        npl = len(self.planes)
        w = [[wins[e * npl + i].as_dict() for i in range(npl)] for e in range(len(evs))]
        return out, w, ident.value

    def forward_batch_device(self, d_depos_ptr, offsets, d_frames_ptr, stream=None, windows=False):
        """Device-buffer batch (one CUDA graph); ``offsets`` host int64 [nevents + 1]."""
        off = np.ascontiguousarray(offsets, dtype=np.int64)
        nev = len(off) - 1
        npl = len(self.planes)
        wins = (PlaneWindow * max(1, nev * npl))() if windows else None
        ident = C.c_int()
        _check(lib().wct_dt_forward_batch_device(self.h, C.c_void_p(d_depos_ptr), off.ctypes.data, nev,
                                                 C.c_void_p(d_frames_ptr),
                                                 C.cast(wins, C.c_void_p) if windows else None, C.byref(ident),
                                                 _dt_stream(stream)))
        if windows:
            return [[wins[e * npl + i].as_dict() for i in range(npl)] for e in range(nev)], ident.value
        return None, ident.value

    BATCH_TUNE_KEYS = ("slots", "raster_per_sm", "fft_threads", "fft_per_sm", "conv_per_sm")

    def batch_tune(self, **kw):
        """Read (no arguments) or change the launch shapes of the batched path."""
        p = (C.c_int * 5)()
        _check(lib().wct_dt_batch_tune(self.h, p, 0))
        cur = dict(zip(self.BATCH_TUNE_KEYS, list(p)))
        if kw:
            cur.update(kw)
            for i, k in enumerate(self.BATCH_TUNE_KEYS):
                p[i] = int(cur[k])
            _check(lib().wct_dt_batch_tune(self.h, p, 1))
        return cur

    def autotune_batch(self, d_depos_ptr, offsets, d_frames_ptr, stream=None):
        """Autotune the batched path on this batch; returns the report (dict)."""
        off = np.ascontiguousarray(offsets, dtype=np.int64)
        buf = C.create_string_buffer(1 << 16)
        _check(lib().wct_dt_autotune_batch(self.h, C.c_void_p(d_depos_ptr), off.ctypes.data, len(off) - 1,
                                           C.c_void_p(d_frames_ptr), _dt_stream(stream), buf, len(buf)))
        return json.loads(buf.value.decode())

    def set_drift_params(self, DL, DT, lifetime):
        _check(lib().wct_dt_set_drift_params(self.h, float(DL), float(DT), float(lifetime)))

    def drift_params(self):
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        _check(lib().wct_dt_get_drift_params(self.h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def patch_records(self, face, plane, n):
        """[n][4] (toffset, poffset, nt, np) per input depo from the last forward call."""
        out = np.zeros((n, 4), dtype=np.int32)
        _check(lib().wct_dt_patch_records(self.h, face, plane, out.ctypes.data, n))
        return out

    def set_profiling(self, on=True):
        _check(lib().wct_dt_set_profiling(self.h, 1 if on else 0))

    def stage_times(self, reset=True):
        """{stage: (ms, launches)} accumulated since the last reset, and the total launch count."""
        ms = np.zeros(len(STAGES))
        nl = np.zeros(len(STAGES), dtype=np.int64)
        tot = C.c_long()
        _check(lib().wct_dt_stage_times(self.h, ms.ctypes.data, nl.ctypes.data, len(STAGES), C.byref(tot),
                                        1 if reset else 0))
        return {STAGES[i]: (float(ms[i]), int(nl[i])) for i in range(len(STAGES))}, tot.value

    def eos(self):
        return lib().wct_dt_eos(self.h)

    def traces(self, frame):
        """IFrame traces: list of (channel, tbin, charges) with Waveform::edge trimming."""
        f = np.ascontiguousarray(frame, dtype=np.float32)
        n = f.shape[0]
        ch = np.zeros(n, np.int32)
        tb = np.zeros(n, np.int32)
        ln = np.zeros(n, np.int32)
        off = np.zeros(n, np.int64)
        k = C.c_int()
        _check(lib().wct_dt_traces(self.h, f.ctypes.data, ch.ctypes.data, tb.ctypes.data, ln.ctypes.data,
                                   off.ctypes.data, C.byref(k)))
        flat = f.reshape(-1)
        return [(int(ch[i]), int(tb[i]), flat[off[i]:off[i] + ln[i]]) for i in range(k.value)]

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.wct_dt_destroy(self.h)
            self.h = None


def _jsonable(o):
    if isinstance(o, dict):
        return {k: _jsonable(v) for k, v in o.items()}
    if isinstance(o, (list, tuple)):
        return [_jsonable(v) for v in o]
    if isinstance(o, np.ndarray):
        return o.tolist()
    if isinstance(o, (np.floating, np.integer)):
        return o.item()
    return o


def binomial_device(seed, ident, n, p, count, d_out_ptr, stream=None):
    """``count`` Binomial(n, p) draws of the stream (seed, ident) into device memory."""
    _check(lib().wct_random_binomial_device(int(seed), int(ident), int(n), float(p), int(count),
                                            C.c_void_p(d_out_ptr), C.c_void_p(stream) if stream else None))


def drifter_json(dr):
    """Drifter configuration with xregions as objects (gen/src/Drifter.cxx:36-52)."""
    d = dict(dr)
    d["xregions"] = [dict(anode=a, response=r, cathode=c) for (a, r, c) in dr["xregions"]]
    return d


def faces_of(cfg):
    """The anode faces of a workload description: cfg["faces"] (a list of
    {"bb": face sensitive box or None, "planes": indices into cfg["planes"]},
    planes of a face consecutive, faces in order) or one face holding every
    plane with cfg["face_bb"]."""
    if cfg.get("faces"):
        return [(f.get("bb"), list(f["planes"])) for f in cfg["faces"]]
    return [(cfg.get("face_bb"), list(range(len(cfg["planes"]))))]


def from_config(cfg, device=0):
    """Build a DepoTransform for a synthetic workload description (see synth.py):
    its faces (faces_of) with cfg["planes"], PIRs from cfg["fr"] and the short
    responses.  Each plane's PIR is built once per distinct field response and
    shared, as the reference shares pirs[plane] across faces."""
    dcfg = {k: cfg[k] for k in ("tick", "start_time", "readout_time", "drift_speed", "nsigma", "fluctuate",
                                 "seed", "first_frame_number") if k in cfg}
    if cfg.get("drifter"):
        dcfg["drifter"] = drifter_json(cfg["drifter"])
    dcfg["device"] = device
    dt = DepoTransform(dcfg)
    pirs = {}
    for bb, idx in faces_of(cfg):
        face = dt.add_face(bb)
        for k in idx:
            p = dt.add_plane(face, cfg["planes"][k])
            fr = cfg["fr"][k]
            key = id(fr)
            if key not in pirs:
                pirs[key] = PlaneImpactResponse(fr, cfg.get("short_responses", []), cfg["overall_short_padding"],
                                                cfg["tick"], cfg["pir_nticks"], cfg.get("long_responses", []),
                                                cfg.get("long_padding", 1.5e6))
            dt.set_response_pir(face, p, pirs[key])
    return dt


_ag = None


def autograd():
    """The libtorch autograd extension (_wct_autograd, built in-tree on first use)."""
    global _ag
    if _ag is None:
        import importlib
        import torch  # noqa: F401  (the extension links libtorch)
        if _build.autograd_stale():
            _build.build_autograd()
        lib()
        _ag = importlib.import_module(__name__ + "._wct_autograd")
    return _ag


def depo_transform(dt, depos, drift_params=None):
    """Differentiable DepoTransform: the dense frame [nrows][nticks] (float32
    torch tensor) of ``depos`` ([n][7] float64 CUDA tensor: t, q, x, y, z,
    extent_long, extent_tran) through the configured component ``dt``, with
    the drifter's (DL, DT, lifetime) taken from ``drift_params`` (float64 CPU
    tensor of 3, may require grad) when given.  Backward goes through the
    hand-written adjoint kernels (torch::autograd::Function in csrc/autograd.cpp)."""
    import torch
    if drift_params is None:
        drift_params = torch.empty(0, dtype=torch.float64)
    return autograd().depo_transform(depos, drift_params, dt.h.value)
