"""TEST INFRASTRUCTURE ONLY -- the parity oracle, never the product.

ctypes front end of ``liboracle.so`` (oracle/wct_oracle.cpp, the CPU
restatement of the reference DepoTransform chain, FP32 and FP64
instantiations) plus an independent FP64 formulation of the same frame in
NumPy (direct linear convolution of the impact-group charge grids), used to
cross-check the restatement's FFT pair-packing.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.
"""

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libref_binning.so")
REF_FUNCS_PATH = os.path.join(HERE, "_ref", "libref_funcs.so")

_lib = None
_ref = None
_ref_funcs = None


def build():
    """Compile liboracle.so (and _ref when the reference tree is present)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = C.CDLL(LIB_PATH)
        _sig(_lib, "orc")
        _lib.orc_fft_best_length.restype = C.c_int
        _lib.orc_fft_best_length.argtypes = [C.c_long, C.c_int]
        _lib.orc_binning_bin.restype = C.c_int
        _lib.orc_binning_bin.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double]
        _lib.orc_sample_bin_range.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                              C.POINTER(C.c_int)]
        _lib.orc_fft_f32.argtypes = [C.c_void_p, C.c_int, C.c_int]
        _lib.orc_fft_f64.argtypes = [C.c_void_p, C.c_int, C.c_int]
        _lib.orc_set_sampling.restype = C.c_int
        _lib.orc_set_sampling.argtypes = [C.c_double] * 5 + [C.c_int, C.c_double, C.c_double, C.c_int, C.c_double,
                                                             C.c_double, C.c_double, C.c_int, C.c_int, C.c_void_p,
                                                             C.c_void_p, C.c_void_p]
        _lib.orc_drift.restype = C.c_int
        _lib.orc_drift.argtypes = [C.c_void_p, C.c_void_p]
        _lib.orc_pir_build.restype = C.c_int
        _lib.orc_pir_build.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.orc_run.restype = C.c_int
        _lib.orc_run.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.orc_edge.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        _lib.orc_binomial_samples.argtypes = [C.c_ulonglong, C.c_int, C.c_double, C.c_long, C.c_void_p]
    return _lib


def ref():
    """The reference-compiled Binning harness, or None when it was not built."""
    global _ref
    if _ref is None and os.path.exists(REF_PATH):
        _ref = C.CDLL(REF_PATH)
        for n, rt, at in [
            ("ref_bin", C.c_int, [C.c_int, C.c_double, C.c_double, C.c_double]),
            ("ref_edge", C.c_double, [C.c_int, C.c_double, C.c_double, C.c_int]),
            ("ref_center", C.c_double, [C.c_int, C.c_double, C.c_double, C.c_int]),
            ("ref_binsize", C.c_double, [C.c_int, C.c_double, C.c_double]),
            ("ref_gcumulative", C.c_double, [C.c_double, C.c_double, C.c_double]),
            ("ref_gbounds", C.c_double, [C.c_double, C.c_double, C.c_double, C.c_double]),
            ("ref_gaussian_sum", C.c_double, [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                              C.c_void_p]),
        ]:
            f = getattr(_ref, n)
            f.restype = rt
            f.argtypes = at
        _ref.ref_sample_bin_range.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                              C.POINTER(C.c_int)]
    return _ref


def ref_funcs():
    """The harness of reference-compiled GausDesc, Waveform::edge and
    Response::coldelec (oracle/ref_funcs_harness.cpp), or None when it was
    not built."""
    global _ref_funcs
    if _ref_funcs is None and os.path.exists(REF_FUNCS_PATH):
        _ref_funcs = C.CDLL(REF_FUNCS_PATH)
        _sig(_ref_funcs, "ref")
    return _ref_funcs


def _sig(L, prefix):
    d, i, p = C.c_double, C.c_int, C.c_void_p
    for n, rt, at in [("_gd_binint", i, [d, d, d, d, i, p]), ("_gd_weight", i, [d, d, d, d, i, p, p]),
                      ("_gd_distance", d, [d, d, d])]:
        f = getattr(L, prefix + n)
        f.restype = rt
        f.argtypes = at
    f = getattr(L, prefix + "_pimpos")
    f.restype = None
    f.argtypes = [i, d, d, p, p, p, i, i, p, p, p]
    f = getattr(L, prefix + "_drift_one")
    f.restype = i
    f.argtypes = [p, i, d, d, d, d, d, p, p]
    f = getattr(L, prefix + "_bdt_add")
    f.restype = i
    f.argtypes = [i, d, d, p, p, p, i, i, d, d, d, p, d, d, p]
    if prefix == "ref":
        L.ref_gd_sigma_range.restype = None
        L.ref_gd_sigma_range.argtypes = [d, d, d, p]
        L.ref_wave_edge.restype = None
        L.ref_wave_edge.argtypes = [p, i, p]
        L.ref_coldelec.restype = d
        L.ref_coldelec.argtypes = [d, d, d]
        L.ref_digitize.restype = None
        L.ref_digitize.argtypes = [p, i, i, p, d, d, d, i, i, p]
        L.ref_noise_resample.restype = i
        L.ref_noise_resample.argtypes = [i, d, i, C.c_float, C.POINTER(d), p, i, p, i, p]
        L.ref_noise_freqs.restype = None
        L.ref_noise_freqs.argtypes = [i, d, p]
        L.ref_noise_interp.restype = i
        L.ref_noise_interp.argtypes = [i, p, p, p, i, d, C.POINTER(d), p]
        L.ref_generator_spec.restype = i
        L.ref_generator_spec.argtypes = [i, p, p, i, p]
        L.ref_group_spectrum.restype = i
        L.ref_group_spectrum.argtypes = [i, d, i, p, p, d, i, d, p]


def gd_binint(L, prefix, center, sigma, start, step, nbins):
    """GausDesc(center, sigma).binint(start, step, nbins) through library L
    (the oracle with prefix "orc", the reference harness with "ref")."""
    out = np.zeros(max(nbins, 1))
    n = getattr(L, prefix + "_gd_binint")(center, sigma, start, step, nbins, out.ctypes.data)
    return out[:n]


def gd_weight(L, prefix, center, sigma, start, step, nbins, pvec):
    pv = np.ascontiguousarray(pvec, dtype=np.float64)
    out = np.zeros(max(nbins, 1))
    n = getattr(L, prefix + "_gd_weight")(center, sigma, start, step, nbins, pv.ctypes.data, out.ctypes.data)
    return out[:n]


def ref_noise_resample(R, fft_length, period, entry):
    """The reference's EmpiricalNoiseModel::resample of one spectra-file entry
    (its float fields rounded as asFloat reads them): (constant, amplitudes)."""
    fr = np.asarray(entry["freqs"], dtype=np.float32)
    am = np.asarray(entry["amps"], dtype=np.float32)
    out = np.zeros(max(fft_length, len(am)), dtype=np.float32)
    c = C.c_double(float(entry.get("const", 0.0)))
    n = R.ref_noise_resample(fft_length, period, int(entry["nsamples"]), float(np.float32(entry["period"])),
                             C.byref(c), fr.ctypes.data, len(fr), am.ctypes.data, len(am), out.ctypes.data)
    return c.value, out[:n]


def ref_group_spectrum(R, freqs, amps, nsamples_orig, period_orig, nsamples, tick, scale=1.0):
    """The reference's GroupNoiseModel treatment of one spectrum (float
    frequencies and amplitudes as asFloat reads them), or None where it throws."""
    fr = np.asarray(freqs, dtype=np.float32)
    am = np.asarray(amps, dtype=np.float32)
    out = np.zeros(int(nsamples), dtype=np.float32)
    rc = R.ref_group_spectrum(int(nsamples_orig), float(period_orig), len(fr), fr.ctypes.data, am.ctypes.data,
                              float(scale), int(nsamples), float(tick), out.ctypes.data)
    return None if rc else out


def drift_one(L, prefix, c):
    """Drifter::insert of one depo (fluctuation off) through library L (the
    oracle "orc" or the reference harness "ref"): (kept, drifted depo)."""
    xr = np.ascontiguousarray(c["xregions"], dtype=np.float64).reshape(-1, 3)
    dep = np.ascontiguousarray(c["depo"], dtype=np.float64)
    out = np.zeros(7)
    k = getattr(L, prefix + "_drift_one")(xr.ctypes.data, xr.shape[0], c["DL"], c["DT"], c["lifetime"], c["speed"],
                                          c["toffset"], dep.ctypes.data, out.ctypes.data)
    return k, out


def bdt_add(L, prefix, c):
    """BinnedDiffusion_transform::add of one depo through library L:
    (added, [outside_time, outside_pitch])."""
    pl = c["plane"]
    w = np.ascontiguousarray(pl["wire"], dtype=np.float64)
    pi = np.ascontiguousarray(pl["pitch"], dtype=np.float64)
    o = np.ascontiguousarray(pl["origin"], dtype=np.float64)
    dep = np.ascontiguousarray(c["depo"], dtype=np.float64)
    cnt = np.zeros(2, dtype=np.int32)
    k = getattr(L, prefix + "_bdt_add")(pl["nwires"], pl["minp"], pl["maxp"], w.ctypes.data, pi.ctypes.data,
                                        o.ctypes.data, pl["nimp"], c["ntbins"], c["tmin"], c["tmax"], c["nsigma"],
                                        dep.ctypes.data, c["sigma_time"], c["sigma_pitch"], cnt.ctypes.data)
    return k, cnt.tolist()


def drift_cases(rng, n):
    """Depos for the Drifter::insert pin: one face, two mirrored faces or a
    region without an anode; positions across and exactly on the anode,
    response and cathode planes; zero, negative and positive charge."""
    out = []
    for k in range(n):
        kind = k % 3
        if kind == 0:
            xr = [[0.0, 100.0, 2700.0]]
        elif kind == 1:
            xr = [[0.0, 100.0, 2700.0], [0.0, -100.0, -2700.0]]
        else:
            xr = [[100.0, 100.0, -2500.0]]  # anode taken from the response plane
        planes = [v for r in xr for v in r]
        x = float(rng.choice(planes)) if k % 5 == 0 else float(rng.uniform(-2800.0, 2800.0))
        q = 0.0 if k % 11 == 0 else float(rng.choice([-1.0, 1.0]) * rng.uniform(1.0, 1e5))
        out.append(dict(xregions=xr, DL=float(rng.uniform(5.0, 10.0) * 1e-7), DT=float(rng.uniform(8.0, 15.0) * 1e-7),
                        lifetime=float(rng.uniform(3.0, 30.0) * 1e6), speed=float(rng.uniform(1.0, 2.0) * 1e-3),
                        toffset=float(rng.choice([0.0, rng.uniform(-1e4, 1e4)])),
                        depo=[float(rng.uniform(-1e5, 3e6)), q, x, float(rng.uniform(-3000.0, 3000.0)),
                              float(rng.uniform(-2300.0, 2300.0)), float(rng.choice([0.0, rng.uniform(0.0, 30.0)])),
                              float(rng.choice([0.0, rng.uniform(0.0, 3.0)]))]))
    return out


def bdt_add_cases(rng, n):
    """Depos for the BinnedDiffusion_transform::add pin: random planes (as
    AnodePlane builds Pimpos), readout windows, widths including 0, centres
    within a few sigma of the window and impact-range edges, some exactly
    nsigma away."""
    out = []
    for k in range(n):
        ang = np.radians(float(rng.choice([0.0, 35.7, -35.7, rng.uniform(-90.0, 90.0)])))
        wire = [0.0, float(np.cos(ang)), float(np.sin(ang))]
        pdir = np.array([0.0, -np.sin(ang), np.cos(ang)])
        nw = int(rng.integers(2, 1000))
        pw = float(rng.uniform(3.0, 5.0))
        minp = -0.5 * pw * (nw - 1)
        plane = dict(nwires=nw, minp=minp, maxp=minp + pw * (nw - 1), wire=wire, pitch=pdir.tolist(),
                     origin=[100.0, 0.0, 0.0], nimp=int(rng.choice([10, 6])))
        ntb = int(rng.choice([6000, 1000]))
        tick = float(rng.choice([500.0, 400.0]))
        tmin = float(rng.choice([0.0, -1000.0]))
        nsigma = float(rng.choice([3.0, 2.5]))
        st = 0.0 if k % 7 == 0 else float(np.exp(rng.uniform(np.log(1.0), np.log(3000.0))))
        sp = 0.0 if k % 5 == 0 else float(np.exp(rng.uniform(np.log(0.01), np.log(10.0))))
        tedge = tmin if rng.random() < 0.5 else tmin + ntb * tick
        t = tedge + (rng.choice([-1.0, 1.0]) * nsigma * st if k % 4 == 0 else rng.uniform(-5.0, 5.0) * (st or 100.0))
        lo, hi = minp - 0.5 * pw, minp + pw * (nw - 1) + 0.5 * pw
        pedge = lo if rng.random() < 0.5 else hi
        c = pedge + (rng.choice([-1.0, 1.0]) * nsigma * sp if k % 6 == 0 else rng.uniform(-5.0, 5.0) * (sp or 1.0))
        pos = np.array(plane["origin"]) + c * pdir + rng.uniform(-1000.0, 1000.0) * np.array(wire)
        out.append(dict(plane=plane, ntbins=ntb, tmin=tmin, tmax=tmin + ntb * tick, nsigma=nsigma,
                        depo=[float(t), -1000.0, float(pos[0]), float(pos[1]), float(pos[2]), 0.0, 0.0],
                        sigma_time=st, sigma_pitch=sp))
    return out


def pimpos(L, prefix, nwires, minp, maxp, wire, pitch, origin, nbins, pts):
    """Pimpos(nwires, minp, maxp, wire, pitch, origin, nbins) through library L:
    ([region nbins, min, max, impact nbins, min, max, axis0, axis1, axis2],
    pitch coordinates of pts [n][3])."""
    w, pd, o = (np.ascontiguousarray(v, dtype=np.float64) for v in (wire, pitch, origin))
    pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
    out = np.zeros(15)
    dist = np.zeros(len(pts))
    getattr(L, prefix + "_pimpos")(nwires, minp, maxp, w.ctypes.data, pd.ctypes.data, o.ctypes.data, nbins, len(pts),
                                   pts.ctypes.data, out.ctypes.data, dist.ctypes.data)
    return out, dist


class OrcPlane(C.Structure):
    _fields_ = [
        ("nwires", C.c_int), ("nimp", C.c_int),
        ("pitchmin", C.c_double), ("pitchmax", C.c_double),
        ("wire", C.c_double * 3), ("pitch", C.c_double * 3), ("origin", C.c_double * 3),
        ("npaths", C.c_int), ("nfr", C.c_int),
        ("pitchpos", C.c_void_p), ("current", C.c_void_p), ("fr_pitch", C.c_double),
    ]


class OrcJob(C.Structure):
    _fields_ = [
        ("start_time", C.c_double), ("readout_time", C.c_double), ("tick", C.c_double),
        ("drift_speed", C.c_double), ("nsigma", C.c_double),
        ("drift", C.c_int),
        ("DL", C.c_double), ("DT", C.c_double), ("lifetime", C.c_double), ("drifter_speed", C.c_double),
        ("toffset", C.c_double),
        ("nxregions", C.c_int), ("xregions", C.c_void_p),
        ("have_bb", C.c_int), ("bb_lo", C.c_double * 3), ("bb_hi", C.c_double * 3),
        ("fr_tstart", C.c_double), ("fr_period", C.c_double),
        ("nshort", C.c_int), ("short_len", C.c_void_p), ("short_wave", C.c_void_p),
        ("overall_short_padding", C.c_double), ("pir_nticks", C.c_int),
        ("nplanes", C.c_int), ("planes", C.c_void_p),
        ("ndepos", C.c_int), ("depos", C.c_void_p),
        ("fp64", C.c_int), ("nthreads", C.c_int),
        ("fluctuate", C.c_int), ("drift_fluctuate", C.c_int), ("seed", C.c_ulonglong),
        ("nlong", C.c_int), ("long_len", C.c_void_p), ("long_wave", C.c_void_p), ("long_padding", C.c_double),
        ("stage_s", C.c_void_p),
        ("nfaces", C.c_int), ("face_bb", C.c_void_p), ("face_have_bb", C.c_void_p), ("plane_face", C.c_void_p),
        ("charge_scale", C.c_void_p),
    ]


class OrcPlaneOut(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("start_ch", "end_ch", "start_tick", "end_tick", "nw", "nt",
                                        "ndepos_added", "outside_time", "outside_pitch")]


class Job:
    """Owns the numpy buffers an OrcJob points into."""

    def __init__(self, cfg, depos, drift=True, fp64=False, nthreads=1, fluctuate=False, drift_fluctuate=False,
                 seed=0, charge_scale=None):
        self.keep = []
        j = OrcJob()
        j.fluctuate = 1 if fluctuate else 0
        j.drift_fluctuate = 1 if drift_fluctuate else 0
        j.seed = int(seed)
        j.start_time = cfg["start_time"]
        j.readout_time = cfg["readout_time"]
        j.tick = cfg["tick"]
        j.drift_speed = cfg["drift_speed"]
        j.nsigma = cfg["nsigma"]
        dr = cfg.get("drifter")
        j.drift = 1 if (drift and dr) else 0
        if dr:
            j.DL, j.DT, j.lifetime = dr["DL"], dr["DT"], dr["lifetime"]
            j.drifter_speed, j.toffset = dr["drift_speed"], dr.get("time_offset", 0.0)
            xr = self._arr(np.array(dr["xregions"], dtype=np.float64).reshape(-1, 3))
            j.nxregions = xr.shape[0]
            j.xregions = xr.ctypes.data
        bb = cfg.get("face_bb")
        if bb is not None:
            j.have_bb = 1
            for i in range(3):
                j.bb_lo[i] = bb[0][i]
                j.bb_hi[i] = bb[1][i]
        j.fr_tstart = cfg["fr"][0]["tstart"]
        j.fr_period = cfg["fr"][0]["period"]
        shorts = [np.asarray(s, dtype=np.float64) for s in cfg.get("short_responses", [])]
        j.nshort = len(shorts)
        if shorts:
            sl = self._arr(np.array([len(s) for s in shorts], dtype=np.int32))
            sw = self._arr(np.concatenate(shorts))
            j.short_len = sl.ctypes.data
            j.short_wave = sw.ctypes.data
        j.overall_short_padding = cfg["overall_short_padding"]
        j.pir_nticks = cfg["pir_nticks"]
        longs = [np.asarray(w, dtype=np.float64) for w in cfg.get("long_responses", [])]
        j.nlong = len(longs)
        j.long_padding = cfg.get("long_padding", 1.5e6)
        if longs:
            ll = self._arr(np.array([len(w) for w in longs], dtype=np.int32))
            lw = self._arr(np.concatenate(longs))
            j.long_len = ll.ctypes.data
            j.long_wave = lw.ctypes.data
        planes = (OrcPlane * len(cfg["planes"]))()
        for i, (pl, fr) in enumerate(zip(cfg["planes"], cfg["fr"])):
            p = planes[i]
            p.nwires = pl["nwires"]
            p.nimp = pl["nimp"]
            p.pitchmin = pl["pitchmin"]
            p.pitchmax = pl["pitchmax"]
            for k in range(3):
                p.wire[k] = pl["wire"][k]
                p.pitch[k] = pl["pitch"][k]
                p.origin[k] = pl["origin"][k]
            pp = self._arr(np.ascontiguousarray(fr["pitchpos"], dtype=np.float64))
            cu = self._arr(np.ascontiguousarray(fr["current"], dtype=np.float64))
            p.npaths = pp.shape[0]
            p.nfr = cu.shape[1]
            p.pitchpos = pp.ctypes.data
            p.current = cu.ctypes.data
            p.fr_pitch = fr["pitch"]
        self.keep.append(planes)
        j.nplanes = len(cfg["planes"])
        j.planes = C.cast(planes, C.c_void_p)
        if cfg.get("faces"):
            # several anode faces: each face's box and each plane's face
            fl = cfg["faces"]
            fb = np.zeros((len(fl), 6), dtype=np.float64)
            fh = np.zeros(len(fl), dtype=np.int32)
            pf = np.full(j.nplanes, -1, dtype=np.int32)
            for f, face in enumerate(fl):
                if face.get("bb") is not None:
                    fb[f, :3] = face["bb"][0]
                    fb[f, 3:] = face["bb"][1]
                    fh[f] = 1
                for k in face["planes"]:
                    pf[k] = f
            assert (pf >= 0).all(), "every plane belongs to a face"
            j.nfaces = len(fl)
            j.face_bb = self._arr(fb).ctypes.data
            j.face_have_bb = self._arr(fh).ctypes.data
            j.plane_face = self._arr(pf).ctypes.data
        if charge_scale is not None:
            cs = self._arr(np.ascontiguousarray(charge_scale, dtype=np.float64))
            assert cs.shape == (len(depos), j.nplanes), cs.shape
            j.charge_scale = cs.ctypes.data
        d = self._arr(np.ascontiguousarray(depos, dtype=np.float64).reshape(-1, 7))
        j.ndepos = d.shape[0]
        j.depos = d.ctypes.data
        j.fp64 = 1 if fp64 else 0
        j.nthreads = nthreads
        self.job = j
        self.cfg = cfg

    def _arr(self, a):
        self.keep.append(a)
        return a


def fft_best_length(n, keep=False):
    return lib().orc_fft_best_length(int(n), 1 if keep else 0)


STAGES = ("drift+cut", "raster+scatter", "response_prep", "fft_convolution", "extraction", "pir_build")
TORCH_FFT_PATH = os.path.join(HERE, "libtorchfft.so")
_torch_fft = None


def set_fft_backend(name):
    """The oracle's transforms: "own" (its scalar Stockham FFTs, the parity
    default) or "mkl" (libtorch-CPU, i.e. Intel MKL, through
    oracle/torch_fft.cpp: the reference's TorchDFT backend).  Process-wide."""
    global _torch_fft
    L = lib()
    L.orc_set_fft_backend.argtypes = [C.c_void_p]
    L.orc_set_fft_backend.restype = None
    if name == "own":
        L.orc_set_fft_backend(None)
        return
    if name != "mkl":
        raise ValueError(name)
    import torch  # noqa: F401  (loads the libtorch_cpu the shim binds to)
    if _torch_fft is None:
        if not os.path.exists(TORCH_FFT_PATH):
            build()
        _torch_fft = C.CDLL(TORCH_FFT_PATH)
    L.orc_set_fft_backend(C.cast(_torch_fft.orc_torch_fft, C.c_void_p))


def run(cfg, depos, drift=True, fp64=False, nthreads=1, records=False, fluctuate=False, drift_fluctuate=False,
        seed=0, stages=False, charge_scale=None):
    """Run the restated DepoTransform. Returns dict(frames=[per-plane
    [nwires][nticks]], windows=[OrcPlaneOut as dict], records=optional,
    stages=optional {STAGES name: seconds, summed over planes}).
    ``fluctuate`` / ``drift_fluctuate`` draw the reference's binomial
    fluctuations with std::mt19937 streams seeded from ``seed``.  Several
    faces: cfg["faces"] (each {"bb", "planes"}), else one face with
    cfg["face_bb"].  ``charge_scale`` [ndepos][nplanes]: modify_depo's
    per-plane charge factor."""
    job = Job(cfg, depos, drift=drift, fp64=fp64, nthreads=nthreads, fluctuate=fluctuate,
              drift_fluctuate=drift_fluctuate, seed=seed, charge_scale=charge_scale)
    st = None
    if stages:
        st = job._arr(np.zeros(len(STAGES), dtype=np.float64))
        job.job.stage_s = st.ctypes.data
    nticks = int(cfg["readout_time"] / cfg["tick"])
    nw = [pl["nwires"] for pl in cfg["planes"]]
    dt = np.float64 if fp64 else np.float32
    frame = np.zeros((sum(nw), nticks), dtype=dt)
    pouts = (OrcPlaneOut * len(nw))()
    rec = None
    if records:
        rec = np.zeros((len(nw), job.job.ndepos, 5), dtype=np.int32)
    rc = lib().orc_run(C.byref(job.job), frame.ctypes.data, C.cast(pouts, C.c_void_p),
                       rec.ctypes.data if rec is not None else None)
    if rc != 0:
        raise RuntimeError("oracle run failed: %d" % rc)
    frames = []
    r0 = 0
    for n in nw:
        frames.append(frame[r0:r0 + n])
        r0 += n
    wins = [{f: getattr(p, f) for f, _ in OrcPlaneOut._fields_} for p in pouts]
    out = dict(frames=frames, windows=wins, records=rec)
    if st is not None:
        out["stages"] = {k: float(v) for k, v in zip(STAGES, st)}
    return out


def binomial_samples(n, p, count, seed=1):
    """``count`` draws of std::binomial_distribution<int>(n, p) over std::mt19937."""
    out = np.zeros(count, dtype=np.int32)
    lib().orc_binomial_samples(int(seed), int(n), float(p), int(count), out.ctypes.data)
    return out


def drift(cfg, depos):
    job = Job(cfg, depos, drift=True)
    out = np.zeros((job.job.ndepos, 8))
    n = lib().orc_drift(C.byref(job.job), out.ctypes.data)
    return out[:n]


def pir_build(cfg, iplane, fp64=False):
    job = Job(cfg, np.zeros((0, 7)), fp64=fp64)
    fr = cfg["fr"][iplane]
    npaths = len(fr["pitchpos"])
    wf = np.zeros((npaths, cfg["pir_nticks"]))
    bywire = np.full((npaths, 16), -1, dtype=np.int32)
    pie = np.zeros(3)
    code = lib().orc_pir_build(C.byref(job.job), iplane, wf.ctypes.data, bywire.ctypes.data, pie.ctypes.data)
    if code < 0:
        raise RuntimeError("pir build failed")
    nwires, nimp = divmod(code, 1000)
    bw = bywire.reshape(-1)[: nwires * nimp].reshape(nwires, nimp)
    return dict(waveforms=wf, bywire=bw, pitch=pie[0], impact=pie[1], half_extent=pie[2])


def set_sampling(t, q, pc, st, sp, tbins, ibins, nsigma=3.0, fp64=False, cap=1 << 16):
    patch = np.zeros(cap)
    w = np.zeros(4096)
    oi = np.zeros(4, dtype=np.int32)
    rc = lib().orc_set_sampling(t, q, pc, st, sp, tbins[0], tbins[1], tbins[2], ibins[0], ibins[1], ibins[2],
                                nsigma, 1 if fp64 else 0, cap, patch.ctypes.data, w.ctypes.data, oi.ctypes.data)
    if rc != 0:
        raise RuntimeError("patch too large")
    to, po, nt, npp = [int(x) for x in oi]
    return dict(toffset=to, poffset=po, nt=nt, np=npp, patch=patch[: nt * npp].reshape(npp, nt), weights=w[:npp])


def edge(wave):
    w = np.ascontiguousarray(wave, dtype=np.float32)
    out = np.zeros(2, dtype=np.int32)
    lib().orc_edge(w.ctypes.data, w.size, out.ctypes.data)
    return int(out[0]), int(out[1])


def traces(frame_rows, channels):
    """DepoTransform trace assembly (gen/src/DepoTransform.cxx:193-208):
    list of (channel, tbin, charges) with exact-zero trimming."""
    out = []
    for iw in range(frame_rows.shape[0]):
        a, b = edge(frame_rows[iw])
        if a == frame_rows.shape[1]:
            continue
        out.append((int(channels[iw]), a, frame_rows[iw, a:b].astype(np.float32)))
    return out


# ---------------------------------------------------------------------------
# Independent FP64 formulation (direct linear convolution), for small cases.
# ---------------------------------------------------------------------------
def direct_fp64(cfg, depos, iplane, pir=None, drift=True):
    """Frame of one plane as V[w,t] = sum_g sum_j sum_tau R_g[j][tau] Q_g[w-j][t-tau],
    with Q_g accumulated in FP64 from FP64 patches and R_g[j] the FP64 PIR
    waveforms selected by the reference's closest() rule.  Independent of the
    restatement's FFT convolution; used to pin it on small inputs."""
    import math
    if pir is None:
        pir = pir_build(cfg, iplane, fp64=True)
    d = drift_fn(cfg, depos) if drift else np.asarray(depos, dtype=np.float64)
    pl = cfg["planes"][iplane]
    nticks = int(cfg["readout_time"] / cfg["tick"])
    nwires = pl["nwires"]
    nimp = pl["nimp"]
    regionsize = (pl["pitchmax"] - pl["pitchmin"]) / (nwires - 1)
    pmin = pl["pitchmin"] - 0.5 * regionsize
    pmax = pl["pitchmax"] + 0.5 * regionsize
    ib = (nwires * nimp, pmin, pmax)
    tb = (int(cfg["readout_time"] / cfg["tick"]), cfg["start_time"], cfg["start_time"] + cfg["readout_time"])
    pdir = np.array(pl["pitch"], dtype=np.float64)
    pdir = pdir / math.sqrt(float(np.dot(pdir, pdir)))
    org = np.array(pl["origin"], dtype=np.float64)
    bb = cfg.get("face_bb")
    G = int(round(pir["pitch"] / pir["impact"])) + 1
    npad = int(round((pir["bywire"].shape[0] - 1) / 2.0))
    Q = np.zeros((G, nwires, nticks))
    for row in d:
        t, q, x, y, z, el, et = row[:7]
        if bb is not None:
            p3 = (x, y, z)
            if any(not (min(bb[0][k], bb[1][k]) <= p3[k] <= max(bb[0][k], bb[1][k])) for k in range(3)
                   if bb[0][k] != bb[1][k]):
                continue
        pc = float(np.dot(pdir, np.array([x, y, z]) - org))
        st = el / cfg["drift_speed"]
        # rejection (gen/src/BinnedDiffusion_transform.cxx:37-76)
        def rej(c, s, lo, hi):
            eff = cfg["nsigma"] if s > 0 else 0.0
            dmin = (lo - c) / s if s else lo - c
            dmax = (hi - c) / s if s else hi - c
            return dmin > eff or dmax < -eff
        if rej(t, st, tb[1], tb[2]) or rej(pc, et, ib[1], ib[2]):
            continue
        P = set_sampling(t, q, pc, st, et, tb, ib, cfg["nsigma"], fp64=True)
        for ip in range(P["np"]):
            k = P["poffset"] + ip
            w = k // nimp
            red = k - (w * nimp + nimp // 2)
            g0 = red + G // 2
            Q[g0, w, P["toffset"]:P["toffset"] + P["nt"]] += P["patch"][ip] * P["weights"][ip]
            Q[g0 + 1, w, P["toffset"]:P["toffset"] + P["nt"]] += P["patch"][ip] * (1.0 - P["weights"][ip])
    # responses R_g[j] by the closest() rule (gen/src/ImpactTransform.cxx:34-74)
    out = np.zeros((nwires, nticks))
    from numpy.fft import rfft, irfft
    nfft = 1
    while nfft < nticks + pir["waveforms"].shape[1]:
        nfft *= 2
    for g in range(G):
        rel = -pir["pitch"] / 2.0 + pir["impact"] * g + (1e-9 if g != G - 1 else -1e-9)
        Qf = rfft(Q[g], nfft, axis=1)
        for j in range(-npad, npad + 1):
            rp = rel - j * pir["pitch"]
            relwire = cround(rp / pir["pitch"])
            wi = pir["bywire"].shape[0] // 2 + relwire
            rem = rp - relwire * pir["pitch"]
            ii = cround(rem / pir["impact"]) + pir["bywire"].shape[1] // 2
            path = pir["bywire"][wi][ii]
            Rf = rfft(pir["waveforms"][path], nfft)
            conv = irfft(Qf * Rf[None, :], nfft, axis=1)[:, :nticks]
            lo, hi = max(0, j), min(nwires, nwires + j)
            out[lo:hi] += conv[lo - j:hi - j]
    return out


def cround(x):
    """C round(): halves away from zero."""
    import math
    return int(math.copysign(math.floor(abs(x) + 0.5), x))


def drift_fn(cfg, depos):
    o = drift(cfg, depos)
    return o[:, :7]


def digitize(frame, row_baseline, gain=1.0, fullscale=(0.0, 2.0e-6), resolution=12, round_adc=False):
    """Gen::Digitizer's per-sample arithmetic (gen/src/Digitizer.cxx:82-141)
    in float64, vectorised: voltage = gain * value + baseline (a float32, as
    the reference reads m_baselines into a float), then digitize (:82-97):
    0 at or below fullscale[0], 2^resolution - 1 at or above fullscale[1],
    otherwise (v - fs0) / (fs1 - fs0) * max, rounded half away from zero
    (C round; the values are positive here) or floored; returned as float32."""
    f = np.asarray(frame, dtype=np.float32).astype(np.float64)
    base = np.asarray(row_baseline, dtype=np.float32).astype(np.float64)[:, None]
    maxv = float((1 << resolution) - 1)
    v = gain * f + base
    with np.errstate(invalid="ignore"):
        fp = ((v - fullscale[0]) / (fullscale[1] - fullscale[0])) * maxv
        fl = np.floor(fp)
        adc = fl + ((fp - fl) >= 0.5) if round_adc else fl
    adc = np.where(v <= fullscale[0], 0.0, np.where(v >= fullscale[1], maxv, adc))
    return adc.astype(np.float32)


def noise_spec(spectrum, normals):
    """The spectrum of one noise waveform as IncoherentAddNoise makes it
    (gen/src/AddNoise.cxx:79-84 and aux/src/NoiseTools.cxx GeneratorN::spec),
    float64: sigma_k = S_k * sqrt(2 / 3.141592); for k <= N/2 + (N even) the
    bin is sigma_k (n_k, n_{k + N/2}); DC and (N even) Nyquist become their
    modulus; the spectrum is made Hermitian.  ``normals`` holds at least
    2 (N/2 + (N even)) + 1 standard normals."""
    S = np.asarray(spectrum, dtype=np.float64)
    n = S.size
    nextra = (n + 1) % 2
    nhalf = n // 2
    sig = S * np.sqrt(2.0 / 3.141592)
    spec = np.zeros(n, dtype=np.complex128)
    for ind in range(min(nhalf + nextra, n - 1) + 1):
        spec[ind] = sig[ind] * complex(normals[ind], normals[ind + nhalf])
    spec[0] = abs(spec[0])
    if nextra:
        spec[nhalf] = abs(spec[nhalf])
    for k in range(1, (n + 1) // 2):  # Hermitian mirror
        spec[n - k] = np.conj(spec[k])
    return spec


def noise_wave(spectrum, normals):
    """One noise waveform as IncoherentAddNoise makes it: the inverse DFT
    (with 1/N) of ``noise_spec``."""
    return np.real(np.fft.ifft(noise_spec(spectrum, normals)))


class OrcSplat(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("tick", "window_start", "window_duration", "nsigma", "drift_speed",
                                          "response_plane")] + \
        [("time_offsets", C.c_double * 3), ("smear_long", C.c_double * 3), ("smear_tran", C.c_double * 3)]


def splat(cfg, depos, scfg, float_sums=False):
    """DepoFluxSplat's dense truth frame (gen/src/DepoFluxSplat.cxx:247-390) of
    drifted depos for the planes of ``cfg`` (its face cut included):
    [sum of nwires][nbins], cells summed in float64, or with ``float_sums``
    in float32 in depo order as the reference's accumulator does.  ``scfg``:
    tick, window_start, window_duration, nsigma, drift_speed, response_plane,
    and optional 3-lists time_offsets, smear_long, smear_tran."""
    job = Job(cfg, depos, drift=False)
    sp = OrcSplat()
    for k in ("tick", "window_start", "window_duration", "nsigma", "drift_speed", "response_plane"):
        setattr(sp, k, float(scfg[k]))
    for k in ("time_offsets", "smear_long", "smear_tran"):
        v = scfg.get(k) or [0.0, 0.0, 0.0]
        for i in range(3):
            getattr(sp, k)[i] = float(v[i])
    nbins = int(scfg["window_duration"] / scfg["tick"])
    nrows = sum(p["nwires"] for p in cfg["planes"])
    out = np.zeros((nrows, nbins), dtype=np.float32 if float_sums else np.float64)
    L = lib()
    f = L.orc_splat_float if float_sums else L.orc_splat
    f.argtypes = [C.POINTER(OrcJob), C.POINTER(OrcSplat), C.c_void_p]
    if f(C.byref(job.job), C.byref(sp), out.ctypes.data) != 0:
        raise RuntimeError("orc_splat failed")
    return out
