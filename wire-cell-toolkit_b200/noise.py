"""Channel noise spectra for ``add_noise``: the empirical (incoherent) noise
model and, at the end of this module, the group (coherent) noise model.

EmpiricalNoiseModel (gen/src/EmpiricalNoiseModel.cxx) holds measured
amplitude spectra per plane at several wire lengths (its "spectra_file":
entries with plane, gain, shaping, wirelen, const, nsamples, period, freqs,
amps).  At configuration (:96-175) every entry is resampled onto the model's
frequency grid of L = fft_best_length(nsamples) bins (:58-70: bin i holds
i / (L period) up to L/2, mirrored above, rounded to float as the reference
stores it), its amplitudes and constant scaled
by sqrt(L / entry nsamples), by linear interpolation between the entry's
frequencies (clamped at both ends).  A channel's spectrum (:250-330) is the
linear interpolation between the plane's entries bracketing the channel's
total wire length (rounded down to wire_length_scale steps; clamped at the
shortest and longest), scaled by the channel's gain over the entries' gain
when they differ by more than 1%, and combined with the interpolated
constant as sqrt(amp^2 + const^2).  A channel whose shaping time differs
from the entries' by more than 1% has its amplitudes scaled by the ratio of
the cold-electronics response magnitudes (util/src/Response.cxx:311-340,
sampled at i * period for i < L) at the two shaping times; responses are
cached by shaping time in 0.1 us steps, the first channel of a step setting
it (as the reference caches them).  Floats stay floats where the reference
holds them so (amplitudes, the frequency grid, the response magnitudes, the
gain factor of Waveform::scale), so the spectra are the reference's bit for
bit except where its single-precision DFT of the response enters.
"""

import numpy as np

from . import fft_best_length

CM = 10.0  # the toolkit's length unit is the mm
US = 1000.0  # and its time unit the ns


def coldelec(time, gain, shaping):
    """Response::coldelec (util/src/Response.cxx:311-340): the cold
    electronics response at ``time`` (array), zero outside (0, 10 us)."""
    t = np.asarray(time, dtype=np.float64)
    r = t / shaping
    g = gain * 10 * 1.012
    e1, e2, e3 = np.exp(-2.94809 * r), np.exp(-2.82833 * r), np.exp(-2.40318 * r)
    c1, s1 = np.cos(1.19361 * r), np.sin(1.19361 * r)
    c2, s2 = np.cos(2.38722 * r), np.sin(2.38722 * r)
    c3, s3 = np.cos(2.5928 * r), np.sin(2.5928 * r)
    c4, s4 = np.cos(5.18561 * r), np.sin(5.18561 * r)
    v = (4.31054 * e1 * g - 2.6202 * e2 * c1 * g - 2.6202 * e2 * c1 * c2 * g + 0.464924 * e3 * c3 * g
         + 0.464924 * e3 * c3 * c4 * g + 0.762456 * e2 * s1 * g - 0.762456 * e2 * c2 * s1 * g
         + 0.762456 * e2 * c1 * s2 * g - 2.620200 * e2 * s1 * s2 * g - 0.327684 * e3 * s3 * g
         + 0.327684 * e3 * c4 * s3 * g - 0.327684 * e3 * c3 * s4 * g + 0.464924 * e3 * s3 * s4 * g)
    return np.where((t <= 0) | (t >= 10 * US), 0.0, v)


class EmpiricalNoiseModel:
    def __init__(self, spectra, nsamples, period, wire_length_scale=1.0 * CM):
        self.nsamples = int(nsamples)
        self.period = float(period)
        self.wlres = float(wire_length_scale)
        self.L = fft_best_length(self.nsamples)
        L = self.L
        i = np.arange(L)
        # the grid is held in floats (m_elec_resp_freq is a Waveform::realseq_t)
        f = np.where(i <= L / 2.0, i / (L * 1.0) / self.period, (L - i) / (L * 1.0) / self.period)
        self.freq = f.astype(np.float32).astype(np.float64)
        self.planes = {}
        self._resp = {}  # shaping step -> response magnitude (L values)
        for e in spectra:  # file order: by wire length within a plane
            ent = dict(plane=int(e["plane"]), gain=float(np.float32(e["gain"])),
                       shaping=float(np.float32(e["shaping"])), wirelen=float(np.float32(e["wirelen"])),
                       const=float(e.get("const", 0.0)), nsamples=int(e["nsamples"]),
                       period=float(np.float32(e["period"])),
                       freqs=np.asarray(e["freqs"], dtype=np.float32).astype(np.float64),
                       amps=np.asarray(e["amps"], dtype=np.float32).astype(np.float64))
            self._resample(ent)
            self.planes.setdefault(ent["plane"], []).append(ent)

    def _resample(self, s):
        """EmpiricalNoiseModel::resample (:96-136)."""
        if s["nsamples"] == self.L and s["period"] == self.period:
            return
        scale = np.sqrt(self.L / (s["nsamples"] * 1.0))
        s["const"] *= scale
        amps = (s["amps"] * scale).astype(np.float32).astype(np.float64)  # amplitude_t holds floats
        fr = s["freqs"]
        out = np.empty(self.L)
        for i, f in enumerate(self.freq):
            if f <= fr[0]:
                lo, hi, mu = 0, 1, 0.0
            elif f >= fr[-1]:
                lo, hi, mu = len(fr) - 2, len(fr) - 1, 1.0
            else:
                lo = int(np.searchsorted(fr, f, side="left")) - 1  # last j with f > fr[j]
                hi = lo + 1
                # the entry's frequencies are floats: their difference is a float subtraction
                mu = (f - fr[lo]) / float(np.float32(fr[hi]) - np.float32(fr[lo]))
            out[i] = (1 - mu) * amps[lo] + mu * amps[hi]
        s["amps"] = out.astype(np.float32).astype(np.float64)

    def interpolate_wire_length(self, plane, wire_length):
        """(constant, amplitudes) at a wire length (:175-210)."""
        sp = self.planes[plane]
        if wire_length <= sp[0]["wirelen"]:
            return sp[0]["const"], sp[0]["amps"].copy()
        if wire_length >= sp[-1]["wirelen"]:
            return sp[-1]["const"], sp[-1]["amps"].copy()
        for k in range(1, len(sp)):
            hi = sp[k]
            if hi["wirelen"] < wire_length:
                continue
            lo = sp[k - 1]
            mu = (wire_length - lo["wirelen"]) / (hi["wirelen"] - lo["wirelen"])
            amp = (lo["amps"] * (1 - mu) + hi["amps"] * mu).astype(np.float32).astype(np.float64)
            return lo["const"] * (1 - mu) + hi["const"] * mu, amp
        raise ValueError("EmpiricalNoiseModel: data corruption")

    def _response(self, shaping):
        """|DFT| (float) of ColdElec(10, shaping) generated on the domain
        [0, L period) in L float samples (Response::Generator::generate,
        util/src/Response.cxx:267-276: t = i (L period) / L), cached per 0.1 us
        step of the shaping time.  The reference transforms the float samples
        with its single-precision IDFT; this one in double, so the magnitudes
        agree to float rounding."""
        key = int(shaping / US / 0.1)
        if key not in self._resp:
            tick = (self.L * self.period - 0.0) / self.L
            sig = coldelec(0.0 + np.arange(self.L) * tick, 10.0, shaping).astype(np.float32)
            self._resp[key] = np.abs(np.fft.fft(sig.astype(np.float64))).astype(np.float32)
        return self._resp[key]

    def channel_spectrum(self, plane, wire_length, gain=None, shaping=None):
        """The amplitude spectrum (L float32 values) of a channel of ``plane``
        whose wires total ``wire_length``; ``gain`` and ``shaping``: the
        channel's preamplifier gain and shaping time when they deviate from
        the spectra's (the channel-status values)."""
        ilen = int(wire_length / self.wlres)
        const, amp = self.interpolate_wire_length(plane, ilen * self.wlres)
        db_gain = self.planes[plane][0]["gain"]
        db_shaping = self.planes[plane][0]["shaping"]
        amp = np.asarray(amp, dtype=np.float32)
        if gain is not None and abs(gain - db_gain) > 0.01 * gain:
            # Waveform::scale(float seq, double) multiplies by the factor cast to float
            amp = amp * np.float32(gain / db_gain)
        if shaping is not None and abs(shaping - db_shaping) > 0.01 * shaping:
            r1, r2 = self._response(shaping), self._response(db_shaping)
            amp = amp * (r1 / r2)  # float amplitudes times a float ratio of float magnitudes
        # sqrt(val * val + constant^2): the square in float, the sum and root in double
        return np.sqrt((amp * amp).astype(np.float64) + const * const).astype(np.float32)

    def frame_spectra(self, row_plane, row_wire_length, row_gain=None, row_shaping=None):
        """Spectra for ``add_noise``: (spectra [k][L] float32, row_spec [rows])
        with one spectrum per distinct (plane, length step, gain, shaping) of the rows."""
        keys, spectra, row_spec = {}, [], np.empty(len(row_plane), dtype=np.int32)
        for r, (p, wl) in enumerate(zip(row_plane, row_wire_length)):
            g = None if row_gain is None else float(row_gain[r])
            sh = None if row_shaping is None else float(row_shaping[r])
            key = (int(p), int(wl / self.wlres), g, sh)
            if key not in keys:
                keys[key] = len(spectra)
                spectra.append(self.channel_spectrum(int(p), wl, g, sh))
            row_spec[r] = keys[key]
        return np.stack(spectra) if spectra else np.zeros((0, self.L), np.float32), row_spec


# ---------------------------------------------------------------------------
# GroupNoiseModel (gen/src/GroupNoiseModel.cxx): coherent noise spectra per
# channel group, for add_noise with one random stream per group.  The float
# arithmetic of the reference's helpers is kept step for step: irrterp and
# linterp (util/inc/WireCellUtil/Interpolate.h, with std::lerp on floats),
# Spectrum::hermitian_mirror, interp, extrap, alias and resample
# (util/inc/WireCellUtil/Spectrum.h).
# ---------------------------------------------------------------------------
F32 = np.float32


def _lerp(a, b, t):
    """std::lerp(a, b, t) on floats as the GNU C++ library evaluates it (exact
    at t = 0 and t = 1, monotonic): the C++20 definition's steps."""
    a, b, t = F32(a), F32(b), F32(t)
    if (a <= 0 and b >= 0) or (a >= 0 and b <= 0):
        return t * b + (F32(1) - t) * a
    if t == F32(1):
        return b
    x = a + t * (b - a)
    if (t > F32(1)) == (b > a):
        return x if b < x else b
    return x if b > x else b


def _irrterp(keys, vals, num, xstep):
    """irrterp<float>(points)(out, num, 0, xstep): num samples from x = 0 in
    float steps of xstep over the sorted irregular points (keys, vals), flat
    beyond both ends (Interpolate.h:73-168)."""
    keys = [F32(k) for k in keys]
    vals = [F32(v) for v in vals]
    n = len(keys)
    xstep = F32(xstep)
    out = np.zeros(num, dtype=np.float32)
    if num == 0:
        return out
    xcur = F32(0)

    def upper_bound(x):
        lo, hi = 0, n
        while lo < hi:
            mid = (lo + hi) // 2
            if x < keys[mid]:
                hi = mid
            else:
                lo = mid + 1
        return lo

    ub = upper_bound(xcur)
    if num == 1:  # the single-point form, operator()(x)
        if ub == 0:
            out[0] = vals[0]
        elif ub == n:
            out[0] = vals[-1]
        else:
            dX = keys[ub] - keys[ub - 1]
            dY = vals[ub] - vals[ub - 1]
            out[0] = vals[ub - 1] + dY * (xcur - keys[ub - 1]) / dX
        return out
    for i in range(num):
        if ub == 0:  # before the domain
            out[i] = vals[0]
            xcur = xcur + xstep
            while xcur > keys[ub]:
                ub += 1
                if ub == n:
                    break
            continue
        if ub == n:  # after the domain
            out[i] = vals[-1]
            xcur = xcur + xstep
            continue
        lb = ub - 1
        delta = (xcur - keys[lb]) / (keys[ub] - keys[lb])
        out[i] = _lerp(vals[lb], vals[ub], delta)
        xcur = xcur + xstep
        while xcur > keys[ub]:
            ub += 1
            if ub == n:
                break
    return out


def _hermitian_mirror(v):
    """Spectrum::hermitian_mirror of a real (amplitude) sequence, in place."""
    n = len(v)
    mid = n // 2
    if n % 2:
        v[mid + 1:] = v[1:mid + 1][::-1]
    else:
        v[mid + 1:] = v[1:mid][::-1]
    return v


def _linterpolate(dat, olen):
    """linterpolate: the input spread over [0, 1) in len(dat) steps (double
    abscissae, float values), sampled at olen steps of 1 / olen."""
    ilen = len(dat)
    step = (1.0 - 0.0) / ilen
    re = 0.0 + step * (ilen - 1)
    newdx = (1.0 - 0.0) / olen
    out = np.zeros(olen, dtype=np.float32)
    for i in range(olen):
        x = 0.0 + i * newdx
        if x <= 0.0:
            out[i] = dat[0]
        elif x >= re:
            out[i] = dat[-1]
        else:
            ind = int((x - 0.0) / step)
            x0 = 0.0 + ind * step
            out[i] = _lerp(dat[ind], dat[ind + 1], F32((x - x0) / step))
    return out


def _spectrum_resample(sorig, olen, relperiod):
    """Spectrum::resample: interp to ceil(olen * relperiod) bins (times
    sqrt(new / old)), then alias (relperiod > 1) or zero-extrapolate."""
    tmpsiz = int(np.ceil(olen * relperiod))
    temp = _linterpolate(sorig, tmpsiz)
    norm = np.sqrt(tmpsiz / float(len(sorig)))
    temp = (temp.astype(np.float64) * norm).astype(np.float32)
    ilen = len(temp)
    out = np.zeros(olen, dtype=np.float32)
    if ilen == olen:
        return temp.copy()
    if relperiod > 1:  # alias
        if ilen < olen:
            raise ValueError("alias requires smaller output than input")
        half = ilen // 2
        L = int(np.ceil(ilen / float(olen)))
        M = olen // 2
        for m in range(M + 1):
            for l in range(L):
                old = m + l * M
                if old > half:
                    break
                out[m] = out[m] + temp[old]
        _hermitian_mirror(out)
        return (out.astype(np.float64) * np.sqrt(olen / float(ilen))).astype(np.float32)
    if ilen > olen:  # extrap
        raise ValueError("extrap requires larger output than input")
    half = ilen // 2
    lo, hi, extra = half, half + 1, 1
    if ilen % 2:
        lo, extra = lo + 1, 0
    out[:lo] = temp[:lo]
    if ilen - hi > 0:
        out[olen - (ilen - hi):] = temp[hi:]
    return out  # the middle olen - ilen + extra bins stay at the constant 0


def group_spectrum(freqs, amps, nsamples_orig, period_orig, nsamples, tick, scale=1.0):
    """One spectrum of GroupNoiseModel's "spectra" (gen/src/GroupNoiseModel.cxx:97-146):
    the points up to Nyquist (amplitudes times ``scale``; a repeated
    frequency keeps its last amplitude) interpolated onto nsamples_orig
    Rayleigh steps, mirrored, and resampled to ``nsamples`` bins at ``tick``."""
    norig, porig = int(nsamples_orig), float(period_orig)
    if not norig:
        raise ValueError("GroupNoiseModel: a spectrum lacks nsamples")
    fnyq = 1.0 / (2 * porig)
    fray = 1.0 / (norig * porig)
    pts = {}
    for f, a in zip(np.asarray(freqs, dtype=np.float32), np.asarray(amps, dtype=np.float32)):
        if float(f) > fnyq:
            continue
        pts[F32(f)] = F32(scale * float(a))
    if not pts:
        raise ValueError("GroupNoiseModel: no spectrum points below Nyquist")
    keys = sorted(pts)
    sorig = _irrterp(keys, [pts[k] for k in keys], norig, F32(fray))
    _hermitian_mirror(sorig)
    return _spectrum_resample(sorig, int(nsamples), float(tick) / porig)


class GroupNoiseModel:
    """GroupNoiseModel (gen/src/GroupNoiseModel.cxx:52-206): ``groups`` =
    [{group (or groupID), channels}], ``spectra`` = [{group (or groupID;
    else the entry's position), nsamples, period, freqs, amps}].  The spectra
    are built at configuration as the reference builds them."""

    def __init__(self, spectra, groups, nsamples=1024, tick=0.5 * US, scale=1.0):
        self.nsamples = int(nsamples)
        self.ch2grp = {}
        for g in groups:
            gid = g.get("group") if g.get("group") is not None else g.get("groupID")
            for ch in g["channels"]:
                self.ch2grp[int(ch)] = int(gid)
        self.grp2amp = {}
        for count, s in enumerate(spectra):
            gid = s.get("group") if s.get("group") is not None else s.get("groupID")
            group = int(gid) if isinstance(gid, (int, np.integer)) and not isinstance(gid, bool) else count
            self.grp2amp[group] = group_spectrum(s["freqs"], s["amps"], s["nsamples"], s["period"], self.nsamples,
                                                 tick, scale)

    def groupid(self, ch):
        return self.ch2grp.get(int(ch), -1)

    def group_spectrum(self, group):
        return self.grp2amp.get(int(group), np.zeros(0, dtype=np.float32))

    def channel_spectrum(self, ch):
        return self.group_spectrum(self.groupid(ch))

    def frame_spectra(self, row_channels):
        """For coherent ``add_noise``: (spectra [k][nsamples] float32, row_spec,
        row_stream): each row's group spectrum (-1: no group or no spectrum,
        the row gets no noise) and the group id as its random stream, so the
        channels of a group share one waveform."""
        keys, spectra = {}, []
        row_spec = np.full(len(row_channels), -1, dtype=np.int32)
        row_stream = np.full(len(row_channels), -1, dtype=np.int32)
        for r, ch in enumerate(row_channels):
            g = self.groupid(ch)
            if g < 0 or g not in self.grp2amp:
                continue
            if g not in keys:
                keys[g] = len(spectra)
                spectra.append(self.grp2amp[g])
            row_spec[r] = keys[g]
            row_stream[r] = g
        out = np.stack(spectra) if spectra else np.zeros((0, self.nsamples), np.float32)
        return out, row_spec, row_stream
