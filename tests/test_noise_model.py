"""EmpiricalNoiseModel's channel spectra (gen/src/EmpiricalNoiseModel.cxx):
frequency grid, resampling (sqrt(L / n) scale, clamped linear
interpolation), wire-length interpolation and clamping, gain scaling, the
constant added in quadrature, and the spectra handed to add_noise."""

import importlib

import numpy as np
import pytest

noise = importlib.import_module("wire-cell-toolkit_b200.noise")
CM = 10.0
US = 1000.0


def _entries(nsamples=256, period=0.5 * US, lengths=(100 * CM, 300 * CM, 600 * CM)):
    out = []
    freqs = np.linspace(0.0, 1.0 / (2 * period), 65)  # up to Nyquist
    for k, wl in enumerate(lengths):
        out.append(dict(plane=0, gain=14.0, shaping=2.0 * US, wirelen=wl, const=0.01 * (k + 1), nsamples=nsamples,
                        period=period, freqs=list(freqs), amps=list(1.0 + (k + 1) * freqs * period)))
    return out


def test_grid_and_resampling(wct):
    ents = _entries()
    m = noise.EmpiricalNoiseModel(ents, nsamples=6000, period=0.5 * US)
    L = wct.fft_best_length(6000)
    assert m.L == L and m.freq.size == L
    assert m.freq[1] == pytest.approx(1.0 / (L * 0.5 * US)) and m.freq[L - 1] == m.freq[1]
    # the entries' amplitudes are linear in frequency: resampling keeps the line, times sqrt(L / 256)
    s = np.sqrt(L / 256.0)
    k = 0
    want = s * (1.0 + (k + 1) * np.minimum(m.freq, 1.0 / (2 * 0.5 * US)) * 0.5 * US)
    np.testing.assert_allclose(m.planes[0][0]["amps"], want, rtol=2e-6)
    assert m.planes[0][0]["const"] == pytest.approx(0.01 * s)


def test_no_resampling_at_the_model_grid(wct):
    L = wct.fft_best_length(6000)
    ents = _entries(nsamples=L)
    ents[0]["amps"] = list(np.arange(L, dtype=np.float64))  # kept as is
    ents[0]["freqs"] = list(np.arange(L, dtype=np.float64))
    for e in ents[1:]:
        e["amps"], e["freqs"] = list(np.ones(L)), list(np.arange(L, dtype=np.float64))
    m = noise.EmpiricalNoiseModel(ents, nsamples=6000, period=0.5 * US)
    assert np.array_equal(m.planes[0][0]["amps"], np.arange(L, dtype=np.float32))


def test_wire_length_interpolation_and_channel_spectrum():
    m = noise.EmpiricalNoiseModel(_entries(), nsamples=6000, period=0.5 * US)
    a, b = m.planes[0][0], m.planes[0][1]
    c, amp = m.interpolate_wire_length(0, 200 * CM)  # halfway between 100 and 300 cm
    np.testing.assert_allclose(amp, 0.5 * (a["amps"] + b["amps"]), rtol=1e-6)
    assert c == pytest.approx(0.5 * (a["const"] + b["const"]))
    c0, amp0 = m.interpolate_wire_length(0, 10 * CM)    # clamped at the shortest
    assert c0 == a["const"] and np.array_equal(amp0, a["amps"])
    s = m.channel_spectrum(0, 200.7 * CM)              # 200.7 cm rounds down to 200 cm steps
    np.testing.assert_allclose(s, np.sqrt(amp * amp + c * c), rtol=1e-6)
    sg = m.channel_spectrum(0, 200 * CM, gain=28.0)    # twice the spectra's gain
    np.testing.assert_allclose(sg, np.sqrt((2 * amp) ** 2 + c * c), rtol=1e-6)
    assert np.array_equal(m.channel_spectrum(0, 200 * CM, gain=14.05), s)  # within 1%: unchanged


def test_coldelec_and_shaping_correction():
    t = np.arange(0, 12 * US, 10.0)
    r = noise.coldelec(t, 10.0, 2.0 * US)
    assert r[0] == 0 and np.all(r[t >= 10 * US] == 0)
    assert 1.0 * US < t[np.argmax(r)] < 3.0 * US          # peaks after about the shaping time
    m = noise.EmpiricalNoiseModel(_entries(), nsamples=6000, period=0.5 * US)
    base = m.channel_spectrum(0, 200 * CM)
    assert np.array_equal(m.channel_spectrum(0, 200 * CM, shaping=2.01 * US), base)  # within 1%
    s1 = m.channel_spectrum(0, 200 * CM, shaping=1.0 * US)
    c, amp = m.interpolate_wire_length(0, 200 * CM)
    tt = np.arange(m.L) * 0.5 * US
    ratio = (np.abs(np.fft.fft(noise.coldelec(tt, 10.0, 1.0 * US).astype(np.float32).astype(np.float64)))
             / np.abs(np.fft.fft(noise.coldelec(tt, 10.0, 2.0 * US).astype(np.float32).astype(np.float64))))
    np.testing.assert_allclose(s1, np.sqrt((amp * ratio) ** 2 + c * c), rtol=1e-5)
    # responses cached per 0.1 us step: 1.03 us reuses the 1.0 us response
    assert np.array_equal(m.channel_spectrum(0, 200 * CM, shaping=1.03 * US), s1)


def test_frame_spectra_groups_rows():
    m = noise.EmpiricalNoiseModel(_entries(), nsamples=6000, period=0.5 * US)
    spectra, row_spec = m.frame_spectra([0, 0, 0, 0], [150 * CM, 150.4 * CM, 400 * CM, 150 * CM])
    assert spectra.shape == (2, m.L) and list(row_spec) == [0, 0, 1, 0]


@pytest.mark.gpu
def test_model_noise_power(wct):
    """add_noise with the model's spectrum: mean power per bin 2 sigma_k^2."""
    m = noise.EmpiricalNoiseModel(_entries(), nsamples=6000, period=0.5 * US)
    rows = 1500
    spectra, row_spec = m.frame_spectra([0] * rows, [250 * CM] * rows)
    if m.L % 2:
        pytest.skip("odd model length")
    frame = np.zeros((rows, m.L), np.float32)
    wct.add_noise(frame, spectra, row_spec, np.arange(rows, dtype=np.int32), seed=3)
    P = (np.abs(np.fft.fft(frame.astype(np.float64), axis=1)) ** 2).mean(axis=0)
    sig2 = 2.0 * (spectra[0].astype(np.float64) * np.sqrt(2.0 / 3.141592)) ** 2
    assert abs((P[: m.L // 2 + 1] / sig2[: m.L // 2 + 1]).mean() - 1.0) < 0.01


def _scalar_resample(freq_grid, nsamples_model, ent):
    """EmpiricalNoiseModel::resample (gen/src/EmpiricalNoiseModel.cxx:96-136) line by line."""
    scale = np.sqrt(nsamples_model / (ent["nsamples"] * 1.0))
    amps = [float(np.float32(a * scale)) for a in np.asarray(ent["amps"], np.float32)]
    freqs = [float(f) for f in np.asarray(ent["freqs"], np.float32)]
    out = []
    for frequency in freq_grid:
        if frequency <= freqs[0]:
            lo, hi, mu = 0, 1, 0.0
        elif frequency >= freqs[-1]:
            lo, hi, mu = len(freqs) - 2, len(freqs) - 1, 1.0
        else:
            lo, hi = 0, 1
            for j in range(len(freqs)):
                if frequency > freqs[j]:
                    lo, hi = j, j + 1
                else:
                    break
            # frequency is a double, the entry's freqs are floats: float - float is a float subtraction
            mu = (frequency - freqs[lo]) / float(np.float32(freqs[hi]) - np.float32(freqs[lo]))
        out.append(float(np.float32((1 - mu) * amps[lo] + mu * amps[hi])))
    return np.array(out)


def test_resample_matches_scalar_loop():
    rng = np.random.default_rng(4)
    ents = _entries()
    ents[1]["freqs"] = list(np.sort(rng.uniform(0, 1.0 / (2 * 0.5 * US), 40)))
    ents[1]["amps"] = list(rng.uniform(0.5, 2.0, 40))
    m = noise.EmpiricalNoiseModel(ents, nsamples=6000, period=0.5 * US)
    for k in range(3):
        np.testing.assert_array_equal(m.planes[0][k]["amps"], _scalar_resample(m.freq, m.L, ents[k]))


def test_channel_spectrum_float_steps():
    """EmpiricalNoiseModel::channel_spectrum (gen/src/EmpiricalNoiseModel.cxx:357-412)
    bin by bin with the reference's types: the gain factor cast to float
    (Waveform::scale), float amplitudes times the float ratio of the float
    response magnitudes, then sqrt(val * val + constant^2) with the square
    in float and the rest in double."""
    import math
    m = noise.EmpiricalNoiseModel(_entries(), nsamples=6000, period=0.5 * US)
    wl, gain, shaping = 250 * CM, 1.3 * 14.0, 3.0 * US
    got = m.channel_spectrum(0, wl, gain, shaping)
    const, amp = m.interpolate_wire_length(0, int(wl / m.wlres) * m.wlres)
    r1, r2 = m._response(shaping), m._response(2.0 * US)
    g = np.float32(gain / 14.0)  # a double quotient cast to float
    for i in range(0, m.L, 7):
        a = np.float32(amp[i]) * g
        a = a * (np.float32(r1[i]) / np.float32(r2[i]))
        assert got[i] == np.float32(math.sqrt(float(a * a) + const * const)), i


def test_group_noise_model_groups():
    """GroupNoiseModel (gen/src/GroupNoiseModel.cxx:84-206): channels map to
    groups by "group" or "groupID"; a spectrum without a group id takes its
    position; channels without a group (or a group without a spectrum) get
    no noise; frame_spectra gives each row its group's spectrum and the group
    as its random stream."""
    freqs = list(np.linspace(0.0, 1.0 / (2 * 0.5 * US), 20))
    spectra = [dict(nsamples=128, period=0.5 * US, freqs=freqs, amps=list(np.linspace(1.0, 2.0, 20))),
               dict(groupID=7, nsamples=128, period=0.5 * US, freqs=freqs, amps=list(np.linspace(3.0, 1.0, 20)))]
    groups = [dict(group=0, channels=[10, 11, 12]), dict(groupID=7, channels=[20, 21]), dict(group=9, channels=[30])]
    m = noise.GroupNoiseModel(spectra, groups, nsamples=256, tick=0.5 * US)
    assert sorted(m.grp2amp) == [0, 7]
    assert m.groupid(11) == 0 and m.groupid(21) == 7 and m.groupid(30) == 9 and m.groupid(99) == -1
    assert m.channel_spectrum(30).size == 0 and m.channel_spectrum(99).size == 0
    assert m.channel_spectrum(12).shape == (256,) and m.channel_spectrum(12).dtype == np.float32
    sp, row_spec, row_stream = m.frame_spectra([10, 20, 11, 30, 99, 21])
    assert sp.shape == (2, 256)
    assert row_spec.tolist() == [0, 1, 0, -1, -1, 1]
    assert row_stream.tolist() == [0, 7, 0, -1, -1, 7]
    assert np.array_equal(sp[1], m.group_spectrum(7))
