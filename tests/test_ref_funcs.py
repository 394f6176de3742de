"""Pins against reference functions compiled here from the reference's own
source (oracle/extract_ref.py + oracle/ref_funcs_harness.cpp): GausDesc bin
integrals, impact weights and distance (gen/src/GaussianDiffusion.cxx:30-92,
gen/inc/WireCellGen/GaussianDiffusion.h:33-49), Waveform::edge
(util/src/Waveform.cxx:136-153), Response::coldelec
(util/src/Response.cxx:311-340), Drifter::insert (gen/src/Drifter.cxx:127-196)
and BinnedDiffusion_transform::add (gen/src/BinnedDiffusion_transform.cxx:37-92),
among others.  Against the committed vectors
(tests/golden/ref_funcs.json, written by tests/golden/make_ref_funcs.py) and,
where the harness was built, live on fresh random cases.  CPU only."""

import json
import os

import numpy as np
import pytest

from conftest import ROOT

GOLDEN = os.path.join(ROOT, "tests", "golden", "ref_funcs.json")


@pytest.fixture(scope="module")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


def test_gausdesc_against_reference_vectors(oracle, golden):
    """The oracle's GausDesc (FP64, the arithmetic of the patch bins and the
    linear impact weights) is bit for bit the reference's."""
    L = oracle.lib()
    for c in golden["gausdesc"]:
        b = oracle.gd_binint(L, "orc", c["center"], c["sigma"], c["start"], c["step"], c["nbins"])
        assert b.tolist() == c["binint"], c
        w = oracle.gd_weight(L, "orc", c["center"], c["sigma"], c["start"], c["step"], len(b), b)
        assert w.tolist() == c["weight"], c
        assert L.orc_gd_distance(c["center"], c["sigma"], c["x"]) == c["distance"]


def test_gausdesc_against_compiled_reference(oracle):
    R = oracle.ref_funcs()
    if R is None:
        pytest.skip("reference function harness not built")
    L = oracle.lib()
    rng = np.random.default_rng(99)
    for _ in range(3000):
        center = rng.uniform(-3000.0, 3000.0)
        sigma = 0.0 if rng.random() < 0.05 else np.exp(rng.uniform(np.log(1e-3), np.log(100.0)))
        step = rng.uniform(0.05, 10.0)
        start = center - rng.uniform(0.0, 6.0 * (sigma or step))
        nbins = 1 if sigma == 0.0 else int(rng.integers(1, 80))
        a = oracle.gd_binint(L, "orc", center, sigma, start, step, nbins)
        b = oracle.gd_binint(R, "ref", center, sigma, start, step, nbins)
        assert np.array_equal(a, b)
        if np.all(a > 0):
            assert np.array_equal(oracle.gd_weight(L, "orc", center, sigma, start, step, len(a), a),
                                  oracle.gd_weight(R, "ref", center, sigma, start, step, len(b), b))


def test_trace_edges_against_reference(oracle, golden):
    """Waveform::edge: first non-zero sample and one past the last (-0.0 is zero)."""
    for e in golden["edge"]:
        w = np.array(e["wave"], dtype=np.float32)
        assert list(oracle.edge(w)) == e["edge"]
    R = oracle.ref_funcs()
    if R is not None:
        rng = np.random.default_rng(5)
        for n in range(0, 64):
            w = rng.normal(size=n).astype(np.float32)
            w[rng.random(n) < 0.7] = 0.0
            out = np.zeros(2, dtype=np.int32)
            R.ref_wave_edge(w.ctypes.data, n, out.ctypes.data)
            assert list(oracle.edge(w)) == out.tolist()


def test_coldelec_against_reference(golden):
    """The noise model's cold-electronics response (noise.coldelec, NumPy)
    against the reference's compiled Response::coldelec: the same terms
    summed in another order, so equal to rounding (1e-12 of the peak); zero
    outside (0, 10 us) exactly as the reference."""
    import importlib
    noise = importlib.import_module("wire-cell-toolkit_b200.noise")
    for c in golden["coldelec"]:
        t = np.array(c["time"])
        want = np.array(c["value"])
        got = noise.coldelec(t, c["gain"], c["shaping"])
        assert np.array_equal(got == 0.0, want == 0.0)
        assert np.max(np.abs(got - want)) <= 1e-12 * np.max(np.abs(want))


def test_pimpos_against_reference(oracle, golden):
    """The oracle's plane geometry (Pimpos: normalised axes, wire and impact
    binning, pitch coordinate of a point) is bit for bit the reference's."""
    L = oracle.lib()
    for c in golden["pimpos"]:
        head, dist = oracle.pimpos(L, "orc", c["nwires"], c["minp"], c["maxp"], c["wire"], c["pitch"], c["origin"],
                                   c["nbins"], c["pts"])
        assert head.tolist() == c["head"], c["nwires"]
        assert dist.tolist() == c["dist"], c["nwires"]
    R = oracle.ref_funcs()
    if R is None:
        return
    rng = np.random.default_rng(123)
    for _ in range(200):
        a = rng.uniform(-np.pi, np.pi)
        wire = [rng.normal() * 1e-3, np.cos(a), np.sin(a)]
        pitch = np.array([0.0, -np.sin(a), np.cos(a)]) * rng.uniform(0.1, 10.0)
        nw = int(rng.integers(2, 3000))
        minp = rng.uniform(-4000.0, 0.0)
        maxp = minp + rng.uniform(1.0, 8000.0)
        pts = rng.uniform(-4000.0, 4000.0, (50, 3))
        origin = rng.uniform(-100.0, 100.0, 3)
        nb = int(rng.integers(1, 12)) * 2
        got = oracle.pimpos(L, "orc", nw, minp, maxp, wire, pitch, origin, nb, pts)
        want = oracle.pimpos(R, "ref", nw, minp, maxp, wire, pitch, origin, nb, pts)
        assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])


def test_digitizer_against_reference(oracle, golden):
    """The oracle's ADC arithmetic (which the GPU digitizer equals bit for bit)
    against the reference's compiled Digitizer::digitize, sample by sample."""
    for c in golden["digitize"]:
        f = np.array(c["frame"], dtype=np.float32)
        got = oracle.digitize(f, np.array(c["baseline"], dtype=np.float32), c["gain"], tuple(c["fullscale"]),
                              c["resolution"], bool(c["round"]))
        assert np.array_equal(got, np.array(c["adc"], dtype=np.float32)), (c["gain"], c["resolution"], c["round"])
    R = oracle.ref_funcs()
    if R is None:
        return
    rng = np.random.default_rng(8)
    volt = 1.0e-6
    for k in range(12):
        f = rng.normal(0.0, rng.uniform(0.05, 1.5) * volt, (16, 200)).astype(np.float32)
        base = rng.uniform(0.0, 1.0, 16).astype(np.float32) * np.float32(volt)
        gain, res, rnd = rng.uniform(0.3, 4.0), int(rng.integers(8, 16)), k % 2
        fs = (0.0, float(rng.uniform(1.0, 3.0)) * volt)
        want = np.zeros_like(f)
        R.ref_digitize(f.ctypes.data, 16, 200, base.ctypes.data, gain, fs[0], fs[1], res, rnd, want.ctypes.data)
        assert np.array_equal(oracle.digitize(f, base, gain, fs, res, bool(rnd)), want)


def _model_entry(e):
    return dict(plane=0, gain=14.0, shaping=2000.0, wirelen=1000.0, const=e["const"], nsamples=e["nsamples"],
                period=e["period"], freqs=e["freqs"], amps=e["amps"])


def test_noise_resampling_against_reference(golden, oracle):
    """The noise model's spectrum resampling (noise.EmpiricalNoiseModel, the
    product's host code) equals the reference's compiled
    EmpiricalNoiseModel::resample bit for bit: float frequency grid, sqrt(L/n)
    scale, clamped linear interpolation, float amplitudes."""
    import importlib
    noise = importlib.import_module("wire-cell-toolkit_b200.noise")
    for e in golden["noise_resample"]:
        m = noise.EmpiricalNoiseModel([_model_entry(e)], nsamples=e["model_nsamples"], period=e["model_period"])
        assert m.L == e["fft_length"]
        s = m.planes[0][0]
        assert s["const"] == e["const_out"]
        assert np.array_equal(np.asarray(s["amps"], dtype=np.float32), np.array(e["amps_out"], dtype=np.float32))
    R = oracle.ref_funcs()
    if R is None:
        return
    rng = np.random.default_rng(21)
    for k in range(20):
        period = float(rng.choice([400.0, 500.0, 1000.0]))
        nyq = 1.0 / (2 * period)
        nf = int(rng.integers(2, 300))
        freqs = np.sort(rng.uniform(-0.1 * nyq, 1.2 * nyq, nf)).astype(np.float32)
        e = dict(const=float(rng.uniform(0, 1)), nsamples=int(rng.integers(16, 2000)), period=period,
                 freqs=list(freqs.astype(float)), amps=list(rng.uniform(0.0, 5.0, nf).astype(np.float32).astype(float)))
        model_n = int(rng.integers(100, 3000))
        m = noise.EmpiricalNoiseModel([_model_entry(e)], nsamples=model_n, period=period)
        const, amps = oracle.ref_noise_resample(R, m.L, period, e)
        assert m.planes[0][0]["const"] == const
        assert np.array_equal(np.asarray(m.planes[0][0]["amps"], dtype=np.float32), amps)


def test_group_noise_spectra_against_reference(golden, oracle):
    """GroupNoiseModel's spectra (noise.group_spectrum, host code) equal the
    reference's bit for bit: irrterp onto Rayleigh steps, the Hermitian
    mirror, Spectrum::resample with its aliasing or extrapolation, in the
    reference's float arithmetic (std::lerp included)."""
    import importlib
    noise = importlib.import_module("wire-cell-toolkit_b200.noise")
    for c in golden["group_spectrum"]:
        got = noise.group_spectrum(c["freqs"], c["amps"], c["nsamples_orig"], c["period_orig"], c["nsamples"],
                                   c["tick"], c["scale"])
        assert np.array_equal(got, np.array(c["spectrum"], dtype=np.float32))
    R = oracle.ref_funcs()
    if R is None:
        return
    rng = np.random.default_rng(17)
    for k in range(40):
        porig = float(rng.choice([400.0, 500.0, 512.0]))
        nyq = 1.0 / (2 * porig)
        nf = int(rng.integers(1, 80))
        f = np.sort(rng.uniform(0.0, 1.3 * nyq, nf)).astype(np.float32)
        if k % 2:
            f[0] = 0.0
        a = rng.uniform(0.0, 3.0, nf).astype(np.float32)
        norig, ns = int(rng.integers(2, 500)), int(rng.integers(2, 600))
        tick = float(rng.choice([200.0, 250.0, 500.0, 1000.0]))
        want = oracle.ref_group_spectrum(R, f, a, norig, porig, ns, tick, 0.8)
        if want is None:
            with pytest.raises(ValueError):
                noise.group_spectrum(f, a, norig, porig, ns, tick, 0.8)
        else:
            assert np.array_equal(noise.group_spectrum(f, a, norig, porig, ns, tick, 0.8), want), k


def test_noise_wire_length_interpolation_against_reference(oracle):
    """EmpiricalNoiseModel::interpolate_wire_length (gen/src/EmpiricalNoiseModel.cxx:232-275):
    clamped at the shortest and longest entries, linear in between (float
    amplitudes, double constant), bit for bit against the compiled reference."""
    import ctypes as C
    import importlib
    noise = importlib.import_module("wire-cell-toolkit_b200.noise")
    R = oracle.ref_funcs()
    if R is None:
        pytest.skip("reference function harness not built")
    rng = np.random.default_rng(5)
    L = 400
    freqs = list(np.linspace(0.0, 1.0 / (2 * 500.0), 60))
    for k in range(10):
        nspec = int(rng.integers(1, 5))
        lens = np.sort(rng.uniform(500.0, 8000.0, nspec)).astype(np.float32).astype(np.float64)
        ents = [dict(plane=0, gain=14.0, shaping=2000.0, wirelen=float(wl), const=float(rng.uniform(0, 0.1)),
                     nsamples=L, period=500.0, freqs=freqs, amps=list(rng.uniform(0.1, 3.0, 60)))
                for wl in lens]
        m = noise.EmpiricalNoiseModel(ents, nsamples=L, period=500.0)
        sp = m.planes[0]
        wls = np.array([s["wirelen"] for s in sp])
        cs = np.array([s["const"] for s in sp])
        am = np.ascontiguousarray(np.stack([np.asarray(s["amps"], dtype=np.float32) for s in sp]))
        for wl in list(rng.uniform(0.0, 9000.0, 20)) + list(wls):
            c = C.c_double()
            out = np.zeros(am.shape[1], dtype=np.float32)
            assert R.ref_noise_interp(len(sp), wls.ctypes.data, cs.ctypes.data, am.ctypes.data, am.shape[1], float(wl),
                                      C.byref(c), out.ctypes.data) == 0
            const, amp = m.interpolate_wire_length(0, float(wl))
            assert const == c.value
            assert np.array_equal(np.asarray(amp, dtype=np.float32), out)


def test_noise_generator_spectrum_against_reference(oracle):
    """The oracle's noise spectrum (oracle.noise_spec, which the GPU noise is
    checked against in distribution) against the reference's compiled
    GeneratorN::spec given the same normals: the same bins draw the same
    normals, DC and Nyquist by modulus, the same Hermitian mirror; equal to
    float rounding (the reference multiplies in float)."""
    R = oracle.ref_funcs()
    if R is None:
        pytest.skip("reference function harness not built")
    rng = np.random.default_rng(12)
    for n in (3, 4, 5, 16, 17, 255, 256, 1000, 1001):
        S = rng.uniform(0.0, 2.0, n)
        nn = 2 * (n // 2 + (n + 1) % 2) + 1
        normals = rng.normal(size=nn).astype(np.float32)
        sig = (S * np.sqrt(2.0 / 3.141592)).astype(np.float32)
        out = np.zeros(2 * n, dtype=np.float32)
        assert R.ref_generator_spec(n, sig.ctypes.data, normals.ctypes.data, nn, out.ctypes.data) == 0
        want = out[0::2].astype(np.float64) + 1j * out[1::2].astype(np.float64)
        got = oracle.noise_spec(sig.astype(np.float64) / np.sqrt(2.0 / 3.141592), normals.astype(np.float64))
        assert np.abs(got - want).max() <= 1e-6 * np.abs(want).max(), n


def test_drift_against_reference_vectors(oracle, golden):
    """Drifter::insert (gen/src/Drifter.cxx:127-196, fluctuation off): which
    depos are kept and their drifted (t, q, x, y, z, extent_long,
    extent_tran), bit for bit the reference's compiled code, over one face,
    two mirrored faces, a region without an anode, and positions exactly on
    the anode, response and cathode planes."""
    L = oracle.lib()
    for c in golden["drift"]:
        k, o = oracle.drift_one(L, "orc", c)
        assert k == c["kept"], c
        if k:
            assert o.tolist() == c["out"], c


def test_drift_against_compiled_reference(oracle):
    R = oracle.ref_funcs()
    if R is None:
        pytest.skip("reference function harness not built")
    L = oracle.lib()
    for c in oracle.drift_cases(np.random.default_rng(1234), 3000):
        ka, a = oracle.drift_one(L, "orc", c)
        kb, b = oracle.drift_one(R, "ref", c)
        assert ka == kb, c
        if ka:
            assert np.array_equal(a, b), c


def test_bdt_add_against_reference_vectors(oracle, golden):
    """BinnedDiffusion_transform::add (gen/src/BinnedDiffusion_transform.cxx:37-92):
    the time and pitch rejections and their counters, bit for bit the
    reference's compiled code, including zero widths and centres exactly
    nsigma outside the window or the impact range."""
    L = oracle.lib()
    for c in golden["bdt_add"]:
        k, cnt = oracle.bdt_add(L, "orc", c)
        assert (k, cnt) == (c["added"], c["counters"]), c


def test_bdt_add_against_compiled_reference(oracle):
    R = oracle.ref_funcs()
    if R is None:
        pytest.skip("reference function harness not built")
    L = oracle.lib()
    for c in oracle.bdt_add_cases(np.random.default_rng(4321), 3000):
        assert oracle.bdt_add(L, "orc", c) == oracle.bdt_add(R, "ref", c), c
