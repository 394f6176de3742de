"""Pins of the CPU oracle (oracle/wct_oracle.cpp) against the reference's own
known-answer tests and against the reference-compiled Binning, plus the
oracle's internal consistency checks.  CPU only."""

import json
import math
import os

import numpy as np
import pytest

from conftest import rel_l2

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "binning_ref.json")


def test_binning_against_reference_golden(oracle):
    """Binning::bin / sample_bin_range (util/inc/WireCellUtil/Binning.h:75,99-102)
    against vectors produced by the reference's compiled Binning."""
    g = json.load(open(GOLDEN))
    L = oracle.lib()
    import ctypes as C
    r = (C.c_int * 2)()
    for c in g["cases"]:
        assert L.orc_binning_bin(c["n"], c["lo"], c["hi"], c["v"]) == c["bin"], c
        L.orc_sample_bin_range(c["n"], c["lo"], c["hi"], c["v"], c["w"], r)
        assert [r[0], r[1]] == c["sbr"], c


def test_binning_against_compiled_reference(oracle):
    """Same comparison live against oracle/_ref (when it was built here)."""
    R = oracle.ref()
    if R is None:
        pytest.skip("reference Binning harness not built")
    L = oracle.lib()
    rng = np.random.default_rng(7)
    for (n, lo, hi) in [(6000, 0.0, 3.0e6), (9600, -2299.2, 2299.2), (8000, -1870.3, 1870.3)]:
        for v in lo + (hi - lo) * rng.uniform(-0.1, 1.1, 2000):
            assert L.orc_binning_bin(n, lo, hi, float(v)) == R.ref_bin(n, lo, hi, float(v))


def test_gaussian_known_answers(oracle):
    """util/test/test_binning.cxx:86-91 known answers, through the reference
    golden values and through the oracle's bin integrals (GausDesc::binint)."""
    g = json.load(open(GOLDEN))
    kat = {("gcumulative", (0, 0, 1)): 0.5, ("gcumulative", (10, 0, 1)): 1.0, ("gcumulative", (5, 5, 30)): 0.5,
           ("gcumulative", (300, 5, 30)): 1.0, ("gbounds", (-1, 1, 0, 1)): 0.682689, ("gbounds", (1, -1, 0, 1)): 0.682689,
           ("gbounds", (0, 10, 0, 1)): 0.5, ("gbounds", (-10, 0, 0, 1)): 0.5}
    for e in g["gauss"]:
        key = (e["kind"], tuple(e["args"]))
        if key in kat:
            assert abs(e["value"] - kat[key]) < 1e-6
        if e["kind"] == "gaussian":
            assert abs(e["value"] - 1.0) < 1e-6
    # oracle bin integral over [-1 sigma, +1 sigma] in two bins of one sigma
    P = oracle.set_sampling(t=0.0, q=-1.0, pc=0.0, st=1.0, sp=1.0, tbins=(2, -1.0, 1.0), ibins=(2, -1.0, 1.0),
                            nsigma=1.0, fp64=True)
    # the patch is normalised to the charge; the raw bins are 0.3413 each
    assert P["nt"] == 2 and P["np"] == 2
    assert abs(P["patch"].sum() + 1.0) < 1e-12


def test_fft_best_length_known_sizes(oracle):
    """util/src/FFTBestLength.cxx:12-59 on the window sizes of the workloads."""
    assert oracle.fft_best_length(964 + 20, True) == 1024
    assert oracle.fft_best_length(964 + 42, True) == 1024
    assert oracle.fft_best_length(3134 + 200, False) == 3584
    assert oracle.fft_best_length(200, False) == 200
    assert oracle.fft_best_length(17000, False) == 17000
    assert oracle.fft_best_length(845, True) == 847
    assert oracle.fft_best_length(846, True) == 896


def _fft_tables():
    with open(os.path.join(os.path.dirname(GOLDEN), "fft_lengths_ref.json")) as f:
        return json.load(f)


def test_fft_length_tables_are_the_references():
    """The three tables of util/src/FFTBestLength.cxx:16-50 (extracted from
    the source text by tests/golden/make_fft_lengths.py) equal csrc/fft_lengths.h,
    which the host window arithmetic and the device batch planner share."""
    g = _fft_tables()
    hdr = open(os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(GOLDEN))), "wire-cell-toolkit_b200", "csrc",
                            "fft_lengths.h")).read()
    for key, macro in (("any", "WCT_FFT_LENGTHS_ANY"), ("even", "WCT_FFT_LENGTHS_EVEN"), ("odd", "WCT_FFT_LENGTHS_ODD")):
        line = next(ln for ln in hdr.splitlines() if ln.startswith("#define " + macro + " "))
        assert [int(x) for x in line.split(None, 2)[2].split(",")] == g[key]


def test_fft_best_length_every_edge(oracle, wct):
    """util/src/FFTBestLength.cxx:52-58: the first table entry >= n while n is
    within the table, else n itself; the even or odd table by n's parity when
    keep_odd_even.  Oracle and product at every table entry and its two
    neighbours, below the first entry, past the last, and at 3000 random n."""
    g = _fft_tables()

    def expect(n, keep):
        t = g["any"] if not keep else (g["even"] if n % 2 == 0 else g["odd"])
        return next((e for e in t if e >= n), n)

    ns = set(range(0, 64)) | set(range(16300, 17001))
    for t in (g["any"], g["even"], g["odd"]):
        for e in t:
            ns |= {e - 2, e - 1, e, e + 1, e + 2}
    ns |= set(int(v) for v in np.random.default_rng(1).integers(0, 17000, 3000))
    for keep in (False, True):
        for n in sorted(v for v in ns if v >= 0):
            e = expect(n, keep)
            assert oracle.fft_best_length(n, keep) == e, (n, keep)
            assert wct.fft_best_length(n, keep) == e, (n, keep)


def test_pimpos_known_answers(oracle):
    """util/test/test_pimpos.cxx:47-70: 2001 wires at 3 mm."""
    pitch = 3.0
    n = 2001
    half = pitch * 0.5 * (n - 1)
    regionsize = (2 * half) / (n - 1)
    lo, hi = -half - 0.5 * regionsize, half + 0.5 * regionsize
    assert lo == -3001.5 and hi == 3001.5
    assert (hi - lo) / n == pitch
    assert oracle.lib().orc_binning_bin(n, lo, hi, 0.0) == n // 2


def _impulse(n):
    x = np.zeros(2 * n)
    x[0] = 1.0
    return x


@pytest.mark.parametrize("n", [64, 200, 1024, 1792, 3584, 6000, 2662, 847])
def test_dft_impulse_flat_roundtrip(oracle, n):
    """aux/test/test_dfttools.cxx:24-34: impulse <-> flat, inverse normalised."""
    x = _impulse(n)
    oracle.lib().orc_fft_f64(x.ctypes.data, n, 0)
    c = x[0::2] + 1j * x[1::2]
    assert np.allclose(c, 1.0, atol=1e-12)
    oracle.lib().orc_fft_f64(x.ctypes.data, n, 1)
    c = x[0::2] + 1j * x[1::2]
    want = np.zeros(n, complex)
    want[0] = 1
    assert np.allclose(c, want, atol=1e-12)


@pytest.mark.parametrize("n", [200, 1792, 3584, 2744])
def test_dft_matches_numpy(oracle, n):
    rng = np.random.default_rng(n)
    z = rng.normal(size=n) + 1j * rng.normal(size=n)
    x = np.empty(2 * n)
    x[0::2], x[1::2] = z.real, z.imag
    oracle.lib().orc_fft_f64(x.ctypes.data, n, 0)
    assert rel_l2(x[0::2] + 1j * x[1::2], np.fft.fft(z)) < 1e-13
    xf = x.astype(np.float32)
    xf[0::2], xf[1::2] = z.real, z.imag
    oracle.lib().orc_fft_f32(xf.ctypes.data, n, 0)
    assert rel_l2(xf[0::2] + 1j * xf[1::2], np.fft.fft(z)) < 2e-6


def test_pir_known_answers(oracle, synth):
    """gen/test/test_pir.cxx:52: 11 impact positions per wire region; the
    symmetrised map puts the mirrored paths in the upper half of each region."""
    cfg = synth.plane1_config(nticks=1000, nwire_half=10)
    pir = oracle.pir_build(cfg, 0, fp64=True)
    assert pir["bywire"].shape == (21, 11)
    assert abs(pir["pitch"] - 4.79) < 1e-12
    assert abs(pir["impact"] - 0.479) < 1e-12
    bw = pir["bywire"]
    for w in range(21):
        k = w - 10
        # direct paths of wire k, then the mirrored paths of wire -k
        assert list(bw[w][:6]) == [6 * (k + 10) + m for m in range(6)]
        assert list(bw[w][6:]) == [6 * (-k + 10) + m for m in (4, 3, 2, 1, 0)]


def test_closest_wire_impact_known_answers():
    """gen/test/test_impcalc.cxx:9-54: the closest_wire_impact arithmetic
    (21 wires, pitch 5 mm, impact 0.5 mm, nimp_per_wire = 6)."""
    import oracle as O
    nwires, pitch, impact = 21, 5.0, 0.5
    nimp = 1 + int(round(pitch / impact)) // 2
    assert nimp == 6
    half = (nwires // 2 + 0.5) * pitch
    rp = -half
    while rp <= half:
        relwire = O.cround(rp / pitch)
        rem = rp - relwire * pitch
        assert -pitch / 2 <= rem <= pitch / 2
        assert abs(O.cround(rem / impact)) <= int(round(pitch / impact)) // 2
        rp += impact


def test_oracle_fp64_matches_direct_convolution(oracle, synth):
    """The restatement's pair-packed 2-D FFT convolution
    (gen/src/ImpactTransform.cxx:120-306) equals an independent FP64 direct
    linear convolution of the impact-group charges."""
    cfg = synth.plane1_config(nticks=1200, nwire_half=10)
    d = synth.plane1_depos(n=12, drift=0.3 * synth.m, span=0.3 * synth.m)
    r64 = oracle.run(cfg, d, fp64=True)
    dd = oracle.direct_fp64(cfg, d, 0)
    assert rel_l2(r64["frames"][0], dd) < 1e-12


def test_oracle_fp32_vs_fp64(oracle, synth):
    cfg = synth.plane1_config(nticks=1500, nwire_half=10)
    d = synth.plane1_depos(n=200, drift=0.8 * synth.m)
    r32 = oracle.run(cfg, d)
    r64 = oracle.run(cfg, d, fp64=True)
    e = rel_l2(r32["frames"][0], r64["frames"][0])
    assert e < 1e-6
    assert r32["windows"] == r64["windows"]


def test_drift_restatement(oracle, synth):
    """Drifter::insert (gen/src/Drifter.cxx:127-196) in closed form."""
    cfg = synth.plane1_config(nticks=1000)
    d = np.array([[0.0, -1000.0, 1100.0, 0.0, 0.0, 0.0, 0.0],
                  [10.0, -1000.0, 50.0, 1.0, 2.0, 0.0, 0.0],     # response region: back-drift
                  [0.0, 0.0, 900.0, 0.0, 0.0, 0.0, 0.0],         # zero charge: dropped
                  [0.0, -5.0, 5000.0, 0.0, 0.0, 0.0, 0.0]])      # outside every region: dropped
    out = oracle.drift(cfg, d)
    dr = cfg["drifter"]
    assert out.shape[0] == 2
    by_index = {int(r[7]): r for r in out}
    dt = 1000.0 / dr["drift_speed"]
    a = by_index[0]
    assert a[0] == dt
    assert abs(a[1] - (-1000.0 * math.exp(-dt / dr["lifetime"]))) < 1e-9
    assert a[2] == 100.0
    assert abs(a[5] - math.sqrt(2 * dr["DL"] * dt)) < 1e-12
    b = by_index[1]
    assert b[0] == 10.0 - 50.0 / dr["drift_speed"] and b[1] == -1000.0 and b[5] == 0.0
