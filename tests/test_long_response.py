"""Long-range response (PlaneImpactResponse long_responses / long_padding,
gen/src/PlaneImpactResponse.cxx:46-47,121-150; ImpactTransform::waveform,
gen/src/ImpactTransform.cxx:327-343).

Every frame row inside the plane's window is circularly convolved with the
long waveform at fft_best_length(nticks + long_padding / tick) and cut back
to nticks.  Checked against the oracle (which follows the reference's
spectra products) at the default padding, whose length 9317 = 7 * 11^3 goes
through Bluestein's transform, and at a 7-smooth length; the adjoint with a
long response equals the adjoint without one applied to the frame gradient
correlated with the long waveform."""

import numpy as np
import pytest

from conftest import rel_l2


def _long_kernel(n=3000, tau=400.0, a=0.004):
    """A unit impulse followed by a small exponential undershoot (an RC-like tail)."""
    k = -a * np.exp(-np.arange(n) / tau)
    k[0] = 1.0
    return k


def test_oracle_long_step_is_circular_convolution(synth, oracle):
    cfg = synth.plane1_config(nticks=1000)
    d = synth.plane1_depos(n=200, seed=3, drift=0.5e3)
    k = _long_kernel(600, 150.0, 0.002)
    f0 = oracle.run(cfg, d, fp64=True)["frames"][0]
    o1 = oracle.run(dict(cfg, long_responses=[k], long_padding=100e3), d, fp64=True)
    f1, w = o1["frames"][0], o1["windows"][0]
    nl = oracle.fft_best_length(1000 + int(100e3 / cfg["tick"]))
    kk = np.zeros(nl)
    kk[:600] = k
    for row in range(cfg["planes"][0]["nwires"]):
        if w["start_ch"] <= row < w["end_ch"]:
            x = np.zeros(nl)
            x[:1000] = f0[row]
            y = np.real(np.fft.ifft(np.fft.fft(x) * np.fft.fft(kk)))[:1000]
            assert np.allclose(f1[row], y, rtol=0, atol=1e-12 * max(1.0, np.abs(y).max()))
        else:
            assert np.all(f1[row] == 0)


@pytest.mark.gpu
@pytest.mark.parametrize("padding", [1.5e6, 100e3])  # 9317 (Bluestein) and a 7-smooth length
def test_long_response_matches_oracle(wct, synth, oracle, padding):
    cfg = dict(synth.plane1_config(nticks=6000), long_responses=[_long_kernel()], long_padding=padding)
    d = synth.plane1_depos(n=2000, seed=5)
    f, wins, _ = wct.from_config(cfg)(d)
    o = oracle.run(cfg, d, fp64=True, nthreads=4)["frames"][0]
    assert rel_l2(f, o) < 1e-5
    o0 = oracle.run(dict(cfg, long_responses=[]), d, fp64=True, nthreads=4)["frames"][0]
    assert rel_l2(o, o0) > 1e-3  # the step is not trivial here
    pir = wct.PlaneImpactResponse(cfg["fr"][0], cfg["short_responses"], cfg["overall_short_padding"], cfg["tick"],
                                  cfg["pir_nticks"], cfg["long_responses"], padding)
    lw, pad = pir.long_waveform()
    assert pad == int(padding / cfg["tick"]) and lw.size == oracle.fft_best_length(6000)
    assert np.allclose(lw[:3000], cfg["long_responses"][0], atol=1e-6)


@pytest.mark.gpu
def test_long_response_batched_matches_single(wct, synth):
    cfg = dict(synth.plane1_config(nticks=6000), long_responses=[_long_kernel()], long_padding=1.5e6)
    dt = wct.from_config(cfg)
    evs = [synth.plane1_depos(n=n, seed=s) for n, s in ((1500, 7), (300, 8), (2000, 9))]
    batch, _, _ = dt.forward_batch(evs)
    for e, d in enumerate(evs):
        f, _, _ = dt(d)
        assert rel_l2(batch[e], f) < 1e-6


@pytest.mark.gpu
def test_long_response_adjoint(wct, synth, oracle):
    cfg = synth.plane1_config(nticks=6000)
    k = _long_kernel()
    pad = 1.5e6
    d = synth.plane1_depos(n=800, seed=11)
    dl = wct.from_config(dict(cfg, long_responses=[k], long_padding=pad))
    d0 = wct.from_config(cfg)
    rng = np.random.default_rng(2)
    nrows, nticks = dl.frame_shape()
    g = rng.standard_normal((nrows, nticks)).astype(np.float32)
    gl, ggl = dl.adjoint(d, g)
    # the long step's transpose on the gradient rows, in float64
    nl = oracle.fft_best_length(nticks + int(pad / cfg["tick"]))
    kk = np.zeros(nl)
    kk[:len(k)] = k
    K = np.fft.fft(kk)
    gp = np.zeros((nrows, nl))
    gp[:, :nticks] = g
    gt = np.real(np.fft.ifft(np.fft.fft(gp, axis=1) * np.conj(K)[None, :], axis=1))[:, :nticks]
    g0, gg0 = d0.adjoint(d, gt.astype(np.float32))
    assert rel_l2(gl, g0) < 1e-4
    assert rel_l2(ggl, gg0) < 1e-4
