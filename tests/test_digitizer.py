"""Digitizer (gen/src/Digitizer.cxx:82-141) on the GPU, bit for bit against
the oracle's float64 restatement, which is itself checked against a scalar
loop that follows Digitizer::digitize line by line."""

import math

import numpy as np
import pytest

VOLT = 1.0e-6


def _scalar_digitize(value, baseline, gain, fs, resolution, rnd):
    """Digitizer::operator() and digitize (gen/src/Digitizer.cxx:82-97,126-131), one sample."""
    adcmaxval = (1 << resolution) - 1
    voltage = gain * float(np.float32(value)) + float(np.float32(baseline))
    if voltage <= fs[0]:
        return 0.0
    if voltage >= fs[1]:
        return float(adcmaxval)
    relvoltage = (voltage - fs[0]) / (fs[1] - fs[0])
    fp_adc = relvoltage * adcmaxval
    if rnd:  # C round, half away from zero (fp_adc > 0 here)
        r = math.floor(fp_adc)
        return float(r + 1 if fp_adc - r >= 0.5 else r)
    return float(math.floor(fp_adc))


def _frame(rng, nrows=40, ncols=300):
    f = rng.normal(0.0, 0.4 * VOLT, (nrows, ncols)).astype(np.float32)
    f[0, :5] = [-5 * VOLT, 5 * VOLT, 0.0, 1.1 * VOLT, -0.9 * VOLT]  # clipped both ways, baseline, edges
    return f


@pytest.mark.parametrize("rnd", [False, True])
def test_oracle_matches_scalar_loop(oracle, rnd):
    rng = np.random.default_rng(1)
    f = _frame(rng, 6, 50)
    base = np.array([0.9, 0.9, 0.9, 0.2, 0.2, 0.2]) * VOLT
    o = oracle.digitize(f, base, 1.3, (0.0, 2.0 * VOLT), 12, rnd)
    for r in range(f.shape[0]):
        for c in range(f.shape[1]):
            assert o[r, c] == _scalar_digitize(f[r, c], base[r], 1.3, (0.0, 2.0 * VOLT), 12, rnd)


@pytest.mark.gpu
@pytest.mark.parametrize("rnd", [False, True])
@pytest.mark.parametrize("gain,resolution", [(1.0, 12), (2.5, 14), (0.7, 10)])
def test_digitizer_bit_exact(wct, oracle, rnd, gain, resolution):
    rng = np.random.default_rng(resolution + int(10 * gain))
    f = _frame(rng)
    dz = wct.Digitizer([15, 15, 10], resolution=resolution, gain=gain, round=rnd)
    got = dz(f)
    ref = oracle.digitize(f, dz.row_baseline, gain, dz.fullscale, resolution, rnd)
    assert np.array_equal(got, ref)


@pytest.mark.gpu
def test_digitizer_on_depo_transform_frame(wct, synth, oracle):
    """The simulated frame of a full-APA event, digitized with the reference's defaults."""
    cfg = synth.apa_config(nticks=6000)
    d = synth.apa_depos(seed=4)[:100000]
    dt = wct.from_config(cfg)
    f, _, _ = dt(d)
    dz = wct.Digitizer([p["nwires"] for p in cfg["planes"]], round=True)
    got = dz(f)
    assert np.array_equal(got, oracle.digitize(f, dz.row_baseline, 1.0, dz.fullscale, 12, True))
    assert got.min() >= 0 and got.max() <= 4095 and np.unique(got).size > 10
    # device entry point, in place
    import torch
    t = torch.from_numpy(f.copy()).cuda()
    b = torch.from_numpy(dz.row_baseline).cuda()
    dz.device(t.data_ptr(), f.shape[1], f.shape[0], f.shape[1], b.data_ptr(), t.data_ptr(), f.shape[1])
    torch.cuda.synchronize()
    assert np.array_equal(t.cpu().numpy(), got)
