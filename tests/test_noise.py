"""Noise (gen/src/AddNoise.cxx IncoherentAddNoise / CoherentAddNoise with the
GeneratorN waveform of aux/src/NoiseTools.cxx).  The reference draws its
normals with std::mt19937 (recycled), so the comparison is of
distributions: every bin's mean power E|X_k|^2 = 2 sigma_k^2 with sigma_k =
S_k sqrt(2/3.141592), which the oracle's restatement (numpy normals) shows
too; plus coherent groups, reproducibility and untouched rows."""

import numpy as np
import pytest

N = 6000


def _spectrum():
    k = np.arange(N)
    f = np.minimum(k, N - k).astype(np.float64)
    return (1.0 + 4.0 * np.exp(-((f - 400.0) / 250.0) ** 2)).astype(np.float32)


def _expected_power(S):
    return 2.0 * (S.astype(np.float64) * np.sqrt(2.0 / 3.141592)) ** 2


def test_oracle_power_spectrum(oracle):
    rng = np.random.default_rng(0)
    S = _spectrum()
    rows = 400
    P = np.zeros(N)
    for _ in range(rows):
        w = oracle.noise_wave(S, rng.standard_normal(2 * (N // 2 + 1) + 1))
        assert w.dtype == np.float64 and w.size == N
        P += np.abs(np.fft.fft(w)) ** 2
    ratio = (P / rows)[: N // 2 + 1] / _expected_power(S)[: N // 2 + 1]
    assert abs(ratio.mean() - 1.0) < 0.02


@pytest.mark.gpu
def test_incoherent_power_spectrum(wct):
    S = _spectrum()
    rows = 2000
    frame = np.zeros((rows, N), np.float32)
    wct.add_noise(frame, S[None, :], np.zeros(rows, np.int32), np.arange(rows, dtype=np.int32), seed=7, ident=3)
    P = (np.abs(np.fft.fft(frame.astype(np.float64), axis=1)) ** 2).mean(axis=0)
    ratio = P[: N // 2 + 1] / _expected_power(S)[: N // 2 + 1]
    assert abs(ratio.mean() - 1.0) < 0.01                               # 3001 bins x 2000 rows
    assert np.abs(ratio[1: N // 2] - 1.0).max() < 6.0 / np.sqrt(rows)  # each bin: exponential power, 2000 draws
    var = frame.astype(np.float64).var()                                 # sum of the bin powers / N^2
    assert abs(var / (_expected_power(S).sum() / N**2) - 1.0) < 0.01


@pytest.mark.gpu
def test_coherent_groups_reproducible_and_untouched(wct):
    S = np.stack([_spectrum(), 0.5 * _spectrum()])
    rows = 12
    base = np.random.default_rng(1).standard_normal((rows, 5000)).astype(np.float32)
    row_spec = np.array([0, 0, 0, 1, 1, 1, -1, 0, 0, 1, 1, -1], np.int32)
    groups = np.array([5, 5, 5, 9, 9, 9, 0, 6, 6, 9, 9, 0], np.int32)
    a = wct.add_noise(base.copy(), S, row_spec, groups, seed=11, ident=2)
    b = wct.add_noise(base.copy(), S, row_spec, groups, seed=11, ident=2)
    c = wct.add_noise(base.copy(), S, row_spec, groups, seed=11, ident=3)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    assert np.array_equal(a[6], base[6]) and np.array_equal(a[11], base[11])  # no spectrum: untouched
    n = a - base
    assert np.allclose(n[0], n[1], atol=1e-6) and np.allclose(n[1], n[2], atol=1e-6)  # coherent group 5
    assert np.allclose(n[7], n[8], atol=1e-6) and not np.allclose(n[0], n[7])
    assert np.allclose(n[3], n[9], atol=1e-6)  # same group and spectrum: same waveform
    assert np.all(np.isfinite(a))
