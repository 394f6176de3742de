"""DepoFluxSplat truth frame (gen/src/DepoFluxSplat.cxx:247-390) on the GPU
against the oracle's restatement: erf-integrated Gaussian patches on the
plane's wire bins and the window's ticks, |charge| added; per-plane smearing
and time offsets; depos outside the window in time skip a plane, depos
outside the wire plane in pitch skip the remaining planes."""

import numpy as np
import pytest

from conftest import rel_l2


def _depos(synth, n=30000, seed=3):
    """Track depos moved to the response plane with drift-like extents."""
    d = synth.apa_depos(seed=seed)[:n].copy()
    rng = np.random.default_rng(seed)
    drift = rng.uniform(0.0, 2500.0, len(d))
    d[:, 0] = drift / 1.6e-3
    d[:, 2] = 100.0
    d[:, 5] = np.sqrt(2 * 7.2e-7 * d[:, 0])
    d[:, 6] = np.sqrt(2 * 1.2e-6 * d[:, 0])
    d[::97, 5] = 0.0          # some point-like in time
    d[::89, 6] = 0.0          # and in pitch
    return d


CFG = dict(tick=500.0, window_start=0.0, window_duration=6000 * 500.0, nsigma=3.0, drift_speed=1.6e-3,
           response_plane=100.0)


def test_oracle_splat_conserves_charge(synth, oracle):
    cfg = synth.apa_config(nticks=6000)
    d = _depos(synth, 5000)
    f = oracle.splat(cfg, d, CFG)
    assert f.min() >= 0
    # every depo lies inside the window and (almost all) over the wire planes:
    # each plane gets its full charge
    np.testing.assert_allclose(f.sum(), 3 * np.abs(d[:, 1]).sum(), rtol=0.02)


@pytest.mark.gpu
@pytest.mark.parametrize("extra", [{}, dict(smear_long=[1.0, 2.0, 0.5], smear_tran=[0.3, 0.0, 1.0],
                                            time_offsets=[-1500.0, 0.0, 2250.0])])
def test_splat_matches_oracle(wct, synth, oracle, extra):
    cfg = synth.apa_config(nticks=6000)
    d = _depos(synth)
    sc = dict(CFG, **extra)
    dt = wct.from_config(cfg)
    f = dt.splat(d, **sc)
    o = oracle.splat(cfg, d, sc)
    assert f.shape == o.shape
    assert rel_l2(f, o) < 1e-6
    assert np.abs(f - o).max() <= 1e-5 * np.abs(o).max()


@pytest.mark.gpu
def test_splat_window_edges(wct, synth, oracle):
    """A short window that cuts patches and drops depos (time misses skip a
    plane; pitch misses skip the remaining planes)."""
    cfg = synth.apa_config(nticks=6000)
    d = _depos(synth, 8000, seed=5)
    d[:50, 4] = 5000.0  # far outside the wire planes in z
    sc = dict(CFG, window_start=1.0e6, window_duration=700 * 500.0)
    f = wct.from_config(cfg).splat(d, **sc)
    o = oracle.splat(cfg, d, sc)
    assert rel_l2(f, o) < 1e-6
    assert wct.from_config(cfg).splat(d[:0], **sc).sum() == 0
