"""Fluctuated forward: binomial draws from counter-based streams.

The reference draws its fluctuations with std::binomial_distribution
(gen/src/Random.cxx); the device draws them with its own sampler from
Philox streams.  The two can only agree in distribution, so these tests
compare distributions: the device sampler against the exact binomial law and
against std::binomial_distribution samples of the oracle, and fluctuated
frames (patch cells redrawn, GaussianDiffusion.cxx:184-213; absorbed electrons
redrawn, Drifter.cxx:177-185) against the oracle's restatement of the same
algorithm drawing with std::mt19937.  Statistical thresholds are chosen so
that a correct sampler fails with probability below about 1e-4 per check."""

import numpy as np
import pytest

from conftest import rel_l2

CASES = [(20, 0.1), (5000, 0.0004), (5000, 0.0019), (5000, 0.05), (100000, 0.3), (60, 0.85), (1000, 0.9995),
         (7, 1.0), (9, 0.0)]


def _chi2_pvalue(counts, expected):
    from scipy import stats
    m = expected >= 5
    obs = np.append(counts[m], counts[~m].sum())
    exp = np.append(expected[m], expected[~m].sum())
    if exp[-1] < 5:
        obs[-2] += obs[-1]
        exp[-2] += exp[-1]
        obs, exp = obs[:-1], exp[:-1]
    exp = exp * obs.sum() / exp.sum()
    return stats.chisquare(obs, exp).pvalue


@pytest.mark.gpu
@pytest.mark.parametrize("n,p", CASES)
def test_device_binomial_matches_exact_law_and_std_sampler(wct, oracle, n, p):
    import torch
    from scipy import stats
    count = 200_000
    out = torch.zeros(count, dtype=torch.int32, device="cuda")
    wct.binomial_device(1234, 7, n, p, count, out.data_ptr())
    torch.cuda.synchronize()
    x = out.cpu().numpy().astype(np.int64)
    assert x.min() >= 0 and x.max() <= n
    if p in (0.0, 1.0):
        assert np.all(x == int(n * p))
        return
    k = np.arange(n + 1)
    pmf = stats.binom.pmf(k, n, p)
    lo, hi = int(stats.binom.ppf(1e-7, n, p)), int(stats.binom.isf(1e-7, n, p))
    sel = slice(lo, hi + 1)
    counts = np.bincount(x, minlength=n + 1).astype(float)
    cnt = np.concatenate([[counts[:lo].sum()], counts[sel], [counts[hi + 1:].sum()]])
    exp = np.concatenate([[pmf[:lo].sum()], pmf[sel], [pmf[hi + 1:].sum()]]) * count
    assert _chi2_pvalue(cnt, exp) > 1e-4
    # two-sample comparison with the reference's generator
    y = oracle.binomial_samples(n, p, count, seed=99).astype(np.int64)
    cy = np.bincount(y, minlength=n + 1).astype(float)
    cy = np.concatenate([[cy[:lo].sum()], cy[sel], [cy[hi + 1:].sum()]])
    both = (cnt + cy) > 10
    table = np.vstack([cnt[both], cy[both]])
    assert stats.chi2_contingency(table)[1] > 1e-4
    assert abs(x.mean() - n * p) < 5 * np.sqrt(n * p * (1 - p) / count)


def _fluc_case(synth, nticks=1200, n=6, seed=3):
    cfg = synth.plane1_config(nticks=nticks)
    rng = np.random.default_rng(seed)
    d = np.zeros((n, 7))
    d[:, 0] = rng.uniform(0, 50e3, n)
    d[:, 1] = -4000.0
    d[:, 2] = rng.uniform(300.0, 600.0, n)
    d[:, 4] = rng.uniform(-50.0, 50.0, n)
    return cfg, d


@pytest.mark.gpu
def test_fluctuated_frames_reproducible_and_fresh(wct, synth):
    cfg, d = _fluc_case(synth)
    cfg = dict(cfg, fluctuate=True, seed=42, first_frame_number=10)
    a = wct.from_config(cfg)
    b = wct.from_config(cfg)
    fa1, _, ia1 = a(d)
    fa2, _, ia2 = a(d)
    fb1, _, _ = b(d)
    assert (ia1, ia2) == (10, 11)
    assert np.array_equal(fa1, fb1)          # same seed and frame ident: the same draws
    assert not np.array_equal(fa1, fa2)      # the next frame draws afresh
    c = wct.from_config(dict(cfg, seed=43))
    fc, _, _ = c(d)
    assert not np.array_equal(fa1, fc)


@pytest.mark.gpu
def test_fluctuated_frame_statistics_match_reference_algorithm(wct, oracle, synth):
    """Mean and per-cell variance of fluctuated frames: device vs the oracle's
    std::binomial_distribution restatement of GaussianDiffusion's fluctuation."""
    cfg, d = _fluc_case(synth)
    det = wct.from_config(cfg)
    f0, _, _ = det(d)
    dt = wct.from_config(dict(cfg, fluctuate=True, seed=5))
    S = 160
    g = np.stack([dt(d)[0].astype(np.float64) for _ in range(S)])
    o = np.stack([oracle.run(cfg, d, fluctuate=True, seed=1000 + k)["frames"][0].astype(np.float64)
                  for k in range(S)])
    nw = cfg["planes"][0]["nwires"]
    f0 = f0[:nw].astype(np.float64)
    g = g[:, :nw]
    # means converge to the unfluctuated frame at the same rate for both
    eg = rel_l2(g.mean(axis=0), f0)
    eo = rel_l2(o.mean(axis=0), f0)
    assert eg < 0.05 and eo < 0.05
    assert 0.6 < eg / eo < 1.6, (eg, eo)
    # total per-cell variance: same law
    vg = g.var(axis=0, ddof=1).sum()
    vo = o.var(axis=0, ddof=1).sum()
    assert vg > 0 and abs(vg / vo - 1.0) < 0.25, (vg, vo)


@pytest.mark.gpu
def test_drift_fluctuation_is_binomial(wct, synth):
    """One depo, drift fluctuation only: the surviving charge Qf = Q - N with
    N ~ Binomial(|Q|, 1 - exp(-dt / lifetime)), read off the frame total."""
    from scipy import stats
    cfg, d = _fluc_case(synth, n=1)
    d[0, 0] = 0.0
    d[0, 2] = 700.0  # 375 us of drift: inside the 600 us readout
    d[0, 4] = 0.0
    det = wct.from_config(cfg)
    f0, _, _ = det(d)
    dr = dict(cfg["drifter"], fluctuate=True)
    fl = wct.from_config(dict(cfg, drifter=dr, seed=11))
    Q = -d[0, 1]
    dtm = abs(d[0, 2] - cfg["drifter"]["xregions"][0][1]) / cfg["drifter"]["drift_speed"]
    pabs = 1.0 - np.exp(-dtm / cfg["drifter"]["lifetime"])
    qdet = Q * (1.0 - pabs)
    s0 = float(f0.astype(np.float64).sum())
    S = 600
    qf = np.array([float(fl(d)[0].astype(np.float64).sum()) / s0 * qdet for _ in range(S)])
    nabs = Q - qf
    assert np.max(np.abs(nabs - np.round(nabs))) < 0.05  # whole electrons
    nabs = np.round(nabs)
    m, v = Q * pabs, Q * pabs * (1 - pabs)
    assert abs(nabs.mean() - m) < 5 * np.sqrt(v / S)
    assert 0.7 < nabs.var(ddof=1) / v < 1.35
    # binned against the exact law
    k = np.arange(int(Q) + 1)
    lo, hi = int(stats.binom.ppf(1e-4, int(Q), pabs)), int(stats.binom.isf(1e-4, int(Q), pabs))
    edges = np.linspace(lo, hi + 1, 9).astype(int)
    cnt = np.histogram(nabs, bins=edges)[0].astype(float)
    exp = np.array([stats.binom.pmf(k[a:b], int(Q), pabs).sum() for a, b in zip(edges[:-1], edges[1:])]) * S
    assert stats.chisquare(cnt, exp * cnt.sum() / exp.sum()).pvalue > 1e-4


@pytest.mark.gpu
def test_batch_fluctuation_matches_per_event(wct, synth):
    """The batched path draws from the same streams as per-event calls (frame
    idents first_frame_number + e), so its fluctuated frames match."""
    cfg = synth.plane1_config(nticks=2000)
    evs = [synth.plane1_depos(n=k, seed=50 + k, drift=0.6 * synth.m) for k in (200, 50, 400)]
    cfg = dict(cfg, fluctuate=True, seed=77, first_frame_number=3)
    a = wct.from_config(cfg)
    per = [a(e)[0] for e in evs]
    b = wct.from_config(cfg)
    frames, _, ident = b.forward_batch(evs)
    assert ident == 3
    for k, f in enumerate(per):
        assert rel_l2(frames[k], f) < 2e-6, k
