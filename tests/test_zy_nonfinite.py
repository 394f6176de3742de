"""Depos with a NaN or infinite value are dropped before the transform.

The reference has no defined result for them (GaussianDiffusion's bin-index
arithmetic, gen/src/GaussianDiffusion.cxx:116-149, and the event window's
min/max reduction, gen/src/BinnedDiffusion_transform.cxx:416-464, take them
as they come).  Here they are dropped like depos outside the drift volume:
appending them to an event leaves its frame and windows bit for bit
unchanged, on the per-event and on the batched path.

Collected after the other GPU tests (test_zz_*)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bad_rows(template):
    """One row per (column, value) with value NaN, +inf or -inf in that column."""
    rows = []
    for col in range(7):
        for v in (np.nan, np.inf, -np.inf):
            r = template.copy()
            r[col] = v
            rows.append(r)
    return np.array(rows)


def test_non_finite_depos_are_dropped(wct, synth):
    cfg = synth.plane1_config(nticks=2000)
    d = synth.plane1_depos(n=400, drift=0.7 * synth.m)
    dt = wct.from_config(cfg)
    f0, w0, _ = dt(d)
    assert np.abs(f0).max() > 0
    dd = np.concatenate([d, _bad_rows(d[0])])
    f1, w1, _ = dt(dd)
    assert np.array_equal(f0, f1)
    assert w0 == w1
    # only bad depos: an empty frame
    f2, w2, _ = dt(_bad_rows(d[0]))
    assert not f2.any() and w2[0]["ndepos_added"] == 0
    # the batched path takes the same prep
    b0, bw0, _ = dt.forward_batch([d, d[:50]])
    b1, bw1, _ = dt.forward_batch([dd, np.concatenate([_bad_rows(d[1]), d[:50]])])
    assert np.array_equal(b0, b1)
    assert bw0 == bw1
