"""Two-face anodes and the modify_depo charge hook.

DepoTransform::operator() loops over IAnodePlane::faces() (each face keeps
the depos inside its sensitive box and frames them on its own planes with
the plane index's PIR) and calls the per-plane modify_depo before
BinnedDiffusion_transform::add (gen/src/DepoTransform.cxx:169-213,
gen/inc/WireCellGen/DepoTransform.h:33-35).  Checked against the oracle's
restatement of both: a two-face APA whose induction wires wrap (channels
shared by the faces), and per-(depo, plane) charge scales on the forward,
the batched forward, the fluctuated forward and the adjoint."""

import numpy as np
import pytest

from conftest import parity_log, rel_l2

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-5


def _face_plane_of(cfg, wct):
    out = []
    for f, (_, idx) in enumerate(wct.faces_of(cfg)):
        for j, k in enumerate(idx):
            out.append((f, j, k))
    return out


def test_two_face_apa(wct, oracle, synth):
    cfg = synth.apa2_config()
    d = synth.apa2_depos()
    dt = wct.from_config(cfg)
    frame, wins, _ = dt(d)
    o = oracle.run(cfg, d, fp64=True, nthreads=6, records=True)
    ref = np.concatenate(o["frames"], axis=0)
    for w, ow in zip(wins, o["windows"]):
        assert (w["start_ch"], w["end_ch"], w["start_tick"], w["end_tick"]) == \
            (ow["start_ch"], ow["end_ch"], ow["start_tick"], ow["end_tick"])
        for k in ("ndepos_added", "outside_time", "outside_pitch"):
            assert w[k] == ow[k]
    assert [(w["face"], w["plane"]) for w in wins] == [(f, j) for f, j, _ in _face_plane_of(cfg, wct)]
    for f, j, k in _face_plane_of(cfg, wct):
        g = dt.patch_records(f, j, len(d))
        r = o["records"][k]
        onz = (r[:, 3] > 0) & (r[:, 4] > 0)
        gnz = (g[:, 2] > 0) & (g[:, 3] > 0)
        assert np.array_equal(onz, gnz)
        assert np.array_equal(g[gnz], r[onz][:, 1:5])
    # both faces see depos
    rows = np.cumsum([0] + [p["nwires"] for p in cfg["planes"]])
    assert np.abs(frame[rows[0]:rows[3]]).max() > 0 and np.abs(frame[rows[3]:rows[6]]).max() > 0
    e = rel_l2(frame, ref)
    print("two-face APA rel-L2 vs FP64:", e)
    parity_log({"config": "two-face APA (wrapped induction channels)", "depos": int(len(d)), "rel_l2_fp64": e})
    assert e < TOL_FP64, e
    # traces: a wrapped channel has one trace from each face, as the reference's frame
    ch, tb, chg = zip(*dt.traces(frame))
    channels = np.concatenate([p["channels"] for p in cfg["planes"]])
    nz = np.nonzero(np.abs(frame).max(axis=1) > 0)[0]
    assert list(ch) == list(channels[nz])
    shared = set(channels[rows[0]:rows[2]]) & set(channels[rows[3]:rows[5]])
    assert len(shared) == 1600
    assert any(list(ch).count(c) == 2 for c in shared)


def _scale(rng, n, nplanes):
    s = rng.uniform(0.5, 1.5, (n, nplanes))
    s[rng.random((n, nplanes)) < 0.05] = 0.0  # a depo that brings nothing to a plane
    return s


def test_charge_scale_forward(wct, oracle, synth):
    cfg = synth.apa_config()
    rng = np.random.default_rng(3)
    d = synth.track_depos(rng, ntracks=3, step=0.5)
    s = _scale(rng, len(d), 3)
    dt = wct.from_config(cfg)
    f0, _, _ = dt(d)
    dt.set_charge_scale(s)
    f1, w1, _ = dt(d)
    o = oracle.run(cfg, d, fp64=True, nthreads=3, records=True, charge_scale=s)
    for w, ow in zip(w1, o["windows"]):
        assert (w["start_ch"], w["end_ch"], w["start_tick"], w["end_tick"]) == \
            (ow["start_ch"], ow["end_ch"], ow["start_tick"], ow["end_tick"])
    e = rel_l2(f1, np.concatenate(o["frames"], axis=0))
    print("charge-scaled forward rel-L2 vs FP64:", e)
    assert e < TOL_FP64, e
    assert rel_l2(f1, f0) > 1e-2  # the scale took effect
    # a call with another depo count is refused while the scale is set
    with pytest.raises(wct.WctError):
        dt(d[:-1])
    dt.set_charge_scale(None)
    f2, _, _ = dt(d)
    assert np.array_equal(f2, f0)


def test_charge_scale_ones_and_zero_plane(wct, synth):
    """Scale 1 is the unmodified forward bit for bit (fluctuation on too: the
    same draws); scale 0 on a plane empties that plane."""
    cfg = dict(synth.apa_config(nticks=3000), fluctuate=True, seed=4)
    rng = np.random.default_rng(5)
    d = synth.track_depos(rng, ntracks=2, step=1.0, hi=(synth.RESPONSE_X + 1500.0, 3000.0, 1150.0))
    a = wct.from_config(cfg)
    b = wct.from_config(cfg)
    fa, _, _ = a(d)
    b.set_charge_scale(np.ones((len(d), 3)))
    fb, _, _ = b(d)
    assert np.array_equal(fa, fb)
    s = np.ones((len(d), 3))
    s[:, 1] = 0.0
    b.set_charge_scale(s)
    fc, _, _ = b(d)
    rows = np.cumsum([0] + [p["nwires"] for p in cfg["planes"]])
    assert not fc[rows[1]:rows[2]].any()
    assert fc[rows[0]:rows[1]].any() and fc[rows[2]:rows[3]].any()


def test_charge_scale_batched(wct, synth):
    cfg = synth.apa_config(nticks=3000)
    rng = np.random.default_rng(8)
    evs = [synth.track_depos(rng, ntracks=2, step=1.0, hi=(synth.RESPONSE_X + 1500.0, 3000.0, 1150.0))
           for _ in range(3)]
    scales = [_scale(rng, len(e), 3) for e in evs]
    dt = wct.from_config(cfg)
    dt.set_charge_scale(np.concatenate(scales))
    frames, _, _ = dt.forward_batch(evs)
    ref = wct.from_config(cfg)
    for k, (e, s) in enumerate(zip(evs, scales)):
        ref.set_charge_scale(s)
        f, _, _ = ref(e)
        assert rel_l2(frames[k], f) < 2e-6, k


def test_charge_scale_adjoint(wct, synth):
    """Per-plane constant scales s_p: with the frame gradient on plane 1's rows
    only, every depo gradient is s_1 times the unscaled one."""
    cfg = synth.apa_config(nticks=3000)
    rng = np.random.default_rng(9)
    d = synth.track_depos(rng, ntracks=2, step=2.0, hi=(synth.RESPONSE_X + 1500.0, 3000.0, 1150.0))
    dt = wct.from_config(cfg)
    nrows, nticks = dt.frame_shape()
    rows = np.cumsum([0] + [p["nwires"] for p in cfg["planes"]])
    g = np.zeros((nrows, nticks), np.float32)
    g[rows[1]:rows[2]] = rng.standard_normal((rows[2] - rows[1], nticks)).astype(np.float32)
    g0, gg0 = dt.adjoint(d, g)
    dt.set_charge_scale(np.tile([0.7, 1.3, 0.4], (len(d), 1)))
    g1, gg1 = dt.adjoint(d, g)
    assert rel_l2(g1, 1.3 * g0) < 1e-6
    assert rel_l2(gg1, 1.3 * gg0) < 1e-6
