"""Batched forward: many events of uneven size in one CUDA graph.

The batched path plans every event's windows on the device and runs the time
FFTs at lengths from a fixed ladder, so its frames equal the per-event
forward's within floating-point rounding (tolerance below), and its windows
equal the per-event windows except for the device FFT length."""

import ctypes as C

import numpy as np
import pytest

from conftest import rel_l2

TOL_VS_EVENT = 2e-6   # batched vs per-event forward (both FP32, FFT lengths differ)
TOL_VS_FP64 = 1e-5    # batched vs the FP64 oracle


def _events_plane1(synth, seed=21):
    rng = np.random.default_rng(seed)
    sizes = [300, 0, 1200, 40, 5000, 700]
    evs = []
    for k, n in enumerate(sizes):
        evs.append(synth.plane1_depos(n=n, seed=seed + k, drift=rng.uniform(0.2, 0.9) * synth.m) if n else
                   np.zeros((0, 7)))
    return evs


def test_batch_argument_checks(wct):
    L = wct.lib()
    off = (C.c_longlong * 2)(0, 1)
    assert L.wct_dt_forward_batch_device(None, None, off, 1, None, None, None, None) == wct.WCT_ERR_ARG
    assert L.wct_dt_batch_tune(None, None, 0) == wct.WCT_ERR_ARG


def _per_event(dt, evs):
    out = []
    for e in evs:
        f, w, _ = dt(e)
        out.append((f, w))
    return out


def _same_windows(wb, we):
    for a, b in zip(wb, we):
        a = dict(a)
        b = dict(b)
        a.pop("nt_gpu")
        b.pop("nt_gpu")
        assert a == b


@pytest.mark.gpu
def test_batch_matches_per_event_plane1(wct, synth):
    cfg = synth.plane1_config(nticks=2000)
    evs = _events_plane1(synth)
    dt = wct.from_config(cfg)
    ref = _per_event(dt, evs)
    frames, wins, _ = dt.forward_batch(evs)
    for k, (f, w) in enumerate(ref):
        if np.abs(f).max() == 0:
            assert np.abs(frames[k]).max() == 0, k
        else:
            assert rel_l2(frames[k], f) < TOL_VS_EVENT, (k, rel_l2(frames[k], f))
        _same_windows(wins[k], w)
        assert wins[k][0]["nt_gpu"] >= w[0]["nt_fft"]


@pytest.mark.gpu
def test_batch_passes_and_graph_replay(wct, synth):
    """Fewer event slots than events (several passes in one graph), replayed
    graphs give the same frames, and a change of drift parameters re-captures."""
    import torch
    cfg = synth.plane1_config(nticks=2000)
    evs = _events_plane1(synth, seed=33)
    dt = wct.from_config(cfg)
    ref = _per_event(dt, evs)
    off = np.zeros(len(evs) + 1, dtype=np.int64)
    off[1:] = np.cumsum([len(e) for e in evs])
    nrows, nticks = dt.frame_shape()
    dd = torch.from_numpy(np.concatenate(evs)).cuda()
    fr = torch.zeros((len(evs), nrows, nticks), dtype=torch.float32, device="cuda")
    s = torch.cuda.Stream()
    dt.batch_tune(slots=2)
    dt.forward_batch_device(dd.data_ptr(), off, fr.data_ptr(), stream=s.cuda_stream)
    a = fr.cpu().numpy().copy()
    fr.fill_(3.0)
    dt.forward_batch_device(dd.data_ptr(), off, fr.data_ptr(), stream=s.cuda_stream)
    b = fr.cpu().numpy()
    assert np.array_equal(a, b)
    for k, (f, _) in enumerate(ref):
        if np.abs(f).max():
            assert rel_l2(a[k], f) < TOL_VS_EVENT
    dl, dtr, lt = dt.drift_params()
    dt.set_drift_params(dl * 0.5, dtr * 2.0, lt)
    ref2 = _per_event(dt, evs)
    dt.forward_batch_device(dd.data_ptr(), off, fr.data_ptr(), stream=s.cuda_stream)
    c = fr.cpu().numpy()
    for k, (f, _) in enumerate(ref2):
        if np.abs(f).max():
            assert rel_l2(c[k], f) < TOL_VS_EVENT
    # torch's default stream (handle 0) is bridged to a capturable stream
    fr.fill_(0.0)
    dt.set_drift_params(dl, dtr, lt)
    dt.forward_batch_device(dd.data_ptr(), off, fr.data_ptr(), stream=0)
    torch.cuda.synchronize()
    assert np.array_equal(fr.cpu().numpy(), a)


@pytest.mark.gpu
def test_batch_apa_uneven_vs_fp64(wct, synth, oracle):
    """Full-APA geometry, uneven track + shower events (small sizes so the FP64
    oracle stays quick)."""
    cfg = synth.apa_config(nticks=3000)
    evs = synth.batch_events(nevents=5, seed=8, lo=2000, hi=30000)
    dt = wct.from_config(cfg)
    frames, wins, _ = dt.forward_batch(evs)
    rows = np.cumsum([0] + [p["nwires"] for p in cfg["planes"]])
    for k in (0, 3):
        o = oracle.run(cfg, evs[k], fp64=True, nthreads=4)
        for ip, f64 in enumerate(o["frames"]):
            err = rel_l2(frames[k][rows[ip]:rows[ip + 1]], f64)
            assert err < TOL_VS_FP64, (k, ip, err)
    ref = _per_event(dt, evs)
    for k, (f, w) in enumerate(ref):
        assert rel_l2(frames[k], f) < TOL_VS_EVENT
        _same_windows(wins[k], w)


@pytest.mark.gpu
def test_autotune_batch(wct, synth):
    import torch
    cfg = synth.plane1_config(nticks=2000)
    evs = _events_plane1(synth, seed=44)
    dt = wct.from_config(cfg)
    off = np.zeros(len(evs) + 1, dtype=np.int64)
    off[1:] = np.cumsum([len(e) for e in evs])
    nrows, nticks = dt.frame_shape()
    dd = torch.from_numpy(np.concatenate(evs)).cuda()
    fr = torch.zeros((len(evs), nrows, nticks), dtype=torch.float32, device="cuda")
    rep = dt.autotune_batch(dd.data_ptr(), off, fr.data_ptr())
    assert rep["best"]["ms"] > 0 and len(rep["tried"]) > 5
    best = {k: rep["best"][k] for k in dt.BATCH_TUNE_KEYS}
    assert dt.batch_tune() == best
    ref = _per_event(dt, evs)
    dt.forward_batch_device(dd.data_ptr(), off, fr.data_ptr())
    got = fr.cpu().numpy()
    for k, (f, _) in enumerate(ref):
        if np.abs(f).max():
            assert rel_l2(got[k], f) < TOL_VS_EVENT
