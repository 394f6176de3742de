"""Parity at the benchmarked sizes: every workload the bench times, forward
frames against the FP64 oracle (rel-L2 <= 1e-5) with windows, depo counters
and per-depo patch placements bit-exact where the oracle records them.

  config 1  one collection plane, 960 wires, 6000 ticks, 2000 point depos
  config 2  the bench's full-APA event: 3 planes, 6000 ticks, 20 muon tracks
            at 0.1 mm steps (519 435 depos), also against the FP32 restatement
  config 3  the bench's 64-event batch (10k-500k depos, tracks + showers)
            through one batched call: every event against its per-event frame,
            the smallest, the largest and the one with the widest patches
            against the FP64 oracle
  config 4  the adjoint workload's forward: full APA, 20 000 track depos
  config 5  one 4M-depo calibration event (cosmic muons + showers), forward
            with fluctuation off

Each rel-L2 is printed and, with WCT_PARITY_LOG set, logged (conftest)."""

import os

import numpy as np
import pytest

from conftest import parity_log, rel_l2

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-5
TOL_FP32 = 1e-5
TOL_BATCH_VS_EVENT = 2e-6
NTH = min(3, os.cpu_count() or 1)  # oracle threads: one per plane


def _windows_match(wins, owins):
    for w, o in zip(wins, owins):
        assert (w["start_ch"], w["end_ch"], w["start_tick"], w["end_tick"]) == \
            (o["start_ch"], o["end_ch"], o["start_tick"], o["end_tick"])
        assert (w["nw_fft"], w["nt_fft"]) == (o["nw"], o["nt"])
        for k in ("ndepos_added", "outside_time", "outside_pitch"):
            assert w[k] == o[k], k


def _records_match(dt, cfg, rec, n):
    for ip in range(len(cfg["planes"])):
        g = dt.patch_records(0, ip, n)
        o = rec[ip]  # added, toffset, poffset, nt, np
        onz = (o[:, 3] > 0) & (o[:, 4] > 0)
        gnz = (g[:, 2] > 0) & (g[:, 3] > 0)
        assert np.array_equal(onz, gnz)
        assert np.array_equal(g[gnz], o[onz][:, 1:5])


def _forward_vs_fp64(wct, oracle, cfg, depos, label, records=True, fp32=False):
    dt = wct.from_config(cfg)
    frame, wins, _ = dt(depos)
    o64 = oracle.run(cfg, depos, fp64=True, nthreads=NTH, records=records)
    _windows_match(wins, o64["windows"])
    if records:
        _records_match(dt, cfg, o64["records"], len(depos))
    e64 = rel_l2(frame, np.concatenate(o64["frames"], axis=0))
    entry = {"config": label, "depos": int(len(depos)), "rel_l2_fp64": e64}
    if fp32:
        o32 = oracle.run(cfg, depos, fp64=False, nthreads=NTH)
        entry["rel_l2_fp32_restatement"] = rel_l2(frame, np.concatenate(o32["frames"], axis=0))
        assert entry["rel_l2_fp32_restatement"] < TOL_FP32, entry
    print(entry)
    parity_log(entry)
    assert e64 < TOL_FP64, entry
    return entry


def test_config1_plane(wct, oracle, synth):
    _forward_vs_fp64(wct, oracle, synth.plane1_config(), synth.plane1_depos(), "1: plane, 2000 depos")


def test_config2_bench_event(wct, oracle, synth):
    """The exact event bench.py times."""
    d = synth.apa_depos(seed=2)
    assert len(d) == 519_435
    _forward_vs_fp64(wct, oracle, synth.apa_config(), d, "2: full APA, 20 tracks", fp32=True)


def test_config3_bench_batch(wct, oracle, synth):
    """The bench's 64-event batch in one batched call."""
    cfg = synth.apa_config()
    evs = synth.batch_events(64)
    dt = wct.from_config(cfg)
    frames, wins, _ = dt.forward_batch(evs)
    worst = 0.0
    for k, e in enumerate(evs):
        f, w, _ = dt(e)
        err = rel_l2(frames[k], f)
        worst = max(worst, err)
        assert err < TOL_BATCH_VS_EVENT, (k, err)
        for a, b in zip(wins[k], w):
            a, b = dict(a), dict(b)
            a.pop("nt_gpu"), b.pop("nt_gpu")
            assert a == b, k
    sizes = np.array([len(e) for e in evs])
    widest = np.array([e[:, 5].max() for e in evs])
    small, large = int(sizes.argmin()), int(sizes.argmax())
    order = [k for k in np.argsort(-widest) if k not in (small, large)]
    picks = [small, large, int(order[0])]
    errs = []
    for k in picks:
        o64 = oracle.run(cfg, evs[k], fp64=True, nthreads=NTH)
        errs.append(rel_l2(frames[k], np.concatenate(o64["frames"], axis=0)))
    entry = {"config": "3: 64-event batch", "depos": int(sizes.sum()), "events_vs_fp64": picks,
             "depos_of_those": [int(sizes[k]) for k in picks], "rel_l2_fp64": max(errs),
             "rel_l2_fp64_each": errs, "rel_l2_batched_vs_per_event_max": worst}
    print(entry)
    parity_log(entry)
    assert max(errs) < TOL_FP64, entry


def test_config4_adjoint_forward(wct, oracle, synth):
    _forward_vs_fp64(wct, oracle, synth.apa_config(), synth.adjoint_depos(n=20_000), "4: full APA, 20k track depos")


def test_config5_calibration_event(wct, oracle, synth):
    """One 4M-depo event of the calibration workload, fluctuation off."""
    d = synth.calibration_events(nevents=1, ndepos=4_000_000)[0]
    _forward_vs_fp64(wct, oracle, synth.apa_config(), d, "5: 4M-depo calibration event", records=False)
