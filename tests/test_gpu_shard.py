"""Sharded work on one GPU: each rank's share run in turn in one process
(the shares never wait on one another), checked against the whole.

* plane split: a DepoTransform configured with a subset of the planes gives
  the full configuration's frame rows of those planes, bit for bit;
* event split: the calibration objective (loss and drift-parameter
  gradients) of all events equals the sum of the objectives of the greedy
  event shards, which is what the per-step all-reduce of a multi-rank fit
  adds up."""

import importlib

import numpy as np
import pytest


@pytest.mark.gpu
def test_plane_split_rows_match(wct, synth):
    shard = importlib.import_module("wire-cell-toolkit_b200.shard")
    cfg = synth.apa_config(nticks=6000)
    depos = synth.apa_depos(seed=11)[:60000]
    full, _, _ = wct.from_config(cfg)(depos)
    nw = [p["nwires"] for p in cfg["planes"]]
    parts = shard.plane_partition(3, 2)
    rows = []
    for planes in parts:
        f, _, _ = wct.from_config(shard.plane_config(cfg, planes))(depos)
        rows.append(np.asarray(f))
    import torch
    stacked = shard.face_order(torch.from_numpy(np.concatenate(rows)), parts, nw).numpy()
    assert np.array_equal(stacked, np.asarray(full))


@pytest.mark.gpu
def test_event_shards_sum_to_whole(wct, synth):
    import torch
    shard = importlib.import_module("wire-cell-toolkit_b200.shard")
    cal = importlib.import_module("wire-cell-toolkit_b200.calibrate")
    cfg = synth.apa_config(nticks=6000)
    events = synth.calibration_events(nevents=5, ndepos=100_000, seed=6)
    dr = cfg["drifter"]
    off = np.zeros(len(events) + 1, dtype=np.int64)
    off[1:] = np.cumsum([len(e) for e in events])
    alld = np.concatenate(events)
    gen = wct.from_config(cfg)
    gen.set_drift_params(dr["DL"] * 0.9, dr["DT"] * 1.1, 8.0e6)
    nrows, nticks = gen.frame_shape()
    d = torch.from_numpy(alld).cuda()
    targets = torch.zeros((len(events), nrows, nticks), dtype=torch.float32, device="cuda")
    gen.forward_batch_device(d.data_ptr(), off, targets.data_ptr())
    torch.cuda.synchronize()

    model = wct.from_config(cfg)
    p = np.array([dr["DL"], dr["DT"], dr["lifetime"]])
    loss, g = cal.batch_objective(model, d, off, targets)(p)
    tot = np.zeros(4)
    for r in range(2):
        ev, rows, loc = shard.local_events(off, r, 2)
        dr_ = torch.from_numpy(alld[rows]).cuda()
        tr_ = targets[torch.from_numpy(ev).cuda()].contiguous()
        lr_, gr_ = cal.batch_objective(model, dr_, loc, tr_)(p)
        tot += np.concatenate([[lr_], gr_])
    assert loss > 0
    np.testing.assert_allclose(tot[0], loss, rtol=1e-6)
    np.testing.assert_allclose(tot[1:], g, rtol=1e-6)
