"""Calibration: gradient-descent fit of DL, DT and lifetime with the adjoint.

Targets are fluctuated frames (patch cells and drift absorption drawn) made
with the true parameters (DL x 0.9, DT x 1.1, lifetime 8 ms); the fit starts
from the nominal values and uses the batched mean forward and the adjoint.
One event's unfluctuated frame is also checked against the FP64 oracle."""

import numpy as np
import pytest

from conftest import rel_l2


@pytest.mark.gpu
def test_fit_recovers_drift_parameters(wct, synth, oracle):
    import importlib
    import torch
    cal = importlib.import_module("wire-cell-toolkit_b200.calibrate")
    cfg = synth.apa_config(nticks=6000)
    events = synth.calibration_events(nevents=3, ndepos=200_000, seed=4)
    dr = cfg["drifter"]
    nominal = np.array([dr["DL"], dr["DT"], dr["lifetime"]])
    truth = np.array([dr["DL"] * 0.9, dr["DT"] * 1.1, 8.0e6])
    off = np.zeros(len(events) + 1, dtype=np.int64)
    off[1:] = np.cumsum([len(e) for e in events])
    d = torch.from_numpy(np.concatenate(events)).cuda()
    gen = wct.from_config(dict(cfg, fluctuate=True, seed=21, drifter=dict(dr, fluctuate=True)))
    gen.set_drift_params(*truth)
    nrows, nticks = gen.frame_shape()
    targets = torch.zeros((len(events), nrows, nticks), dtype=torch.float32, device="cuda")
    gen.forward_batch_device(d.data_ptr(), off, targets.data_ptr())
    torch.cuda.synchronize()

    model = wct.from_config(cfg)
    # float32 forward of one event against the FP64 oracle
    f, _, _ = model(events[0])
    o = oracle.run(cfg, events[0], fp64=True, nthreads=4)
    rows = np.cumsum([0] + [p["nwires"] for p in cfg["planes"]])
    for ip, f64 in enumerate(o["frames"]):
        assert rel_l2(f[rows[ip]:rows[ip + 1]], f64) < 1e-5

    hist, final = cal.fit_drift_params(model, d, off, targets, steps=25, lr=0.05)
    losses = [h[2] for h in hist]
    assert losses[-1] < 0.6 * losses[0], losses
    err0 = np.abs(np.log(nominal / truth))
    err1 = np.abs(np.log(np.array(final) / truth))
    assert np.all(err1 < 0.5 * err0 + 0.02), (final, truth)
