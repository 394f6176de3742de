"""Calibration of the drifter's diffusion and electron lifetime.

Fits DL, DT and the electron lifetime of a configured DepoTransform (one with
a "drifter") to target frames by gradient descent: every step runs the
batched forward of all events (one CUDA graph; the drift parameters are
kernel arguments, so a change re-captures it), the loss
L = sum over events and frame cells of (F - T)^2 with its frame gradient
2 (F - T) on the device, and the adjoint of every event, which returns
dL/d(DL, DT, lifetime).  Parameters move in log space with Adam steps (the
three gradients differ by orders of magnitude) of decaying size.  The model is the mean
(unfluctuated) forward; targets may be fluctuated frames.

Several ranks (one process per GPU) fit together when a torch.distributed
process group is initialised: each rank holds its share of the events (see
shard.local_events), and the loss and the three gradients are summed over
ranks once per step, so every rank takes the same step.
"""

import numpy as np

from . import shard


def adam_fit(evaluate, p0, steps=10, lr=0.05, decay=0.93, reduce=None, callback=None):
    """Adam in log space with step size lr * decay**k.

    evaluate(p) -> (loss, dL/dp) at the positive parameters p (numpy);
    reduce(vector) -> the vector summed over ranks, applied to
    [loss, dL/dp...] before the step (None: a single rank).
    Returns (history of (step, params, loss), final params)."""
    theta = np.log(np.asarray(p0, dtype=np.float64))
    m1 = np.zeros_like(theta)
    m2 = np.zeros_like(theta)
    b1, b2 = 0.9, 0.999
    history = []
    for it in range(steps):
        p = np.exp(theta)
        loss, g = evaluate(p)
        v = np.concatenate([[float(loss)], np.asarray(g, dtype=np.float64)])
        if reduce is not None:
            v = reduce(v)
        loss, g = float(v[0]), v[1:]
        history.append((it, tuple(p), loss))
        if callback:
            callback(it, p, loss, g)
        gt = g * p  # d/d log p
        m1 = b1 * m1 + (1 - b1) * gt
        m2 = b2 * m2 + (1 - b2) * gt * gt
        mh = m1 / (1 - b1 ** (it + 1))
        vh = m2 / (1 - b2 ** (it + 1))
        theta = theta - lr * decay ** it * mh / (np.sqrt(vh) + 1e-30)
    return history, tuple(np.exp(theta))


def batch_objective(dt, d_depos, offsets, d_targets, stream=None):
    """evaluate(p) for ``adam_fit``: sets the drift parameters p, runs the
    batched forward and the per-event adjoint of this process's events and
    returns (L, dL/d(DL, DT, lifetime)).

    d_depos    device tensor [n][7] float64 of the events, concatenated
    offsets    host int64 [nevents + 1]: event e holds depos offsets[e] .. offsets[e+1]
    d_targets  device tensor [nevents][nrows][nticks] float32"""
    import torch
    off = np.ascontiguousarray(offsets, dtype=np.int64)
    nev = len(off) - 1
    nrows, nticks = dt.frame_shape()
    dev = d_depos.device
    s = stream if stream is not None else torch.cuda.Stream(device=dev)
    sid = s.cuda_stream
    frames = torch.empty((nev, nrows, nticks), dtype=torch.float32, device=dev)
    gframe = torch.empty((nrows, nticks), dtype=torch.float32, device=dev)
    nmax = int(max(1, np.diff(off).max())) if nev else 1
    gdep = torch.empty((nmax, 7), dtype=torch.float64, device=dev)
    gglob = torch.zeros(3, dtype=torch.float64, device=dev)
    gsum = torch.zeros(3, dtype=torch.float64, device=dev)

    def evaluate(p):
        dt.set_drift_params(*p)
        if nev == 0:
            return 0.0, np.zeros(3)
        with torch.cuda.stream(s):
            dt.forward_batch_device(d_depos.data_ptr(), off, frames.data_ptr(), stream=sid)
            diff = frames - d_targets
            loss = (diff * diff).sum()
            gsum.zero_()
            for e in range(nev):
                n = int(off[e + 1] - off[e])
                torch.mul(diff[e], 2.0, out=gframe)
                dt.adjoint_device(d_depos[off[e]:off[e + 1]].data_ptr() if n else d_depos.data_ptr(), n,
                                  gframe.data_ptr(), gdep.data_ptr(), gglob.data_ptr(), stream=sid)
                gsum.add_(gglob)
            out = torch.cat([loss.double().reshape(1), gsum]).cpu().numpy()
        return float(out[0]), out[1:].copy()

    return evaluate


def fit_drift_params(dt, d_depos, offsets, d_targets, steps=10, lr=0.05, decay=0.93, stream=None, callback=None,
                     group=None):
    """Fit in place.

    dt         DepoTransform with a drifter; its current DL, DT, lifetime are the start
    d_depos    device tensor [n][7] float64 of this rank's events, concatenated
    offsets    host int64 [nevents + 1]: event e holds depos offsets[e] .. offsets[e+1]
    d_targets  device tensor [nevents][nrows][nticks] float32
    lr, decay  step k moves log-parameters by about lr * decay**k (Adam)
    group      process group whose ranks share the fit (the default group when
               torch.distributed is initialised; each rank passes its own events)
    Returns a list of (step, (DL, DT, lifetime), loss) before each update, and
    the final parameters; every rank returns the same."""
    evaluate = batch_objective(dt, d_depos, offsets, d_targets, stream)
    reduce = None
    if shard.world()[1] > 1:
        def reduce(v):
            return shard.allreduce_sum(v, group)
    history, final = adam_fit(evaluate, dt.drift_params(), steps, lr, decay, reduce, callback)
    dt.set_drift_params(*final)
    return history, final
