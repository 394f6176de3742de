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
"""

import numpy as np


def fit_drift_params(dt, d_depos, offsets, d_targets, steps=10, lr=0.05, decay=0.93, stream=None, callback=None):
    """Fit in place.

    dt         DepoTransform with a drifter; its current DL, DT, lifetime are the start
    d_depos    device tensor [n][7] float64 of all events, concatenated
    offsets    host int64 [nevents + 1]: event e holds depos offsets[e] .. offsets[e+1]
    d_targets  device tensor [nevents][nrows][nticks] float32
    lr, decay  step k moves log-parameters by about lr * decay**k (Adam)
    Returns a list of (step, (DL, DT, lifetime), loss) before each update, and
    the final parameters."""
    import torch
    off = np.ascontiguousarray(offsets, dtype=np.int64)
    nev = len(off) - 1
    nrows, nticks = dt.frame_shape()
    s = stream if stream is not None else torch.cuda.Stream()
    sid = s.cuda_stream
    frames = torch.empty((nev, nrows, nticks), dtype=torch.float32, device=d_depos.device)
    gframe = torch.empty((nrows, nticks), dtype=torch.float32, device=d_depos.device)
    nmax = int(max(1, np.diff(off).max()))
    gdep = torch.empty((nmax, 7), dtype=torch.float64, device=d_depos.device)
    gglob = torch.zeros(3, dtype=torch.float64, device=d_depos.device)
    theta = np.log(np.array(dt.drift_params(), dtype=np.float64))
    m1 = np.zeros(3)
    m2 = np.zeros(3)
    b1, b2 = 0.9, 0.999
    history = []
    with torch.cuda.stream(s):
        for it in range(steps):
            p = np.exp(theta)
            dt.set_drift_params(*p)
            dt.forward_batch_device(d_depos.data_ptr(), off, frames.data_ptr(), stream=sid)
            diff = frames - d_targets
            loss = float((diff * diff).sum())
            g = np.zeros(3)
            for e in range(nev):
                n = int(off[e + 1] - off[e])
                torch.mul(diff[e], 2.0, out=gframe)
                dt.adjoint_device(d_depos[off[e]:off[e + 1]].data_ptr() if n else d_depos.data_ptr(), n,
                                  gframe.data_ptr(), gdep.data_ptr(), gglob.data_ptr(), stream=sid)
                g += gglob.cpu().numpy()
            history.append((it, tuple(p), loss))
            if callback:
                callback(it, p, loss, g)
            gt = g * p  # d/d log p
            m1 = b1 * m1 + (1 - b1) * gt
            m2 = b2 * m2 + (1 - b2) * gt * gt
            mh = m1 / (1 - b1 ** (it + 1))
            vh = m2 / (1 - b2 ** (it + 1))
            theta = theta - lr * decay ** it * mh / (np.sqrt(vh) + 1e-30)
    final = tuple(np.exp(theta))
    dt.set_drift_params(*final)
    return history, final
