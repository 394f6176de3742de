"""Differentiable forward + adjoint.

The adjoint (wct_dt_adjoint*, csrc/adjoint.cu) is the reverse-mode derivative
of the forward with the piecewise-constant choices held fixed: which depos reach
a plane, patch sample ranges and event windows.  Its FP64 oracle is
oracle/adjoint.py (a NumPy restatement of the same model, checked here against
the C restatement of the reference and against central finite differences).

Loss used throughout: L = sum over frame cells of (F - T)^2, with T the frame
simulated with DT x 1.1, DL x 0.9 and lifetime 8 ms.

Finite-difference steps are 1e-4 relative: to the tick for times, to the
impact-plane pitch for positions and extents, and to the value for charge and
for DL, DT and lifetime.

Tolerances: gradients within 1e-4 (relative L2 over each parameter column, and
relative per global parameter) of the FP64 gradient and of FP64 finite
differences.
"""

import copy

import numpy as np
import pytest

from conftest import rel_l2

GRAD_TOL = 1e-4
COLS = ("t", "q", "x", "y", "z", "extent_long", "extent_tran")


def _adjoint_oracle():
    import adjoint
    return adjoint


def _small_case(synth, nticks=1200, n=60, seed=5):
    cfg = synth.plane1_config(nticks=nticks)
    rng = np.random.default_rng(seed)
    d = np.zeros((n, 7))
    d[:, 0] = rng.uniform(0, 100e3, n)
    d[:, 1] = -5000.0 * rng.uniform(0.5, 1.5, n)
    d[:, 2] = rng.uniform(110.0, 900.0, n)
    d[:, 4] = rng.uniform(-200.0, 200.0, n)
    return cfg, d


def _target_glob(glob):
    return np.array([glob[0] * 0.9, glob[1] * 1.1, 8.0e6])


PITCH = 4.79  # mm, the collection-plane pitch


def _fd_steps(cfg, d):
    return [1e-4 * cfg["tick"], 1e-4 * abs(d[1])] + [1e-4 * PITCH] * 5


# ---------------------------------------------------------------------------
# CPU: the FP64 oracle of the adjoint
# ---------------------------------------------------------------------------
def test_frozen_model_frames_match_oracle(synth, oracle):
    A = _adjoint_oracle()
    cfg, d = _small_case(synth)
    M = A.FrozenModel(cfg, d)
    F = M.frames()
    for f, b in zip(F, M.base_frames):
        assert np.abs(b).max() > 0
        assert rel_l2(f, b) < 1e-12


def test_frozen_model_frames_match_oracle_apa(synth, oracle):
    A = _adjoint_oracle()
    cfg = synth.apa_config(nticks=1500)
    rng = np.random.default_rng(11)
    d = synth.track_depos(rng, ntracks=2, step=5.0, lo=np.array((110.0, -800.0, -400.0)),
                          hi=np.array((700.0, 800.0, 400.0)))
    M = A.FrozenModel(cfg, d)
    F = M.frames()
    for f, b in zip(F, M.base_frames):
        assert np.abs(b).max() > 0
        assert rel_l2(f, b) < 1e-12


def test_correlate_is_transpose_of_convolve(synth, oracle):
    """<conv(Q), G> == <Q, corr(G)> for random Q and G (dot-product test)."""
    A = _adjoint_oracle()
    cfg, d = _small_case(synth, n=20)
    M = A.FrozenModel(cfg, d)
    P = M.planes[0]
    rng = np.random.default_rng(3)
    w0, t0 = 400, 300
    Qb = rng.normal(size=(P.G, 30, 80))
    lo, tt, V = M._conv_block(0, w0, t0, Qb)
    G = rng.normal(size=(P.nwires, M.nticks))
    lhs = float(np.sum(V * G[lo:lo + V.shape[0], tt:tt + V.shape[1]]))
    dQ = M.correlate(0, G)
    rhs = float(np.sum(Qb * dQ[:, w0:w0 + 30, t0:t0 + 80]))
    assert abs(lhs - rhs) <= 1e-11 * abs(lhs)


def test_fp64_gradient_matches_finite_differences(synth, oracle):
    A = _adjoint_oracle()
    cfg, d = _small_case(synth)
    M = A.FrozenModel(cfg, d)
    F = M.frames()
    T = M.frames(glob=_target_glob(M.glob))
    gd, gg = M.gradient([2.0 * (f - t) for f, t in zip(F, T)])
    added = np.nonzero(M.records[0, :, 0])[0]
    assert len(added) > 10
    for i in added[:4]:
        steps = _fd_steps(cfg, d[i])
        for k in (0, 1, 2, 4):
            fd = M.fd_depo(i, k, steps[k], T, F)
            assert abs(gd[i, k] - fd) <= GRAD_TOL * abs(fd) + 1e-12 * np.abs(gd[:, k]).max(), (i, COLS[k])
    for k in range(3):
        fd = M.fd_global(k, 1e-4 * M.glob[k], T)
        assert abs(gg[k] - fd) <= 1e-6 * abs(fd), k


# ---------------------------------------------------------------------------
# GPU: the adjoint kernels
# ---------------------------------------------------------------------------
def _gpu_pair(wct, cfg, glob_target):
    dt = wct.from_config(cfg)
    dtt = wct.from_config(cfg)
    dtt.set_drift_params(*glob_target)
    return dt, dtt


def _check_columns(g, ref, what):
    for k, name in enumerate(COLS):
        if np.abs(ref[:, k]).max() == 0:
            assert np.abs(g[:, k]).max() <= 1e-30, (what, name)
            continue
        err = rel_l2(g[:, k], ref[:, k])
        assert err < GRAD_TOL, (what, name, err)


@pytest.mark.gpu
def test_adjoint_matches_fp64_gradient_plane1(wct, synth, oracle):
    A = _adjoint_oracle()
    cfg, d = _small_case(synth, nticks=2000, n=400, seed=7)
    dr = cfg["drifter"]
    glob = np.array([dr["DL"], dr["DT"], dr["lifetime"]])
    dt, dtt = _gpu_pair(wct, cfg, _target_glob(glob))
    F, _, _ = dt(d)
    T, _, _ = dtt(d)
    gF = 2.0 * (F - T)
    gd, gg = dt.adjoint(d, gF)
    M = A.FrozenModel(cfg, d)
    nw = cfg["planes"][0]["nwires"]
    rd, rg = M.gradient([gF[:nw].astype(np.float64)])
    _check_columns(gd, rd, "plane1")
    for k in range(3):
        assert abs(gg[k] - rg[k]) <= GRAD_TOL * abs(rg[k]), (k, gg[k], rg[k])


def _apa_adjoint_case(wct, synth, nticks, n):
    cfg = synth.apa_config(nticks=nticks)
    d = synth.adjoint_depos(n=n)
    dr = cfg["drifter"]
    glob = np.array([dr["DL"], dr["DT"], dr["lifetime"]])
    dt, dtt = _gpu_pair(wct, cfg, _target_glob(glob))
    F, _, _ = dt(d)
    T, _, _ = dtt(d)
    return cfg, d, dt, F, T


@pytest.mark.gpu
def test_adjoint_config4_fp64_gradient_and_finite_differences(wct, synth, oracle):
    """Full-APA geometry, 6000 ticks, 20k track depos: GPU gradient of the
    GPU loss against the FP64 gradient of the FP64 loss (same target frame)
    and against FP64 central finite differences for a sample of depos."""
    A = _adjoint_oracle()
    cfg, d, dt, F, T = _apa_adjoint_case(wct, synth, 6000, 20_000)
    gd, gg = dt.adjoint(d, 2.0 * (F - T))
    M = A.FrozenModel(cfg, d)
    F64 = M.frames()
    rows = np.cumsum([0] + [p["nwires"] for p in cfg["planes"]])
    T64 = [T[rows[i]:rows[i + 1]].astype(np.float64) for i in range(len(F64))]
    for i, f in enumerate(F64):
        assert rel_l2(F[rows[i]:rows[i + 1]], f) < 1e-5
    rd, rg = M.gradient([2.0 * (f - t) for f, t in zip(F64, T64)])
    _check_columns(gd, rd, "config4")
    for k in range(3):
        assert abs(gg[k] - rg[k]) <= GRAD_TOL * abs(rg[k]), (k, gg[k], rg[k])
    rng = np.random.default_rng(0)
    added = np.nonzero(M.records.any(axis=0)[:, 0])[0]
    sample = rng.choice(added, size=6, replace=False)
    got, want = [], []
    for i in sample:
        steps = _fd_steps(cfg, d[i])
        for k in (0, 1, 2, 3, 4):
            got.append(gd[i, k])
            want.append(M.fd_depo(i, k, steps[k], T64, F64))
    got, want = np.array(got), np.array(want)
    assert rel_l2(got, want) < GRAD_TOL, (got, want)


@pytest.mark.gpu
def test_adjoint_global_finite_differences_apa(wct, synth, oracle):
    """DL, DT and lifetime gradients of the GPU against FP64 central differences
    (full frozen forward twice per parameter) on a smaller APA case."""
    A = _adjoint_oracle()
    cfg, d, dt, F, T = _apa_adjoint_case(wct, synth, 3000, 3000)
    _, gg = dt.adjoint(d, 2.0 * (F - T))
    M = A.FrozenModel(cfg, d)
    rows = np.cumsum([0] + [p["nwires"] for p in cfg["planes"]])
    T64 = [T[rows[i]:rows[i + 1]].astype(np.float64) for i in range(len(cfg["planes"]))]
    for k in range(3):
        fd = M.fd_global(k, 1e-4 * M.glob[k], T64)
        assert abs(gg[k] - fd) <= GRAD_TOL * abs(fd), (k, gg[k], fd)


@pytest.mark.gpu
def test_adjoint_without_drifter(wct, synth, oracle):
    """Undrifted input (drifted on the host by the oracle): positions enter
    through the pitch coordinate only; no global gradients."""
    A = _adjoint_oracle()
    cfg, d = _small_case(synth, nticks=2000, n=300, seed=9)
    dd = oracle.drift_fn(cfg, d)[:, :7]
    cfg2 = copy.deepcopy(cfg)
    cfg2.pop("drifter")
    dt = wct.from_config(cfg2)
    F, _, _ = dt(dd)
    rng = np.random.default_rng(1)
    T = F * (1.0 + 0.1 * rng.standard_normal(F.shape)).astype(np.float32)
    gF = 2.0 * (F - T)
    gd, gg = dt.adjoint(dd, gF)
    assert np.all(gg == 0)
    M = A.FrozenModel(cfg2, dd)
    rd, _ = M.gradient([gF.astype(np.float64)])
    _check_columns(gd, rd, "undrifted")


@pytest.mark.gpu
def test_adjoint_empty_and_zero(wct, synth):
    cfg, d = _small_case(synth, nticks=2000, n=50)
    dt = wct.from_config(cfg)
    nrows, nticks = dt.frame_shape()
    gd, gg = dt.adjoint(np.zeros((0, 7)), np.ones((nrows, nticks), np.float32))
    assert gd.shape == (0, 7) and np.all(gg == 0)
    gd, gg = dt.adjoint(d, np.zeros((nrows, nticks), np.float32))
    assert np.all(gd == 0) and np.all(gg == 0)


@pytest.mark.gpu
def test_autograd_function_matches_adjoint(wct, synth):
    import torch
    cfg, d = _small_case(synth, nticks=2000, n=400, seed=7)
    dr = cfg["drifter"]
    glob = np.array([dr["DL"], dr["DT"], dr["lifetime"]])
    dt, dtt = _gpu_pair(wct, cfg, _target_glob(glob))
    T, _, _ = dtt(d)
    dev = torch.device("cuda", 0)
    depos = torch.tensor(d, dtype=torch.float64, device=dev, requires_grad=True)
    dp = torch.tensor(glob, dtype=torch.float64, requires_grad=True)
    frame = wct.depo_transform(dt, depos, dp)
    Tt = torch.from_numpy(T).to(dev)
    loss = ((frame - Tt) ** 2).sum()
    loss.backward()
    F, _, _ = dt(d)
    assert np.array_equal(frame.detach().cpu().numpy(), F)  # the forward is bit-reproducible
    gd, gg = dt.adjoint(d, 2.0 * (F - T))
    assert np.array_equal(depos.grad.cpu().numpy(), gd)     # so is the per-depo gradient
    assert rel_l2(dp.grad.numpy(), gg) < 1e-12              # global sums: atomics in any order
    # the drift parameters passed in are the ones the forward used
    frame2 = wct.depo_transform(dt, depos.detach(), torch.tensor(_target_glob(glob)))
    assert np.array_equal(frame2.cpu().numpy(), T)
