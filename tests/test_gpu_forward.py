"""GPU parity of the DepoTransform forward path against the oracle.

Frames are compared dense (channel x tick) by relative L2 against the FP64
oracle (tolerance 1e-5, the target precision) and against the FP32
restatement; window indices, depo counters and patch placements are compared
bit-exactly."""

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-5   # rel-L2 of the frame against the FP64 oracle
TOL_FP32 = 1e-5   # rel-L2 against the FP32 restatement of the reference


def _windows_match(wins, owins):
    for w, o in zip(wins, owins):
        assert (w["start_ch"], w["end_ch"], w["start_tick"], w["end_tick"]) == \
            (o["start_ch"], o["end_ch"], o["start_tick"], o["end_tick"])
        assert (w["nw_fft"], w["nt_fft"]) == (o["nw"], o["nt"])
        assert w["ndepos_added"] == o["ndepos_added"]
        assert w["outside_time"] == o["outside_time"]
        assert w["outside_pitch"] == o["outside_pitch"]


def _records_match(dt, cfg, rec, n):
    for ip in range(len(cfg["planes"])):
        g = dt.patch_records(0, ip, n)
        o = rec[ip]  # added, toffset, poffset, nt, np
        onz = (o[:, 3] > 0) & (o[:, 4] > 0)
        gnz = (g[:, 2] > 0) & (g[:, 3] > 0)
        assert np.array_equal(onz, gnz)
        assert np.array_equal(g[gnz], o[onz][:, 1:5])


def _run(wct, oracle, cfg, depos, fp64_tol=TOL_FP64, check_fp32=True, records=True):
    dt = wct.from_config(cfg)
    frame, wins, ident = dt(depos)
    o64 = oracle.run(cfg, depos, fp64=True, records=records)
    ref64 = np.concatenate(o64["frames"], axis=0)
    _windows_match(wins, o64["windows"])
    if records:
        _records_match(dt, cfg, o64["records"], len(depos))
    e64 = rel_l2(frame, ref64)
    assert e64 < fp64_tol, e64
    if check_fp32:
        o32 = oracle.run(cfg, depos, fp64=False)
        e32 = rel_l2(frame, np.concatenate(o32["frames"], axis=0))
        assert e32 < TOL_FP32, e32
    return dt, frame, wins, e64


@pytest.mark.parametrize("nwire_half", [21, 10])
def test_plane1_full(wct, oracle, synth, nwire_half):
    """One collection plane, 960 wires, 6000 ticks, 2000 point depos."""
    cfg = synth.plane1_config(nwire_half=nwire_half)
    d = synth.plane1_depos()
    dt, frame, wins, e = _run(wct, oracle, cfg, d)
    assert np.abs(frame).max() > 0
    print("plane1 rel-L2 vs FP64:", e)


def test_plane1_odd_pad(wct, oracle, synth):
    """A 15-wire response exercises the run-time-pad convolution kernel."""
    cfg = synth.plane1_config(nticks=2000, nwire_half=7)
    d = synth.plane1_depos(n=300, drift=0.7 * synth.m)
    _run(wct, oracle, cfg, d)


def test_apa_tracks(wct, oracle, synth):
    """Three planes with induction responses, two muon tracks."""
    cfg = synth.apa_config(nticks=6000)
    rng = np.random.default_rng(11)
    d = synth.track_depos(rng, ntracks=2, step=1.0)
    _run(wct, oracle, cfg, d)


def test_frame_ident_and_determinism(wct, synth):
    cfg = synth.plane1_config(nticks=2000)
    cfg["first_frame_number"] = 7
    d = synth.plane1_depos(n=400, drift=0.7 * synth.m)
    dt = wct.from_config(cfg)
    f1, w1, i1 = dt(d)
    f2, w2, i2 = dt(d)
    assert (i1, i2) == (7, 8)
    assert w1 == w2
    # integer accumulation (charge grid and its fixed-point bounds): bit-reproducible
    assert np.array_equal(f1, f2)


def test_empty_and_rejected_inputs(wct, oracle, synth):
    cfg = synth.plane1_config(nticks=2000)
    dt = wct.from_config(cfg)
    f, w, _ = dt(np.zeros((0, 7)))
    assert not f.any() and w[0]["ndepos_added"] == 0
    # every depo outside the pitch range or dropped by the drifter
    d = synth.plane1_depos(n=50)
    d[:, 4] += 1.0e5
    d[5:10, 2] = 5000.0
    f, w, _ = dt(d)
    o = oracle.run(cfg, d, fp64=True)
    assert not f.any()
    _windows_match(w, o["windows"])


def test_clipped_patches_at_readout_edges(wct, oracle, synth):
    """Depos whose +-3 sigma windows cross the first/last tick and the first/last
    impact bin: clipped patches are renormalised to the full charge
    (gen/src/GaussianDiffusion.cxx:176-182)."""
    cfg = synth.plane1_config(nticks=1500)
    rng = np.random.default_rng(5)
    n = 200
    d = np.zeros((n, 7))
    d[:, 1] = -3000.0
    d[:, 2] = synth.RESPONSE_X + rng.uniform(1.0, 2400.0, n)
    pmin = -0.5 * 4.79 * 960
    d[:, 4] = np.where(rng.random(n) < 0.5, pmin + rng.uniform(-3.0, 6.0, n), -pmin + rng.uniform(-6.0, 3.0, n))
    # times that put the drifted arrival near tick 0 and near the readout end
    drift_t = (d[:, 2] - synth.RESPONSE_X) / cfg["drifter"]["drift_speed"]
    end = cfg["readout_time"]
    d[:, 0] = np.where(rng.random(n) < 0.5, -drift_t + rng.uniform(-2000, 2000, n),
                       end - drift_t + rng.uniform(-2000, 2000, n))
    _run(wct, oracle, cfg, d)


def test_undrifted_point_and_extended_depos(wct, oracle, synth):
    """Without a drifter the depos are used as given: zero-extent depos make
    single-bin patches (sigma = 0 branch of GausDesc::binint/weight); large
    extents make patches of ~40 impact bins x ~200 ticks."""
    cfg = synth.plane1_config(nticks=3000)
    cfg.pop("drifter")
    rng = np.random.default_rng(9)
    n = 300
    d = np.zeros((n, 7))
    d[:, 0] = rng.uniform(1e5, 1.3e6, n)
    d[:, 1] = -rng.uniform(100, 5000, n)
    d[:, 2] = synth.RESPONSE_X
    d[:, 4] = rng.uniform(-2000, 2000, n)
    d[: n // 3, 5:7] = 0.0
    d[n // 3: 2 * n // 3, 5] = rng.uniform(0.5, 3.0, n // 3)
    d[n // 3: 2 * n // 3, 6] = rng.uniform(0.1, 2.0, n // 3)
    d[2 * n // 3:, 5] = rng.uniform(10.0, 25.0, n - 2 * n // 3)
    d[2 * n // 3:, 6] = rng.uniform(2.0, 3.2, n - 2 * n // 3)
    _run(wct, oracle, cfg, d)


def test_response_region_backdrift(wct, oracle, synth):
    """Depos between the anode and the response plane are drifted backwards in
    time without attenuation or diffusion (gen/src/Drifter.cxx:144-151)."""
    cfg = synth.plane1_config(nticks=2000)
    rng = np.random.default_rng(13)
    n = 100
    d = np.zeros((n, 7))
    d[:, 0] = rng.uniform(2e5, 8e5, n)
    d[:, 1] = -2000.0
    d[:, 2] = rng.uniform(1.0, 99.0, n)
    d[:, 4] = rng.uniform(-2000, 2000, n)
    d[:, 5:7] = rng.uniform(0.2, 1.0, (n, 2))
    _run(wct, oracle, cfg, d)


def test_device_api_matches_host_api(wct, synth):
    import torch
    cfg = synth.plane1_config(nticks=2000)
    d = synth.plane1_depos(n=500, drift=0.7 * synth.m)
    dt = wct.from_config(cfg)
    fh, wh, _ = dt(d)
    dd = torch.from_numpy(d).cuda()
    nrows, nticks = dt.frame_shape()
    fd = torch.empty((nrows, nticks), dtype=torch.float32, device="cuda")
    wd, _ = dt.forward_device(dd.data_ptr(), len(d), fd.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert wd == wh
    assert rel_l2(fd.cpu().numpy(), fh) < 1e-6


@pytest.mark.parametrize("case", ["apa", "one_plane_empty", "long_response"])
def test_host_frame_fully_written(wct, synth, case):
    """The host forward downloads each plane's zero rest early and its
    written block after the plane: every element of the caller's buffer is
    set (a NaN-filled buffer), and bit for bit the device frame."""
    import torch
    cfg = synth.apa_config(nticks=6000)
    d = synth.apa_depos(seed=6)[:40000]
    if case == "one_plane_empty":  # a 10-wire second plane that no depo reaches: its rows hold no window
        planes = list(cfg["planes"])
        planes[1] = synth._plane(10, 4.67 * synth.mm, -35.7, 1, 800, synth.RESPONSE_X)
        cfg = dict(cfg, planes=planes)
        d = d.copy()
        d[:, 3] = -2500.0  # its pitch coordinate is then above 500 mm, beyond the 10 wires
    if case == "long_response":
        k = -0.004 * np.exp(-np.arange(3000) / 400.0)
        k[0] = 1.0
        cfg = dict(cfg, long_responses=[k], long_padding=100e3)
    dt = wct.from_config(cfg)
    nrows, nticks = dt.frame_shape()
    out = np.full((nrows, nticks), np.nan, dtype=np.float32)
    fh, _, _ = dt(d, out=out)
    assert not np.isnan(fh).any()
    dd = torch.from_numpy(np.ascontiguousarray(d)).cuda()
    fd = torch.empty((nrows, nticks), dtype=torch.float32, device="cuda")
    dt.forward_device(dd.data_ptr(), len(d), fd.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert np.array_equal(fd.cpu().numpy(), fh)
    empty = synth.apa_depos(seed=6)[:0]
    out2 = np.full((nrows, nticks), np.nan, dtype=np.float32)
    f0, _, _ = dt(empty, out=out2)
    assert np.all(f0 == 0)


def test_traces_follow_waveform_edge(wct, oracle, synth):
    """Trace assembly (gen/src/DepoTransform.cxx:193-208): every non-zero wire
    becomes one trace spanning its first..last non-zero tick."""
    cfg = synth.plane1_config(nticks=2000)
    d = synth.plane1_depos(n=200, drift=0.7 * synth.m)
    dt = wct.from_config(cfg)
    frame, w, _ = dt(d)
    tr = dt.traces(frame)
    assert len(tr) > 0
    for ch, tbin, q in tr:
        row = frame[ch]
        a, b = oracle.edge(row)
        assert (tbin, tbin + len(q)) == (a, b)
        assert np.array_equal(q, row[a:b])
    nz = [i for i in range(frame.shape[0]) if frame[i].any()]
    assert sorted(t[0] for t in tr) == nz


def test_forward_traces_match_dense_frame(wct, synth):
    """wct_dt_forward_traces gives the trace list of the dense forward's frame
    (channels, first ticks, lengths and samples, bit for bit), bringing back
    only the window blocks; a short buffer is refused."""
    cfg = synth.apa_config(nticks=6000)
    d = synth.apa_depos(seed=7)[:100_000]
    dt = wct.from_config(cfg)
    frame, wins, _ = dt(d)
    want = dt.traces(frame)
    got, wins2, _, nsamp = dt.forward_traces(d)
    assert [dict(w) for w in wins2] == [dict(w) for w in wins]
    assert [(c, t, len(q)) for c, t, q in got] == [(c, t, len(q)) for c, t, q in want]
    assert all(np.array_equal(a[2], b[2]) for a, b in zip(got, want))
    nrows, nticks = dt.frame_shape()
    assert 0 < nsamp < nrows * nticks
    with pytest.raises(wct.WctError):
        dt.forward_traces(d, charge=np.empty(nsamp - 1, np.float32))
    # no depos: no traces
    t0, _, _, n0 = dt.forward_traces(d[:0])
    assert t0 == [] and n0 == 0
