#!/usr/bin/env python
"""Throughput of the DepoTransform signal-simulation path on B200.

Workload (default): the full-APA plain forward -- three planes (U/V 800 wires
at 4.67 mm, W 960 wires at 4.79 mm, +-35.7 deg), 6000 ticks, 20 seeded
straight muon tracks with one depo per 0.1 mm (~520k depos), drift + diffusion
+ erf patches + FFT convolution + frame.  One step = one event through
DepoTransform::operator() with its depos already resident in HBM.

Output: one JSON line (rank 0).  Multi-GPU: one process per GPU; `--gpus N`
starts the N ranks itself (torch.distributed.run on 127.0.0.1) unless a
launcher already did, and refuses a launcher's world that is not N.  Every
rank simulates its own event (events are independent: weak scaling, no
data-path collective); times are the slowest rank's.

"cpu_baseline": the CPU restatement of the reference (oracle/, FP32) on the
same event, one thread, transforms by libtorch-CPU (MKL; the reference's
TorchDFT backend), plane responses built once; 1 warm-up, median of 5, split
by stage.  "parity": that leg's checker run, the FP64 oracle's frame of the
same event against the GPU frame (rel-L2, windows), outside the timed region.

On one GPU the line also carries "patterns": forward + adjoint on 20k track
depos (full-APA geometry), a batch of 64 uneven full-APA events through one
captured CUDA graph against per-event calls (and a batch of small events),
a full-APA event with fluctuation on, and the large batched calibration (16
events x 4M depos, fluctuated targets, DL/DT/lifetime fit steps) -- each timed
with CUDA events on the launch stream (skip with --no-patterns,
--no-calibration).

``--impl reference`` times the CPU restatement of the reference (oracle/,
FP32, MKL transforms, one event per step) on every host core instead.
"""

import argparse
import csv
import importlib
import io
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "depos/s fwd & fwd+adjoint on 1 B200 vs plain GPU fwd, rel-L2≤1e-5 vs FP64"
UNIT = "depos/s"


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.p = None
        self.lines = []

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.lines = []
            import threading
            self.th = threading.Thread(target=self._reader, daemon=True)
            self.th.start()
        except Exception:
            self.p = None

    def _reader(self):
        for line in self.p.stdout:
            self.lines.append(line)

    def wait_first_sample(self, timeout=3.0):
        t0 = time.perf_counter()
        while self.p is not None and not self.lines and time.perf_counter() - t0 < timeout:
            time.sleep(0.01)

    def nsamples(self):
        return len(self.lines)

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.th.join(timeout=5)
        rows = [[c.strip() for c in r] for r in csv.reader(io.StringIO("".join(self.lines))) if len(r) >= 9]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for k, nm in enumerate(names):
                if r[5 + k].strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def dist_setup(args):
    """Rank, world size and local rank of this process (torch.distributed.run
    sets them; a plain run is rank 0 of 1).  A world that is not the --gpus
    count the caller asked for is an error, never a relabelled result."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args is not None and world != args.gpus:
        raise SystemExit("bench.py: --gpus %d but WORLD_SIZE=%d" % (args.gpus, world))
    return rank, world, local


def free_port():
    import socket
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def relaunch(nproc, script, argv, timeout_s=None):
    """Run `script argv` as nproc ranks of one node (one process per GPU)
    under torch.distributed.run on 127.0.0.1 and return its exit status."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", str(nproc),
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()), script] + list(argv)
    env = dict(os.environ, OMP_NUM_THREADS=os.environ.get("OMP_NUM_THREADS", "4"))
    return subprocess.run(cmd, env=env, timeout=timeout_s).returncode


def init_group(world, backend="nccl", timeout_s=120):
    """The process group of a multi-rank run (a short timeout, so ranks that
    wait for a missing peer end with an error)."""
    if world <= 1:
        return
    import datetime
    import torch.distributed as dist
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))


def max_over_ranks(x, world, device="cuda"):
    """The largest of each rank's x (the whole job's time is the slowest rank's)."""
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


STAGE_KERNELS = {"raster": "k_fill + k_raster_wires", "time_fft": "k_rfft_rows x planes",
                 "wire_conv": "k_wire_conv x planes", "inverse_fft+frame": "k_irfft_rows x planes",
                 "drift+prep": "k_prep_all + k_scan_*"}


def stage_bytes(wins, cfg, n_depos, G=11):
    """Per-stage algorithmic bytes of one event (sum over planes):
    raster    32 B patch record per depo-plane + the group grids written once
    time_fft  group grids read + packed spectra written
    wire_conv group spectra read + one plane spectrum written
    inverse   plane spectrum read + frame window written."""
    nticks = int(round(cfg["readout_time"] / cfg["tick"]))
    out = {"raster": 0, "time_fft": 0, "wire_conv": 0, "inverse_fft+frame": 0}
    for w, pl in zip(wins, cfg["planes"]):
        if w["ndepos_added"] == 0:
            continue
        N = w["nt_gpu"]
        M = N // 2
        nin = w["charge_rows"]
        nout = nin + 2 * w["npad"]
        grid = G * nin * N * 4
        out["raster"] += 32 * n_depos + grid
        out["time_fft"] += 2 * grid
        out["wire_conv"] += G * nin * M * 8 + nout * M * 8
        rows = max(0, min(pl["nwires"], w["end_ch"]) - max(0, w["start_ch"]))
        cols = max(0, min(nticks, w["end_tick"]) - max(0, w["start_tick"]))
        out["inverse_fft+frame"] += nout * M * 8 + rows * cols * 4
    return out


WORKLOAD_TEXT = {
    "apa": "full-APA plain forward: U/V 800 + W 960 wires, 6000 ticks, 20 muon tracks, %d depos per event per GPU, "
           "drift+diffusion+FFT convolution",
    "plane": "one collection plane (960 wires, 4.79 mm, 6000 ticks), %d point depos per event per GPU (5000 "
             "electrons each, uniform in wire coordinate and drift distance), drift+diffusion+FFT convolution",
}


def run_b200(args):
    import torch
    rank, world, local = dist_setup(args)
    torch.cuda.set_device(local)
    init_group(world, "nccl")
    wct = importlib.import_module("wire-cell-toolkit_b200")
    synth = importlib.import_module("wire-cell-toolkit_b200.synth")
    if args.workload == "plane":
        cfg = synth.plane1_config()
        depos = synth.plane1_depos(seed=1 + rank)
    else:
        cfg = synth.apa_config()
        depos = synth.apa_depos(seed=2 + rank)
    if args.depos:  # a smaller workload (profiling): the event's first depos
        depos = np.ascontiguousarray(depos[:args.depos])
    n = len(depos)
    dt = wct.from_config(cfg, device=local)
    # a dedicated (non-default) stream: the library and the timing events share it
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    d_depos = torch.from_numpy(depos).to("cuda")
    nrows, nticks = dt.frame_shape()
    d_frame = torch.empty((nrows, nticks), dtype=torch.float32, device="cuda")
    flush = torch.empty(320 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")  # > L2 (126 MB)

    def step():
        return dt.forward_device(d_depos.data_ptr(), n, d_frame.data_ptr(), stream.cuda_stream)

    for _ in range(args.warmup):
        flush.fill_(1.0)
        wins, _ = step()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clocks.start()
    clocks.wait_first_sample()
    evs = []
    for k in range(args.steps):
        flush.fill_(float(k))  # L2 flush between timed steps, outside the timed events
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        wins, _ = step()
        b.record(stream)
        evs.append((a, b))
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    # The timed region is far shorter than the 200 ms sampling period: keep
    # running identical steps until the sampler has seen the GPU under load.
    t_load = time.perf_counter()
    while clocks.nsamples() < 4 and time.perf_counter() - t_load < 5.0:
        for _ in range(20):
            step()
        torch.cuda.synchronize()
    clk = clocks.stop()
    total_ms = sum(a.elapsed_time(b) for a, b in evs)
    # stage breakdown: the same steps again with the library's stage timers on
    # (the planes' chains then run one after another on the launch stream)
    dt.stage_times(reset=True)
    dt.set_profiling(True)
    for k in range(args.steps):
        flush.fill_(float(k))
        step()
    torch.cuda.synchronize()
    dt.set_profiling(False)
    stages, launches = dt.stage_times(reset=True)
    max_ms = max_over_ranks(total_ms, world)
    gpu_frame = d_frame.cpu().numpy() if rank == 0 else None  # the last timed step's frame
    total_depos = n * world
    value = total_depos * args.steps / (max_ms / 1e3)

    # --- end to end through the public host API (the call a Wire-Cell adapter
    # makes): pinned host depos in, the frame's trace list out (the reference's
    # output, SimpleFrame of Waveform::edge-trimmed traces); host<->device
    # copies inside the timed region.  Also the dense-frame call for comparison.
    h_depos = torch.from_numpy(depos).pin_memory()
    h_charge = torch.empty(nrows * nticks, dtype=torch.float32).pin_memory()
    h_frame = torch.empty((nrows, nticks), dtype=torch.float32).pin_memory()
    hd, hc, hf = h_depos.numpy(), h_charge.numpy(), h_frame.numpy()
    meta = dt.trace_meta()
    nsamples = 0
    for _ in range(max(1, args.warmup)):
        _, nsamples, _ = dt.forward_traces_raw(hd, hc, meta)
    if world > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        _, nsamples, _ = dt.forward_traces_raw(hd, hc, meta)
    e2e_s = time.perf_counter() - t0
    e2e_value = total_depos * args.steps / max_over_ranks(e2e_s, world)
    for _ in range(max(1, args.warmup)):
        dt(hd, out=hf)
    if world > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        dt(hd, out=hf)
    dense_value = total_depos * args.steps / max_over_ranks(time.perf_counter() - t0, world)

    # --- roofline of the dominant stage (live CUDA events on the launch stream).
    # A "launch" here is one execution of the stage for one event (all planes):
    # algorithmic bytes of the event's stage over the stage's event time.
    peak, peak_kind = load_peaks()
    sb = stage_bytes(wins, cfg, n)
    dom = max((k for k in sb), key=lambda k: stages[k][0])
    bytes_per_launch = sb[dom]
    ms_per_launch = stages[dom][0] / args.steps
    achieved = bytes_per_launch / (ms_per_launch / 1e3) / 1e9 if ms_per_launch > 0 else 0.0
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        try:
            traffic = json.load(open(tp))["stages"].get(dom)
        except Exception:
            traffic = None

    result = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": max_ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {
            "workload": (WORKLOAD_TEXT[args.workload] % n),
            "depos_per_event": n,
            "planes": [dict(w) for w in wins],
            "l2": "flushed between timed steps (320 MB write, untimed)",
            "parallelism": "events sharded over %d GPU(s), no collective" % world,
        },
        "roofline": {
            "bound": "hbm",
            "kernel": dom + " (" + STAGE_KERNELS.get(dom, dom) + ")",
            "achieved": achieved,
            "peak": peak,
            "unit": "GB/s",
            "frac": achieved / peak,
            "peak_kind": peak_kind,
            "traffic": traffic,
            "algorithmic_bytes_per_launch": bytes_per_launch,
            "ms_per_launch": ms_per_launch,
            "launch": "one execution of the stage for one event (all planes)",
        },
        "stages_ms_per_step": {k: v[0] / args.steps for k, v in stages.items() if not k.startswith("adj_")},
        "stages_note": "stage times from the same steps run again with the stage timers on (planes one after "
                       "another); the timed steps run each plane's FFT chain on its own stream",
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(depos.nbytes),
                "d2h_bytes_per_step": int(nsamples * 4 + nrows * 8),
                "call": "wct_dt_forward_traces: host depos in, the trace list out (window blocks + trace edges)",
                "dense_frame": {"value": dense_value, "unit": UNIT, "call": "wct_dt_forward: host depos in, "
                                "the dense frame out", "d2h_bytes_per_step": int(nrows * nticks * 4)}},
        "gpu_launches": launches,
        "clocks": clk,
    }
    result["frame_ticks_per_s"] = world * nrows * nticks * args.steps / (max_ms / 1e3)
    if rank == 0 and world == 1 and not args.no_patterns and args.workload == "apa":
        try:
            result["patterns"] = patterns(wct, synth, torch, stream, local)
        except Exception as e:  # the headline line must print whatever happens here
            result["patterns"] = {"error": repr(e)[:300]}
        try:
            result["patterns"]["downstream"] = downstream(wct, synth, torch, stream, local)
        except Exception as e:
            result["patterns"]["downstream"] = {"error": repr(e)[:300]}
        if not args.no_calibration:
            try:
                result["patterns"]["calibration"] = calibration(wct, synth, torch, local)
            except Exception as e:
                result["patterns"]["calibration"] = {"error": repr(e)[:300]}
    if rank == 0 and not args.no_cpu_baseline:
        result["cpu_baseline"], result["parity"] = cpu_baseline(cfg, depos, gpu_frame, wins, timed=world == 1)
    if rank == 0:
        print(json.dumps(result), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def _time_ms(torch, stream, fn, reps=5, warm=2, spread=False):
    """Median milliseconds of fn() (device time, CUDA events on the launch stream);
    with spread, also the fastest and slowest repetition."""
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        b.synchronize()
        ts.append(a.elapsed_time(b))
    med = float(statistics.median(ts))
    return (med, float(min(ts)), float(max(ts))) if spread else med


def patterns(wct, synth, torch, stream, local):
    """The two patterns beside the plain forward, and the fluctuated forward:
    forward + adjoint on 20k track depos (full-APA geometry), a batch of 64
    uneven events through one captured graph against per-event calls (and the
    same for a batch of small events), and one full-APA event with
    fluctuation on."""
    out = {}
    cfg = synth.apa_config()
    nrows, nticks = wct.from_config(cfg, device=local).frame_shape()

    # forward + adjoint (gradients of every depo coordinate and of DL, DT, lifetime)
    d = synth.adjoint_depos(n=20_000)
    dt = wct.from_config(cfg, device=local)
    dd = torch.from_numpy(d).cuda()
    fr = torch.zeros((nrows, nticks), dtype=torch.float32, device="cuda")
    gf = torch.randn((nrows, nticks), dtype=torch.float32, device="cuda")
    gd = torch.zeros_like(dd)
    gg = torch.zeros(3, dtype=torch.float64, device="cuda")
    sid = stream.cuda_stream
    fwd = lambda: dt.forward_device(dd.data_ptr(), len(d), fr.data_ptr(), sid)  # noqa: E731
    adj = lambda: dt.adjoint_device(dd.data_ptr(), len(d), gf.data_ptr(), gd.data_ptr(), gg.data_ptr(), sid)  # noqa
    t_f = _time_ms(torch, stream, fwd)
    t_fa = _time_ms(torch, stream, lambda: (fwd(), adj()))
    out["fwd_adjoint"] = {
        "workload": "full-APA geometry, 6000 ticks, 20000 track depos; adjoint of every depo coordinate and of "
                    "DL, DT, lifetime with patches recomputed",
        "fwd_ms": t_f, "fwd_adj_ms": t_fa, "ratio_fwd_adj_over_fwd": t_fa / t_f,
        "depos_per_s_fwd_adj": len(d) / (t_fa / 1e3), "target_ratio": "<= 3"}
    del dd, fr, gf, gd, gg

    def batch_case(events, label):
        dtb = wct.from_config(cfg, device=local)
        off = np.zeros(len(events) + 1, dtype=np.int64)
        off[1:] = np.cumsum([len(e) for e in events])
        db = torch.from_numpy(np.concatenate(events)).cuda()
        frames = torch.zeros((len(events), nrows, nticks), dtype=torch.float32, device="cuda")

        def per_event():
            for k in range(len(events)):
                if off[k + 1] > off[k]:
                    dtb.forward_device(db[off[k]:off[k + 1]].data_ptr(), int(off[k + 1] - off[k]),
                                       frames[k].data_ptr(), sid)
        # both forms end with a host synchronisation per call (the per-event
        # call also one per event), so host-side delays on a busy machine
        # land in these device times: five repetitions, the median reported
        # with the range beside it
        t_pe, pe_lo, pe_hi = _time_ms(torch, stream, per_event, reps=5, warm=1, spread=True)
        rep = dtb.autotune_batch(db.data_ptr(), off, frames.data_ptr(), stream=sid)
        t_b, b_lo, b_hi = _time_ms(torch, stream,
                                   lambda: dtb.forward_batch_device(db.data_ptr(), off, frames.data_ptr(), sid),
                                   reps=5, warm=2, spread=True)
        nd = int(off[-1])
        r = {"workload": label, "events": len(events), "depos": nd, "per_event_ms": t_pe, "batched_ms": t_b,
             "per_event_ms_range": [pe_lo, pe_hi], "batched_ms_range": [b_lo, b_hi],
             "speedup_batched_over_per_event": t_pe / t_b, "depos_per_s_batched": nd / (t_b / 1e3),
             "frame_ticks_per_s_batched": len(events) * nrows * nticks / (t_b / 1e3),
             "autotuned": rep["best"], "target_speedup": ">= 2"}
        del db, frames
        torch.cuda.empty_cache()
        return r

    out["batched"] = batch_case(synth.batch_events(64),
                                "64 full-APA events, depo counts log-uniform in [10k, 500k], tracks + shower blobs, "
                                "patches 3x10 .. 40x200 bins; one captured graph, autotuned launch shapes")
    out["batched_small"] = batch_case(synth.batch_events(64, seed=5, lo=500, hi=5000),
                                      "64 full-APA events, depo counts log-uniform in [500, 5000] (launch-bound "
                                      "regime)")

    # fluctuated forward (patch cells and drift), one full-APA event
    dfl = wct.from_config(dict(cfg, fluctuate=True, seed=1, drifter=dict(cfg["drifter"], fluctuate=True)),
                          device=local)
    d = synth.apa_depos(seed=2)
    dd = torch.from_numpy(d).cuda()
    fr = torch.zeros((nrows, nticks), dtype=torch.float32, device="cuda")
    t_fl = _time_ms(torch, stream, lambda: dfl.forward_device(dd.data_ptr(), len(d), fr.data_ptr(), sid))
    out["fluctuated"] = {"workload": "full-APA event (%d depos), patch-cell and drift fluctuation on" % len(d),
                         "ms": t_fl, "depos_per_s": len(d) / (t_fl / 1e3)}
    return out


def downstream(wct, synth, torch, stream, local):
    """The components beside the DepoTransform path, device-timed (CUDA events
    on the launch stream, median of 5): the DepoFluxSplat truth frame of a
    full-APA event's depos at the response plane, noise (three plane spectra)
    and digitization of the full-APA frame, and IDFT 2-D transforms."""
    peak, kind = load_peaks()
    out = {}
    sid = stream.cuda_stream
    cfg = synth.apa_config()
    dt = wct.from_config(cfg, device=local)
    nrows, nticks = dt.frame_shape()
    # splat: depos as the drifter leaves them (times and extents of their drift distance)
    d = synth.apa_depos(seed=2).copy()
    drift = np.abs(d[:, 2] - synth.RESPONSE_X)
    d[:, 0] = drift / (1.6 * synth.mm / synth.us)
    d[:, 2] = synth.RESPONSE_X
    d[:, 5] = np.sqrt(2 * cfg["drifter"]["DL"] * d[:, 0])
    d[:, 6] = np.sqrt(2 * cfg["drifter"]["DT"] * d[:, 0])
    sc = dict(tick=cfg["tick"], window_start=0.0, window_duration=nticks * cfg["tick"], nsigma=3.0,
              drift_speed=1.6 * synth.mm / synth.us, response_plane=synth.RESPONSE_X)
    sr, st = dt.splat_shape(**sc)
    dd = torch.from_numpy(d).cuda()
    sf = torch.empty((sr, st), dtype=torch.float32, device="cuda")
    t = _time_ms(torch, stream, lambda: dt.splat_device(dd.data_ptr(), len(d), sf.data_ptr(), sid, **sc))
    out["splat"] = {"workload": "DepoFluxSplat frame of %d depos, %d x %d" % (len(d), sr, st), "ms": t,
                    "depos_per_s": len(d) / (t / 1e3)}
    # noise + digitizer on the full frame
    frame = torch.zeros((nrows, nticks), dtype=torch.float32, device="cuda")
    k = np.arange(nticks)
    f = np.minimum(k, nticks - k).astype(np.float64)
    spec = np.stack([(0.02 + 0.05 * np.exp(-((f - 300.0 * (p + 1)) / 400.0) ** 2)) * 1e-6 for p in range(3)])
    dspec = torch.from_numpy(spec.astype(np.float32)).cuda()
    row_spec = torch.from_numpy(np.concatenate([np.full(p["nwires"], i, np.int32)
                                                for i, p in enumerate(cfg["planes"])])).cuda()
    row_stream = torch.arange(nrows, dtype=torch.int32, device="cuda")
    t_n = _time_ms(torch, stream, lambda: wct.add_noise_device(frame.data_ptr(), nticks, nrows, nticks,
                                                               dspec.data_ptr(), nticks, row_spec.data_ptr(),
                                                               row_stream.data_ptr(), seed=1, stream=sid))
    dz = wct.Digitizer([p["nwires"] for p in cfg["planes"]], round=True)
    base = torch.from_numpy(dz.row_baseline).cuda()
    adc = torch.empty_like(frame)
    t_d = _time_ms(torch, stream, lambda: dz.device(frame.data_ptr(), nticks, nrows, nticks, base.data_ptr(),
                                                    adc.data_ptr(), nticks, stream=sid))
    fb = nrows * nticks * 4
    out["noise"] = {"workload": "incoherent noise on %d x %d" % (nrows, nticks), "ms": t_n,
                    "gbs": 2 * fb / (t_n / 1e3) / 1e9, "peak_gbs": peak, "peak_kind": kind}
    out["digitizer"] = {"workload": "Digitizer on %d x %d" % (nrows, nticks), "ms": t_d,
                        "gbs": 2 * fb / (t_d / 1e3) / 1e9, "frac": 2 * fb / (t_d / 1e3) / 1e9 / peak,
                        "peak_gbs": peak, "peak_kind": kind}
    # IDFT: 2-D forward transforms
    for (nr, nc) in ((1024, 1024), (2560, 6000)):
        x = torch.randn((nr, nc), dtype=torch.complex64, device="cuda")
        y = torch.empty_like(x)
        t2 = _time_ms(torch, stream, lambda: wct.dft_2d_device(x.data_ptr(), y.data_ptr(), nr, nc, stream=sid))
        n = nr * nc
        out["idft_2d_%dx%d" % (nr, nc)] = {"ms": t2, "gflops_5nlog2n": 5 * n * np.log2(n) / (t2 / 1e3) / 1e9}
        del x, y
    return out


def calibration(wct, synth, torch, local, nevents=16, ndepos=4_000_000, steps=20):
    """Large batched calibration: nevents events of ndepos depos (cosmic muons +
    exponential-spectrum showers, mean 1 GeV), targets drawn with fluctuation
    on (patch cells and drift) at DL x 0.9, DT x 1.1, lifetime 8 ms, then
    gradient-descent steps of DL, DT, lifetime (batched mean forward + adjoint
    of every event per step), timed with CUDA events."""
    cal = importlib.import_module("wire-cell-toolkit_b200.calibrate")
    cfg = synth.apa_config()
    dr = cfg["drifter"]
    truth = (dr["DL"] * 0.9, dr["DT"] * 1.1, 8.0e6)
    t0 = time.perf_counter()
    events = synth.calibration_events(nevents, ndepos)
    t_gen = time.perf_counter() - t0
    off = np.zeros(nevents + 1, dtype=np.int64)
    off[1:] = np.cumsum([len(e) for e in events])
    d = torch.from_numpy(np.concatenate(events)).to("cuda")
    del events
    gen = wct.from_config(dict(cfg, fluctuate=True, seed=5, drifter=dict(dr, fluctuate=True)), device=local)
    gen.set_drift_params(*truth)
    nrows, nticks = gen.frame_shape()
    targets = torch.zeros((nevents, nrows, nticks), dtype=torch.float32, device="cuda")
    s = torch.cuda.Stream()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(s)
    gen.forward_batch_device(d.data_ptr(), off, targets.data_ptr(), stream=s.cuda_stream)
    b.record(s)
    b.synchronize()
    t_target = a.elapsed_time(b)
    del gen
    model = wct.from_config(cfg, device=local)
    marks = []

    def cb(it, p, loss, g):
        ev = torch.cuda.Event(enable_timing=True)
        ev.record(s)
        marks.append(ev)

    hist, final = cal.fit_drift_params(model, d, off, targets, steps=steps, lr=0.05, stream=s, callback=cb)
    torch.cuda.synchronize()
    per_step = [marks[k].elapsed_time(marks[k + 1]) for k in range(len(marks) - 1)]
    ms_step = float(statistics.median(per_step)) if per_step else None
    ndep = int(off[-1])
    out = {
        "workload": "%d full-APA events x %d depos (cosmic muons + showers, exponential spectrum of mean 1 GeV); "
                    "targets with patch and drift fluctuation at DL x 0.9, DT x 1.1, lifetime 8 ms; fit of "
                    "DL, DT, lifetime by batched forward + per-event adjoint, Adam in log space" % (nevents, ndepos),
        "depos": ndep, "generation_s": t_gen, "fluctuated_target_ms": t_target,
        "fluctuated_depos_per_s": ndep / (t_target / 1e3),
        "ms_per_fit_step": ms_step,
        "fwd_adj_depos_per_s": ndep / (ms_step / 1e3) if ms_step else None,
        "loss_first": hist[0][2], "loss_last": hist[-1][2],
        "params_start": list(hist[0][1]), "params_final": list(final), "params_truth": list(truth)}
    del d, targets
    torch.cuda.empty_cache()
    return out


def host_cpu():
    """Model name and logical core count of this host."""
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"model": model, "logical_cores": os.cpu_count()}


def cpu_baseline(cfg, depos, gpu_frame=None, gpu_windows=None, timed=True, reps=5):
    """The CPU restatement of the reference (oracle/, FP32) on the bench's own
    full event, one thread: its transforms through libtorch-CPU (Intel MKL),
    the reference's TorchDFT backend, the plane responses built once as the
    reference's configured PlaneImpactResponse is; one warm-up run, then the
    median of `reps` runs, split into the reference's stages.  Also the
    checker of this event: the FP64 oracle's frame against the GPU frame
    (rel-L2, windows), outside every timed region.  Returns (baseline or
    None when not timed, parity)."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.lib()
    parity = None
    if gpu_frame is not None:
        ref = O.run(cfg, depos, fp64=True, nthreads=min(3, os.cpu_count() or 1))
        r = np.concatenate(ref["frames"])
        g = gpu_frame.astype(np.float64)
        keys = ("start_ch", "end_ch", "start_tick", "end_tick", "ndepos_added", "outside_time", "outside_pitch")
        same = all(all(w[k] == o[k] for k in keys) for w, o in zip(gpu_windows, ref["windows"]))
        parity = {"rel_l2_vs_fp64": float(np.linalg.norm(g - r) / np.linalg.norm(r)), "tolerance": 1e-5,
                  "windows_and_counters_equal": bool(same),
                  "event": "the benchmarked event (%d depos), last timed step's frame" % len(depos)}
    if not timed:
        return None, parity
    nth0 = torch.get_num_threads()
    torch.set_num_threads(1)
    O.set_fft_backend("mkl")
    try:
        O.run(cfg, depos, nthreads=1)  # warm-up: plane responses, transform plans
        runs = []
        for _ in range(reps):
            t0 = time.perf_counter()
            res = O.run(cfg, depos, nthreads=1, stages=True)
            runs.append((time.perf_counter() - t0, res["stages"]))
    finally:
        O.set_fft_backend("own")
        torch.set_num_threads(nth0)
    med = statistics.median(t for t, _ in runs)
    stages = {k: statistics.median(st[k] for _, st in runs) for k in O.STAGES}
    return ({"value": len(depos) / med, "unit": UNIT, "cores": 1, "kind": "port",
             "sample": "the benchmarked event (%d depos), FP32 restatement, one thread; transforms by "
                       "libtorch-CPU (MKL, the reference's TorchDFT backend); plane responses built once; 1 warm-up, "
                       "median of %d runs (%.2f s)" % (len(depos), reps, med),
             "seconds_median": med, "seconds_runs": [t for t, _ in runs],
             "stages_s_median": stages, "host_cpu": host_cpu()}, parity)


def run_reference(args):
    rank, world, local = dist_setup(args)
    if rank != 0:
        return
    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.lib()
    # transforms through libtorch-CPU (MKL), the reference's TorchDFT backend;
    # one intra-op thread per call, the parallelism is over planes and events
    torch.set_num_threads(1)
    O.set_fft_backend("mkl")
    synth = importlib.import_module("wire-cell-toolkit_b200.synth")
    if args.workload == "plane":
        cfg, depos = synth.plane1_config(), synth.plane1_depos(seed=1)
    else:
        cfg, depos = synth.apa_config(), synth.apa_depos(seed=2)
    # every host core: each event's planes on their own threads, and as many
    # independent events at once as the remaining cores take (events share
    # nothing, as they do in the reference), bounded by a quarter of the free
    # host memory at ~0.7 GB per event in flight
    ncpu = os.cpu_count() or 1
    nth = max(1, min(len(cfg["planes"]), ncpu))
    nev = max(1, ncpu // nth)
    try:
        import psutil
        nev = max(1, min(nev, int(psutil.virtual_memory().available * 0.25 // (700 << 20))))
    except Exception:
        nev = min(nev, 4)
    nev = min(nev, 64)
    import concurrent.futures as cf
    pool = cf.ThreadPoolExecutor(nev)  # the oracle's C call releases the GIL

    def step():
        list(pool.map(lambda _: O.run(cfg, depos, nthreads=nth), range(nev)))

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = time.perf_counter() - t0
    pool.shutdown()
    value = len(depos) * nev * args.steps / dt
    sample = ("%d events (%d depos each) at once per step, FP32 restatement, each event's planes on %d "
              "threads, transforms by libtorch-CPU (MKL), plane responses built once" % (nev, len(depos), nth))
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD_TEXT[args.workload] % len(depos)},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nth * nev, "kind": "port", "sample": sample,
                         "host_cpu": host_cpu()},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-patterns", action="store_true", help="skip the adjoint / batched / fluctuated lines")
    ap.add_argument("--no-calibration", action="store_true", help="skip the large batched calibration")
    ap.add_argument("--workload", default="apa", choices=["apa", "plane"],
                    help="apa: the full-APA event (default); plane: the single collection-plane workload")
    ap.add_argument("--depos", type=int, default=0,
                    help="time only the event's first DEPOS depos (a small case for profilers); 0: the whole event")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.gpus < 1:
        raise SystemExit("bench.py: --gpus must be at least 1")
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # one process per GPU: start the ranks here when no launcher did
        sys.exit(relaunch(args.gpus, os.path.abspath(__file__), sys.argv[1:]))
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
