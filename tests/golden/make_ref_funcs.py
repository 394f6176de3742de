"""Generate tests/golden/ref_funcs.json from reference code compiled here:
GausDesc::binint / weight / distance (gen/src/GaussianDiffusion.cxx:30-92,
gen/inc/WireCellGen/GaussianDiffusion.h:33-49), Waveform::edge
(util/src/Waveform.cxx:136-153), Response::coldelec
(util/src/Response.cxx:311-340), Pimpos (util/src/Pimpos.cxx:5-68),
Digitizer::digitize (gen/src/Digitizer.cxx:77-93), EmpiricalNoiseModel's
resampling (gen/src/EmpiricalNoiseModel.cxx:55-147), GroupNoiseModel's
spectra (gen/src/GroupNoiseModel.cxx:97-146), Drifter::insert
(gen/src/Drifter.cxx:127-196) and BinnedDiffusion_transform::add
(gen/src/BinnedDiffusion_transform.cxx:37-92), from
oracle/_ref/libref_funcs.so (built by
oracle/Makefile with extract_ref.py and ref_funcs_harness.cpp).

Run from the repository root:  python tests/golden/make_ref_funcs.py"""

import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

US = 1000.0  # ns


def gausdesc_cases(rng, n):
    """Bin ranges as GaussianDiffusion::set_sampling takes them: the bins
    covering +-nsigma around the centre on a grid of the given step."""
    out = []
    for k in range(n):
        center = float(rng.uniform(-100.0, 100.0))
        step = float(rng.uniform(0.1, 5.0))
        if k % 10 == 0:
            sigma, nbins = 0.0, 1
            start = center - float(rng.uniform(0.0, step))
        else:
            sigma = float(np.exp(rng.uniform(np.log(1e-2), np.log(50.0))))
            nsig = float(rng.choice([1.0, 3.0, 5.0]))
            lo = center - nsig * sigma
            start = np.floor(lo / step) * step
            nbins = int(np.ceil((center + nsig * sigma - start) / step))
            nbins = max(1, min(nbins, 120))
        out.append(dict(center=center, sigma=sigma, start=float(start), step=step, nbins=nbins,
                        x=float(center + rng.normal() * (sigma or 1.0))))
    return out


def pimpos_cases(rng, n):
    """Wire planes as AnodePlane builds Pimpos (gen/src/AnodePlane.cxx:200-219):
    wire directions at an angle in the (y, z) plane, the pitch direction
    normal to it (not always unit length), and points in a 2.5 m x 6 m x 2.3 m
    volume."""
    out = []
    for k in range(n):
        ang = float(rng.choice([0.0, 35.7, -35.7, 60.0])) if k % 4 else float(rng.uniform(-90.0, 90.0))
        a = np.radians(ang)
        wire = [0.0, float(np.cos(a)), float(np.sin(a))]
        s = float(rng.choice([1.0, 3.0, 0.25]))
        pitch = [0.0, float(-np.sin(a) * s), float(np.cos(a) * s)]
        nw = int(rng.integers(2, 1200))
        pw = float(rng.uniform(3.0, 5.0))
        minp = float(-0.5 * pw * (nw - 1) + rng.uniform(-10.0, 10.0))
        pts = np.column_stack([rng.uniform(-50.0, 2500.0, 20), rng.uniform(-3000.0, 3000.0, 20),
                               rng.uniform(-1150.0, 1150.0, 20)])
        out.append(dict(nwires=nw, minp=minp, maxp=minp + pw * (nw - 1), wire=wire, pitch=pitch,
                        origin=[float(rng.uniform(-10.0, 100.0)), 0.0, float(rng.uniform(-5.0, 5.0))],
                        nbins=int(rng.choice([10, 6, 20])), pts=pts.tolist()))
    return out


def main():
    O.build()
    R = O.ref_funcs()
    if R is None:
        raise SystemExit("reference function harness not built (reference tree absent)")
    rng = np.random.default_rng(2024)
    gd = []
    for c in gausdesc_cases(rng, 100):
        b = O.gd_binint(R, "ref", c["center"], c["sigma"], c["start"], c["step"], c["nbins"])
        w = O.gd_weight(R, "ref", c["center"], c["sigma"], c["start"], c["step"], len(b), b)
        d = R.ref_gd_distance(c["center"], c["sigma"], c["x"])
        gd.append(dict(c, binint=[float(v) for v in b], weight=[float(v) for v in w], distance=d))

    edges = []
    for k in range(60):
        n = int(rng.integers(0, 120))
        w = rng.normal(size=n).astype(np.float32)
        w[rng.random(n) < rng.uniform(0.0, 1.0)] = 0.0
        if n and k % 3 == 0:
            a, b = sorted(rng.integers(0, n, 2))
            w[:a] = 0.0
            w[b:] = 0.0
        if n and k % 7 == 0:
            w[rng.random(n) < 0.3] = -0.0
        out = np.zeros(2, dtype=np.int32)
        R.ref_wave_edge(w.ctypes.data, n, out.ctypes.data)
        edges.append(dict(wave=[float(v) for v in w], edge=[int(out[0]), int(out[1])]))

    cold = []
    times = list(np.linspace(-1.0, 12.0, 131) * US) + [0.0, 10.0 * US, 10.0 * US - 1e-9]
    for gain in (7.8, 14.0):
        for shaping in (0.5 * US, 1.0 * US, 2.0 * US, 3.0 * US):
            cold.append(dict(gain=gain, shaping=shaping, time=[float(t) for t in times],
                             value=[R.ref_coldelec(float(t), gain, shaping) for t in times]))

    digi = []
    drng = np.random.default_rng(31)
    volt = 1.0e-6
    for gain, resolution in ((1.0, 12), (2.5, 14), (0.7, 10)):
        for rnd in (0, 1):
            f = drng.normal(0.0, 0.4 * volt, (8, 24)).astype(np.float32)
            f[0, :5] = [-5 * volt, 5 * volt, 0.0, 1.1 * volt, -0.9 * volt]
            base = (np.array([0.9, 0.9, 0.9, 0.9, 0.2, 0.2, 0.2, 0.2]) * volt).astype(np.float32)
            adc = np.zeros_like(f)
            R.ref_digitize(f.ctypes.data, f.shape[0], f.shape[1], base.ctypes.data, gain, 0.0, 2.0 * volt, resolution,
                           rnd, adc.ctypes.data)
            digi.append(dict(gain=gain, resolution=resolution, round=rnd, fullscale=[0.0, 2.0 * volt],
                             baseline=[float(v) for v in base], frame=f.astype(float).tolist(),
                             adc=adc.astype(float).tolist()))

    nm = []
    nrng = np.random.default_rng(55)
    us = 1000.0
    for nsamples, period, model_n, kind in ((256, 0.5 * us, 600, "line"), (128, 0.4 * us, 400, "random"),
                                            (300, 0.5 * us, 500, "inner"), (0, 0.5 * us, 200, "same"),
                                            (200, 1.0 * us, 560, "random")):
        L = O.fft_best_length(model_n)
        nyq = 1.0 / (2 * period)
        if kind == "line":
            freqs = np.linspace(0.0, nyq, nsamples // 2 + 1)
        elif kind == "inner":  # the model grid reaches past both ends: clamped
            freqs = np.linspace(0.1 * nyq, 0.8 * nyq, 50)
        elif kind == "same":  # the model's own sampling: kept as given
            nsamples = L
            freqs = np.linspace(0.0, nyq, L)
        else:
            freqs = np.sort(nrng.uniform(0.0, nyq, 40))
        amps = nrng.uniform(0.2, 3.0, len(freqs))
        ent = dict(nsamples=nsamples, period=period, const=float(nrng.uniform(0.0, 0.1)),
                   freqs=[float(v) for v in np.float32(freqs)], amps=[float(v) for v in np.float32(amps)])
        const, out = O.ref_noise_resample(R, L, period, ent)
        nm.append(dict(ent, model_nsamples=model_n, model_period=period, fft_length=L, const_out=const,
                       amps_out=[float(v) for v in out]))

    grp = []
    grng = np.random.default_rng(91)
    for porig, norig, ns, tick in ((500.0, 256, 300, 500.0), (500.0, 400, 150, 1000.0), (400.0, 300, 200, 250.0),
                                   (512.0, 128, 128, 512.0), (500.0, 333, 257, 800.0), (500.0, 200, 301, 200.0)):
        nf = int(grng.integers(5, 60))
        f = np.sort(grng.uniform(0.0, 1.2 / (2 * porig), nf)).astype(np.float32)
        f[0] = 0.0
        a = grng.uniform(0.0, 3.0, nf).astype(np.float32)
        out = O.ref_group_spectrum(R, f, a, norig, porig, ns, tick, 1.5)
        grp.append(dict(freqs=[float(v) for v in f], amps=[float(v) for v in a], nsamples_orig=norig,
                        period_orig=porig, nsamples=ns, tick=tick, scale=1.5, spectrum=[float(v) for v in out]))

    pim = []
    prng = np.random.default_rng(77)
    for c in pimpos_cases(prng, 12):
        head, dist = O.pimpos(R, "ref", c["nwires"], c["minp"], c["maxp"], c["wire"], c["pitch"], c["origin"],
                              c["nbins"], c["pts"])
        pim.append(dict(c, head=[float(v) for v in head], dist=[float(v) for v in dist]))

    drift = []
    for c in O.drift_cases(np.random.default_rng(13), 120):
        k, o = O.drift_one(R, "ref", c)
        drift.append(dict(c, kept=int(k), out=[float(v) for v in o]))
    bdt = []
    for c in O.bdt_add_cases(np.random.default_rng(17), 200):
        k, cnt = O.bdt_add(R, "ref", c)
        bdt.append(dict(c, added=int(k), counters=cnt))

    out = {"source": ["gen/src/GaussianDiffusion.cxx", "util/src/Waveform.cxx", "util/src/Response.cxx",
                      "util/src/Pimpos.cxx", "gen/src/Digitizer.cxx", "gen/src/EmpiricalNoiseModel.cxx",
                      "gen/src/GroupNoiseModel.cxx", "gen/src/Drifter.cxx", "gen/src/BinnedDiffusion_transform.cxx"],
           "gausdesc": gd, "edge": edges, "coldelec": cold, "pimpos": pim, "digitize": digi, "noise_resample": nm,
           "group_spectrum": grp, "drift": drift, "bdt_add": bdt}
    with open(os.path.join(ROOT, "tests", "golden", "ref_funcs.json"), "w") as f:
        json.dump(out, f)
    print("%d GausDesc cases, %d edges, %d coldelec curves, %d planes, %d digitizer frames, %d noise spectra, "
          "%d group spectra, %d drifted depos, %d add decisions" % (len(gd), len(edges), len(cold), len(pim),
                                                                    len(digi), len(nm), len(grp), len(drift),
                                                                    len(bdt)))


if __name__ == "__main__":
    main()
