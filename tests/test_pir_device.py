"""PlaneImpactResponse::build_responses on the GPU
(gen/src/PlaneImpactResponse.cxx:89-269): the reference's single-precision
chain (field response binned onto ticks, spectrum x short-response spectrum,
real inverse; long responses as a spectrum product) through the library's
transforms.  Against the host build (double-precision direct circular
convolution) and the oracle's FP32 restatement of the reference build, with
the same grouping; frames built on either PIR agree.  Host and device build
times are printed (and logged with WCT_PARITY_LOG)."""

import time

import numpy as np
import pytest

from conftest import parity_log, rel_l2

pytestmark = pytest.mark.gpu


def _pirs(wct, cfg, ip, longs=()):
    args = (cfg["fr"][ip], cfg.get("short_responses", []), cfg["overall_short_padding"], cfg["tick"],
            cfg["pir_nticks"])
    t0 = time.perf_counter()
    host = wct.PlaneImpactResponse(*args, long_responses=longs)
    t1 = time.perf_counter()
    dev = wct.PlaneImpactResponse(*args, long_responses=longs, device=True)
    t2 = time.perf_counter()
    return host, dev, t1 - t0, t2 - t1


@pytest.mark.parametrize("ip", [0, 2])
def test_device_build_matches_host_and_oracle(wct, oracle, synth, ip):
    cfg = synth.apa_config()
    _pirs(wct, cfg, ip)  # warm: transform plans, context
    host, dev, th, td = _pirs(wct, cfg, ip)
    assert dev.info() == host.info()
    n = host.info()["npaths"]
    wh = np.stack([host.waveform(p) for p in range(n)])
    wd = np.stack([dev.waveform(p) for p in range(n)])
    e = rel_l2(wd, wh)
    assert e < 1e-6, e
    for r in (-30.0, -2.4, 0.0, 1.1, 17.3):
        assert dev.closest(r) == host.closest(r)
    # the oracle's FP32 restatement of the reference build
    ob = oracle.pir_build(cfg, ip, fp64=False)
    eo = rel_l2(wd, ob["waveforms"][:, :wd.shape[1]])
    assert eo < 1e-5, eo
    entry = {"pir_build": "plane %d, %d paths, %d ticks" % (ip, n, wh.shape[1]), "host_s": th, "device_s": td,
             "rel_l2_device_vs_host_fp64": e, "rel_l2_device_vs_oracle_fp32": eo}
    print(entry)
    parity_log(entry)


def test_device_long_responses(wct, synth):
    cfg = synth.plane1_config(nticks=2000)
    k = -0.004 * np.exp(-np.arange(2500) / 400.0)
    k[0] = 1.0
    host, dev, _, _ = _pirs(wct, cfg, 0, longs=[k, k[:700]])
    lh, ph = host.long_waveform()
    ld, pd = dev.long_waveform()
    assert ph == pd and len(lh) == len(ld) > 0
    assert rel_l2(ld, lh) < 1e-6


def test_frames_on_device_built_pir(wct, synth):
    cfg = synth.apa_config(nticks=6000)
    d = synth.apa_depos(seed=3)[:50_000]
    a = wct.from_config(cfg)
    fa, _, _ = a(d)
    b = wct.DepoTransform({k: cfg[k] for k in ("tick", "start_time", "readout_time", "drift_speed", "nsigma")}
                          | {"drifter": wct.drifter_json(cfg["drifter"])})
    face = b.add_face(cfg["face_bb"])
    for pl, fr in zip(cfg["planes"], cfg["fr"]):
        p = b.add_plane(face, pl)
        b.set_response_pir(face, p, wct.PlaneImpactResponse(fr, cfg["short_responses"], cfg["overall_short_padding"],
                                                            cfg["tick"], cfg["pir_nticks"], device=True))
    fb, _, _ = b(d)
    assert rel_l2(fb, fa) < 1e-6
