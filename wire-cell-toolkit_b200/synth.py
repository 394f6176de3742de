"""Seeded synthetic inputs for the DepoTransform workloads.

The reference is exercised on detector field-response files and depo samples
from the external wire-cell-data repository, which are not available here.
These generators build stand-ins with the shapes, sizes and value
distributions of the five workloads:

* ``plane1``   one collection plane, 960 wires, 2 000 point depos;
* ``apa``      a full three-plane APA face with 20 straight muon tracks;
* ``batch``    many events of APA geometry with uneven depo counts;
* ``adjoint``  APA geometry with 20k track depos and a perturbed target;
* ``calib``    large events with cosmic tracks and EM showers.

Everything is in the Wire-Cell system of units (util/inc/WireCellUtil/Units.h:
mm = 1, ns = 1, positron charge = 1, megavolt = 1).

The field response follows the Response::Schema layout
(util/inc/WireCellUtil/Response.h:28-110, util/src/Response.cxx:32-72) with the
path ordering PlaneImpactResponse expects (gen/src/PlaneImpactResponse.cxx:155-174):
six paths per wire region, from half a pitch below the wire up to the wire,
in increasing pitch.
"""

import math
import numpy as np

# Units (util/inc/WireCellUtil/Units.h)
mm = 1.0
cm = 10.0
m = 1000.0
ns = 1.0
us = 1000.0
ms = 1.0e6
second = 1.0e9
volt = 1.0e-6
mV = 1.0e-3 * volt
fC = 1.0e-15 / 1.602176487e-19
cm2_per_s = cm * cm / second

TICK = 0.5 * us


def elec_crrc2(gain=14.0 * mV / fC, peaking=2.0 * us, tick=TICK, nsamples=200):
    """CR-RC^2 shaper response to a unit-charge impulse, peak value ``gain``
    at ``peaking``, sampled at tick centres (util/src/Response.cxx:277-286)."""
    t = (np.arange(nsamples) + 0.5) * tick
    x = t / peaking
    return gain * x * x * np.exp(2.0 * (1.0 - x))


def field_response(pitch, nwire_half=21, kind="collection", sigma=2.0 * us, t_peak=50.0 * us,
                   period=0.1 * us, nsamples=1000):
    """Synthetic per-path induced currents for one plane.

    Paths: for relative wire k in [-nwire_half, nwire_half], six impact
    positions (k - 0.5 + m/10) * pitch, m = 0..5.  The current at pitch
    position p is a Gaussian pulse (collection) or its time derivative
    (induction) scaled by exp(-|p/pitch|/2), so it is mirror symmetric in p
    as the reference's response symmetrisation assumes.
    Returns dict(pitchpos[npaths], current[npaths][nsamples], pitch, tstart, period).
    """
    pp = []
    # A common offset of 1e-9 pitch keeps every path robustly inside its wire
    # region under the reference's ceil() grouping
    # (gen/src/PlaneImpactResponse.cxx:186-201), which is otherwise sensitive
    # to the last bit of k * pitch.
    nudge = 1e-9 * pitch
    for k in range(-nwire_half, nwire_half + 1):
        for mm_ in range(6):
            pp.append((k - 0.5 + mm_ / 10.0) * pitch - nudge)
    pp = np.array(pp, dtype=np.float64)
    t = (np.arange(nsamples) + 0.5) * period
    u = (t - t_peak) / sigma
    g = np.exp(-0.5 * u * u) / (sigma * math.sqrt(2.0 * math.pi))
    if kind == "collection":
        shape = g
    else:
        shape = -u * g * 1.5
    cur = np.exp(-np.abs(pp / pitch) / 2.0)[:, None] * shape[None, :]
    return dict(pitchpos=pp, current=np.ascontiguousarray(cur), pitch=float(pitch), tstart=0.0,
                period=float(period))


def _plane(nwires, pitch, angle_deg, ident, channel0, response_x):
    a = math.radians(angle_deg)
    wire = (0.0, math.cos(a), -math.sin(a))
    pdir = (0.0, math.sin(a), math.cos(a))
    half = 0.5 * pitch * (nwires - 1)
    return dict(ident=ident, nwires=nwires, pitchmin=-half, pitchmax=half, wire=wire, pitch=pdir,
                origin=(response_x, 0.0, 0.0), nimp=10,
                channels=np.arange(channel0, channel0 + nwires, dtype=np.int32), wire_pitch=pitch)


DRIFT = dict(DL=7.2 * cm2_per_s, DT=12.0 * cm2_per_s, lifetime=10.0 * ms, drift_speed=1.6 * mm / us,
             time_offset=0.0)
ANODE_X, RESPONSE_X, CATHODE_X = 0.0, 100.0 * mm, 2700.0 * mm


def base_config(nticks=6000, planes=None, fr_kinds=None, nwire_half=21):
    """DepoTransform + Drifter + PIR configuration dict shared by all workloads."""
    cfg = dict(
        tick=TICK,
        start_time=0.0,
        readout_time=nticks * TICK,
        drift_speed=1.6 * mm / us,
        nsigma=3.0,
        fluctuate=False,
        first_frame_number=0,
        drifter=dict(DRIFT, xregions=[(ANODE_X, RESPONSE_X, CATHODE_X)]),
        face_bb=((ANODE_X, -3000.0 * mm, -2300.0 * mm), (CATHODE_X, 3000.0 * mm, 2300.0 * mm)),
        planes=planes,
        overall_short_padding=100.0 * us,
        pir_nticks=nticks,
        short_responses=[elec_crrc2()],
    )
    frs = []
    for pl, kind in zip(planes, fr_kinds):
        frs.append(field_response(pl["wire_pitch"], nwire_half=nwire_half, kind=kind))
    cfg["fr"] = frs
    return cfg


def plane1_config(nticks=6000, nwire_half=21):
    planes = [_plane(960, 4.79 * mm, 0.0, 2, 0, RESPONSE_X)]
    return base_config(nticks, planes, ["collection"], nwire_half)


def apa_config(nticks=6000, nwire_half=21):
    planes = [
        _plane(800, 4.67 * mm, 35.7, 0, 0, RESPONSE_X),
        _plane(800, 4.67 * mm, -35.7, 1, 800, RESPONSE_X),
        _plane(960, 4.79 * mm, 0.0, 2, 1600, RESPONSE_X),
    ]
    return base_config(nticks, planes, ["induction", "induction", "collection"], nwire_half)


def apa2_config(nticks=6000, nwire_half=21):
    """A two-face APA: face 0 drifts from x = +2700 mm to its response plane
    at +100 mm, face 1 from -2700 mm to -100 mm, the wire planes at x = 0
    between them (one Drifter x-region per face).  Face 1 sees the
    induction wires wrapped around the frame: its U and V wires run at the
    mirrored angles and keep the channel numbers of face 0's U and V (a
    channel then has a trace from each face, as in the reference's frame);
    its collection plane has channels of its own.  pirs are per plane index
    and shared by the faces (DepoTransform.cxx:188)."""
    f0 = [
        _plane(800, 4.67 * mm, 35.7, 0, 0, RESPONSE_X),
        _plane(800, 4.67 * mm, -35.7, 1, 800, RESPONSE_X),
        _plane(960, 4.79 * mm, 0.0, 2, 1600, RESPONSE_X),
    ]
    f1 = [
        _plane(800, 4.67 * mm, -35.7, 0, 0, -RESPONSE_X),
        _plane(800, 4.67 * mm, 35.7, 1, 800, -RESPONSE_X),
        _plane(960, 4.79 * mm, 0.0, 2, 2560, -RESPONSE_X),
    ]
    cfg = base_config(nticks, f0 + f1, ["induction", "induction", "collection"] * 2, nwire_half)
    cfg["fr"] = cfg["fr"][:3] * 2  # the same response objects: one PIR per plane index
    cfg["drifter"]["xregions"] = [(ANODE_X, RESPONSE_X, CATHODE_X), (ANODE_X, -RESPONSE_X, -CATHODE_X)]
    cfg["faces"] = [
        dict(bb=((ANODE_X, -3000.0 * mm, -2300.0 * mm), (CATHODE_X, 3000.0 * mm, 2300.0 * mm)), planes=[0, 1, 2]),
        dict(bb=((-CATHODE_X, -3000.0 * mm, -2300.0 * mm), (ANODE_X, 3000.0 * mm, 2300.0 * mm)), planes=[3, 4, 5]),
    ]
    cfg.pop("face_bb", None)
    return cfg


def apa2_depos(seed=6, ntracks=8, step=0.5 * mm):
    """Muon tracks through both drift volumes of the two-face APA (some cross
    the wire planes at x = 0)."""
    rng = np.random.default_rng(seed)
    return track_depos(rng, ntracks=ntracks, step=step, lo=(-RESPONSE_X - 2500.0, -3000.0, -1150.0),
                       hi=(RESPONSE_X + 2500.0, 3000.0, 1150.0))


def plane1_depos(n=2000, seed=1, charge=-5000.0, span=4.6 * m, drift=2.5 * m):
    """Point depos uniform in the wire (pitch) coordinate over ``span`` from the
    first wire region edge and in drift distance over [0, drift]."""
    rng = np.random.default_rng(seed)
    pitch = 4.79 * mm
    pmin = -0.5 * pitch * 960
    z = pmin + rng.uniform(0.0, span, n)
    x = RESPONSE_X + rng.uniform(0.0, drift, n)
    d = np.zeros((n, 7))
    d[:, 0] = 0.0
    d[:, 1] = charge
    d[:, 2] = x
    d[:, 3] = 0.0
    d[:, 4] = z
    return d


def moyal(rng, n):
    """Standard Moyal variates (a Landau approximation): -ln(Z^2), Z ~ N(0,1)."""
    z = rng.standard_normal(n)
    return -np.log(z * z + 1e-300)


def track_depos(rng, ntracks=20, step=0.1 * mm, lo=None, hi=None, dedx_mpv=2.1, dedx_width=0.1,
                wion=23.6e-6, recomb=0.7, t0=0.0, max_depos=None):
    """Straight tracks with endpoints uniform in [lo, hi], one depo per ``step``,
    charge from Moyal-distributed dE/dx (MeV/cm) -> electrons."""
    lo = np.array(lo if lo is not None else (RESPONSE_X, -3000.0, -1150.0))
    hi = np.array(hi if hi is not None else (RESPONSE_X + 2500.0, 3000.0, 1150.0))
    out = []
    for _ in range(ntracks):
        a = lo + (hi - lo) * rng.random(3)
        b = lo + (hi - lo) * rng.random(3)
        length = float(np.linalg.norm(b - a))
        n = max(1, int(length / step))
        s = (np.arange(n) + 0.5) / n
        pos = a[None, :] + s[:, None] * (b - a)[None, :]
        dedx = np.clip(dedx_mpv + dedx_width * moyal(rng, n), 0.2, 200.0)  # MeV/cm
        de = dedx * (step / cm)  # MeV
        q = -(de / wion) * recomb
        d = np.zeros((n, 7))
        d[:, 0] = t0
        d[:, 1] = q
        d[:, 2:5] = pos
        out.append(d)
    d = np.concatenate(out, axis=0)
    if max_depos is not None and len(d) > max_depos:
        d = d[:max_depos]
    return d


def apa_depos(seed=2, ntracks=20):
    rng = np.random.default_rng(seed)
    return track_depos(rng, ntracks=ntracks)


def shower_depos(rng, n, center=None, radius=300.0 * mm, energy_mev=1000.0, ext_long_max=26.0 * mm,
                 ext_tran_max=2.4 * mm):
    """A Gaussian blob of n depos around ``center`` carrying ``energy_mev``, with
    initial extents uniform up to ``ext_long_max`` along the drift and
    ``ext_tran_max`` across it: with diffusion over 0-2.5 m of drift the patches
    span from ~3 x 10 up to ~40 impact bins x ~200 ticks."""
    if center is None:
        center = np.array([RESPONSE_X + rng.uniform(200, 2300), rng.uniform(-2500, 2500), rng.uniform(-900, 900)])
    pos = center[None, :] + rng.normal(0.0, radius / 3.0, (n, 3))
    pos[:, 0] = np.clip(pos[:, 0], RESPONSE_X + 1.0, CATHODE_X - 1.0)
    e = rng.exponential(1.0, n)
    e *= energy_mev / e.sum()
    d = np.zeros((n, 7))
    d[:, 1] = -(e / 23.6e-6) * 0.7
    d[:, 2:5] = pos
    d[:, 5] = rng.uniform(0.0, ext_long_max, n)
    d[:, 6] = rng.uniform(0.0, ext_tran_max, n)
    return d


def batch_events(nevents=64, seed=3, lo=10_000, hi=500_000):
    """Events of APA geometry with log-uniform depo counts in [lo, hi], each a
    mix of tracks and shower blobs."""
    rng = np.random.default_rng(seed)
    events = []
    for _ in range(nevents):
        n = int(math.exp(rng.uniform(math.log(lo), math.log(hi))))
        ntr = int(n * 0.6)
        tr = track_depos(rng, ntracks=max(1, ntr // 20000 + 1), max_depos=ntr)
        nsh = n - len(tr)
        parts = [tr]
        while nsh > 0:
            k = min(nsh, int(rng.integers(2000, 20000)))
            parts.append(shower_depos(rng, k, energy_mev=float(rng.exponential(1000.0)) + 10.0))
            nsh -= k
        events.append(np.ascontiguousarray(np.concatenate(parts, axis=0)))
    return events


def adjoint_depos(seed=4, n=20_000, ntracks=20):
    """APA-geometry track depos with the step chosen so that the 20 tracks hold
    ``n`` depos in total."""
    rng = np.random.default_rng(seed)
    probe = np.random.default_rng(seed)
    lo = np.array((RESPONSE_X, -3000.0, -1150.0))
    hi = np.array((RESPONSE_X + 2500.0, 3000.0, 1150.0))
    total = 0.0
    for _ in range(ntracks):
        a = lo + (hi - lo) * probe.random(3)
        b = lo + (hi - lo) * probe.random(3)
        total += float(np.linalg.norm(b - a))
        probe.standard_normal(1)
    step = total / n
    d = track_depos(rng, ntracks=ntracks, step=step, lo=lo, hi=hi)
    return d[:n]


def cosmic_depos(rng, ntracks, step=0.1 * mm, t0_spread=0.0):
    """Cosmic-ray muons crossing the volume from top (y = +3 m) to bottom
    (y = -3 m), entry and exit x, z uniform; Moyal dE/dx as track_depos."""
    out = []
    for _ in range(ntracks):
        a = np.array((RESPONSE_X + 2500.0 * rng.random(), 3000.0, -1150.0 + 2300.0 * rng.random()))
        b = np.array((RESPONSE_X + 2500.0 * rng.random(), -3000.0, -1150.0 + 2300.0 * rng.random()))
        t0 = float(rng.uniform(0.0, t0_spread)) if t0_spread else 0.0
        out.append(_segment(rng, a, b, step, t0))
    return np.concatenate(out, axis=0)


def _segment(rng, a, b, step, t0, dedx_mpv=2.1, dedx_width=0.1, wion=23.6e-6, recomb=0.7):
    length = float(np.linalg.norm(b - a))
    n = max(1, int(length / step))
    s = (np.arange(n) + 0.5) / n
    d = np.zeros((n, 7))
    d[:, 0] = t0
    d[:, 2:5] = a[None, :] + s[:, None] * (b - a)[None, :]
    dedx = np.clip(dedx_mpv + dedx_width * moyal(rng, n), 0.2, 200.0)
    d[:, 1] = -(dedx * (step / cm) / wion) * recomb
    return d


def calibration_events(nevents=16, ndepos=4_000_000, seed=9, depos_per_gev=40_000):
    """Events of about ``ndepos`` depos: half cosmic-ray muons, half EM shower
    blobs with energies drawn from an exponential spectrum of mean 1 GeV (a
    shower of E GeV holds depos_per_gev * E depos)."""
    rng = np.random.default_rng(seed)
    events = []
    for _ in range(nevents):
        parts, n = [], 0
        while n < ndepos // 2:
            c = cosmic_depos(rng, 1)
            parts.append(c)
            n += len(c)
        while n < ndepos:
            e_gev = float(rng.exponential(1.0)) + 0.01
            k = min(ndepos - n, max(10, int(depos_per_gev * e_gev)))
            parts.append(shower_depos(rng, k, energy_mev=1000.0 * e_gev))
            n += k
        events.append(np.ascontiguousarray(np.concatenate(parts, axis=0)[:ndepos]))
    return events
