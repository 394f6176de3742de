"""TEST INFRASTRUCTURE ONLY -- the FP64 oracle of the adjoint, never the product.

An FP64 NumPy restatement of the DepoTransform forward as a differentiable
function of the depos (t, q, x, y, z, extent_long, extent_tran) and of the
drifter's DL, DT and lifetime, with every piecewise-constant choice -- which
depos reach a plane, the patch sample ranges, the event windows -- frozen at a
base point taken from the restated reference (``oracle.run(..., records=True)``).
On top of it:

* ``FrozenModel.frames``     the frame of every plane (checked against
                               ``oracle.run`` at the base point),
* ``FrozenModel.gradient``   the analytic reverse-mode gradient in FP64,
* ``FrozenModel.fd_depo`` /
  ``FrozenModel.fd_global``  central finite differences of the FP64 loss.

Model, per plane (gen/src/Drifter.cxx:164-192, gen/src/DepoTransform.cxx:180-186,
gen/src/GaussianDiffusion.cxx:30-92,116-182,
gen/src/BinnedDiffusion_transform.cxx:296-367, gen/src/ImpactTransform.cxx):

  drift (bulk region):  dt = |x_resp - x| / v,  t' = t + dt + t_off,
                        q' = q exp(-dt / lifetime),
                        sL = sqrt(2 DL dt + el^2),  sT = sqrt(2 DT dt + et^2)
  (response region: t' = t - dt + t_off, nothing else changes; x' = x_resp)
  patch:  tv_tau = Phi(v_{tau+1}) - Phi(v_tau), v = (edge - t') / (sL / v_d)
          p_k    = Phi(u_{k+1}) - Phi(u_k),     u = (edge - c) / sT
          a_k    = p_k * weight_k = [sT (phi(u_{k+1}) - phi(u_k)) + (e_{k+1} - c) p_k] / bs
          Q_l[w][tau]   += q' tv a_k / (sum tv * sum p)
          Q_l+1[w][tau] += q' tv (p_k - a_k) / (sum tv * sum p)
  frame:  F[w][t] = window(w, t) * sum_g sum_j (R_g[j] (x) Q_g[w - j])[t]

Only tests/ import this module.
"""

import math

import numpy as np
from scipy.signal import fftconvolve
from scipy.special import ndtr

import oracle

SQ2PI = math.sqrt(2.0 * math.pi)


def _pdf(u):
    return np.exp(-0.5 * u * u) / SQ2PI


def drift_state(cfg, row, DL, DT, lifetime):
    """Drifted (t', q', x', sL, sT) of one depo and the Jacobian of those with
    respect to (t, q, x, y, z, el, et, DL, DT, lifetime) (rows: t', q', x', sL, sT)."""
    t, q, x, y, z, el, et = [float(v) for v in row[:7]]
    J = np.zeros((5, 10))
    dr = cfg.get("drifter")
    if dr is None:
        J[0, 0] = J[1, 1] = J[2, 2] = J[3, 5] = J[4, 6] = 1.0
        return (t, q, x, el, et), J
    v = dr["drift_speed"]
    toff = dr.get("time_offset", 0.0)
    found, sgn = None, 0.0
    for a, rp, c in dr["xregions"]:
        if (a < x < rp) or (rp < x < a):
            found, sgn = rp, -1.0
            break
    if found is None:
        for a, rp, c in dr["xregions"]:
            if (rp < x < c) or (c < x < rp):
                found, sgn = rp, 1.0
                break
    if found is None:
        return None, None
    dt = abs((found - x) / v)
    dtdx = (1.0 if x > found else -1.0) / v
    if sgn > 0:
        ex = math.exp(-dt / lifetime)
        qd = q * ex
        sL = math.sqrt(2.0 * DL * dt + el * el)
        sT = math.sqrt(2.0 * DT * dt + et * et)
        tp = t + dt + toff
        J[0, 0] = 1.0
        J[0, 2] = dtdx
        J[1, 1] = ex
        J[1, 2] = -qd / lifetime * dtdx
        J[1, 9] = qd * dt / lifetime ** 2
        if sL > 0:
            J[3, 2] = DL / sL * dtdx
            J[3, 5] = el / sL
            J[3, 7] = dt / sL
        if sT > 0:
            J[4, 2] = DT / sT * dtdx
            J[4, 6] = et / sT
            J[4, 8] = dt / sT
        return (tp, qd, found, sL, sT), J
    tp = t - dt + toff
    J[0, 0] = 1.0
    J[0, 2] = -dtdx
    J[1, 1] = 1.0
    J[3, 5] = 1.0
    J[4, 6] = 1.0
    return (tp, q, found, el, et), J


class _Plane:
    def __init__(self, cfg, ip, window):
        pl = cfg["planes"][ip]
        self.nwires = pl["nwires"]
        self.nimp = pl["nimp"]
        regionsize = (pl["pitchmax"] - pl["pitchmin"]) / (self.nwires - 1)
        self.imp_min = pl["pitchmin"] - 0.5 * regionsize
        imp_max = pl["pitchmax"] + 0.5 * regionsize
        self.imp_bs = (imp_max - self.imp_min) / (self.nwires * self.nimp)
        pdir = np.array(pl["pitch"], dtype=np.float64)
        self.axis = pdir / math.sqrt(float(np.dot(pdir, pdir)))
        self.origin = np.array(pl["origin"], dtype=np.float64)
        pir = oracle.pir_build(cfg, ip, fp64=True)
        self.G = int(round(pir["pitch"] / pir["impact"])) + 1
        self.npad = int(round((pir["bywire"].shape[0] - 1) / 2.0))
        nt = pir["waveforms"].shape[1]
        # K[g][jj][tau] = R_g[jj - npad][tau] by the closest() rule (gen/src/ImpactTransform.cxx:34-74)
        K = np.zeros((self.G, 2 * self.npad + 1, nt))
        for g in range(self.G):
            rel = -pir["pitch"] / 2.0 + pir["impact"] * g + (1e-9 if g != self.G - 1 else -1e-9)
            for jj in range(2 * self.npad + 1):
                rp = rel - (jj - self.npad) * pir["pitch"]
                relwire = oracle.cround(rp / pir["pitch"])
                wi = pir["bywire"].shape[0] // 2 + relwire
                rem = rp - relwire * pir["pitch"]
                ii = oracle.cround(rem / pir["impact"]) + pir["bywire"].shape[1] // 2
                K[g, jj] = pir["waveforms"][pir["bywire"][wi][ii]]
        last = np.nonzero(np.any(K != 0, axis=(0, 1)))[0]
        self.K = K[:, :, : (last[-1] + 1 if len(last) else 1)]
        self.win = window

    def mask(self, nticks):
        w = self.win
        m = np.zeros((self.nwires, nticks), dtype=bool)
        w0, w1 = max(0, w["start_ch"]), min(self.nwires, w["end_ch"])
        t0, t1 = max(0, w["start_tick"]), min(nticks, w["end_tick"])
        if w["ndepos_added"] > 0 and w1 > w0 and t1 > t0:
            m[w0:w1, t0:t1] = True
        return m


class FrozenModel:
    """FP64 forward, gradient and finite differences with the discrete
    choices of the reference frozen at (cfg, depos)."""

    def __init__(self, cfg, depos):
        self.cfg = cfg
        self.depos = np.array(depos, dtype=np.float64).reshape(-1, 7)
        self.nticks = int(cfg["readout_time"] / cfg["tick"])
        self.tbs = cfg["readout_time"] / self.nticks
        self.tmin = cfg["start_time"]
        base = oracle.run(cfg, self.depos, drift=cfg.get("drifter") is not None, fp64=True, records=True)
        self.base_frames = base["frames"]
        self.records = base["records"]  # [plane][depo] (added, toff, poff, nt, np)
        self.windows = base["windows"]
        self.planes = [_Plane(cfg, ip, base["windows"][ip]) for ip in range(len(cfg["planes"]))]
        self.masks = [p.mask(self.nticks) for p in self.planes]
        dr = cfg.get("drifter") or {}
        self.glob = np.array([dr.get("DL", 0.0), dr.get("DT", 0.0), dr.get("lifetime", 1.0)])

    # ---- patches ---------------------------------------------------------
    def _patch(self, ip, i, state, row):
        """Patch values and derivatives of depo i (input row ``row``, drifted
        ``state``) on plane ip; None where the depo adds nothing there."""
        added, toff, poff, nt, npp = (int(v) for v in self.records[ip, i])
        if not added or nt <= 0 or npp <= 0:
            return None
        P = self.planes[ip]
        tp, qp, xp, sL, sT = state
        cp = float(np.dot(P.axis, np.array([xp, row[3], row[4]]) - P.origin))
        st = sL / self.cfg["drift_speed"]
        sp = sT
        te = self.tmin + (toff + np.arange(nt + 1)) * self.tbs - tp
        pe = P.imp_min + (poff + np.arange(npp + 1)) * P.imp_bs - cp
        out = dict(toff=toff, poff=poff, nt=nt, np=npp)
        if st > 0:
            v = te / st
            Phi, ph = ndtr(v), _pdf(v)
            out["tv"] = np.diff(Phi)
            out["dtv_c"] = -np.diff(ph) / st
            out["dtv_s"] = -np.diff(v * ph) / st
            out["St"] = Phi[-1] - Phi[0]
            out["dSt_c"] = -(ph[-1] - ph[0]) / st
            out["dSt_s"] = -(v[-1] * ph[-1] - v[0] * ph[0]) / st
        else:
            out["tv"] = np.ones(1)
            out["dtv_c"] = np.zeros(1)
            out["dtv_s"] = np.zeros(1)
            out["St"], out["dSt_c"], out["dSt_s"] = 1.0, 0.0, 0.0
        bs = P.imp_bs
        if sp > 0:
            u = pe / sp
            Phi, ph = ndtr(u), _pdf(u)
            p = np.diff(Phi)
            x2 = pe[1:]
            dpc = -np.diff(ph) / sp
            dps = -np.diff(u * ph) / sp
            out["p"] = p
            out["a"] = (sp * np.diff(ph) + x2 * p) / bs
            out["dp_c"], out["dp_s"] = dpc, dps
            out["da_c"] = (np.diff(u * ph) - p + x2 * dpc) / bs
            out["da_s"] = (np.diff(ph) + np.diff(u * u * ph) + x2 * dps) / bs
            out["Sp"] = Phi[-1] - Phi[0]
            out["dSp_c"] = -(ph[-1] - ph[0]) / sp
            out["dSp_s"] = -(u[-1] * ph[-1] - u[0] * ph[0]) / sp
        else:
            out["p"] = np.ones(1)
            out["a"] = np.array([pe[1] / bs])
            out["dp_c"] = np.zeros(1)
            out["dp_s"] = np.zeros(1)
            out["da_s"] = np.zeros(1)
            out["da_c"] = np.array([-1.0 / bs])
            out["Sp"], out["dSp_c"], out["dSp_s"] = 1.0, 0.0, 0.0
        out["qn"] = qp / (out["St"] * out["Sp"])
        k = poff + np.arange(npp)
        out["wire"] = k // P.nimp
        out["l"] = k - out["wire"] * P.nimp
        return out

    def _block(self, ip, pt):
        """Charge block of one patch: (first wire, first tick, Q[G][nw][nt])."""
        P = self.planes[ip]
        w0 = int(pt["wire"][0])
        nw = int(pt["wire"][-1]) - w0 + 1
        Qb = np.zeros((P.G, nw, pt["nt"]))
        tq = pt["qn"] * pt["tv"]
        for k in range(pt["np"]):
            w, l = pt["wire"][k] - w0, pt["l"][k]
            Qb[l, w] += pt["a"][k] * tq
            Qb[l + 1, w] += (pt["p"][k] - pt["a"][k]) * tq
        return w0, pt["toff"], Qb

    def _conv_block(self, ip, w0, t0, Qb):
        """Windowed frame contribution of a charge block: (first wire, first tick, V)."""
        P = self.planes[ip]
        V = None
        for g in range(P.G):
            f = fftconvolve(Qb[g], P.K[g])
            V = f if V is None else V + f
        o0 = w0 - P.npad
        lo, hi = max(0, o0), min(P.nwires, o0 + V.shape[0])
        t1 = min(self.nticks, t0 + V.shape[1])
        V = V[lo - o0:hi - o0, : t1 - t0] * self.masks[ip][lo:hi, t0:t1]
        return lo, t0, V

    # ---- forward ---------------------------------------------------------
    def frames(self, depos=None, glob=None):
        """Frame of every plane [nwires][nticks]."""
        depos = self.depos if depos is None else depos
        glob = self.glob if glob is None else glob
        out = []
        for ip, P in enumerate(self.planes):
            Q = np.zeros((P.G, P.nwires, self.nticks))
            for i in range(len(depos)):
                st, _ = drift_state(self.cfg, depos[i], *glob)
                if st is None:
                    continue
                pt = self._patch(ip, i, st, depos[i])
                if pt is None:
                    continue
                w0, t0, Qb = self._block(ip, pt)
                Q[:, w0:w0 + Qb.shape[1], t0:t0 + Qb.shape[2]] += Qb
            V = np.zeros((P.nwires, self.nticks))
            rows = np.nonzero(np.any(Q != 0, axis=(0, 2)))[0]
            if len(rows):
                r0, r1 = rows[0], rows[-1] + 1
                lo, t0, Vb = self._conv_block(ip, r0, 0, Q[:, r0:r1])
                V[lo:lo + Vb.shape[0], t0:t0 + Vb.shape[1]] = Vb
            out.append(V)
        return out

    @staticmethod
    def loss(frames, targets):
        return sum(float(np.sum((f - t) ** 2)) for f, t in zip(frames, targets))

    # ---- reverse ---------------------------------------------------------
    def correlate(self, ip, gF):
        """dL/dQ_g[w][t] = sum_j sum_tau gF[w + j][t + tau] R_g[j][tau] (the transpose of the convolution)."""
        P = self.planes[ip]
        g = gF * self.masks[ip]
        dQ = np.zeros((P.G, P.nwires, self.nticks))
        rows = np.nonzero(np.any(g != 0, axis=1))[0]
        if len(rows) == 0:
            return dQ
        r0, r1 = rows[0], rows[-1] + 1
        L = P.K.shape[2]
        for gi in range(P.G):
            full = fftconvolve(g[r0:r1], P.K[gi][::-1, ::-1])
            w0 = r0 - P.npad          # full row a <-> charge row r0 - npad + a
            lo, hi = max(0, w0), min(P.nwires, w0 + full.shape[0])
            nt = min(self.nticks, full.shape[1] - (L - 1))  # full column b <-> tick b - (L - 1)
            dQ[gi, lo:hi, :nt] = full[lo - w0:hi - w0, L - 1:L - 1 + nt]
        return dQ

    def gradient(self, grad_frames):
        """(dL/d depos [n][7], dL/d (DL, DT, lifetime)) for dL/d(frame) of every plane."""
        n = len(self.depos)
        gd = np.zeros((n, 7))
        gg = np.zeros(3)
        vd = self.cfg["drift_speed"]
        states = [drift_state(self.cfg, r, *self.glob) for r in self.depos]
        for ip, P in enumerate(self.planes):
            dQ = self.correlate(ip, grad_frames[ip])
            for i in range(n):
                st, J = states[i]
                if st is None:
                    continue
                pt = self._patch(ip, i, st, self.depos[i])
                if pt is None:
                    continue
                toff, nt = pt["toff"], pt["nt"]
                D0 = dQ[pt["l"], pt["wire"], toff:toff + nt]          # [np][nt]
                D1 = dQ[pt["l"] + 1, pt["wire"], toff:toff + nt]
                U = pt["a"] @ (D0 - D1) + pt["p"] @ D1                  # [nt]
                Ac = pt["da_c"] @ (D0 - D1) + pt["dp_c"] @ D1
                As = pt["da_s"] @ (D0 - D1) + pt["dp_s"] @ D1
                qn = pt["qn"]
                gqn = float(pt["tv"] @ U)
                gcp = qn * float(pt["tv"] @ Ac) - gqn * qn / pt["Sp"] * pt["dSp_c"]
                gsp = qn * float(pt["tv"] @ As) - gqn * qn / pt["Sp"] * pt["dSp_s"]
                gct = qn * float(pt["dtv_c"] @ U) - gqn * qn / pt["St"] * pt["dSt_c"]
                gst = qn * float(pt["dtv_s"] @ U) - gqn * qn / pt["St"] * pt["dSt_s"]
                gq = gqn / (pt["St"] * pt["Sp"])
                # back through (t', q', x', sL, sT) and c = axis . ((x', y, z) - origin)
                gstate = np.array([gct, gq, gcp * P.axis[0], gst / vd, gsp])
                gfull = gstate @ J
                gfull[3] += gcp * P.axis[1]
                gfull[4] += gcp * P.axis[2]
                gd[i] += gfull[:7]
                gg += gfull[7:]
        if self.cfg.get("drifter") is None:
            gg[:] = 0.0
        return gd, gg

    # ---- finite differences ---------------------------------------------
    def fd_depo(self, i, k, h, targets, frames0):
        """Central difference of the loss in depos[i][k] with step h.  Only depo
        i changes, so the frame changes by its own (block-local) contribution."""
        out = 0.0
        for ip in range(len(self.planes)):
            blocks = []
            for sgn in (+1.0, -1.0, 0.0):
                row = self.depos[i].copy()
                row[k] += sgn * h
                st, _ = drift_state(self.cfg, row, *self.glob)
                pt = None if st is None else self._patch(ip, i, st, row)
                if pt is None:
                    blocks = None
                    break
                blocks.append(self._conv_block(ip, *self._block(ip, pt)))
            if blocks is None:
                continue
            (lo, t0, Ap), (_, _, Am), (_, _, A0) = blocks
            sl = (slice(lo, lo + Ap.shape[0]), slice(t0, t0 + Ap.shape[1]))
            R0 = frames0[ip][sl] - targets[ip][sl] - A0
            out += float(np.sum((Ap - Am) * (2.0 * R0 + Ap + Am)))
        return out / (2.0 * h)

    def fd_global(self, k, h, targets):
        gp = self.glob.copy()
        gm = self.glob.copy()
        gp[k] += h
        gm[k] -= h
        return (self.loss(self.frames(glob=gp), targets) - self.loss(self.frames(glob=gm), targets)) / (2.0 * h)
