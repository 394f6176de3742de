"""Depo and frame files in the toolkit's numpy formats (the sio package).

Two containers, the same arrays:

* ``.npz`` archives, members appended per save (sio/src/NumpyDepoSaver.cxx,
  NumpyDepoTools.cxx, NumpyFrameSaver.cxx);
* tar streams (plain, .gz or .bz2) of ``.npy`` members, one group per event
  (sio/src/DepoFileSink.cxx, DepoFileSource.cxx, FrameFileSink.cxx).

Arrays:

* ``depo_data_<n>``: float32 [N][7] = time, charge, x, y, z, extent_long,
  extent_tran; ``depo_info_<n>``: int32 [N][4] = id, pdg, generation, child.
  Rows of generation > 0 are the "prior" depos of row ``child`` and are not
  simulated (NumpyDepoTools::load keeps the generation-0 rows).  Files that
  hold the transposed [7][N] / [4][N] layout are read too.
* ``frame_<tag>_<n>``: float32 (int16 when digitized) [channels][ticks];
  ``channels_<tag>_<n>``: int32 channel numbers (sorted) of the rows;
  ``tickinfo_<tag>_<n>``: float64 [frame time, tick, first tick bin].

The dense frames of this package map to traces as the DepoTransform
component emits them (gen/src/DepoTransform.cxx:193-215): each non-zero
row, from its first to its last non-zero sample.
"""

import io
import os
import tarfile
import zipfile

import numpy as np


def _npy_bytes(a):
    b = io.BytesIO()
    np.lib.format.write_array(b, np.ascontiguousarray(a), allow_pickle=False)
    return b.getvalue()


def _npz_write(path, members, mode="a"):
    """Add (or, mode "w", write afresh) .npy members to an .npz archive, as
    cnpy::npz_save does (a member of the same name is replaced)."""
    if mode == "a" and os.path.exists(path):
        with zipfile.ZipFile(path) as z:
            keep = {n: z.read(n) for n in z.namelist() if n[:-4] not in members}
    else:
        keep = {}
    with zipfile.ZipFile(path, "w", zipfile.ZIP_STORED) as z:
        for n, data in keep.items():
            z.writestr(n, data)
        for name, a in members.items():
            z.writestr(name + ".npy", _npy_bytes(a))


def _rows(a, ncols):
    """[N][ncols] from an [N][ncols] or transposed [ncols][N] array."""
    a = np.asarray(a)
    if a.ndim != 2:
        raise ValueError("expected a 2-D array")
    if a.shape[1] == ncols:
        return a
    if a.shape[0] == ncols:
        return a.T
    raise ValueError("array of shape %s has no axis of length %d" % (a.shape, ncols))


def depo_arrays(data, info):
    """(depos [n][7] float64, info [n][4] int32) of the generation-0 rows."""
    d = _rows(data, 7).astype(np.float64)
    i = _rows(info, 4).astype(np.int32)
    if len(d) != len(i):
        raise ValueError("depo data and info hold different counts")
    keep = i[:, 2] == 0
    return np.ascontiguousarray(d[keep]), np.ascontiguousarray(i[keep])


def load_depos(path, index=0):
    """depo_data_<index> / depo_info_<index> of an .npz archive (NumpyDepoTools::load)."""
    z = np.load(path)
    return depo_arrays(z["depo_data_%d" % index], z["depo_info_%d" % index])


def save_depos(path, depos, info=None, index=0, mode="a"):
    """NumpyDepoSaver: depo_data_<index> (float32 [N][7]) and depo_info_<index>
    (int32 [N][4]; default: id = row, pdg 0, generation 0, child 0)."""
    d = np.asarray(depos, dtype=np.float32).reshape(-1, 7)
    if info is None:
        info = np.zeros((len(d), 4), dtype=np.int32)
        info[:, 0] = np.arange(len(d))
    _npz_write(path, {"depo_data_%d" % index: d, "depo_info_%d" % index: np.asarray(info, dtype=np.int32)}, mode)


def frame_traces(frame, channels):
    """[(channel, first tick, samples)] of the non-zero rows of a dense frame."""
    out = []
    for r, ch in enumerate(channels):
        nz = np.flatnonzero(frame[r])
        if nz.size:
            out.append((int(ch), int(nz[0]), np.asarray(frame[r, nz[0]:nz[-1] + 1], dtype=np.float32)))
    return out


def frame_arrays(frame, channels, tick, time=0.0, baseline=0.0, scale=1.0, offset=0.0, digitize=False):
    """NumpyFrameSaver's arrays (sio/src/NumpyFrameSaver.cxx:107-160) of a
    dense frame: the traces' channels (sorted) by the traces' tick range,
    (baseline + samples) * scale + offset, int16 (truncated) when digitize.
    Returns (frame array, channels, tickinfo) or None without traces."""
    tr = frame_traces(np.asarray(frame), channels)
    if not tr:
        return None
    chans = np.array(sorted({c for c, _, _ in tr}), dtype=np.int32)
    t0 = min(t for _, t, _ in tr)
    t1 = max(t + len(s) for _, t, s in tr)
    arr = np.zeros((len(chans), t1 - t0), dtype=np.float32) + np.float32(baseline)
    row = {c: k for k, c in enumerate(chans)}
    for c, t, s in tr:
        arr[row[c], t - t0:t - t0 + len(s)] += s
    arr = arr * np.float32(scale) + np.float32(offset)
    if digitize:
        arr = arr.astype(np.int16)
    tickinfo = np.array([time, tick, float(t0)], dtype=np.float64)
    return arr, chans, tickinfo


def save_frame(path, frame, channels, tick, time=0.0, tag="", index=0, baseline=0.0, scale=1.0, offset=0.0,
               digitize=False, mode="a"):
    """NumpyFrameSaver: frame_<tag>_<index>, channels_<tag>_<index>, tickinfo_<tag>_<index>."""
    a = frame_arrays(frame, channels, tick, time, baseline, scale, offset, digitize)
    if a is None:
        return False
    f, c, ti = a
    _npz_write(path, {"frame_%s_%d" % (tag, index): f, "channels_%s_%d" % (tag, index): c,
                      "tickinfo_%s_%d" % (tag, index): ti}, mode)
    return True


def load_frame(path, tag="", index=0):
    """(frame, channels, tickinfo) of an .npz archive."""
    z = np.load(path)
    return (z["frame_%s_%d" % (tag, index)], z["channels_%s_%d" % (tag, index)],
            z["tickinfo_%s_%d" % (tag, index)])


def _tar_mode(path, write):
    ext = {".gz": "gz", ".tgz": "gz", ".bz2": "bz2", ".xz": "xz"}.get(os.path.splitext(path)[1], "")
    return ("w" if write else "r") + (":" + ext if ext else "")


def write_tar(path, members):
    """A tar stream of .npy members: ``members`` maps file names (without
    .npy) to arrays, written in order."""
    with tarfile.open(path, _tar_mode(path, True)) as t:
        for name, a in members.items():
            data = _npy_bytes(a)
            ti = tarfile.TarInfo(name + ".npy")
            ti.size = len(data)
            t.addfile(ti, io.BytesIO(data))


def read_tar(path):
    """{name without .npy: array} of a tar stream, in stream order."""
    out = {}
    with tarfile.open(path, _tar_mode(path, False)) as t:
        for m in t:
            if m.isfile() and m.name.endswith(".npy"):
                out[m.name[:-4]] = np.load(io.BytesIO(t.extractfile(m).read()), allow_pickle=False)
    return out


def save_depo_stream(path, events):
    """DepoFileSink: for each (ident, depos[, info]) the members
    depo_data_<ident> and depo_info_<ident>."""
    members = {}
    for ev in events:
        ident, d = ev[0], np.asarray(ev[1], dtype=np.float32).reshape(-1, 7)
        info = ev[2] if len(ev) > 2 else None
        if info is None:
            info = np.zeros((len(d), 4), dtype=np.int32)
            info[:, 0] = np.arange(len(d))
        members["depo_data_%d" % ident] = d
        members["depo_info_%d" % ident] = np.asarray(info, dtype=np.int32)
    write_tar(path, members)


def load_depo_stream(path):
    """DepoFileSource: [(ident, depos, info)] of the generation-0 rows, in stream order."""
    m = read_tar(path)
    out = []
    for name in m:
        if name.startswith("depo_data_"):
            ident = int(name.split("_")[2])
            d, i = depo_arrays(m[name], m["depo_info_%d" % ident])
            out.append((ident, d, i))
    return out


def save_frame_stream(path, frames, tag=""):
    """FrameFileSink: for each (ident, dense frame, channels, tick[, time])
    the members frame_<tag>_<ident>, channels_<tag>_<ident> and
    tickinfo_<tag>_<ident> (frames without traces are skipped)."""
    members = {}
    for fr in frames:
        ident, frame, chans, tick = fr[:4]
        time = fr[4] if len(fr) > 4 else 0.0
        a = frame_arrays(frame, chans, tick, time)
        if a is None:
            continue
        members["frame_%s_%d" % (tag, ident)] = a[0]
        members["channels_%s_%d" % (tag, ident)] = a[1]
        members["tickinfo_%s_%d" % (tag, ident)] = a[2]
    write_tar(path, members)


def load_frame_stream(path):
    """FrameFileSource: [(ident, tag, frame, channels, tickinfo)] of the
    frames in a tar stream, in stream order."""
    m = read_tar(path)
    out = []
    for name in m:
        if not name.startswith("frame_"):
            continue
        tag, ident = name[len("frame_"):].rsplit("_", 1)
        out.append((int(ident), tag, m[name], m["channels_%s_%s" % (tag, ident)],
                    m["tickinfo_%s_%s" % (tag, ident)]))
    return out


def dense_frame(frame, channels, tickinfo, channel_rows, nticks, baseline=0.0, scale=1.0, offset=0.0):
    """A saved frame put back on a dense [rows][nticks] float32 array:
    ``channel_rows`` maps channel number -> row (the component's frame rows);
    the saved (value - offset) / scale - baseline lands at ticks
    tickinfo[2] + k; ticks outside [0, nticks) and unknown channels are dropped."""
    nrows = max(channel_rows.values()) + 1 if channel_rows else 0
    out = np.zeros((nrows, nticks), dtype=np.float32)
    t0 = int(tickinfo[2])
    vals = (np.asarray(frame, dtype=np.float32) - np.float32(offset)) / np.float32(scale) - np.float32(baseline)
    lo, hi = max(0, t0), min(nticks, t0 + vals.shape[1])
    for k, ch in enumerate(channels):
        r = channel_rows.get(int(ch))
        if r is not None and hi > lo:
            out[r, lo:hi] = vals[k, lo - t0:hi - t0]
    return out
