"""sio formats (sio/src/NumpyDepoSaver.cxx, NumpyDepoTools.cxx,
NumpyFrameSaver.cxx, DepoFileSink/Source, FrameFileSink): the reference's
sample depo file (its first depos, tests/golden/muon_depos_head.npz, written
by tests/golden/make_sio_fixture.py), round trips through .npz archives and
tar streams, and the frame saver's trace layout."""

import importlib
import os

import numpy as np
import pytest

sio = importlib.import_module("wire-cell-toolkit_b200.sio")
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "muon_depos_head.npz")


def test_reference_sample_depos():
    d, info = sio.load_depos(GOLDEN)
    z = np.load(GOLDEN)
    assert d.shape == (300, 7) and info.shape == (300, 4)
    assert np.array_equal(d, z["depo_data_0"].T.astype(np.float64))
    assert np.array_equal(info, z["depo_info_0"].T)
    assert np.all(d[:, 1] < 0)          # electrons: negative charge
    assert set(np.unique(info[:, 1])) <= {11, 13}  # muon depos and their delta electrons


def test_depo_npz_round_trip_and_priors(tmp_path):
    rng = np.random.default_rng(0)
    p = str(tmp_path / "depos.npz")
    d0 = rng.normal(size=(50, 7)).astype(np.float32)
    sio.save_depos(p, d0, index=0, mode="w")
    d1 = rng.normal(size=(20, 7)).astype(np.float32)
    info1 = np.zeros((20, 4), np.int32)
    info1[:, 0] = np.arange(20)
    info1[[5, 6], 2] = 1       # two priors of rows 3 and 4
    info1[[5, 6], 3] = [3, 4]
    sio.save_depos(p, d1, info1, index=1)
    a, ia = sio.load_depos(p, 0)
    b, ib = sio.load_depos(p, 1)
    assert np.array_equal(a, d0.astype(np.float64)) and np.array_equal(ia[:, 0], np.arange(50))
    keep = np.ones(20, bool)
    keep[[5, 6]] = False
    assert np.array_equal(b, d1[keep].astype(np.float64)) and np.all(ib[:, 2] == 0)


def _frame():
    f = np.zeros((6, 40), np.float32)
    f[1, 10:15] = [1, 2, 3, 0, 5]
    f[4, 3] = -7
    f[5, 20:38] = 0.5
    return f


def test_frame_saver_layout(tmp_path):
    f = _frame()
    chans = np.array([100, 105, 101, 102, 104, 103])
    arr, ch, ti = sio.frame_arrays(f, chans, tick=500.0, time=1.0e3, baseline=1.0, scale=2.0, offset=-0.5)
    assert list(ch) == [103, 104, 105]          # non-zero rows, sorted channel numbers
    assert list(ti) == [1.0e3, 500.0, 3.0]      # first tick bin of the traces
    assert arr.shape == (3, 35)                 # ticks 3 .. 37
    ref = np.full((3, 35), 1.0, np.float32)
    ref[2, 7:12] += [1, 2, 3, 0, 5]             # channel 105 (row 1)
    ref[1, 0] += -7                             # channel 104 (row 4)
    ref[0, 17:35] += 0.5                        # channel 103 (row 5)
    assert np.array_equal(arr, ref * 2.0 - 0.5)
    p = str(tmp_path / "frames.npz")
    assert sio.save_frame(p, f, chans, 500.0, tag="orig", index=2, mode="w")
    g, c, t = sio.load_frame(p, "orig", 2)
    assert np.array_equal(g, sio.frame_arrays(f, chans, 500.0)[0]) and list(c) == [103, 104, 105]
    dig = sio.frame_arrays(f * 3.3, chans, 500.0, digitize=True)[0]
    assert dig.dtype == np.int16 and dig[2, 9] == 9   # 3 * 3.3 = 9.9 truncated
    assert not sio.save_frame(p, np.zeros((2, 5)), [1, 2], 500.0)


@pytest.mark.parametrize("ext", [".tar", ".tar.gz", ".tar.bz2"])
def test_tar_streams(tmp_path, ext):
    rng = np.random.default_rng(1)
    p = str(tmp_path / ("depos" + ext))
    evs = [(7, rng.normal(size=(30, 7))), (9, rng.normal(size=(0, 7))), (12, rng.normal(size=(5, 7)))]
    sio.save_depo_stream(p, evs)
    back = sio.load_depo_stream(p)
    assert [b[0] for b in back] == [7, 9, 12]
    for (i, d), (j, e, _) in zip(evs, back):
        assert np.array_equal(e, d.astype(np.float32).astype(np.float64))
    q = str(tmp_path / ("frames" + ext))
    sio.save_frame_stream(q, [(3, _frame(), np.arange(6), 500.0), (4, np.zeros((6, 40)), np.arange(6), 500.0)],
                          tag="sim")
    m = sio.read_tar(q)
    assert sorted(m) == ["channels_sim_3", "frame_sim_3", "tickinfo_sim_3"]
    assert np.array_equal(m["frame_sim_3"], sio.frame_arrays(_frame(), np.arange(6), 500.0)[0])


def test_frame_stream_back_to_dense(tmp_path):
    f = _frame()
    chans = np.array([100, 105, 101, 102, 104, 103])
    q = str(tmp_path / "frames.tar.bz2")
    sio.save_frame_stream(q, [(3, f, chans, 500.0, 2.0e3)], tag="sim")
    (ident, tag, arr, ch, ti), = sio.load_frame_stream(q)
    assert (ident, tag) == (3, "sim") and list(ti) == [2.0e3, 500.0, 3.0]
    rows = {int(c): r for r, c in enumerate(chans)}
    assert np.array_equal(sio.dense_frame(arr, ch, ti, rows, 40), f)
