"""Multi-rank host logic on CPU: gloo process groups of world size 2.

Events (and the planes of one event) are independent, so the forward needs no
collective; these tests cover the event balance, the plane split with its row
gather, and the drift-parameter fit whose loss and gradients are summed over
ranks once per step.  The objective here is a host-side stand-in with the
same shape as the GPU one (a sum of per-event terms), so the fit logic runs
without a GPU."""

import importlib
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402

shard = importlib.import_module("wire-cell-toolkit_b200.shard")
cal = importlib.import_module("wire-cell-toolkit_b200.calibrate")

TRUE = np.array([0.9, 1.1, 8.0])
P0 = np.array([1.0, 1.0, 10.0])


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _event_weights(nev, seed=3):
    rng = np.random.default_rng(seed)
    return rng.uniform(0.5, 2.0, (nev, 3)), rng.integers(1000, 50000, nev)


def _objective(events, w):
    """sum over events e of sum_i w[e,i] (log p_i - log t_i)^2 and its gradient in p."""
    def evaluate(p):
        lp = np.log(p) - np.log(TRUE)
        loss = 0.0
        g = np.zeros(3)
        for e in events:
            loss += float(np.sum(w[e] * lp * lp))
            g += 2.0 * w[e] * lp / p
        return loss, g
    return evaluate


def _run(rank, world, port, nev, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        w, counts = _event_weights(nev)
        off = np.zeros(nev + 1, dtype=np.int64)
        off[1:] = np.cumsum(counts)
        ev, rows, loc = shard.local_events(off, rank, world)
        res = {"events": ev.tolist(), "nrows": len(rows), "loc": loc.tolist()}
        # the fit: every rank evaluates its own events, the step uses the sums
        hist, final = cal.adam_fit(_objective(ev, w), P0, steps=40, lr=0.1, decay=0.97,
                                   reduce=lambda v: shard.allreduce_sum(v))
        res["final"] = list(final)
        res["losses"] = [h[2] for h in hist]
        # plane split of one event: rank r holds its planes' rows, rank 0 stacks them
        nw = [800, 800, 960]
        mine = shard.plane_partition(3, world)[rank]
        rows_r = torch.cat([torch.full((nw[p], 16), float(p), dtype=torch.float32) for p in mine])
        got = shard.gather_rows(rows_r, dst=0)
        if rank == 0:
            res["gathered"] = got.numpy()
        else:
            res["gathered"] = got
        np.save(os.path.join(out, "r%d.npy" % rank), np.array([res], dtype=object), allow_pickle=True)
    finally:
        dist.destroy_process_group()


def _spawn(tmp_path, nev, world=2):
    port = _free_port()
    mp.start_processes(_run, args=(world, port, nev, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    return [np.load(tmp_path / ("r%d.npy" % r), allow_pickle=True)[0] for r in range(world)]


def test_greedy_partition_balance():
    rng = np.random.default_rng(5)
    for nranks in (1, 2, 3, 8):
        counts = np.exp(rng.uniform(np.log(1e4), np.log(5e5), 64)).astype(np.int64)
        parts = shard.greedy_partition(counts, nranks)
        allev = np.sort(np.concatenate(parts))
        assert np.array_equal(allev, np.arange(64))
        loads = [int(counts[p].sum()) for p in parts]
        assert max(loads) - min(loads) <= int(counts.max())
        # largest-first greedy is within 4/3 of the best possible makespan
        assert max(loads) <= (4.0 / 3.0) * max(counts.sum() / nranks, counts.max()) + 1
        # same call, same answer
        again = shard.greedy_partition(counts, nranks)
        assert all(np.array_equal(a, b) for a, b in zip(parts, again))


def test_greedy_partition_edges():
    assert [p.tolist() for p in shard.greedy_partition([], 3)] == [[], [], []]
    assert [p.tolist() for p in shard.greedy_partition([5], 2)] == [[0], []]
    assert [p.tolist() for p in shard.greedy_partition([0, 0, 0, 0], 2)] == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        shard.greedy_partition([1, 2], 0)


def test_local_events_rows():
    off = np.array([0, 3, 3, 10, 12])
    ev, rows, loc = shard.local_events(off, 0, 2)
    ev1, rows1, loc1 = shard.local_events(off, 1, 2)
    assert sorted(ev.tolist() + ev1.tolist()) == [0, 1, 2, 3]
    assert sorted(rows.tolist() + rows1.tolist()) == list(range(12))
    for e, r, lo in ((ev, rows, loc), (ev1, rows1, loc1)):
        for k, evk in enumerate(e):
            assert r[lo[k]:lo[k + 1]].tolist() == list(range(off[evk], off[evk + 1]))
    with pytest.raises(ValueError):
        shard.local_events([0, 5, 2], 0, 2)


def test_plane_config_subset():
    synth = importlib.import_module("wire-cell-toolkit_b200.synth")
    cfg = synth.apa_config(nticks=600)
    sub = shard.plane_config(cfg, [2])
    assert sub["planes"] == [cfg["planes"][2]] and len(sub["fr"]) == 1
    assert len(cfg["planes"]) == 3
    assert shard.plane_partition(3, 2) == [[0, 2], [1]]
    assert shard.plane_partition(3, 4) == [[0], [1], [2], []]


def test_two_rank_fit_and_gather(tmp_path):
    nev = 16
    res = _spawn(tmp_path, nev)
    # every event on exactly one rank
    assert sorted(res[0]["events"] + res[1]["events"]) == list(range(nev))
    _, counts = _event_weights(nev)
    loads = [int(counts[r["events"]].sum()) for r in res]
    assert abs(loads[0] - loads[1]) <= int(counts.max())
    # both ranks took identical steps
    assert res[0]["final"] == res[1]["final"]
    assert res[0]["losses"] == res[1]["losses"]
    # and the same fit as one rank holding all events (sums differ only in order)
    w, _ = _event_weights(nev)
    hist1, final1 = cal.adam_fit(_objective(range(nev), w), P0, steps=40, lr=0.1, decay=0.97)
    np.testing.assert_allclose(res[0]["final"], final1, rtol=1e-10)
    np.testing.assert_allclose(res[0]["losses"], [h[2] for h in hist1], rtol=1e-10)
    # the fit converges towards the truth
    np.testing.assert_allclose(final1, TRUE, rtol=0.05)
    assert hist1[-1][2] < 1e-2 * hist1[0][2]
    # rank 0 holds planes 0 and 2, rank 1 plane 1: stacked in rank order
    g = res[0]["gathered"]
    assert g.shape == (800 + 960 + 800, 16)
    assert np.all(g[:800] == 0) and np.all(g[800:1760] == 2) and np.all(g[1760:] == 1)
    assert res[1]["gathered"] is None
    f = shard.face_order(torch.from_numpy(g), shard.plane_partition(3, 2), [800, 800, 960]).numpy()
    assert np.all(f[:800] == 0) and np.all(f[800:1600] == 1) and np.all(f[1600:] == 2)
