"""bench.py --gpus N starts its own N ranks (one process per GPU) when no
launcher did, and refuses a world that is not the N it was asked for.  The
plumbing is checked on CPU: bench.relaunch starts two gloo ranks of a stub
(tests/bench_launch_stub.py) that use bench.py's own rank setup and
max-over-ranks reduction."""

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_relaunch_two_ranks(tmp_path):
    stub = os.path.join(ROOT, "tests", "bench_launch_stub.py")
    rc = bench.relaunch(2, stub, ["--gpus", "2", "--out", str(tmp_path)], timeout_s=240)
    assert rc == 0
    got = [json.load(open(tmp_path / ("rank%d.json" % r))) for r in range(2)]
    assert [g["rank"] for g in got] == [0, 1]
    assert all(g["world"] == 2 for g in got)
    assert sorted(g["local"] for g in got) == [0, 1]
    worst = max(g["ms"] for g in got)
    # every rank holds the slowest rank's time
    assert all(abs(g["max_ms"] - worst) < 1e-9 for g in got)
    assert got[1]["ms"] > got[0]["ms"]


def test_world_mismatch_is_refused():
    env = dict(os.environ, WORLD_SIZE="1", RANK="0", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--steps", "1"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode != 0
    assert "--gpus 2 but WORLD_SIZE=1" in r.stderr


def test_dist_setup_plain_run(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)

    class A:
        gpus = 1
    assert bench.dist_setup(A()) == (0, 1, 0)
    A.gpus = 3
    with pytest.raises(SystemExit):
        bench.dist_setup(A())
