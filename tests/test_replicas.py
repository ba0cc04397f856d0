"""Replica parallelism (one process per GPU, whole pairs per GPU) on CPU: pair ranges, the
collectives a replica job uses (max over ranks for timing, sums, gathered statistics) with two
gloo ranks, and least-loaded dispatch of requests over devices."""
import json
import os
import socket
import subprocess
import sys

import pytest

from piv_b200.replicas import MultiDeviceServer, least_loaded, pair_range

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_pair_ranges_partition_the_pairs():
    for n in (0, 1, 7, 32, 1999):
        for world in (1, 2, 3, 4, 8):
            got = [pair_range(n, r, world) for r in range(world)]
            assert got[0][0] == 0 and got[-1][1] == n
            for (a, b), (c, d) in zip(got, got[1:]):
                assert b == c  # contiguous, disjoint
            sizes = [b - a for a, b in got]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        pair_range(10, 2, 2)


WORKER = r"""
import json, sys
sys.path.insert(0, sys.argv[1])
from piv_b200.replicas import Ranks, pair_range
r = Ranks(backend="gloo", timeout_s=60)
t = 10.0 + 5.0 * r.rank                  # this rank's timed region (ms)
out = {"rank": r.rank, "world": r.world, "max": r.max(t), "sum": r.sum(r.rank + 1),
       "gather": r.gather({"rank": r.rank, "pairs": pair_range(1999, r.rank, r.world)})}
r.close()
print(json.dumps(out))
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_agree_on_time_and_statistics():
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", WORKER, ROOT], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            so, se = p.communicate(timeout=120)
        except subprocess.TimeoutExpired:
            p.kill()
            raise
        assert p.returncode == 0, se
        outs.append(json.loads(so.strip().splitlines()[-1]))
    for o in outs:
        assert o["world"] == 2
        assert o["max"] == 15.0           # the slower rank's time
        assert o["sum"] == 3.0
        assert [g["rank"] for g in o["gather"]] == [0, 1]
        ranges = [tuple(g["pairs"]) for g in o["gather"]]
        assert ranges == [(0, 1000), (1000, 1999)]


class _FakeServer:
    def __init__(self, device):
        self.device = device
        self.pending = {}
        self.n = 0

    def submit(self, a, b, cfg=None, pre=None):
        self.n += 1
        self.pending[self.n] = (a, b)
        return self.n

    def wait(self, t):
        a, b = self.pending.pop(t)
        return ("done", self.device, len(a))

    def reserve(self, nbytes):
        self.held = getattr(self, "held", 0) + nbytes
        return self.held


class _Buf:
    def __init__(self, nbytes):
        self.nbytes = nbytes

    def __len__(self):
        return self.nbytes


def test_least_loaded_dispatch_keeps_requests_whole():
    assert least_loaded([3, 1, 1, 5]) == 1
    ms = MultiDeviceServer([0, 1, 2], make_server=_FakeServer)
    t1 = ms.submit(_Buf(100), _Buf(100))    # -> device 0 (all idle, lowest index)
    t2 = ms.submit(_Buf(10), _Buf(10))      # -> device 1
    t3 = ms.submit(_Buf(10), _Buf(10))      # -> device 2
    t4 = ms.submit(_Buf(10), _Buf(10))      # -> device 1 (20 outstanding, ties broken by index)
    assert [ms.device_of(t) for t in (t1, t2, t3, t4)] == [0, 1, 2, 1]
    assert ms.wait(t1) == ("done", 0, 100)
    t5 = ms.submit(_Buf(1), _Buf(1))       # device 0 is idle again
    assert ms.device_of(t5) == 0
    for t in (t2, t3, t4, t5):
        ms.wait(t)
    assert ms.load == [0, 0, 0]


def test_reserve_reaches_every_device():
    ms = MultiDeviceServer([0, 1], make_server=_FakeServer)
    assert ms.reserve(1 << 20) == [1 << 20, 1 << 20]
    assert ms.reserve(0) == [1 << 20, 1 << 20]
