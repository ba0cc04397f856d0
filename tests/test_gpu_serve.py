"""The serving form: continuous batching of mixed requests. Each result must be the same alone
and in the mix (bit-identical: window pairs are independent inside a launch and every launch
variant of a window size computes the same arithmetic), and must equal PivAnalyzer.analyze of
that pair. Admission must respect the device-memory budget."""
import numpy as np
import pytest

from conftest import same_floats

pytestmark = pytest.mark.gpu


def _pin(a):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a).view(np.int16) if a.dtype == np.uint16 else np.ascontiguousarray(a))
    return t.pin_memory().numpy().view(a.dtype)


def _pair(h, w, seed, shear=0.01, offset=2.0):
    from piv_b200 import synthetic as S
    f = lambda X, Y: (np.float32(offset) + shear * (np.asarray(Y, np.float32) - h / 2), np.float32(0.5 * offset))
    a, b = S.baseline_pair(h, w, seed, f, ppp=0.05, dmin=2.0, dmax=4.0, bits=12)
    return _pin(a), _pin(b)


SCHEDULES = ([32], [64, 32], [64, 32, 16])


def _cfg(sched):
    import piv_b200 as P
    return P.PivConfig(windows=list(sched), overlap=0.5, final_iterations=1)


def _same(r, q):
    assert np.array_equal(r.field.flags, q.field.flags)
    assert same_floats(r.field.dx, q.field.dx) and same_floats(r.field.dy, q.field.dy)
    assert same_floats(r.field.peak_ratio, q.field.peak_ratio)
    assert r.summary.as_dict() == q.summary.as_dict()


def test_results_are_the_same_alone_and_in_the_mix():
    import piv_b200 as P
    rng = np.random.default_rng(0)
    sizes = [(256, 256), (384, 288), (512, 512)]
    reqs = []
    for i in range(18):
        h, w = sizes[i % 3]
        sched = SCHEDULES[int(rng.integers(0, 3))]
        reqs.append((h, w, sched, _pair(h, w, 100 + i, shear=float(rng.uniform(0, 0.02)), offset=float(rng.uniform(0, 4)))))
    # alone: a fresh server per request
    alone = []
    for h, w, sched, (a, b) in reqs[:4]:
        sv = P.PivServer(memory_budget_bytes=1 << 30, max_in_flight=4)
        t = sv.submit(a, b, _cfg(sched))
        alone.append(sv.wait(t)[0])
        sv.close()
    # in the mix: everything at once on one server
    sv = P.PivServer(memory_budget_bytes=1 << 30, max_in_flight=64)
    tickets = [sv.submit(a, b, _cfg(sched)) for h, w, sched, (a, b) in reqs]
    mixed = [sv.wait(t) for t in tickets]
    st = sv.stats()
    sv.close()
    for r, (q, lat) in zip(alone, mixed[:4]):
        _same(r, q)
    assert all(lat > 0 for _, lat in mixed)
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["steps"] < sum(len(s) for _, _, s, _ in reqs)  # passes of different requests shared steps
    # and every request equals the per-pair analysis
    for (h, w, sched, (a, b)), (q, _) in zip(reqs, mixed):
        an = P.PivAnalyzer(_cfg(sched))
        r = an.analyze(an.prepare(a, P.RAW), an.prepare(b, P.RAW))
        _same(r, q)


def test_admission_respects_the_memory_budget():
    import piv_b200 as P
    a, b = _pair(512, 512, 7)
    sv = P.PivServer(memory_budget_bytes=12 << 20, max_in_flight=64)  # room for about two requests
    tickets = [sv.submit(a, b, _cfg([64, 32, 16])) for _ in range(6)]
    res = [sv.wait(t) for t in tickets]
    st = sv.stats()
    assert st["completed"] == 6
    for q, _ in res[1:]:
        _same(res[0][0], q)
    big_a, big_b = _pair(2048, 2048, 9)
    with pytest.raises(P.UnsupportedError):
        sv.submit(big_a, big_b, _cfg([32]))
    sv.close()


def test_one_fused_launch_per_step_gives_the_per_size_results():
    """The FP32 windows of 8-64 px of all requests, uniform and deformed, run in one fused
    correlation launch per step; results are bit-identical to one launch per (size, kind), and
    the steps launch fewer kernels."""
    import piv_b200 as P
    rng = np.random.default_rng(3)
    reqs = []
    for i in range(9):
        h, w = ((256, 256), (384, 288), (512, 512))[i % 3]
        sched = ([32], [64, 32], [64, 32, 16], [32, 16, 8])[i % 4]
        cfg = P.PivConfig(windows=list(sched), overlap=0.5, final_iterations=1, deform=bool(i % 2))
        reqs.append((cfg, _pair(h, w, 500 + i, shear=float(rng.uniform(0, 0.02)), offset=float(rng.uniform(0, 4)))))
    out = {}
    for fused in (True, False):
        sv = P.PivServer(memory_budget_bytes=1 << 30, max_in_flight=64)
        sv.set_fused(fused)
        sv.set_manual(True)  # everything admitted at once: every step mixes sizes and kinds
        tickets = [sv.submit(a, b, cfg) for cfg, (a, b) in reqs]
        sv.advance(3)
        out[fused] = ([sv.wait(t)[0] for t in tickets], sv.stats())
        sv.close()
    for r, q in zip(out[True][0], out[False][0]):
        _same(r, q)
    assert out[True][1]["steps"] == out[False][1]["steps"] == 3
    assert out[True][1]["kernel_launches"] < out[False][1]["kernel_launches"]
    for (cfg, (a, b)), r in zip(reqs, out[True][0]):
        an = P.PivAnalyzer(cfg)
        _same(an.analyze(an.prepare(a, P.RAW), an.prepare(b, P.RAW)), r)


def test_reserved_pool_serves_admissions_without_growing():
    """piv_server_reserve grows the server's own pool ahead of time: a burst of requests whose
    memory in flight stays below the reservation is admitted without the pool mapping more
    memory, and its results equal PivAnalyzer.analyze of each pair."""
    import piv_b200 as P
    sv = P.PivServer(memory_budget_bytes=1 << 30, max_in_flight=64)
    assert sv.reserve(0) == 0
    held = sv.reserve(256 << 20)
    assert held >= 256 << 20
    reqs = [(256, 256, SCHEDULES[i % 3], _pair(256, 256, 300 + i)) for i in range(12)]
    tickets = [sv.submit(a, b, _cfg(sched)) for _, _, sched, (a, b) in reqs]
    results = [sv.wait(t)[0] for t in tickets]
    assert sv.reserve(0) == held, "the pool grew although the burst fitted the reservation"
    for (h, w, sched, (a, b)), r in zip(reqs, results):
        an = P.PivAnalyzer(_cfg(sched))
        _same(r, an.analyze(an.prepare(a, P.RAW), an.prepare(b, P.RAW)))
    with pytest.raises(P.PivError):
        sv.reserve(-1)
    sv.close()


def test_pinned_and_pageable_result_buffers_give_the_same_result():
    """Results land in the caller's buffers whether those are pinned (written by the download
    directly) or pageable (staged through the server's pinned blocks and copied out at retire)."""
    import piv_b200 as P
    sv = P.PivServer(memory_budget_bytes=1 << 30, max_in_flight=16)
    reqs = [(SCHEDULES[i % 3], _pair(256, 256, 400 + i)) for i in range(6)]
    got = []
    for pinned in (False, True):
        outs, tickets = [], []
        for sched, (a, b) in reqs:
            g = P.Grid.new(256, 256, sched[-1], 0.5)
            shape = (g.ny, g.nx)
            if pinned:
                o = tuple(_pin(np.zeros(shape, t)) for t in (np.float32, np.float32, np.float32, np.uint8))
            else:
                o = tuple(np.zeros(shape, t) for t in (np.float32, np.float32, np.float32, np.uint8))
            outs.append(o)
            tickets.append(sv.submit(a, b, _cfg(sched), out=o))
        got.append([(sv.wait(t)[0], o) for t, o in zip(tickets, outs)])
    sv.close()
    for (rp, op), (rq, oq) in zip(*got):
        _same(rp, rq)
        for x, y in zip(op, oq):
            assert np.array_equal(np.asarray(x).view(np.uint8), np.asarray(y).view(np.uint8))
