"""The serving form's failure paths and its continuous admission, all made on the host: malformed
requests refused at submit, cancellation of queued and admitted requests, bounded waits, device
allocation failures injected into admission (the allocator is not called), and requests that
arrive while others are mid-pass joining them at the next pass boundary. No test makes the GPU
fail; each keeps using the server afterwards and checks its results against the analyzer alone.

Manual stepping (piv_server_set_manual / piv_server_advance) makes the step-level tests
deterministic: the scheduler admits and launches only the steps a test grants.
"""
import numpy as np
import pytest

from test_gpu_serve import _cfg, _pair, _same

pytestmark = pytest.mark.gpu


def _alone(a, b, sched):
    import piv_b200 as P
    an = P.PivAnalyzer(_cfg(sched))
    return an.analyze(an.prepare(a, P.RAW), an.prepare(b, P.RAW))


def test_malformed_requests_are_refused_at_submit_and_the_server_keeps_serving():
    import piv_b200 as P
    a, b = _pair(256, 256, 31)
    sv = P.PivServer(memory_budget_bytes=1 << 30, max_in_flight=8)
    with pytest.raises(P.ConfigError):  # odd window (multipass.rs:98-104)
        sv.submit(a, b, P.PivConfig(windows=[33], overlap=0.5))
    with pytest.raises(P.ConfigError):  # window below 8
        sv.submit(a, b, P.PivConfig(windows=[6], overlap=0.5))
    with pytest.raises(P.ConfigError):  # overlap outside [0, 1)
        sv.submit(a, b, P.PivConfig(windows=[32], overlap=1.0))
    with pytest.raises(P.ConfigError):
        sv.submit(a, b, P.PivConfig(windows=[32], overlap=0.5, final_iterations=0))
    with pytest.raises(P.ImageTooSmallError):  # window larger than the image (grid.rs:27-33)
        sv.submit(a[:48, :48].copy(), b[:48, :48].copy(), P.PivConfig(windows=[64, 32], overlap=0.5))
    with pytest.raises(P.ShapeMismatchError):
        sv.submit(a, b[:128].copy(), _cfg([32]))
    st = sv.stats()
    assert st["submitted"] == 0 and st["queued"] == 0
    r, _ = sv.wait(sv.submit(a, b, _cfg([64, 32])))
    _same(_alone(a, b, [64, 32]), r)
    sv.close()


def test_cancelling_a_queued_request_drops_it_and_the_others_finish():
    import piv_b200 as P
    pairs = [_pair(384, 384, 40 + k) for k in range(3)]
    sv = P.PivServer(memory_budget_bytes=1 << 30, max_in_flight=8)
    sv.set_manual(True)
    t = [sv.submit(a, b, _cfg([64, 32, 16])) for a, b in pairs]
    sv.cancel(t[1])  # nothing admitted yet
    with pytest.raises(P.CancelledError):
        sv.wait(t[1])
    sv.advance(3)
    sv.set_manual(False)
    for k in (0, 2):
        r, _ = sv.wait(t[k])
        _same(_alone(*pairs[k], [64, 32, 16]), r)
    st = sv.stats()
    assert st["cancelled"] == 1 and st["completed"] == 2 and st["failed"] == 0
    sv.close()


def test_cancelling_an_admitted_request_stops_it_at_a_step_boundary():
    import piv_b200 as P
    (a, b), (c, d) = _pair(512, 512, 50), _pair(512, 512, 51)
    sv = P.PivServer(memory_budget_bytes=1 << 30, max_in_flight=8)
    sv.set_manual(True)
    out = tuple(np.full(len(P.Grid.new(512, 512, 16, 0.5)), 7.0, np.float32) for _ in range(3))
    out = out + (np.full(out[0].size, 200, np.uint8),)
    g = P.Grid.new(512, 512, 16, 0.5)
    out = tuple(x.reshape(g.ny, g.nx) for x in out)
    t0 = sv.submit(a, b, _cfg([64, 32, 16]), out=out)
    t1 = sv.submit(c, d, _cfg([64, 32, 16]))
    sv.advance(1)  # both admitted, pass 0 of both launched
    assert sv.stats()["in_flight"] == 2
    sv.cancel(t0)
    sv.advance(2)  # t1 runs its passes 1 and 2; t0 launches nothing more
    with pytest.raises(P.CancelledError):
        sv.wait(t0)
    assert np.all(out[0] == 7.0) and np.all(out[3] == 200)  # a cancelled request's outputs are not written
    r, _ = sv.wait(t1)
    _same(_alone(c, d, [64, 32, 16]), r)
    st = sv.stats()
    assert st["cancelled"] == 1 and st["completed"] == 1 and st["in_flight"] == 0
    assert st["memory_in_use_bytes"] == 0
    sv.set_manual(False)
    r, _ = sv.wait(sv.submit(a, b, _cfg([64, 32, 16])))
    _same(_alone(a, b, [64, 32, 16]), r)
    sv.close()


def test_a_bounded_wait_runs_out_and_the_request_stays_pending():
    import time

    import piv_b200 as P
    a, b = _pair(256, 256, 60)
    sv = P.PivServer(memory_budget_bytes=1 << 30, max_in_flight=8)
    sv.set_manual(True)
    t = sv.submit(a, b, _cfg([64, 32]))
    t_start = time.perf_counter()
    with pytest.raises(P.TimeoutError):
        sv.wait(t, timeout_ms=50.0)
    assert time.perf_counter() - t_start >= 0.045
    sv.advance(2)
    r, _ = sv.wait(t, timeout_ms=30000.0)
    _same(_alone(a, b, [64, 32]), r)
    sv.close()


def test_an_allocation_failure_with_nothing_in_flight_fails_only_that_request():
    import piv_b200 as P
    a, b = _pair(256, 256, 70)
    sv = P.PivServer(memory_budget_bytes=1 << 30, max_in_flight=8)
    sv.fail_next_allocations(1)
    t0 = sv.submit(a, b, _cfg([64, 32]))
    with pytest.raises(P.CudaError, match="out of memory"):
        sv.wait(t0)
    r, _ = sv.wait(sv.submit(a, b, _cfg([64, 32])))
    _same(_alone(a, b, [64, 32]), r)
    st = sv.stats()
    assert st["failed"] == 1 and st["completed"] == 1 and st["memory_in_use_bytes"] == 0
    sv.close()


def test_an_allocation_failure_while_others_run_is_retried_after_one_finishes():
    import piv_b200 as P
    (a, b), (c, d) = _pair(384, 384, 80), _pair(384, 384, 81)
    sv = P.PivServer(memory_budget_bytes=1 << 30, max_in_flight=8)
    sv.set_manual(True)
    t0 = sv.submit(a, b, _cfg([64, 32]))
    sv.advance(1)  # t0 admitted, pass 0 launched
    sv.fail_next_allocations(1)
    t1 = sv.submit(c, d, _cfg([32]))
    sv.advance(1)  # t1's admission fails and is put back; t0 runs its last pass
    st = sv.stats()
    assert st["deferred"] == 1 and st["queued"] == 1 and st["failed"] == 0
    r0, _ = sv.wait(t0)
    sv.advance(1)  # t0 has given its memory back: t1 is admitted and runs
    r1, _ = sv.wait(t1, timeout_ms=30000.0)
    _same(_alone(a, b, [64, 32]), r0)
    _same(_alone(c, d, [32]), r1)
    st = sv.stats()
    assert st["completed"] == 2 and st["failed"] == 0
    sv.close()


def test_a_request_arriving_mid_pass_joins_at_the_next_pass_boundary():
    """Continuous batching: B arrives while A is between its passes, is admitted at the next step
    and shares that step's launches with A's next pass, and finishes first although it came
    later; both results equal the analyzer's alone."""
    import piv_b200 as P
    (a, b), (c, d) = _pair(512, 384, 90), _pair(256, 256, 91)
    sv = P.PivServer(memory_budget_bytes=1 << 30, max_in_flight=8)
    sv.set_manual(True)
    ta = sv.submit(a, b, _cfg([64, 32, 16]))
    sv.advance(1)
    s = sv.stats()
    assert s["steps"] == 1 and s["last_step_requests"] == 1 and s["admitted"] == 1
    tb = sv.submit(c, d, _cfg([64, 32]))  # A is mid-way: pass 0 done, passes 1-2 to go
    sv.advance(1)
    s = sv.stats()
    assert s["steps"] == 2 and s["last_step_requests"] == 2 and s["admitted"] == 2  # joined A's pass 1
    sv.advance(1)
    rb, _ = sv.wait(tb, timeout_ms=30000.0)  # B's last pass ran beside A's pass 2
    rb_stats = sv.stats()
    assert rb_stats["last_step_requests"] == 2 and rb_stats["completed"] >= 1
    ra, _ = sv.wait(ta, timeout_ms=30000.0)
    _same(_alone(a, b, [64, 32, 16]), ra)
    _same(_alone(c, d, [64, 32]), rb)
    sv.close()


def test_arrivals_over_time_overlap_on_the_device_and_match_the_analyzer():
    """Free-running server, requests submitted one by one with gaps while earlier ones are still
    on the GPU: steps are shared, and every result equals its analysis alone."""
    import time

    import piv_b200 as P
    rng = np.random.default_rng(5)
    reqs = []
    for i in range(12):
        h, w = ((2048, 2048), (768, 1024), (512, 512))[i % 3]
        sched = ([32], [64, 32], [64, 32, 16])[int(rng.integers(0, 3))]
        reqs.append((sched, _pair(h, w, 300 + i)))
    sv = P.PivServer(memory_budget_bytes=4 << 30, max_in_flight=64)
    tickets = []
    for sched, (a, b) in reqs:
        tickets.append(sv.submit(a, b, _cfg(sched)))
        time.sleep(0.0002)
    res = [sv.wait(t)[0] for t in tickets]
    st = sv.stats()
    sv.close()
    assert st["completed"] == len(reqs)
    assert st["max_step_requests"] >= 2  # some step advanced requests that had arrived apart
    for (sched, (a, b)), r in zip(reqs, res):
        _same(_alone(a, b, sched), r)
