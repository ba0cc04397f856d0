"""The batching form (one launch per stage for many pairs, replayed from a CUDA graph) against
the per-pair analysis: results must be bit-identical, on the eager first run, on graph replays
and on new data written into the same input slab."""
import ctypes

import numpy as np
import pytest

from conftest import same_floats

pytestmark = pytest.mark.gpu


def _frames(n, h, w, seed):
    from piv_b200 import synthetic as S
    out = []
    for i in range(n):
        x, y, s, a = S._blobs(h, w, seed + i, 0.04, 2.0, 5.0, 0.47 * 4095, 4095)
        xb, yb = S.displace(x, y, lambda X, Y: (np.float32(2.5) + 0.01 * Y, np.float32(-1.2) + 0.005 * X))
        f = S.render(h, w, x if i % 2 == 0 else xb, y if i % 2 == 0 else yb, s, a)
        out.append(S.quantise(S.add_noise(f, 16.0, seed + 100 + i), 4095, np.uint16))
    return np.stack(out)


def _reference(an, frames, pairs):
    import piv_b200 as P
    res = []
    for ia, ib in pairs:
        fa, fb = an.prepare(frames[ia], P.RAW), an.prepare(frames[ib], P.RAW)
        res.append(an.analyze(fa, fb))
    return res


def _same(r, q):
    assert np.array_equal(r.field.flags, q.field.flags)
    assert same_floats(r.field.dx, q.field.dx) and same_floats(r.field.dy, q.field.dy)
    assert same_floats(r.field.peak_ratio, q.field.peak_ratio)
    assert r.summary.as_dict() == q.summary.as_dict()


@pytest.mark.parametrize("sequential", [True, False])
def test_batch_matches_per_pair_analysis(sequential):
    import piv_b200 as P
    h, w, k = 200, 264, 5
    cfg = P.PivConfig(windows=[64, 32], overlap=0.5, final_iterations=1)
    an = P.PivAnalyzer(cfg)
    nframes = k + 1 if sequential else 2 * k
    pairs = [(i, i + 1) for i in range(k)] if sequential else [(2 * i, 2 * i + 1) for i in range(k)]
    batch = P.PivBatch(an, h, w, k, sequential=sequential)
    for run, seed in enumerate((3, 3, 11)):  # eager run, graph replay, new data through the graph
        frames = _frames(nframes, h, w, seed)
        got = batch.run_host(frames)
        ref = _reference(an, frames, pairs)
        for r, q in zip(got, ref):
            _same(r, q)
    assert batch.kernels() > 0


def test_batch_device_entry_matches():
    import torch

    import piv_b200 as P
    h, w, k = 160, 160, 3
    an = P.PivAnalyzer(P.PivConfig(windows=[32, 16], overlap=0.5, final_iterations=2))
    frames = _frames(2 * k, h, w, 5)
    ref = _reference(an, frames, [(2 * i, 2 * i + 1) for i in range(k)])
    fr = [an.prepare(f, P.RAW) for f in frames]
    g = an.output_grid(h, w)
    c = g.nx * g.ny
    dev = torch.device("cuda", 0)
    dx, dy, ppr = (torch.empty(k * c, device=dev) for _ in range(3))
    fl = torch.empty(k * c, device=dev, dtype=torch.uint8)
    import ctypes
    arr = (ctypes.c_void_p * k)
    a = arr(*[f._h.value for f in fr[0::2]])
    b = arr(*[f._h.value for f in fr[1::2]])
    lib = P.load_library()
    assert lib.piv_analyze_batch_device(an._h, a, b, k, dx.data_ptr(), dy.data_ptr(), ppr.data_ptr(), fl.data_ptr(),
                                        None) == 0
    an.sync()
    for i, r in enumerate(ref):
        sl = slice(i * c, (i + 1) * c)
        assert np.array_equal(fl[sl].cpu().numpy().reshape(g.ny, g.nx), r.field.flags)
        assert same_floats(dx[sl].cpu().numpy().reshape(g.ny, g.nx), r.field.dx)


@pytest.mark.parametrize("depth", [1, 2, 3])
def test_pipeline_matches_per_pair_analysis(depth):
    """Pipelined pairs equal PivAnalyzer.analyze bit for bit, also when more pairs are submitted
    than there are slots (a slot is reused before its ticket is collected) and when tickets are
    collected out of order."""
    import piv_b200 as P
    h, w, k = 200, 264, 5
    an = P.PivAnalyzer(P.PivConfig(windows=[64, 32], overlap=0.5, final_iterations=2))
    frames = _frames(2 * k, h, w, 17)
    ref = _reference(an, frames, [(2 * i, 2 * i + 1) for i in range(k)])
    pl = P.PivPipeline(an, h, w, depth=depth)
    tickets = [pl.submit(frames[2 * i], frames[2 * i + 1]) for i in range(k)]
    order = list(range(k))[::-1]
    for i in order:
        _same(pl.wait(tickets[i]), ref[i])
    # steady state: wait for the oldest before each new submission
    live = []
    for i in range(2 * k):
        if len(live) == depth:
            j, t = live.pop(0)
            _same(pl.wait(t), ref[j % k])
        live.append((i, pl.submit(frames[2 * (i % k)], frames[2 * (i % k) + 1])))
    for j, t in live:
        _same(pl.wait(t), ref[j % k])
    pl.close()


def test_asynchronous_host_submission_alternating_batches():
    """submit_host / wait_host on two batches in turn give the run_host results."""
    import piv_b200 as P
    h, w, k = 160, 192, 3
    an = P.PivAnalyzer(P.PivConfig(windows=[32, 16], overlap=0.5, final_iterations=1))
    frames = [_frames(k + 1, h, w, s) for s in (31, 32)]
    ref = [_reference(an, f, [(i, i + 1) for i in range(k)]) for f in frames]
    bs = [P.PivBatch(an, h, w, k, sequential=True) for _ in range(2)]
    for rnd in range(3):
        for b, f in zip(bs, frames):
            b.submit_host(f)
        for b, r in zip(bs, ref):
            for x, y in zip(b.wait_host(), r):
                _same(x, y)


def test_batches_sharing_one_compute_stream():
    """Two batches replaying on one shared stream (their copies on private streams) give the
    run_host results, submitted back to back and alternating."""
    import piv_b200 as P
    h, w, k = 160, 192, 3
    an = P.PivAnalyzer(P.PivConfig(windows=[32, 16], overlap=0.5, final_iterations=1))
    frames = [_frames(k + 1, h, w, s) for s in (41, 42)]
    ref = [_reference(an, f, [(i, i + 1) for i in range(k)]) for f in frames]
    bs = [P.PivBatch(an, h, w, k, sequential=True) for _ in range(2)]
    bs[1].set_stream(bs[0].stream())
    assert bs[1].stream() == bs[0].stream()
    for rnd in range(3):
        for b, f in zip(bs, frames):
            b.submit_host(f)
        with pytest.raises(P.PivError):
            bs[0].set_stream(None)  # a submission is pending
        for b, r in zip(bs, ref):
            for x, y in zip(b.wait_host(), r):
                _same(x, y)
    bs[1].set_stream(None)
    assert bs[1].stream() != bs[0].stream()
    for b in bs:
        b.close()


def test_repeated_single_pair_calls_replay_the_pass_graph_on_current_data():
    """From the second identical call on, an analyzer replays its passes as a captured CUDA graph.
    The graph reads the frames' current contents: new samples prepared into the same frames,
    swapped frame order (a new key) and a pinned launch variant (new launch choices) all give
    exactly what a fresh analyzer gives."""
    import piv_b200 as P
    from piv_b200 import synthetic as S
    h = w = 256
    cfg = P.PivConfig(windows=[64, 32, 16], overlap=0.5, final_iterations=1)
    pairs = [S.baseline_pair(h, w, 40 + j, lambda x, y, j=j: (1.3 + 0.4 * j, -0.8 + 0.002 * x), ppp=0.05,
                             dmin=2.0, dmax=4.0, bits=12) for j in range(2)]

    def fresh(a, b):
        an0 = P.PivAnalyzer(cfg)
        r = an0.analyze(an0.prepare(a, P.RAW), an0.prepare(b, P.RAW))
        an0.close()
        return r

    def same(r, q):
        for name in ("dx", "dy", "peak_ratio"):
            x, y = getattr(r.field, name), getattr(q.field, name)
            assert np.array_equal(np.isnan(x), np.isnan(y)) and np.array_equal(x[~np.isnan(x)], y[~np.isnan(y)])
        assert np.array_equal(r.field.flags, q.field.flags)
        assert r.summary == q.summary

    refs = [fresh(a, b) for a, b in pairs]
    an = P.PivAnalyzer(cfg)
    fa, fb = an.frame(h, w), an.frame(h, w)
    per_call = None
    for rep in range(3):
        for j, (a, b) in enumerate(pairs):
            fa.prepare(a, P.RAW)
            fb.prepare(b, P.RAW)
            l0 = an.launches()
            same(an.analyze(fa, fb), refs[j])
            n = an.launches() - l0
            per_call = n if per_call is None else per_call
            assert n == per_call  # replays count the kernels they run
    swapped = fresh(pairs[1][1], pairs[1][0])
    for _ in range(3):
        same(an.analyze(fb, fa), swapped)
    an.set_variant(32, P.PivAnalyzer.num_variants(32) - 1)
    for _ in range(3):
        same(an.analyze(fa, fb), refs[1])
    an.close()


def test_pipeline_background_and_clip_match_piv_analyze():
    """A pipeline-wide background (the per-pixel minimum of the run's frames) and a percentile
    clip give each pair exactly what piv_analyze gives with the same background and settings."""
    import torch

    import piv_b200 as P
    h, w, k = 192, 256, 3
    frames = _frames(k + 1, h, w, 77)
    cfg = P.PivConfig(windows=[32, 16], overlap=0.5, final_iterations=1)
    pre = P.PreprocessConfig(smooth_sigma=0.0, normalize_radius=0, normalize_eps=0.0, clip_percentile=99.0)
    an = P.PivAnalyzer(cfg)
    # background over all frames on the device (BackgroundEstimator, min mode)
    dev = torch.from_numpy(frames.view(np.int16)).to("cuda:0")
    bg = torch.empty((h, w), dtype=torch.float32, device="cuda:0")
    st = P.load_library().piv_background_device(an._h, ctypes.c_void_p(dev.data_ptr()), P.api._dtype_code(frames[0]),
                                                k + 1, h, w, 0, ctypes.c_void_p(bg.data_ptr()))
    assert st == 0
    torch.cuda.synchronize()
    bg_host = bg.cpu().numpy()
    assert np.array_equal(bg_host, (frames.min(axis=0).astype(np.float32) / np.float32(65535)).astype(np.float32))
    ref = [an.analyze(an.prepare(frames[i], pre, background=bg_host), an.prepare(frames[i + 1], pre, background=bg_host))
           for i in range(k)]
    pl = P.PivPipeline(an, h, w, dtype=np.uint16, cfg=pre, depth=2)
    pl.set_background(bg.data_ptr())
    tickets = [pl.submit(frames[i], frames[i + 1]) for i in range(k)]
    for t, r in zip(tickets, ref):
        _same(pl.wait(t), r)
    pl.close()


def test_batch_device_calls_replay_their_graph_on_new_frame_contents():
    """piv_analyze_batch_device over K pairs, called repeatedly (eager, captured, replayed), and
    again after new samples were prepared into the same frames: every call equals per-pair
    analysis of the frames' current contents."""
    import torch

    import piv_b200 as P
    h, w, k = 160, 192, 3
    an = P.PivAnalyzer(P.PivConfig(windows=[32, 16], overlap=0.5, final_iterations=1))
    sets = [_frames(2 * k, h, w, 51), _frames(2 * k, h, w, 52)]
    refs = [_reference(an, f, [(2 * i, 2 * i + 1) for i in range(k)]) for f in sets]
    fr = [an.frame(h, w) for _ in range(2 * k)]
    g = an.output_grid(h, w)
    c = g.nx * g.ny
    dev = torch.device("cuda", 0)
    dx, dy, ppr = (torch.empty(k * c, device=dev) for _ in range(3))
    fl = torch.empty(k * c, device=dev, dtype=torch.uint8)
    arr = ctypes.c_void_p * k
    a = arr(*[f._h.value for f in fr[0::2]])
    b = arr(*[f._h.value for f in fr[1::2]])
    lib = P.load_library()
    for s in (0, 0, 0, 1, 1, 0):
        for f, raw in zip(fr, sets[s]):
            f.prepare(raw, P.RAW)
        assert lib.piv_analyze_batch_device(an._h, a, b, k, dx.data_ptr(), dy.data_ptr(), ppr.data_ptr(),
                                            fl.data_ptr(), None) == 0
        an.sync()
        for i, r in enumerate(refs[s]):
            sl = slice(i * c, (i + 1) * c)
            assert np.array_equal(fl[sl].cpu().numpy().reshape(g.ny, g.nx), r.field.flags)
            assert same_floats(dx[sl].cpu().numpy().reshape(g.ny, g.nx), r.field.dx)
            assert same_floats(dy[sl].cpu().numpy().reshape(g.ny, g.nx), r.field.dy)


def test_batch_background_matches_per_pair_analysis_and_can_change():
    """A batch-wide background image (and a percentile clip) gives each pair what analyze gives
    with that background; clearing it re-records the batch, which then matches analysis without
    one."""
    import torch

    import piv_b200 as P
    h, w, k = 160, 224, 3
    frames = _frames(k + 1, h, w, 91)
    pre = P.PreprocessConfig(smooth_sigma=0.0, normalize_radius=0, normalize_eps=0.0, clip_percentile=99.0)
    an = P.PivAnalyzer(P.PivConfig(windows=[32, 16], overlap=0.5, final_iterations=1))
    bg_host = (frames.min(axis=0).astype(np.float32) / np.float32(65535)).astype(np.float32)
    bg = torch.from_numpy(bg_host).to("cuda:0")
    with_bg = [an.analyze(an.prepare(frames[i], pre, background=bg_host), an.prepare(frames[i + 1], pre, background=bg_host))
               for i in range(k)]
    without = [an.analyze(an.prepare(frames[i], pre), an.prepare(frames[i + 1], pre)) for i in range(k)]
    bt = P.PivBatch(an, h, w, k, sequential=True, cfg=pre)
    bt.set_background(bg.data_ptr())
    for _ in range(3):  # eager, captured, replayed
        for x, y in zip(bt.run_host(frames), with_bg):
            _same(x, y)
    bt.set_background(None)
    for _ in range(2):
        for x, y in zip(bt.run_host(frames), without):
            _same(x, y)
    bt.close()
