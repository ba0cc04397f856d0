"""The split-precision tensor-core correlation (precisions "bf16x3" and "fp16x3").

1. The tcgen05 building blocks: a 128 x n x k GEMM with the operand layouts the correlation uses
   (A K-major and MN-major, B K-major, FP32 accumulators read back from TMEM), exact on small
   integers.
2. One pass of tensor-core correlation against the FP64 oracle on the same origins: NO_SIGNAL
   decisions identical, integer peaks identical, sub-pixel error far below the 0.01 px gate.
3. The whole pipeline within 0.01 px RMS of the FP64 oracle, and the batching and serving forms
   bit-identical to the analyzer.
"""
import ctypes

import numpy as np
import pytest

from conftest import same_floats
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("a_mn", [0, 1])
@pytest.mark.parametrize("n,k", [(16, 16), (32, 32), (64, 64), (32, 64), (128, 32), (256, 16)])
def test_tensor_core_gemm_layouts(a_mn, n, k):
    import torch

    import piv_b200 as P
    rng = np.random.default_rng(n * 1000 + k + a_mn)
    a = rng.integers(-8, 9, (128, k)).astype(np.float32)
    b = rng.integers(-8, 9, (n, k)).astype(np.float32)
    dev = torch.device("cuda", 0)
    ta, tb = torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)
    td = torch.full((128, n), float("nan"), device=dev)
    lib = P.load_library()
    st = lib.piv_tc_selftest(0, a_mn, n, k, ctypes.c_void_p(ta.data_ptr()), ctypes.c_void_p(tb.data_ptr()),
                             ctypes.c_void_p(td.data_ptr()))
    assert st == 0, P._lib.last_error()
    assert np.array_equal(td.cpu().numpy(), a @ b.T)


def _pair(h, seed=4, vmax=6.0):
    from piv_b200 import synthetic as S
    f = S.vortex_shear_field(h, h, vmax=vmax, shear=0.01)
    return S.baseline_pair(h, h, seed, f, ppp=0.05, dmin=2.0, dmax=4.0, bits=12)


def _one_pass_errors(n, precision):
    import piv_b200 as P
    h = 320
    a, b = _pair(h)
    an = P.PivAnalyzer(P.PivConfig(windows=[n], overlap=0.5, final_iterations=1, precision=precision))
    fa, fb = an.prepare(a, P.RAW), an.prepare(b, P.RAW)
    g = an.output_grid(h, h)
    # shifted, fractional origins exercise the bilinear sampler
    base = an.place_windows(h, h, g)
    rng = np.random.default_rng(n)
    sh = rng.uniform(-3, 3, (len(g), 2)).astype(np.float32)
    o = base.copy()
    o[:, 2:] = np.clip(base[:, :2] + sh, 0, h - n - 1)
    dx, dy, ppr, fl = an.correlate_origins(fa, fb, n, o)
    ia, ib = O.u16_to_f32(a), O.u16_to_f32(b)
    odx, ody, oppr, ofl = O.correlate_pass(ia, ib, ia, ib, n, o, mode=O.FP64)
    assert np.array_equal(fl, ofl)
    fin = np.isfinite(odx)
    gd, od = np.r_[dx[fin], dy[fin]], np.r_[odx[fin], ody[fin]]
    oo = np.r_[o[fin, 2] - o[fin, 0], o[fin, 3] - o[fin, 1]]
    # peaks whose sub-pixel offset sits at +-0.5 may round either way
    ambiguous = np.abs(np.abs(od - oo - np.round(od - oo)) - 0.5) < 1e-3
    assert np.mean((np.round(gd - oo) == np.round(od - oo)) | ambiguous) == 1.0
    return np.abs(gd - od)


@pytest.mark.parametrize("precision", ["bf16x3", "fp16x3"])
@pytest.mark.parametrize("n", [64, 32, 16])
def test_one_pass_against_fp64_oracle(n, precision):
    err = _one_pass_errors(n, precision)
    assert np.sqrt(np.mean(err ** 2)) < 1e-3, np.sqrt(np.mean(err ** 2))
    assert np.quantile(err, 0.999) < 0.01


@pytest.mark.parametrize("n", [64, 32, 16])
def test_fp16_halves_are_more_accurate_than_bf16(n):
    e16 = _one_pass_errors(n, "fp16x3")
    eb = _one_pass_errors(n, "bf16x3")
    assert np.sqrt(np.mean(e16 ** 2)) < 0.5 * np.sqrt(np.mean(eb ** 2))


@pytest.mark.parametrize("precision", ["bf16x3", "fp16x3"])
@pytest.mark.parametrize("windows,overlap", [([64, 32, 16], 0.5), ([128, 64, 32, 16], 0.75), ([32, 16], 0.5)])
def test_pipeline_within_0p01_px_rms_of_fp64(windows, overlap, precision):
    import piv_b200 as P
    from piv_b200 import synthetic as S
    h = 512
    f = S.vortex_shear_field(h, h, vmax=8.0, shear=0.01)
    a, b = S.baseline_pair(h, h, 9, f, ppp=0.05, dmin=2.0, dmax=4.0, bits=12)
    an = P.PivAnalyzer(P.PivConfig(windows=windows, overlap=overlap, final_iterations=1, precision=precision))
    r = an.analyze(an.prepare(a, P.RAW), an.prepare(b, P.RAW))
    ref, _, _ = O.analyze(O.OracleConfig(windows, overlap, 1), O.u16_to_f32(a), O.u16_to_f32(b), mode=O.FP64)
    ok = (ref["flags"] == 0) & (r.field.flags == 0)
    d = np.hypot(r.field.dx[ok] - ref["dx"][ok], r.field.dy[ok] - ref["dy"][ok])
    assert ok.mean() > 0.9
    assert np.sqrt(np.mean(d * d)) <= 0.01, np.sqrt(np.mean(d * d))
    assert np.mean(ref["flags"] == r.field.flags) > 0.99


@pytest.mark.parametrize("precision", ["bf16x3", "fp16x3"])
def test_batch_and_server_forms_match_the_analyzer(precision):
    import piv_b200 as P
    h = w = 256
    frames = np.stack([x for s in range(3) for x in _pair(h, seed=20 + s)])
    cfg = P.PivConfig(windows=[64, 32, 16], overlap=0.5, final_iterations=1, precision=precision)
    an = P.PivAnalyzer(cfg)
    ref = [an.analyze(an.prepare(frames[2 * k], P.RAW), an.prepare(frames[2 * k + 1], P.RAW)) for k in range(3)]
    batch = P.PivBatch(an, h, w, 3, sequential=False)
    for _ in range(2):
        for r, q in zip(batch.run_host(frames), ref):
            assert np.array_equal(r.field.flags, q.field.flags)
            assert same_floats(r.field.dx, q.field.dx) and same_floats(r.field.dy, q.field.dy)
    sv = P.PivServer(memory_budget_bytes=1 << 30, max_in_flight=8)
    plain = P.PivConfig(windows=[64, 32, 16], overlap=0.5, final_iterations=1)
    tickets = [(sv.submit(frames[2 * k], frames[2 * k + 1], cfg), sv.submit(frames[2 * k], frames[2 * k + 1], plain))
               for k in range(3)]
    for (tt, tp), q in zip(tickets, ref):
        r, _ = sv.wait(tt)
        sv.wait(tp)
        assert np.array_equal(r.field.flags, q.field.flags)
        assert same_floats(r.field.dx, q.field.dx) and same_floats(r.field.dy, q.field.dy)
    sv.close()


@pytest.mark.parametrize("precision", ["bf16x3", "fp16x3"])
def test_deformed_windows_on_tensor_cores_within_0p01_px_of_fp64(precision):
    """Window deformation (the predictor's bilinear blend over each window) with the 32 and 16 px
    passes on the tensor cores: the final field within 0.01 px RMS of the FP64 oracle's deformed
    analysis, and close to the FP32 kernel's."""
    import piv_b200 as P
    h = 384
    a, b = _pair(h, seed=6, vmax=7.0)
    cfg = dict(windows=[64, 32, 16], overlap=0.5, final_iterations=1, deform=True)
    an = P.PivAnalyzer(P.PivConfig(precision=precision, **cfg))
    assert all("tensor-core" in an.variant(n) for n in (64, 32, 16))
    r = an.analyze(an.prepare(a, P.RAW), an.prepare(b, P.RAW))
    an32 = P.PivAnalyzer(P.PivConfig(**cfg))
    r32 = an32.analyze(an32.prepare(a, P.RAW), an32.prepare(b, P.RAW))
    ref, _, _ = O.analyze(O.OracleConfig((64, 32, 16), 0.5, 1, deform=1), O.u16_to_f32(a), O.u16_to_f32(b),
                          mode=O.FP64)
    ok = (ref["flags"] == 0) & (r.field.flags == 0)
    assert ok.mean() > 0.9
    d = np.hypot(r.field.dx[ok] - ref["dx"][ok], r.field.dy[ok] - ref["dy"][ok])
    assert np.sqrt(np.mean(d * d)) <= 0.01
    assert np.mean(ref["flags"] == r.field.flags) > 0.99
    both = ok & (r32.field.flags == 0)
    d32 = np.hypot(r.field.dx[both] - r32.field.dx[both], r.field.dy[both] - r32.field.dy[both])
    assert np.sqrt(np.mean(d32 * d32)) <= 1e-3


def test_bounded_wait_runs_out_reports_and_leaves_the_device_usable():
    """The tensor-core kernel's mbarrier waits are bounded. On a barrier that nothing completes,
    the wait gives up after the kernel's own bound (about a second), records the timeout in its
    status word and returns; tensor-core work on the same context then runs normally."""
    import piv_b200 as P
    lib = P.load_library()
    timings = {}
    for log2_iters in (10, 18):
        t, ms = ctypes.c_int32(-1), ctypes.c_float(-1.0)
        assert lib.piv_tc_wait_probe(0, log2_iters, ctypes.byref(t), ctypes.byref(ms)) == 0, P._lib.last_error()
        assert t.value == 1
        timings[log2_iters] = ms.value
    assert 0.0 < timings[10] < timings[18] < 5000.0
    t = ctypes.c_int32()
    ms = ctypes.c_float()
    assert lib.piv_tc_wait_probe(0, 19, ctypes.byref(t), ctypes.byref(ms)) != 0  # beyond the kernel's bound
    test_tensor_core_gemm_layouts(0, 32, 32)
    err = _one_pass_errors(32, "bf16x3")  # a correlation pass, whose status checks read the error word
    assert np.sqrt(np.mean(err ** 2)) < 1e-3
