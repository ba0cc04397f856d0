"""Edge cases on the GPU: the reference's errors (error.rs:4-19: ShapeMismatch, ImageTooSmall,
Config), ragged odd-sized and non-square frames through every stage against the oracle, windows
as large as the frame allows, and u8 input."""
import numpy as np
import pytest

from test_gpu_parity import _stage_check

pytestmark = pytest.mark.gpu


def test_shape_mismatch_and_too_small_images_raise_the_reference_errors():
    import piv_b200 as P
    an = P.PivAnalyzer(P.PivConfig(windows=[32, 16], final_iterations=1))
    a = np.zeros((64, 64), np.float32)
    b = np.zeros((64, 80), np.float32)
    fa, fb = an.prepare(a, P.RAW), an.prepare(b, P.RAW)
    with pytest.raises(P.ShapeMismatchError):
        an.analyze(fa, fb)
    small = np.zeros((20, 40), np.float32)
    with pytest.raises(P.ImageTooSmallError):
        an.analyze(an.prepare(small, P.RAW), an.prepare(small, P.RAW))
    with pytest.raises(P.ConfigError):
        P.PivAnalyzer(P.PivConfig(windows=[33]))
    with pytest.raises(P.ConfigError):
        P.PivAnalyzer(P.PivConfig(windows=[32], overlap=1.0))
    with pytest.raises(P.ConfigError):
        P.PivAnalyzer(P.PivConfig(windows=[32], final_iterations=0))


@pytest.mark.parametrize("h,w,windows,overlap", [(203, 317, [48, 24], 0.5), (131, 97, [32, 16, 8], 0.5),
                                                 (257, 129, [64, 32], 0.75), (65, 65, [64], 0.0),
                                                 (96, 200, [96, 48, 24], 0.5)])
def test_ragged_frames_match_the_oracle_stage_by_stage(h, w, windows, overlap):
    import piv_b200 as P
    from piv_b200 import synthetic as S
    a, b = S.particle_pair(h, w, 13, 0.05, 0.75, lambda x, y: (1.7 + 0.01 * y, -0.9 + 0.004 * x))
    an = P.PivAnalyzer(P.PivConfig(windows=windows, overlap=overlap, final_iterations=2))
    fa, fb = an.prepare(a, P.RAW), an.prepare(b, P.RAW)
    _, traces = an.analyze_traced(fa, fb)
    _stage_check(an, traces, a, b, windows, overlap=overlap)


def test_u8_frames_are_scaled_as_the_reference_decodes_them():
    """u8 samples become v / 255 (decode.rs:227-234): analysing u8 frames equals analysing their
    f32 conversion, bit for bit."""
    import piv_b200 as P
    from piv_b200 import synthetic as S
    f = lambda x, y: (2.3, -1.7)
    a, b = S.baseline_pair(256, 256, 3, f, ppp=0.05, dmin=2.0, dmax=4.0, bits=8)
    assert a.dtype == np.uint8
    an = P.PivAnalyzer(P.PivConfig(windows=[32], overlap=0.5, final_iterations=1))
    r8 = an.analyze(an.prepare(a, P.RAW), an.prepare(b, P.RAW))
    af = (a.astype(np.float32) / np.float32(255)).astype(np.float32)
    bf = (b.astype(np.float32) / np.float32(255)).astype(np.float32)
    rf = an.analyze(an.prepare(af, P.RAW), an.prepare(bf, P.RAW))
    assert np.array_equal(r8.field.flags, rf.field.flags)
    assert np.array_equal(np.nan_to_num(r8.field.dx, nan=9e9), np.nan_to_num(rf.field.dx, nan=9e9))
    ok = r8.field.flags == 0
    assert ok.mean() > 0.9
    # one 32 px pass on 8-bit particles: peak locking leaves a bias of a few hundredths of a pixel
    err = np.hypot(r8.field.dx[ok] - 2.3, r8.field.dy[ok] + 1.7)
    assert np.sqrt(np.mean(err ** 2)) < 0.1 and err.max() < 0.3


@pytest.mark.parametrize("dtype", [np.uint8, np.uint16])
def test_every_code_decodes_as_the_reference_divides(dtype):
    """Every u8 / u16 code becomes exactly f32(code) / 255 or / 65535, correctly rounded as
    decode.rs:227-234 divides, through the vectorised path (aligned buffers) and the per-code path
    (a device pointer one code past an aligned address, and a ragged frame size)."""
    import torch

    import piv_b200 as P
    top = np.iinfo(dtype).max
    h, w = 257, 259  # 66,563 samples: every code, then the sequence again, ragged against 16 bytes
    frame = np.resize(np.arange(top + 1, dtype=np.uint32).astype(dtype), (h, w))
    ref = (frame.astype(np.float32) / np.float32(top)).astype(np.float32)
    an = P.PivAnalyzer(P.PivConfig(windows=[32], final_iterations=1))
    img = an.prepare(frame, P.RAW).image
    assert np.array_equal(img.view(np.uint32), ref.view(np.uint32))
    # the same codes from a device buffer that starts one code past a 16-byte boundary
    flat = np.concatenate([np.zeros(1, dtype), frame.ravel()])
    dev = torch.from_numpy(flat.view(np.int8 if dtype == np.uint8 else np.int16)).to("cuda:0")
    f = an.frame(h, w)
    f.prepare_device(dev.data_ptr() + flat.itemsize, P.api._dtype_code(frame), P.RAW)
    torch.cuda.synchronize()
    assert np.array_equal(f.image.view(np.uint32), ref.view(np.uint32))
