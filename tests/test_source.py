"""Frame sources (rust/crates/piv-io/src/decode.rs): the decoder command line, the raw-frame
stream and its errors, FrameRate parsing (piv-core/src/frame.rs tests), and the stream of pairs
through the GPU pipeline.

ffmpeg is not installed here, so a stand-in decoder (a small Python program written by the test)
takes its place: it records the arguments it was given, emulates the seek, crop and frame count
of that command line on frames the test supplies, and writes them as rawvideo gray / gray16le
to stdout, or fails the ways a decoder fails (a truncated last frame, an error exit with a
message on stderr)."""
import json
import os
import stat
import sys

import numpy as np
import pytest

from piv_b200 import source as SRC

FAKE = r'''#!{python}
import json, os, sys
import numpy as np
args = sys.argv[1:]
with open(os.environ["FAKE_DECODER_LOG"], "w") as f:
    json.dump(args, f)
mode = os.environ.get("FAKE_DECODER_MODE", "ok")
if mode == "fail":
    sys.stderr.write("clip.mp4: Invalid data found when processing input\n")
    sys.exit(1)
frames = np.load(os.environ["FAKE_DECODER_FRAMES"])
rate = float(os.environ.get("FAKE_DECODER_RATE", "50"))
start = 0
if "-ss" in args:
    start = int(float(args[args.index("-ss") + 1]) * rate + 0.5)
vf = args[args.index("-vf") + 1].split(",")
for flt in vf:
    if flt.startswith("crop="):
        w, h, x, y = map(int, flt[5:].split(":"))
        frames = frames[:, y:y + h, x:x + w]
count = int(args[args.index("-frames:v") + 1]) if "-frames:v" in args else len(frames) - start
pix = args[args.index("-pix_fmt") + 1]
dtype = "<u2" if pix == "gray16le" else "u1"
out = sys.stdout.buffer
sel = frames[start:start + count]
for k, fr in enumerate(sel):
    data = np.ascontiguousarray(fr.astype(dtype)).tobytes()
    if mode == "truncate" and k == len(sel) - 1:
        out.write(data[: len(data) // 2])
        out.flush()
        sys.stderr.write("Error while decoding stream #0:0\n")
        sys.exit(0)
    out.write(data)
    if mode == "fail_after" and k == 1:
        out.flush()
        sys.stderr.write("corrupt frame\n")
        sys.exit(1)
out.flush()
'''


@pytest.fixture
def decoder(tmp_path, monkeypatch):
    prog = tmp_path / "ffmpeg"
    prog.write_text(FAKE.replace("{python}", sys.executable))
    prog.chmod(prog.stat().st_mode | stat.S_IXUSR)
    log = tmp_path / "args.json"
    monkeypatch.setenv("FAKE_DECODER_LOG", str(log))

    def setup(frames, mode="ok", rate=50):
        np.save(tmp_path / "frames.npy", frames)
        monkeypatch.setenv("FAKE_DECODER_FRAMES", str(tmp_path / "frames.npy"))
        monkeypatch.setenv("FAKE_DECODER_MODE", mode)
        monkeypatch.setenv("FAKE_DECODER_RATE", str(rate))
        return str(prog), (lambda: json.loads(log.read_text()))
    return setup


def _frames(n, h, w, dtype, seed=0):
    rng = np.random.default_rng(seed)
    hi = 255 if dtype == np.uint8 else 4095
    return rng.integers(0, hi + 1, (n, h, w)).astype(dtype)


def _opts(**kw):
    base = dict(frame_size=(48, 64), container_rate=SRC.FrameRate.new(50, 1))
    base.update(kw)
    return SRC.DecodeOptions(**base)


def test_command_line_is_the_reference_decoders():
    """FfmpegSource::open's arguments (decode.rs:100-171), option by option."""
    cmd, dims, dtype = SRC.ffmpeg_args("clip.mp4", _opts())
    assert cmd == ["ffmpeg", "-nostdin", "-hide_banner", "-v", "error", "-i", "clip.mp4", "-map", "0:v:0", "-an",
                   "-sn", "-dn", "-vf", "format=gray", "-fps_mode", "passthrough", "-f", "rawvideo", "-pix_fmt",
                   "gray", "-"]
    assert dims == (48, 64) and dtype == np.uint8
    o = _opts(start=10, count=5, roi=SRC.Roi(2, 3, 32, 16), channel=SRC.Channel.GREEN, high_bit_depth=True)
    cmd, dims, dtype = SRC.ffmpeg_args("clip.mp4", o)
    # seek half a frame early: frame 9.5 at 50 fps
    assert cmd == ["ffmpeg", "-nostdin", "-hide_banner", "-v", "error", "-ss", "0.190000", "-i", "clip.mp4", "-map",
                   "0:v:0", "-an", "-sn", "-dn", "-vf", "crop=32:16:2:3,format=gbrp16le,extractplanes=g,format=gray16le",
                   "-frames:v", "5", "-fps_mode", "passthrough", "-f", "rawvideo", "-pix_fmt", "gray16le", "-"]
    assert dims == (16, 32) and dtype == np.dtype("<u2")
    cmd, _, _ = SRC.ffmpeg_args("clip.mp4", _opts(channel=SRC.Channel.YPLANE, roi=SRC.Roi(1, 1, 8, 8)))
    assert cmd[cmd.index("-vf") + 1] == "extractplanes=y,crop=8:8:1:1,format=gray"
    with pytest.raises(ValueError, match="exceeds"):
        SRC.ffmpeg_args("clip.mp4", _opts(roi=SRC.Roi(40, 0, 32, 16)))


def test_roi_parsing():
    assert SRC.Roi.parse("10, 20,300,400") == SRC.Roi(10, 20, 300, 400)
    for bad in ("1,2,3", "a,b,c,d", "0,0,0,5", "1,2,3,4,5"):
        with pytest.raises(ValueError):
            SRC.Roi.parse(bad)


@pytest.mark.parametrize("dtype,hbd", [(np.uint8, False), (np.uint16, True)])
def test_frames_stream_through_the_pipe(decoder, dtype, hbd):
    frames = _frames(7, 48, 64, dtype)
    prog, args = decoder(frames)
    with SRC.FfmpegSource("clip.mp4", _opts(high_bit_depth=hbd), program=prog, pinned=False) as src:
        got = [(i, f.copy()) for i, f in src]
    assert [i for i, _ in got] == list(range(7))
    for (_, f), ref in zip(got, frames):
        assert f.dtype == np.dtype(dtype) and np.array_equal(f, ref)
    assert args()[-2] == ("gray16le" if hbd else "gray")


def test_seek_count_and_roi(decoder):
    frames = _frames(20, 48, 64, np.uint8, seed=1)
    prog, args = decoder(frames, rate=50)
    o = _opts(start=6, count=4, roi=SRC.Roi(8, 4, 32, 24))
    with SRC.FfmpegSource("clip.mp4", o, program=prog, pinned=False) as src:
        assert src.dims() == (24, 32)
        got = [(i, f.copy()) for i, f in src]
    assert [i for i, _ in got] == [6, 7, 8, 9]
    for i, f in got:
        assert np.array_equal(f, frames[i, 4:28, 8:40])
    assert np.array_equal(SRC.read_frame("clip.mp4", 13, _opts(), program=prog), frames[13])


def test_truncated_frame_and_failing_decoder_are_errors(decoder):
    frames = _frames(3, 48, 64, np.uint8, seed=2)
    prog, _ = decoder(frames, mode="truncate")
    with SRC.FfmpegSource("clip.mp4", _opts(), program=prog, pinned=False) as src:
        assert src.next_frame()[0] == 0 and src.next_frame()[0] == 1
        with pytest.raises(SRC.DecodeError, match="truncated frame.*Error while decoding"):
            src.next_frame()
    prog, _ = decoder(frames, mode="fail")
    with SRC.FfmpegSource("clip.mp4", _opts(), program=prog, pinned=False) as src:
        with pytest.raises(SRC.DecodeError, match="Invalid data found"):
            src.next_frame()
    prog, _ = decoder(frames, mode="fail_after")
    with SRC.FfmpegSource("clip.mp4", _opts(), program=prog, pinned=False) as src:
        assert src.next_frame()[0] == 0 and src.next_frame()[0] == 1
        with pytest.raises(SRC.DecodeError, match="corrupt frame"):
            src.next_frame()
    with pytest.raises(SRC.DecodeError, match="failed to start"):
        SRC.FfmpegSource("clip.mp4", _opts(), program=os.path.join(os.path.dirname(prog), "no-such-decoder"))


def test_frame_rate_known_answers():
    """The reference's own FrameRate tests (piv-core/src/frame.rs:122-168)."""
    R = SRC.FrameRate
    for s, want in (("240", (240, 1)), ("1000p", (1000, 1)), ("240p", (240, 1)), (" 50P ", (50, 1)),
                    ("120fps", (120, 1)), ("240000/1001", (240000, 1001)), ("50000/1000", (50, 1)),
                    ("239.76", (240000, 1001)), ("29.97", (30000, 1001)), ("23.98", (24000, 1001)),
                    ("119.88p", (120000, 1001)), ("12.5", (25, 2)), ("1000.0", (1000, 1))):
        assert R.parse(s) == R.new(*want), s
    for s in ("", "0", "abc", "-5", "1/0", "0/7", "1.", "nan"):
        with pytest.raises(SRC.FrameRateError):
            R.parse(s)
    assert abs(R.parse("1000").dt(1) - 1e-3) < 1e-15
    assert abs(R.parse("1000").dt(3) - 3e-3) < 1e-15
    assert abs(R.parse("240").dt(1) - 1.0 / 240.0) < 1e-15
    assert abs(R.parse("239.76").dt(2) - 2.0 * 1001.0 / 240000.0) < 1e-15
    assert abs(R.parse("50").time_of(3720.0) - 74.4) < 1e-9


@pytest.mark.gpu
def test_stream_of_pairs_through_the_pipeline_equals_the_analyzer(decoder):
    """analyze_stream (the CLI's pair loop, analyze.rs:388-441) on decoded u16 frames: every
    pair (i, i + stride) equals PivAnalyzer.analyze of the same frames."""
    import piv_b200 as P
    from piv_b200 import synthetic as S
    h, w, n = 256, 320, 7
    f = lambda X, Y: (np.float32(2.5), np.float32(-1.25))
    frames = [S.baseline_pair(h, w, 40 + k, f, ppp=0.05, dmin=2.0, dmax=4.0, bits=12)[0] for k in range(n)]
    frames = np.stack(frames).astype(np.uint16)
    prog, _ = decoder(frames)
    cfg = P.PivConfig(windows=[64, 32], overlap=0.5, final_iterations=1)
    an = P.PivAnalyzer(cfg)
    ref = P.PivAnalyzer(cfg)
    opts = SRC.DecodeOptions(frame_size=(h, w), container_rate=SRC.FrameRate.new(1000, 1), high_bit_depth=True)
    for stride in (1, 2):
        src = SRC.FfmpegSource("clip.mp4", opts, program=prog)
        got = list(SRC.analyze_stream(src, an, stride=stride, depth=3))
        src.close()
        assert [(a, b) for a, b, _ in got] == [(k, k + stride) for k in range(n - stride)]
        for a, b, r in got:
            q = ref.analyze(ref.prepare(frames[a], P.RAW), ref.prepare(frames[b], P.RAW))
            assert np.array_equal(r.field.flags, q.field.flags)
            assert np.array_equal(r.field.dx, q.field.dx, equal_nan=True)
            assert np.array_equal(r.field.dy, q.field.dy, equal_nan=True)
