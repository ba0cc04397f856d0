"""Frame sources: raw grayscale frames from a video decoder process, handed to the GPU path.

Mirrors the reference's `piv-io` decoding (rust/crates/piv-io/src/decode.rs):
  Channel, Roi ("x,y,w,h")         decode.rs:11-58
  FrameSource (next_frame, dims)   decode.rs:60-66
  DecodeOptions                    decode.rs:68-84
  FfmpegSource                     decode.rs:86-255: the same `ffmpeg` command line (filters,
                                   seek half a frame early, -frames:v, rawvideo gray / gray16le
                                   on stdout), the same errors for a truncated frame or a
                                   failing decoder (with its stderr)
  read_frame                       decode.rs:257-267
  FrameRate                        rust/crates/piv-core/src/frame.rs:14-91
and differs in one place, by design: a frame is returned as its raw u8 / u16 samples (in a
reusable, optionally pinned host buffer) instead of an f32 image, because the conversion v/255 or
v/65535 (decode.rs:227-234) runs on the GPU inside piv_frame_prepare, bit for bit, and the raw
samples are half or a quarter of the bytes to upload.

analyze_stream() runs the reference CLI's pair loop (piv-cli/src/analyze.rs:388-441: a decoder
thread feeding frames, pairs (i, i + stride) analysed in order) through PivPipeline, so the pipe
reads, the uploads and the GPU passes of successive pairs overlap.
"""
import math
import os
import subprocess
import threading
from dataclasses import dataclass, replace
from enum import Enum
from fractions import Fraction
from queue import Queue
from typing import Iterator, Optional, Tuple

import numpy as np

from .api import PivError


class FrameRateError(PivError):
    """PivError::FrameRate (error.rs:4-6)."""


class DecodeError(PivError):
    """The decoder process failed, or a frame was truncated (decode.rs:199-211)."""


@dataclass(frozen=True)
class FrameRate:
    """An exact rational frame rate (frame.rs:14-53)."""
    num: int
    den: int

    @staticmethod
    def new(num: int, den: int) -> "FrameRate":
        if num <= 0 or den <= 0:
            raise FrameRateError(f"{num}/{den}")
        g = math.gcd(num, den)
        return FrameRate(num // g, den // g)

    @staticmethod
    def parse(s: str) -> "FrameRate":
        """`240`, `239.76`, `240000/1001`, `1000p`, `59.94i`, `240fps`; decimals within 0.006 of
        an NTSC rate n*1000/1001 snap to it (frame.rs:55-91)."""
        t = s.strip().lower()
        for suffix in ("fps", "p", "i"):
            if t.endswith(suffix):
                t = t[: -len(suffix)]
                break
        t = t.strip()
        try:
            if "/" in t:
                n, d = t.split("/", 1)
                return FrameRate.new(int(n.strip()), int(d.strip()))
            if "." in t:
                whole, frac = t.split(".", 1)
                f = float(t)
                if not math.isfinite(f) or f <= 0 or not frac or not frac.isdigit():
                    raise ValueError
                n = _round_half_away(f * 1001.0 / 1000.0)
                if n >= 1.0 and abs(n * 1000.0 / 1001.0 - f) < 0.006:
                    return FrameRate.new(int(n) * 1000, 1001)
                return FrameRate.new(int(whole + frac), 10 ** len(frac))
            return FrameRate.new(int(t), 1)
        except (ValueError, FrameRateError):
            raise FrameRateError(s) from None

    def fps(self) -> float:
        return self.num / self.den

    def dt(self, stride: int) -> float:
        """Seconds between frame i and frame i + stride."""
        return stride * self.den / self.num

    def time_of(self, index: float) -> float:
        """Time of (possibly fractional) frame `index` from frame 0, in seconds."""
        return index * self.den / self.num

    def as_fraction(self) -> Fraction:
        return Fraction(self.num, self.den)


def _round_half_away(v: float) -> float:
    return math.floor(v + 0.5) if v >= 0 else math.ceil(v - 0.5)


class Channel(Enum):
    """Which image plane to analyse (decode.rs:11-25)."""
    LUMA = "luma"      # ffmpeg's `gray` conversion
    GREEN = "green"    # the green channel after conversion to RGB
    YPLANE = "yplane"  # the Y plane exactly as stored (extractplanes=y)


@dataclass(frozen=True)
class Roi:
    """Region of interest in full-frame pixels (decode.rs:27-58)."""
    x: int
    y: int
    width: int
    height: int

    @staticmethod
    def parse(s: str) -> "Roi":
        try:
            v = [int(p.strip()) for p in s.split(",")]
        except ValueError:
            raise ValueError(f"invalid ROI {s!r}; expected x,y,w,h") from None
        if len(v) != 4 or v[2] <= 0 or v[3] <= 0 or min(v) < 0:
            raise ValueError(f"invalid ROI {s!r}; expected x,y,w,h with w,h > 0")
        return Roi(*v)


@dataclass(frozen=True)
class DecodeOptions:
    """decode.rs:68-84."""
    frame_size: Tuple[int, int]          # full (height, width), to validate the ROI
    container_rate: FrameRate            # stream rate, used to seek to `start` by timestamp
    start: int = 0
    count: Optional[int] = None          # None: to the end
    channel: Channel = Channel.LUMA
    roi: Optional[Roi] = None
    high_bit_depth: bool = False         # gray16le (sources deeper than 8 bits)


def ffmpeg_args(path: str, opts: DecodeOptions, program: str = "ffmpeg"):
    """The decoder command line of FfmpegSource::open (decode.rs:100-171), the output geometry
    and the sample type."""
    full_h, full_w = opts.frame_size
    if opts.roi is not None:
        r = opts.roi
        if r.x + r.width > full_w or r.y + r.height > full_h:
            raise ValueError(f"ROI {r} exceeds the {full_w}x{full_h} frame")
        x, y, width, height = r.x, r.y, r.width, r.height
    else:
        x, y, width, height = 0, 0, full_w, full_h
    pix, dtype = ("gray16le", np.dtype("<u2")) if opts.high_bit_depth else ("gray", np.dtype(np.uint8))
    filters = []
    # Y before cropping, so odd ROI offsets don't interact with chroma subsampling
    if opts.channel == Channel.YPLANE:
        filters.append("extractplanes=y")
    if opts.roi is not None:
        filters.append(f"crop={width}:{height}:{x}:{y}")
    if opts.channel == Channel.GREEN:
        filters.append("format=" + ("gbrp16le" if opts.high_bit_depth else "gbrp"))
        filters.append("extractplanes=g")
    filters.append(f"format={pix}")
    cmd = [program, "-nostdin", "-hide_banner", "-v", "error"]
    if opts.start > 0:
        # seek half a frame early: the first frame emitted is `start`
        cmd += ["-ss", f"{opts.container_rate.time_of(opts.start - 0.5):.6f}"]
    cmd += ["-i", str(path), "-map", "0:v:0", "-an", "-sn", "-dn", "-vf", ",".join(filters)]
    if opts.count is not None:
        cmd += ["-frames:v", str(opts.count)]
    cmd += ["-fps_mode", "passthrough", "-f", "rawvideo", "-pix_fmt", pix, "-"]
    return cmd, (height, width), dtype


class FfmpegSource:
    """Streams raw grayscale frames from a decoder process (decode.rs:86-255).

    next_frame() returns (index, samples) with samples an [H, W] u8 or u16 array that the source
    reuses: it stays valid until the `buffers`-th next call (a ring of host buffers, pinned when
    torch is available and `pinned` is set, so that uploads from it are asynchronous)."""

    def __init__(self, path: str, opts: DecodeOptions, program: Optional[str] = None, buffers: int = 4,
                 pinned: bool = True):
        program = program or os.environ.get("PIV_FFMPEG", "ffmpeg")
        self.cmd, (self.height, self.width), self.dtype = ffmpeg_args(path, opts, program)
        self.path = str(path)
        self.frame_bytes = self.height * self.width * self.dtype.itemsize
        self._ring = [_host_buffer(self.frame_bytes, pinned) for _ in range(max(1, buffers))]
        self._slot = 0
        self.next_index = opts.start
        self.remaining = opts.count
        try:
            self.child = subprocess.Popen(self.cmd, stdin=subprocess.DEVNULL, stdout=subprocess.PIPE,
                                          stderr=subprocess.PIPE, bufsize=0)
        except OSError as e:
            raise DecodeError(f"failed to start {program} ({e}) - is FFmpeg installed and on PATH?") from None
        self._stderr = []
        self._errt = threading.Thread(target=self._drain_stderr, daemon=True)
        self._errt.start()

    def _drain_stderr(self):
        for chunk in iter(lambda: self.child.stderr.read(4096), b""):
            self._stderr.append(chunk)

    def dims(self):
        return self.height, self.width

    def _fail(self, what):
        self.child.kill()
        self.child.wait()
        self._errt.join(timeout=5)
        err = b"".join(self._stderr).decode(errors="replace").strip()
        return DecodeError(f"{what} decoding {self.path}: {err}")

    def next_frame(self):
        """(index, samples) of the next frame, or None at the end."""
        if self.remaining == 0:
            return None
        buf = self._ring[self._slot]
        view = memoryview(buf)
        filled = 0
        while filled < self.frame_bytes:
            n = self.child.stdout.readinto(view[filled:])
            if not n:
                break
            filled += n
        if filled == 0:
            if self.child.wait() != 0:
                raise self._fail("ffmpeg failed")
            return None
        if filled < self.frame_bytes:
            raise self._fail("truncated frame: ffmpeg failed")
        self._slot = (self._slot + 1) % len(self._ring)
        frame = np.frombuffer(buf, dtype=self.dtype, count=self.height * self.width).reshape(self.height, self.width)
        index = self.next_index
        self.next_index += 1
        if self.remaining is not None:
            self.remaining -= 1
        return index, frame

    def __iter__(self) -> Iterator:
        while True:
            f = self.next_frame()
            if f is None:
                return
            yield f

    def close(self):
        if getattr(self, "child", None) is not None and self.child.poll() is None:
            self.child.kill()
        if getattr(self, "child", None) is not None:
            self.child.wait()
            for s in (self.child.stdout, self.child.stderr):
                if s:
                    s.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def _host_buffer(nbytes, pinned):
    if pinned:
        try:
            import torch
            if torch.cuda.is_available():
                return torch.empty(nbytes, dtype=torch.uint8).pin_memory().numpy()
        except Exception:
            pass
    return np.empty(nbytes, np.uint8)


def read_frame(path: str, index: int, opts: DecodeOptions, program: Optional[str] = None) -> np.ndarray:
    """The single frame at `index` (decode.rs:257-267), as a fresh array of raw samples."""
    with FfmpegSource(path, replace(opts, start=index, count=1), program=program, buffers=1, pinned=False) as src:
        f = src.next_frame()
        if f is None:
            raise DecodeError(f"frame {index} not found in {path}")
        return f[1].copy()


def analyze_stream(source, analyzer, pre=None, background=None, stride: int = 1, depth: int = 3):
    """Yields (index_a, index_b, PairResult) for the pairs (i, i + stride) of the source's frames,
    in order (analyze.rs:388-441). A decoder thread reads frames from the pipe ahead of the GPU;
    PivPipeline uploads, prepares and analyses the pairs with `depth` in flight. `background` is
    a DEVICE image pointer (see PivPipeline.set_background), or None."""
    from .api import RAW, PivPipeline
    h, w = source.dims()
    pl = PivPipeline(analyzer, h, w, dtype=source.dtype, cfg=RAW if pre is None else pre, depth=depth)
    if background is not None:
        pl.set_background(background)
    q: Queue = Queue(maxsize=2 * (stride + depth) + 2)
    done = object()
    errors = []

    def reader():
        try:
            for idx, f in source:
                q.put((idx, f.copy()))  # the source's ring buffer is reused
        except Exception as e:  # reported in the consumer
            errors.append(e)
        q.put(done)

    t = threading.Thread(target=reader, daemon=True)
    t.start()
    window = []
    pending = []
    try:
        while True:
            item = q.get()
            if item is done:
                break
            window.append(item)
            if len(window) > stride:
                (ia, fa), (ib, fb) = window[0], window[stride]
                window.pop(0)
                pending.append((ia, ib, pl.submit(fa, fb)))
                if len(pending) >= depth:
                    a, b, tk = pending.pop(0)
                    yield a, b, pl.wait(tk)
        while pending:
            a, b, tk = pending.pop(0)
            yield a, b, pl.wait(tk)
        if errors:
            raise errors[0]
    finally:
        for _, _, tk in pending:
            try:
                pl.wait(tk)
            except Exception:
                pass
        pl.close()
        t.join(timeout=5)
