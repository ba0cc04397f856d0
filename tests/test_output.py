"""NPZ output (write.rs:113-165): the reference's per-pair file name and array names, derived
velocities in f32 as the reference computes them, grid centres with the ROI offset, run.json.
Mirrors the reference's own writer test (piv-io/tests/write.rs `npz_writes_pairs_and_run_json`)."""
import json
import os

import numpy as np

import piv_b200 as P
from piv_b200.output import NpzWriter


def _field(k):
    g = P.Grid.new(96, 128, 32, 0.5)
    dx = np.full((g.ny, g.nx), 1.5 * k, np.float32)
    dy = np.full((g.ny, g.nx), -0.5 * k, np.float32)
    ppr = np.full((g.ny, g.nx), 3.0, np.float32)
    fl = np.zeros((g.ny, g.nx), np.uint8)
    fl[0, 0] = P.flags.NO_SIGNAL
    dx[0, 0] = np.nan
    return P.VectorField(g, dx, dy, ppr, fl)


META = {"tool_version": "test", "frame_width": 1920, "frame_height": 1080,
        "roi": {"x": 100, "y": 50, "width": 128, "height": 96}, "dt_s": 0.002,
        "scale": {"m_per_px": 0.0002452407}, "piv": {"windows": [96, 64]}}


def test_npz_writes_pairs_and_run_json(tmp_path):
    out = tmp_path / "npz"
    w = NpzWriter(out, META)
    f = _field(1.0)
    p = w.write(10, 12, 0.011, f)
    w.finish()
    assert os.path.basename(p) == "pair_000010_000012.npz"
    assert json.load(open(out / "run.json"))["piv"]["windows"] == [96, 64]
    z = np.load(p)
    assert set(z.files) == {"x", "y", "dx", "dy", "u", "v", "u_mps", "v_mps", "peak_ratio", "flags", "frames", "t"}
    assert z["dx"][1, 1] == 1.5 and np.isnan(z["dx"][0, 0])
    assert abs(z["u"][1, 1] - 750.0) < 1e-3          # 1.5 px over 2 ms
    assert abs(z["u_mps"][1, 1] - 750.0 * 0.0002452407) < 1e-4
    assert z["flags"][0, 0] == P.flags.NO_SIGNAL
    assert z["x"][0] == 100.0 + 15.5                  # ROI offset added back
    assert z["y"][0] == 50.0 + 15.5
    assert list(z["frames"]) == [10, 12] and z["frames"].dtype == np.uint64
    assert z["t"].shape == () and abs(float(z["t"]) - 0.011) < 1e-15
    # f32 arithmetic of write.rs: u = dx * f32(1 / dt)
    assert np.array_equal(z["u"][1:], (f.dx[1:] * np.float32(1 / 0.002)).astype(np.float32))


def test_npz_without_scale_has_no_physical_fields(tmp_path):
    meta = dict(META)
    del meta["scale"]
    w = NpzWriter(tmp_path, meta)
    z = np.load(w.write(0, 2, 0.001, _field(2.0)))
    assert "u_mps" not in z.files and "u" in z.files
    assert z["dx"][2, 1] == 3.0
