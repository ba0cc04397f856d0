"""The C ABI driven by a plain C99 program (tests/c_driver/piv_c_driver.c) that includes
include/piv_b200.h and links libpivb200.so, the way a Rust or C host binds it, with no Python or
ctypes between them.

- host mode (no GPU): Grid::new on the reference's own test cases (grid.rs:81-108) and
  PivAnalyzer::new's config errors (multipass.rs:91-119) through the header's status codes;
- analyze mode (GPU): the reference's golden pairs, prepared on the host as the reference's
  PreparedFrame holds them (image + IntegralImage f64 tables, preprocess.rs:76-135), analysed
  through piv_frame_set_prepared_tables + piv_analyze, against the Rust-written final fields.
"""
import os
import struct
import subprocess

import numpy as np
import pytest

from conftest import Golden, same_floats

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "c_driver", "piv_c_driver.c")


def reference_integral_tables(base):
    """IntegralImage::new (preprocess.rs:84-103) in the reference's f64 operation order: running
    row sums of v and v*v, each added to the entry above. np.add.accumulate is sequential."""
    v = np.asarray(base, np.float32).astype(np.float64)
    h, w = v.shape
    t1 = np.zeros((h + 1, w + 1), np.float64)
    t2 = np.zeros((h + 1, w + 1), np.float64)
    t1[1:, 1:] = np.add.accumulate(np.add.accumulate(v, axis=1), axis=0)
    t2[1:, 1:] = np.add.accumulate(np.add.accumulate(v * v, axis=1), axis=0)
    return t1, t2


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    import piv_b200 as P
    P.load_library()  # built in-tree
    exe = str(tmp_path_factory.mktemp("c_driver") / "piv_c_driver")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-O2", "-I", os.path.join(ROOT, "include"), SRC,
                    "-L", os.path.join(ROOT, "piv_b200"), "-lpivb200",
                    "-Wl,-rpath," + os.path.join(ROOT, "piv_b200"), "-o", exe], check=True)
    return exe


def test_c_program_host_calls(driver):
    r = subprocess.run([driver, "host"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == "host ok"


def _request(g, path, tables):
    m = g.piv["mask"]
    with open(path, "wb") as f:
        f.write(struct.pack("<qqi", g.h, g.w, len(g.piv["windows"])))
        f.write(struct.pack(f"<{len(g.piv['windows'])}i", *g.piv["windows"]))
        f.write(struct.pack("<fiffi", g.piv["overlap"], g.piv["final_iterations"], m["min_mean"], m["min_std"],
                            int(tables)))
        f.write(np.ascontiguousarray(g.prepared_a, np.float32).tobytes())
        f.write(np.ascontiguousarray(g.prepared_b, np.float32).tobytes())
        if tables:
            for base in (g.base_a, g.base_b):
                for t in reference_integral_tables(base):
                    f.write(t.tobytes())
        else:
            f.write(np.ascontiguousarray(g.base_a, np.float32).tobytes())
            f.write(np.ascontiguousarray(g.base_b, np.float32).tobytes())


def _result(path):
    with open(path, "rb") as f:
        ny, nx = struct.unpack("<qq", f.read(16))
        n = ny * nx
        dx, dy, ppr = (np.frombuffer(f.read(4 * n), np.float32).reshape(ny, nx) for _ in range(3))
        fl = np.frombuffer(f.read(n), np.uint8).reshape(ny, nx)
        summary = struct.unpack("<5q", f.read(40))
    return dx, dy, ppr, fl, summary


@pytest.mark.gpu
@pytest.mark.parametrize("tables", [True, False])
def test_c_program_analyzes_the_golden_pairs(driver, golden, tables, tmp_path):
    g = golden
    # the driver uses the reference's default validation, as every golden case does
    assert (np.float32(g.val["median_eps"]), g.val["median_threshold"], np.float32(g.val["ppr_threshold"])) == (
        np.float32(0.1), 2.0, np.float32(1.3))
    req, res = str(tmp_path / "req.bin"), str(tmp_path / "res.bin")
    _request(g, req, tables)
    r = subprocess.run([driver, "analyze", req, res], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    dx, dy, ppr, fl, summary = _result(res)
    ref = g.passes[-1]
    assert np.array_equal(fl, ref["flags"]), g.name
    fin = np.isfinite(ref["dx"])
    assert np.array_equal(fin, np.isfinite(dx))
    d = np.r_[dx[fin] - ref["dx"][fin], dy[fin] - ref["dy"][fin]]
    # RustParityGPUTests.swift:105-123: final field within 1e-4 px RMS of the reference's
    assert np.sqrt(np.mean(d * d)) < 1e-4 and np.abs(d).max(initial=0) < 1e-3, g.name
    s = g.meta["summary"]
    assert summary == (s["no_signal"], s["low_ppr"], s["median_outliers"], s["out_of_range"], s["replaced"])


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["fog_background_mask", "particles_blank_half"])
def test_reference_tables_give_the_same_field_as_the_base_image(case):
    """piv_frame_set_prepared_tables (the reference's f64 tables) and piv_frame_set_prepared (the
    base image, exact integer tables built on the device) agree bit for bit on the cases with a
    signal mask, and both equal the reference's final field."""
    import piv_b200 as P
    g = Golden(case)
    m = g.piv["mask"]
    cfg = P.PivConfig(windows=list(g.piv["windows"]), overlap=g.piv["overlap"],
                      final_iterations=g.piv["final_iterations"], mask=P.MaskConfig(m["min_mean"], m["min_std"]))
    an = P.PivAnalyzer(cfg)
    fa = an.frame(g.h, g.w).set_prepared_tables(g.prepared_a, *reference_integral_tables(g.base_a))
    fb = an.frame(g.h, g.w).set_prepared_tables(g.prepared_b, *reference_integral_tables(g.base_b))
    r1 = an.analyze(fa, fb)
    ga = an.frame(g.h, g.w).set_prepared(g.prepared_a, g.base_a)
    gb = an.frame(g.h, g.w).set_prepared(g.prepared_b, g.base_b)
    r2 = an.analyze(ga, gb)
    assert np.array_equal(r1.field.flags, r2.field.flags)
    assert same_floats(r1.field.dx, r2.field.dx) and same_floats(r1.field.dy, r2.field.dy)
    assert np.array_equal(r1.field.flags, g.passes[-1]["flags"])
    assert r1.summary.no_signal == g.meta["summary"]["no_signal"]
    bad = reference_integral_tables(g.base_a)[0]
    bad[3, 4] = np.inf
    with pytest.raises(P.PivError, match="non-finite"):
        an.frame(g.h, g.w).set_prepared_tables(g.prepared_a, bad, bad)
