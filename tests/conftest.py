import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def golden_names():
    with open(os.path.join(GOLDEN, "index.json")) as f:
        return json.load(f)


class Golden:
    """One of the reference's golden cases (rust/crates/piv-core/examples/fixtures.rs:44-116)."""

    def __init__(self, name):
        z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
        self.name = name
        self.z = z
        self.meta = json.loads(bytes(z["meta_json"]).decode())
        self.h, self.w = self.meta["height"], self.meta["width"]
        self.frame_a, self.frame_b = z["frame_a"], z["frame_b"]
        self.background = z["background"] if "background" in z else None
        self.prepared_a = z["prepared_a"] if "prepared_a" in z else self.frame_a
        self.prepared_b = z["prepared_b"] if "prepared_b" in z else self.frame_b
        self.pre = self.meta["preprocess"]
        self.piv = self.meta["piv"]
        self.val = self.piv["validation"]
        self.passes = []
        for i, p in enumerate(self.meta["passes"]):
            d = {"grid": p["grid"], "origins": z[f"pass{i}_origins"]}
            for k in ("dx", "dy", "ppr", "flags"):
                d["raw_" + k] = z[f"pass{i}_raw_{k}"]
                d[k] = z[f"pass{i}_{k}"]
            self.passes.append(d)

    @property
    def base_a(self):
        if self.background is None:
            return self.frame_a
        return np.maximum(self.frame_a - self.background, np.float32(0)).astype(np.float32)

    @property
    def base_b(self):
        if self.background is None:
            return self.frame_b
        return np.maximum(self.frame_b - self.background, np.float32(0)).astype(np.float32)

    @property
    def max_displacement(self):
        return self.piv["windows"][0] / 2.0


@pytest.fixture(params=golden_names())
def golden(request):
    return Golden(request.param)


def same_floats(a, b):
    """Bitwise equality that treats NaN == NaN (RustFixtures.swift `sameFloats`)."""
    a, b = np.asarray(a, np.float32), np.asarray(b, np.float32)
    return a.shape == b.shape and bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))
