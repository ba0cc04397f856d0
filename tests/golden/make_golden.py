"""Regenerates tests/golden/*.npz from the reference's own golden fixtures.

The reference's Rust fixture generator (rust/crates/piv-core/examples/fixtures.rs:44-201) wrote
seven cases, stage by stage, to swift/Tests/PIVKitTests/Fixtures/cases/<case>/ as raw
little-endian .f32/.u8 arrays plus meta.json. This script packs each case into one compressed
.npz so that the tests can run where the reference tree is absent. Arrays are copied unchanged;
`prepared_a`/`prepared_b` are omitted when they equal the raw frames bit for bit (cases run with
no preprocessing and no background), and the tests then use the frames.

Usage: python tests/golden/make_golden.py <reference_root>
   or: PIV_REFERENCE_ROOT=<reference_root> python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

CASES_REL = "swift/Tests/PIVKitTests/Fixtures/cases"
HERE = os.path.dirname(os.path.abspath(__file__))


def load_case(case_dir):
    with open(os.path.join(case_dir, "meta.json")) as f:
        meta = json.load(f)
    h, w = meta["height"], meta["width"]

    def f32(name, shape=None):
        a = np.fromfile(os.path.join(case_dir, name), dtype="<f4")
        return a.reshape(shape) if shape is not None else a

    def u8(name, shape=None):
        a = np.fromfile(os.path.join(case_dir, name), dtype=np.uint8)
        return a.reshape(shape) if shape is not None else a

    out = {
        "frame_a": f32(meta["frame_a"], (h, w)),
        "frame_b": f32(meta["frame_b"], (h, w)),
    }
    if meta.get("background"):
        out["background"] = f32(meta["background"], (h, w))
    pa = f32(meta["prepared_a"], (h, w))
    pb = f32(meta["prepared_b"], (h, w))
    same = np.array_equal(pa.view(np.uint32), out["frame_a"].view(np.uint32)) and np.array_equal(
        pb.view(np.uint32), out["frame_b"].view(np.uint32)
    )
    if not same:
        out["prepared_a"] = pa
        out["prepared_b"] = pb
    for i, p in enumerate(meta["passes"]):
        g = p["grid"]
        shape = (g["ny"], g["nx"])
        out[f"pass{i}_origins"] = f32(p["origins"], (g["ny"] * g["nx"], 4))
        for kind, key in (("raw", "raw"), ("validated", "")):
            fld = p[kind]
            pre = f"pass{i}_raw_" if key else f"pass{i}_"
            out[pre + "dx"] = f32(fld["dx"], shape)
            out[pre + "dy"] = f32(fld["dy"], shape)
            out[pre + "ppr"] = f32(fld["peak_ratio"], shape)
            out[pre + "flags"] = u8(fld["flags"], shape)
    meta["prepared_is_frame"] = bool(same)
    out["meta_json"] = np.frombuffer(json.dumps(meta, sort_keys=True).encode(), dtype=np.uint8)
    return out


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PIV_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: make_golden.py <reference_root> (or set PIV_REFERENCE_ROOT): the checkout of the reference "
                 "whose " + CASES_REL + " holds the cases")
    cases_dir = os.path.join(root, CASES_REL)
    with open(os.path.join(cases_dir, "index.json")) as f:
        names = json.load(f)
    for name in names:
        arrays = load_case(os.path.join(cases_dir, name))
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **arrays)
        print(name, sorted(k for k in arrays if not k.startswith("pass")))
    with open(os.path.join(HERE, "index.json"), "w") as f:
        json.dump(names, f, indent=2)


if __name__ == "__main__":
    main()
