"""Build recipe for the CPU oracle library (test infrastructure only).

Compiles oracle/piv_oracle.cpp into oracle/_build/libpivoracle.so with OpenMP and
-ffp-contract=off (no FMA contraction, matching the Rust reference's f32 rounding).
The reference itself is Rust and cannot be compiled here (no cargo), so there is no
oracle/_ref build; this restatement is the oracle.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "piv_oracle.cpp")
OUT_DIR = os.path.join(HERE, "_build")
OUT = os.path.join(OUT_DIR, "libpivoracle.so")


def build(force: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    deps = [SRC, os.path.join(HERE, "piv_oracle.h")]
    if not force and os.path.exists(OUT) and all(os.path.getmtime(OUT) >= os.path.getmtime(d) for d in deps):
        return OUT
    cmd = [
        "g++", "-O3", "-std=c++17", "-fPIC", "-shared", "-fopenmp",
        "-march=x86-64-v3", "-ffp-contract=off", "-fno-fast-math",
        SRC, "-o", OUT + ".tmp",
    ]
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
