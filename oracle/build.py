"""Builds the CPU oracle into oracle/_build/liboracle.so (test infrastructure).

The reference's Elixir/Nx and Rust code has no compiler in this image; the
oracle is this directory's C restatement of it, and build_ref.py compiles
the reference's compute shaders as C++ to pin that restatement. -ffp-contract=off keeps every f32 operation rounded on its own,
in source order, as the reference evaluates it.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
LIBRARY = os.path.join(BUILD, "liboracle.so")
SOURCES = ["nxs_oracle.c", "nxs_oracle_fast.c", "nxs_oracle_band.c"]


def build(force=False):
    sources = [os.path.join(HERE, s) for s in SOURCES + ["nxs_oracle.h"]]
    if not force and os.path.exists(LIBRARY):
        newest = max(os.path.getmtime(s) for s in sources)
        if os.path.getmtime(LIBRARY) >= newest:
            return LIBRARY
    os.makedirs(BUILD, exist_ok=True)
    command = ["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math",
               "-pthread", "-o", LIBRARY + ".tmp"] + [os.path.join(HERE, s) for s in SOURCES] + ["-lm"]
    subprocess.run(command, check=True)
    os.replace(LIBRARY + ".tmp", LIBRARY)
    return LIBRARY


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
