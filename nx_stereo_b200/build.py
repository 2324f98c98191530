"""Builds the CUDA library nx_stereo_b200/libnxs_b200.so for B200 (sm_100a).

`python -m nx_stereo_b200.build [--force]`. The library is built in-tree so
it travels with the sources; nvcc cross-compiles without a GPU.

-fmad=false: no multiply-add is ever contracted, so every f32 step rounds on
its own as the reference evaluates it (the kernels also spell those steps
with __f*_rn intrinsics).
"""
import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBRARY = os.path.join(HERE, "libnxs_b200.so")
PORT = os.path.join(HERE, "nxs_port")
SOURCES = ["matcher.cu", "stages.cu", "abi.cu", "matcher_static.cu", "batch.cu", "band.cu"]
HEADERS = ["nxs_device.cuh", "nxs_kernels.h", "nxs_matcher.cuh", "port_records.h", "port.cpp"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
         "-fmad=false", "-Xcompiler", "-fPIC,-O2", "--expt-relaxed-constexpr"]


def _stale():
    if not os.path.exists(LIBRARY) or not os.path.exists(PORT):
        return True
    inputs = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    inputs.append(os.path.join(ROOT, "include", "nx_stereo_b200.h"))
    inputs.append(os.path.abspath(__file__))
    return os.path.getmtime(LIBRARY) < max(os.path.getmtime(f) for f in inputs)


def build(force=False, verbose=False):
    if not force and not _stale():
        return LIBRARY
    build_dir = os.path.join(HERE, "_build")
    os.makedirs(build_dir, exist_ok=True)
    commands, objects = [], []
    for source in SOURCES:
        obj = os.path.join(build_dir, source.replace(".cu", ".o"))
        cmd = [NVCC] + FLAGS + ["-c", os.path.join(CSRC, source), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd))
        commands.append(cmd)
        objects.append(obj)
    with concurrent.futures.ThreadPoolExecutor(len(commands)) as pool:
        for done in pool.map(lambda c: subprocess.run(c, check=True), commands):
            pass
    tmp = LIBRARY + ".tmp"
    subprocess.run([NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", tmp]
                   + objects + ["-lcudart_static", "-lrt", "-ldl", "-lpthread"], check=True)
    os.replace(tmp, LIBRARY)
    # nxs_port: the stereo_match Port protocol over the library (found beside it).
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", PORT + ".tmp", os.path.join(CSRC, "port.cpp"),
                    "-L", HERE, "-lnxs_b200", "-Wl,-rpath,$ORIGIN", "-lpthread"], check=True)
    os.replace(PORT + ".tmp", PORT)
    return LIBRARY


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
