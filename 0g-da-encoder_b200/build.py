"""Build recipe of the B200 encoder library (nvcc, sm_100a, in-tree).

The library is a single translation unit, csrc/zg_encoder.cu, compiled to
_build/libzg_encoder_b200.so. nvcc cross-compiles without a GPU.
"""
import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "libzg_encoder_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
]


def _sources():
    out = [os.path.join(INCLUDE, "zg_encoder.h")]
    for name in sorted(os.listdir(CSRC)):
        if name.endswith((".cu", ".cuh", ".h", ".hpp")):
            out.append(os.path.join(CSRC, name))
    return out


def _host_compiler():
    # the system g++ (an environment CXX wrapper may lack OpenMP specs)
    for cand in ("/usr/bin/g++", shutil.which("g++")):
        if cand and os.path.exists(cand):
            return cand
    return None


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(p) > t for p in _sources())


def build(force=False, verbose=False):
    """Compile the library if a source is newer than it; returns its path."""
    if not force and not needs_build():
        return LIB
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    os.makedirs(BUILD, exist_ok=True)
    cmd = [nvcc] + NVCC_FLAGS
    cc = _host_compiler()
    if cc:
        cmd += ["-ccbin", cc]
    tmp = LIB + ".tmp"
    cmd += ["-o", tmp, os.path.join(CSRC, "zg_encoder.cu")]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + res.stdout + res.stderr)
    if verbose:
        print(res.stdout + res.stderr)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True, verbose=True))
