"""Builds the device-view consumer kernel (test code) into
``tests/consumer/lib/libview_consumer.so`` with nvcc for sm_100a."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
SRC = os.path.join(HERE, "view_consumer.cu")
LIB = os.path.join(HERE, "lib", "libview_consumer.so")


def ensure_built() -> str:
    header = os.path.join(ROOT, "include", "octopus_b200.h")
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(SRC), os.path.getmtime(header)):
        return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    nvcc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    subprocess.run([nvcc if os.path.exists(nvcc) else "nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3",
                    "-std=c++17", "-fmad=false", "-shared", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include"),
                    SRC, "-o", LIB], check=True)
    return LIB


if __name__ == "__main__":
    print(ensure_built())
