"""Build the in-tree CUDA library for sm_100a.

    python -m tmol_b200.build

Compiles ``tmol_b200/csrc/*.cu`` with nvcc into
``tmol_b200/lib/libtmol_b200_ljlk.so`` (static CUDA runtime, so the library
does not depend on the runtime version torch bundles).
"""

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "lib", "libtmol_b200_ljlk.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["ljlk.cu", "ljlk_noalloc.cu", "screen.cu", "bondsep.cu"]
HEADERS = ["ljlk_potentials.cuh", "elec_potentials.cuh", "bondsep.cuh"]


def nvcc_path():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise FileNotFoundError("nvcc not found")


def _stale():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(SRC, f) for f in SOURCES + HEADERS]
    for h in ("tmol_b200_ljlk.h", "tmol_b200_screen.h", "tmol_b200_elec.h", "tmol_b200_pose.h"):
        deps.append(os.path.join(HERE, "..", "include", h))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False, extra=()):
    if not force and not _stale():
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cmd = (
        [nvcc_path()]
        + ARCH
        + [
            "-O3",
            "-lineinfo",
            "--use_fast_math",
            "-std=c++17",
            "-Xcompiler",
            "-fPIC",
            "-shared",
            "-cudart",
            "static",
            "-o",
            OUT + ".tmp",
        ]
        + list(extra)
        + [os.path.join(SRC, f) for f in SOURCES]
    )
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, extra=[a for a in sys.argv[1:] if a != "--force"]))
