"""Compile tmol's own CPU implementation of the LJ/LK pose-scoring op from its
sources, for use as a test oracle and as the timed CPU baseline.

This is test infrastructure: only tests, the smoke check and the benchmark's
CPU-baseline leg use what it builds.

The op is two translation units of the reference,
``tmol/score/ljlk/potentials/compiled.ops.cpp`` (the ``torch::autograd``
wrapper registering ``torch.ops.tmol_ljlk.ljlk_pose_scores``) and
``tmol/score/ljlk/potentials/ljlk_pose_score.cpu.cpp`` (the CPU instantiation
of the pose-score dispatch), plus header-only code under ``tmol/`` and the
vendored Eigen / moderngpu headers in ``tmol/extern``.  They are compiled in
place with g++ -O3 through torch's extension builder (no reference build
system is run); the shared library lands in ``oracle/_ref/``.

Usage: ``python oracle/build_ref.py [/path/to/tmol/checkout]``
"""

import os
import sys
import time

REF_DEFAULT = "/root/reference"
HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
LIB_NAME = "tmol_ljlk_ref"


def lib_path():
    return os.path.join(OUT, LIB_NAME + ".so")


def build(ref=REF_DEFAULT, verbose=False):
    from torch.utils.cpp_extension import load

    src = os.path.join(ref, "tmol", "score", "ljlk", "potentials")
    if not os.path.isdir(src):
        raise FileNotFoundError(f"reference sources not found under {src}")
    os.makedirs(OUT, exist_ok=True)
    t0 = time.time()
    load(
        name=LIB_NAME,
        sources=[
            os.path.join(src, "compiled.ops.cpp"),
            os.path.join(src, "ljlk_pose_score.cpu.cpp"),
        ],
        extra_include_paths=[ref, os.path.join(ref, "tmol", "extern")],
        extra_cflags=["-O3", "-w"],
        is_python_module=False,
        build_directory=OUT,
        verbose=verbose,
    )
    return time.time() - t0


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else REF_DEFAULT
    print(f"built {lib_path()} in {build(ref, verbose=True):.1f}s")
