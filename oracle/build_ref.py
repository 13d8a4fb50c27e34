"""Compile tmol's own CPU implementation of the LJ/LK pose-scoring op from its
sources, for use as a test oracle and as the timed CPU baseline.

This is test infrastructure: only tests, the smoke check and the benchmark's
CPU-baseline leg use what it builds.

The LJ/LK op is two translation units of the reference,
``tmol/score/ljlk/potentials/compiled.ops.cpp`` (the ``torch::autograd``
wrapper registering ``torch.ops.tmol_ljlk.ljlk_pose_scores`` and
``ljlk_rotamer_scores``) and
``tmol/score/ljlk/potentials/ljlk_pose_score.cpu.cpp`` (the CPU instantiation
of the dispatch); the elec op (``torch.ops.tmol_elec.elec_pose_scores``) is
the two matching files under ``tmol/score/elec/potentials``; the stacked
all-pairs-shortest-paths op (``torch.ops.tmol_apsp.apsp_op``, the PoseStack
builder's bond-separation step) is ``tmol/pose/compiled/apsp_vestibule.ops.cpp``
with ``apsp.cpu.cpp``; the LK-ball ops (``torch.ops.tmol_lk_ball``: water
generation and pose / rotamer scores) are ``tmol/score/lk_ball/potentials/
compiled.ops.cpp`` with ``lk_ball_pose_score.cpu.cpp`` and
``gen_pose_waters.cpu.cpp``.  All use
header-only code under ``tmol/`` and the
vendored Eigen / moderngpu headers in ``tmol/extern``.  They are compiled in
place with g++ -O3 through torch's extension builder (no reference build
system is run); the shared library lands in ``oracle/_ref/``.

Usage: ``python oracle/build_ref.py [/path/to/tmol/checkout]``.  Without an
argument the checkout is taken from the ``TMOL_REFERENCE`` environment
variable, else from a ``reference`` directory beside this repository.
"""

import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
LIB_NAME = "tmol_ljlk_ref"
ELEC_LIB_NAME = "tmol_elec_ref"
APSP_LIB_NAME = "tmol_apsp_ref"
LKBALL_LIB_NAME = "tmol_lk_ball_ref"


def reference_root():
    """The tmol checkout the reference ops are compiled from: ``$TMOL_REFERENCE``,
    else ``reference/`` beside this repository's directory."""
    env = os.environ.get("TMOL_REFERENCE")
    if env:
        return env
    return os.path.normpath(os.path.join(HERE, "..", "..", "reference"))


def lib_path():
    return os.path.join(OUT, LIB_NAME + ".so")


def elec_lib_path():
    return os.path.join(OUT, "elec", ELEC_LIB_NAME + ".so")


def apsp_lib_path():
    return os.path.join(OUT, "apsp", APSP_LIB_NAME + ".so")


def lk_ball_lib_path():
    return os.path.join(OUT, "lk_ball", LKBALL_LIB_NAME + ".so")


def build(ref=None, verbose=False):
    from torch.utils.cpp_extension import load

    ref = ref or reference_root()
    t0 = time.time()
    # each op in its own build directory: both have a compiled.ops.cpp
    for name, sub, srcs, out in (
        (LIB_NAME, "score/ljlk/potentials", ["compiled.ops.cpp", "ljlk_pose_score.cpu.cpp"], OUT),
        (
            ELEC_LIB_NAME,
            "score/elec/potentials",
            ["compiled.ops.cpp", "elec_pose_score.cpu.cpp"],
            os.path.join(OUT, "elec"),
        ),
        (APSP_LIB_NAME, "pose/compiled", ["apsp_vestibule.ops.cpp", "apsp.cpu.cpp"], os.path.join(OUT, "apsp")),
        (
            LKBALL_LIB_NAME,
            "score/lk_ball/potentials",
            ["compiled.ops.cpp", "lk_ball_pose_score.cpu.cpp", "gen_pose_waters.cpu.cpp"],
            os.path.join(OUT, "lk_ball"),
        ),
    ):
        src = os.path.join(ref, "tmol", *sub.split("/"))
        if not os.path.isdir(src):
            raise FileNotFoundError(f"reference sources not found under {src}")
        os.makedirs(out, exist_ok=True)
        load(
            name=name,
            sources=[os.path.join(src, f) for f in srcs],
            extra_include_paths=[ref, os.path.join(ref, "tmol", "extern")],
            extra_cflags=["-O3", "-w"],
            is_python_module=False,
            build_directory=out,
            verbose=verbose,
        )
    return time.time() - t0


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else reference_root()
    t = build(ref, verbose=True)
    print(f"built {lib_path()}, {elec_lib_path()}, {apsp_lib_path()} and {lk_ball_lib_path()} in {t:.1f}s")
