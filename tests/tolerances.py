"""Parity tolerances of the CUDA path, shared by the GPU tests.

Energies, per pose:
    |E - E_ref| <= 1e-3 kcal/mol + 1e-5 |E_ref|

Gradients, per component (no component exempt, no scaling by the largest):
    |g - g_ref| <= 1e-4 |g_ref| + 1e-3 kcal/mol/A          (g_close)

against the oracle in float64, i.e. the exact value of the reference's
algorithm for the same float32 inputs.  The relative part is the parity bar
for this path; the absolute floor covers float32 summation order.  A
coordinate's gradient is a sum of one signed contribution per neighbouring
atom, and on these synthetic poses (hard clashes: per-atom contributions of
10^3 kcal/mol/A that cancel to a net of a few kcal/mol/A) the float32 sum
loses up to ~1e-3 kcal/mol/A whichever order it is taken in.  The
reference's own float32 op, measured against its float64 result on eight
150-residue poses (oracle/ljlk_oracle.c is bit-exact with it), has a largest
error of 1.4e-3 kcal/mol/A and no component outside this band.  The scoring
kernels sum in another order (per-atom partial sums in shared memory, then
one global atomic per atom and work item).

Comparing two float32 results of the same sums (the reference op's stored
float32 output, or the GPU path against itself) doubles both terms, since
each side carries its own rounding (g_close_f32).

Rotamer-set gradients (the packer's ops) sum several times more
contributions per coordinate (a rotamer meets every rotamer of each
neighbouring block), and the reference's own float32 rotamer op lands up to
3.5e-3 kcal/mol/A from its float64 result on the test sets: they are held to
the float32-vs-float32 band (g_close_rotamers).

float64 paths are held to 1e-9 relative + 1e-9 absolute.
"""

import numpy

E_RTOL, E_ATOL = 1e-5, 1e-3
G_RTOL, G_FLOOR = 1e-4, 1e-3


def _report(what, err, ref, rtol, floor):
    nz = numpy.abs(ref) > 0
    rel = err[nz] / numpy.abs(ref[nz]) if nz.any() else numpy.zeros(1)
    over = err > rtol * numpy.abs(ref) + floor
    print(
        f"[parity] {what}: {err.size} components, max |dg| {err.max() if err.size else 0:.3e}, "
        f"max rel {rel.max():.3e}, median rel {numpy.median(rel):.3e}, "
        f"beyond 1e-4 rel {(rel > 1e-4).mean():.2e} (within the floor), outside the bar {int(over.sum())}"
    )
    return over


def E_close(E, ref, rtol=E_RTOL, atol=E_ATOL, what="energies"):
    E = numpy.asarray(E, dtype=numpy.float64)
    ref = numpy.asarray(ref, dtype=numpy.float64)
    assert E.shape == ref.shape, (E.shape, ref.shape)
    err = numpy.abs(E - ref)
    over = err > atol + rtol * numpy.abs(ref)
    if err.size:
        print(f"[parity] {what}: {err.size} values, max |dE| {err.max():.3e}, "
              f"max rel {(err / numpy.maximum(numpy.abs(ref), 1e-30)).max():.3e}")
    assert not over.any(), (
        f"{what}: {int(over.sum())} of {err.size} outside |dE| <= {atol} + {rtol}|E|; "
        f"worst {numpy.sort(err[over])[-3:]}"
    )


def g_close(g, ref, rtol=G_RTOL, floor=None, what="gradient"):
    """Per-component gradient check: |g - ref| <= rtol |ref| + floor, with
    floor = 1e-3 for float32 (rtol >= 1e-6) and floor = rtol for float64."""
    if floor is None:
        floor = G_FLOOR if rtol >= 1e-6 else rtol
    g = numpy.asarray(g, dtype=numpy.float64)
    ref = numpy.asarray(ref, dtype=numpy.float64)
    assert g.shape == ref.shape, (g.shape, ref.shape)
    assert numpy.isfinite(g).all(), f"{what}: non-finite components"
    err = numpy.abs(g - ref)
    over = _report(what, err, ref, rtol, floor)
    if over.any():
        idx = numpy.argsort(numpy.where(over, err, 0).ravel())[-3:]
        raise AssertionError(
            f"{what}: {int(over.sum())} of {err.size} components outside |dg| <= {rtol}|g| + {floor}; "
            f"worst (got, ref): {list(zip(g.ravel()[idx], ref.ravel()[idx]))}"
        )


def g_close_f32(g, ref, what="gradient (float32 vs float32)"):
    """Two float32 results of the same sums: each side's band, added."""
    g_close(g, ref, rtol=2 * G_RTOL, floor=2 * G_FLOOR, what=what)


def g_close_rotamers(g, ref, what="rotamer-set gradient"):
    """Rotamer-set gradients against the float64 oracle: the doubled band."""
    g_close(g, ref, rtol=2 * G_RTOL, floor=2 * G_FLOOR, what=what)
