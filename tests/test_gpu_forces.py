"""Lift and drag on the GPU (fb_forces), checked against the oracle's FP64 restatement of the same
definition (the reference computes no forces, so parity is to this library's own definition),
and against symmetry: a symmetric section at zero incidence carries no lift.

Tolerances: device vs restatement 1e-10 relative (FP64 sums in different orders); zero-lift
|C_L| < 1e-9; float32 fields with the FP64-refined pressure vs the FP64 path 1e-3 relative
on C_L and C_D after a few steps (velocity agrees to about 1e-6, the coefficients to the
pressure solve's tolerance, 1e-6 here: the viscosity solve borrows that tolerance, as in the
reference, and float32 Jacobi cannot reach much below it)."""

import numpy as np
import pytest

from foilbench_b200 import workloads
from foilbench_b200.geometry import NacaFoil
from foilbench_b200.solver import StableFluidsSolver
from oracle.stable_fluids import Grid, surface_forces

pytestmark = pytest.mark.gpu


def _run(sc, steps):
    s = StableFluidsSolver()
    s.initialize(sc, NacaFoil(sc.foil), 0)
    for k in range(steps):
        s.advance(sc.control_at((k + 1) * sc.output_dt), sc.output_dt)
    return s


def _oracle_forces(s, sc):
    u, v = s.face_velocities()
    ctl = sc.control_at(0.0)
    return surface_forces(u, v, s.pressure(), s.solid_mask(), Grid.from_domain(sc.domain), 1.0 / sc.reynolds,
                          ctl.angular_velocity_degrees, sc.foil.pivot, sc.freestream, sc.foil.chord)


@pytest.mark.parametrize("precision", ["float64", "float32"])
def test_device_forces_match_the_restatement(precision):
    sc = workloads.single("f", 256, 128, "2412", 8.0, 1000.0, precision=precision, tolerance=1e-6)
    s = _run(sc, 4)
    got, ref = s.forces(), _oracle_forces(s, sc)
    for k, want in ref.items():
        assert got[k] == pytest.approx(want, rel=1e-10, abs=1e-12), k


def test_symmetric_section_at_zero_incidence_has_no_lift():
    sc = workloads.single("sym", 256, 128, "0012", 0.0, 1000.0, precision="float64", tolerance=1e-10)
    f = _run(sc, 4).forces()
    assert abs(f["lift_coefficient"]) < 1e-9
    assert f["drag_coefficient"] > 0.0


def test_mirrored_incidence_mirrors_lift_and_fp32_tracks_fp64():
    """The reference's angle turns the section counter-clockwise about its pivot (trailing edge
    up), so +8 deg meets the stream nose-down: negative lift, and -8 deg the mirror image."""
    c = {}
    for prec, angle in (("float64", 8.0), ("float64", -8.0), ("float32", 8.0)):
        sc = workloads.single("lift", 256, 128, "0012", angle, 1000.0, precision=prec, tolerance=1e-6)
        c[(prec, angle)] = _run(sc, 4).forces()
    up, down = c[("float64", 8.0)], c[("float64", -8.0)]
    assert up["lift_coefficient"] < -0.05 and up["drag_coefficient"] > 0.0
    assert down["lift_coefficient"] == pytest.approx(-up["lift_coefficient"], rel=1e-6)
    assert down["drag_coefficient"] == pytest.approx(up["drag_coefficient"], rel=1e-6)
    for k in ("lift_coefficient", "drag_coefficient"):
        assert c[("float32", 8.0)][k] == pytest.approx(up[k], rel=1e-3), k
