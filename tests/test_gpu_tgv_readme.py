"""End-to-end pin against the reference's own published number.

README.md:13-16 quotes the Taylor-Green dissipation peak of a 64^3 run as
eps = 0.01265 at t = 9.13; docs/figures/readme_header.jl:24-95 is the run
(Re 1600, c0 10, artificial properties off, cfl 0.6, filter every step, to
t = 12, kinetic energy every 10 steps, centred difference and a 5-point
mean).  The device solver, in FP64 and in mixed precision, must reproduce
both numbers to the digits quoted."""
import pytest

import compactles_b200 as cl
from compactles_b200 import tgv_study

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_readme_dissipation_peak(precision):
    res, times, energy = tgv_study.run_case(cl, "readme64", 64, precision)
    assert res["t_end"] == 12.0
    assert round(res["eps_peak"], 5) == 0.01265, res
    assert round(res["t_peak"], 2) == 9.13, res
