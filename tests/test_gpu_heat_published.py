"""The reference's benchmark 00 (heat equation, error_report.py:4-15) on the
GPU through the C-ABI: the 21 published relative errors of the 10-step decay
of uMean (ARS_111, ARS_222, ARS_443 at seven dt), reproduced by the device's
mean systems, factorisations and time stepping -- pinned to the reference's
own numbers, not to the oracle."""
import json
import math
import os

import numpy as np
import pytest

from tests.heat_problem import heat_equations, heat_params

pytestmark = pytest.mark.gpu

GOLD = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                   "heat_equation_published.json")))


def _heat_equations_with_profile():
    """the benchmark's recipe plus a full variable holding uMean, read back in
    physical space"""
    t = heat_equations()
    a = ">>linear_variable_full_build :: + w <<\n"
    assert t.count(a) == 1
    return t.replace(a, a + ">>linear_variable_full :: uProfile <<\n>>linear_variable_full_build :: + uMean <<\n")


@pytest.mark.parametrize("scheme,key", [("ARS_111", "err111"), ("ARS_222", "err222"), ("ARS_443", "err443")])
def test_heat_equation_published_errors_on_gpu(scheme, key):
    from coral_b200.solver import PlaneLayer
    eq = _heat_equations_with_profile()
    errs = []
    for idx, dt in enumerate(GOLD["dt"]):
        pl = PlaneLayer(eq, heat_params(128, dt, scheme))
        z = 0.5 + np.cos(np.pi * (2 * np.arange(1, pl.NZAA + 1) - 1) / (2 * pl.NZAA)) * 0.5
        pl.set_mean_var_profile(0, 0, 1.34e-4 * np.sin(9 * (z - 1) * np.pi / 2))
        pl.set_mean_var_profile(1, 0, -2.3e-2 * np.sin(7 * z * np.pi / 2))
        pl.set_mean_var_profile(2, 0, np.pi * 1e-3 * np.sin(5 * z * np.pi))
        # the restart's first step at dt / 50 (timeKeeping.f90:108), then 8 + 10 steps
        pl.march_forward(dt / 50, nsteps=1)
        pl.march_forward(dt, nsteps=8)
        u1 = pl.full_phys(1)[0, 0, :].copy()
        pl.march_forward(dt, nsteps=10)
        u2 = pl.full_phys(1)[0, 0, :].copy()
        pl.close()
        rate = 0.33 * (9 * np.pi / 2) ** 2
        err = math.sqrt(np.sum((u2 - u1 * np.exp(-rate * 10 * dt)) ** 2) / np.sum(u1 ** 2))
        errs.append(err)
    # the reference prints four significant digits
    for idx, (e, g) in enumerate(zip(errs, GOLD[key])):
        assert e == pytest.approx(g, rel=2e-3), (scheme, GOLD["dt"][idx], e, g)
