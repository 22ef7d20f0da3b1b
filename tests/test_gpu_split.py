"""The split-precision form of the time step: the z (Chebyshev) transforms as
int8-digit contractions on the tensor cores (coral_set_z_transform(h, 1)),
everything else FP64.

Its target: every spectral field within 1e-9 relative L2 of the FP64 oracle
after 100 steps.  The oracle itself is checked over a few steps (it needs
seconds per step at NZ = 192); the 100-step comparison is against the FP64
form on the GPU, which matches the oracle to 1e-10 (test_gpu_parity.py,
test_gpu_parity_sizes.py).  Recipe and initial condition are the benchmark's:
no-slip Rayleigh-Benard at Ra = 1e8, seeded white-noise temperature
(PCG64 seed 2), dt = 1e-6, at 32 x 32 x 192 (the same z length, so the same
kernel instances as at 384 x 384 x 192).
"""
import os
import tempfile

import numpy as np
import pytest

from oracle import coral_oracle as co
from tests.problems import equations, params

pytestmark = pytest.mark.gpu

TOL = 1e-9


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _cfg(name):
    from coral_b200 import CONFIG_DIR
    with open(os.path.join(CONFIG_DIR, name)) as f:
        return f.read()


def _bench_case(d):
    from coral_b200 import initial_conditions as ic
    eq = _cfg("rbc_noslip_ra1e8.equations")
    par = _cfg("rbc_noslip_ra1e8_32x32x192.parameters.in")
    ic.white_noise_temperature(d, 32, 32, 192, seed=2)
    return eq, par


def _field_errors(pl, field, zfields, lay):
    """Relative L2 error per spectral field.  A field whose norm is below 1e-9 of
    the coupled state's (the mean horizontal flow of no-slip convection, which
    carries no net momentum: ~1e-12 of the state here) has no significant digits
    at the 1e-9 level in any finite-precision transform; its error is measured
    against 1e-9 of the state norm instead."""
    f = pl.get_field(0)
    scale = 1e-9 * np.linalg.norm(field)
    errs = {}
    for v in range(lay.nV):
        idx = lay.var_pos[v]
        b = field[..., idx]
        errs["kxky%d" % v] = float(np.linalg.norm(f[..., idx] - b) / max(np.linalg.norm(b), scale))
    for s, z in enumerate(zfields):
        errs["mean%d" % s] = float(np.linalg.norm(pl.get_mean_field(s) - z) / max(np.linalg.norm(z), scale))
    return errs


def test_split_steps_match_oracle():
    from coral_b200.solver import PlaneLayer
    with tempfile.TemporaryDirectory() as d:
        eq, par = _bench_case(d)
        ref = co.Solver(eq, par)
        ref.import_quicksave(d)
        pl = PlaneLayer(eq, par)
        pl.set_z_transform(1)
        pl.import_quicksave(d)
    for _ in range(3):
        ref.step(1e-6)
    pl.march_forward(1e-6, 3)
    pl.synchronize()
    errs = _field_errors(pl, ref.field[0], ref.zfield, ref.lay[0])
    assert max(errs.values()) < TOL, errs
    pl.close()


def test_split_100_steps_within_1e9_of_fp64():
    from coral_b200.solver import PlaneLayer
    with tempfile.TemporaryDirectory() as d:
        eq, par = _bench_case(d)
        a = PlaneLayer(eq, par)
        a.import_quicksave(d)
        b = PlaneLayer(eq, par)
        b.set_z_transform(1)
        b.import_quicksave(d)
    a.march_forward(1e-6, 100)
    b.march_forward(1e-6, 100)
    a.synchronize()
    b.synchronize()
    lay = co.SystemLayout(192, co.parse_equations(eq).kxky[0])
    errs = _field_errors(b, a.get_field(0), [a.get_mean_field(s) for s in range(a.n_zero)], lay)
    assert max(errs.values()) < TOL, errs
    # diagnostics of the split form: same CFL step and kinetic energy to the same bound
    da, db = a.diagnostics(), b.diagnostics()
    assert abs(db["cfl_dt"] - da["cfl_dt"]) <= TOL * da["cfl_dt"]
    assert abs(db["KE"] - da["KE"]) <= TOL * da["KE"]
    a.close()
    b.close()


def test_split_timeseries_and_form_switch():
    """Timeseries objects in the split form match the FP64 form's; switching the
    form back to 0 restores the FP64 path (bit-identical steps)."""
    from coral_b200.solver import PlaneLayer
    ts = (">>Volume_average :: uu <<\n>>Volume_average :: ww <<\n>>Horizontal_avg :: tFull ;; Position= 1 <<\n"
          ">>Horizontal_avg :: tw ;; Position= 7 <<\n>>Volume_average :: tFull <<\n>>EOF<<\n")
    with tempfile.TemporaryDirectory() as d:
        eq, par = _bench_case(d)
        a = PlaneLayer(eq, par)
        a.import_quicksave(d)
        b = PlaneLayer(eq, par)
        b.import_quicksave(d)
    a.set_timeseries(ts)
    b.set_timeseries(ts)
    b.set_z_transform(1)
    a.march_forward(1e-6, 2)
    b.march_forward(1e-6, 2)
    va, vb = a.timeseries()[:5], b.timeseries()[:5]
    assert np.all(np.abs(vb - va) <= 1e-8 * np.abs(va) + 1e-14), (va, vb)
    # back to FP64 on both: b now differs from a only by its two split steps
    b.set_z_transform(0)
    c = PlaneLayer(eq, par)
    c.set_field(0, b.get_field(0))
    for s in range(b.n_zero):
        c.set_mean_field(s, b.get_mean_field(s))
    b.march_forward(1e-6, 1)
    c.march_forward(1e-6, 1)
    assert np.array_equal(b.get_field(0), c.get_field(0))
    for x in (a, b, c):
        x.close()


def test_split_rejects_unsupported_nz():
    from coral_b200.solver import PlaneLayer, CoralError
    pl = PlaneLayer(equations(), params(16, 16, 48))
    with pytest.raises(CoralError) as e:
        pl.set_z_transform(1)
    assert e.value.code == -8
    pl.close()
