"""Parity of the kernel instances the benchmark configurations run, at their sizes.

The transform kernels are compiled per FFT length with their own plans (two
passes of radix 24 x 24 for 576 and 18 x 16 for 288, three-pass plans
elsewhere), so each length used by a benchmark grid is its own code path:

* 384 x 384 x 192 (grid 576 x 576 x 288): k_inv_y<576>, k_inv_x<576>,
  k_fwd_x<576>, k_fwd_y_pipe<576> in x / y and the z passes at 288;
* 192 x 192 x 96 (grid 288 x 288 x 144): the 288-point x / y passes, 144 in z;
* the fused z kernel of the time step, k_z_fused<288>, runs at NZ = 192 and
  k_z_fused<144> at NZ = 96: a few steps at 32 x 32 x 192 (the benchmark's
  recipe and Rayleigh number) and at 24 x 24 x 96 (the rotating stress-free
  recipe at Ekman 1e-4, Ra 5e7, its box size and time step) are compared with
  the oracle.

Tolerances as in the other parity tests: transforms to 1e-13 of the field's
maximum, steps to 1e-11 relative L2 per coupled variable.
"""
import os

import numpy as np
import pytest

from oracle import coral_oracle as co
from tests.problems import equations, params

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _cfg(name):
    from coral_b200 import CONFIG_DIR
    with open(os.path.join(CONFIG_DIR, name)) as f:
        return f.read()


@pytest.mark.parametrize("eqname,parname", [
    ("rbc_noslip_ra1e8.equations", "rbc_noslip_ra1e8_384x384x192.parameters.in"),
    ("rrbc_stressfree_ek1e-4_ra5e7.equations", "rrbc_stressfree_192x192x96.parameters.in"),
])
def test_transforms_at_benchmark_sizes(eqname, parname):
    from coral_b200.solver import PlaneLayer
    eq, par = _cfg(eqname), _cfg(parname)
    p = co.read_parameters_text(par)
    g = co.Geometry(p["NX"], p["NY"], p["NZ"], p["Lx"], p["Ly"], p["gap"], p["center"])
    pl = PlaneLayer(eq, par)
    rng = np.random.default_rng(17)
    spec = rng.standard_normal((g.NXH, g.NYAA, g.NZ)) + 1j * rng.standard_normal((g.NXH, g.NYAA, g.NZ))
    p_gpu = pl.spec_to_phys(spec)
    p_ref = co.spec_to_phys(spec, g)
    assert np.abs(p_gpu - p_ref).max() <= 1e-13 * np.abs(p_ref).max()
    del p_gpu, spec
    s_gpu = pl.phys_to_spec(p_ref)
    s_ref = co.phys_to_spec(p_ref, g)
    assert np.abs(s_gpu - s_ref).max() <= 1e-13 * np.abs(s_ref).max()
    pl.close()


def _random_state(solver, pl, seed, amp):
    rng = np.random.default_rng(seed)
    for s, lay in enumerate(solver.lay):
        f = amp * (rng.standard_normal((pl.NXH, pl.NYAA, lay.T)) + 1j * rng.standard_normal((pl.NXH, pl.NYAA, lay.T)))
        solver.field[s] = f.copy()
        pl.set_field(s, f)
    for s, lay in enumerate(solver.zlay):
        z = amp * rng.standard_normal(lay.T)
        solver.zfield[s] = z.copy()
        pl.set_mean_field(s, z)


def _steps_match(eq, par, dt, nsteps, seed, amp):
    from coral_b200.solver import PlaneLayer
    ref = co.Solver(eq, par)
    pl = PlaneLayer(eq, par)
    _random_state(ref, pl, seed, amp)
    for _ in range(nsteps):
        ref.step(dt)
    pl.march_forward(dt, nsteps)
    pl.synchronize()
    f_gpu = pl.get_field(0)
    lay = ref.lay[0]
    for v in range(lay.nV):
        idx = lay.var_pos[v]
        assert _rel(f_gpu[..., idx], ref.field[0][..., idx]) < 1e-11, ref.recipe.kxky[0].vars[v]
    for s in range(len(ref.zlay)):
        assert _rel(pl.get_mean_field(s), ref.zfield[s]) < 1e-11
    pl.close()


def test_steps_rbc_ra1e8_nz192_match_oracle():
    """3 ARS_222 steps of the benchmark recipe (no-slip, Ra = 1e8) at 32 x 32 x 192:
    the fused z kernel at NZAA = 288 (radix 18 x 16)."""
    _steps_match(_cfg("rbc_noslip_ra1e8.equations"), _cfg("rbc_noslip_ra1e8_32x32x192.parameters.in"),
                 dt=1e-6, nsteps=3, seed=21, amp=1e-2)


def test_steps_rrbc_cfg1_parameters_match_oracle():
    """3 ARS_222 steps of the rotating stress-free recipe at its configured
    Ekman 1e-4 and Ra 5e7, box 2.9164 and dt 5e-6, at 24 x 24 x 96 (z length 144
    as in the 192 x 192 x 96 configuration)."""
    p = co.read_parameters_text(_cfg("rrbc_stressfree_192x192x96.parameters.in"))
    par = params(24, 24, 96, dt=5e-6, Lx=p["Lx"], Ly=p["Ly"])
    _steps_match(_cfg("rrbc_stressfree_ek1e-4_ra5e7.equations"), par, dt=5e-6, nsteps=3, seed=22, amp=1e-2)


@pytest.mark.parametrize("n", [(128, 128, 128), (256, 256, 128)])
def test_transforms_at_the_closure_grids(n):
    """The closure's grids: x / y lengths 192 and 384, z length 192 (the
    instances whose static plus dynamic shared memory crosses 48 KB without
    either alone doing so)."""
    from coral_b200.solver import PlaneLayer
    eq = _cfg("rbc_noslip_ra1e8.equations")
    par = params(*n, dt=1e-6)
    p = co.read_parameters_text(par)
    g = co.Geometry(p["NX"], p["NY"], p["NZ"], p["Lx"], p["Ly"], p["gap"], p["center"])
    pl = PlaneLayer(eq, par)
    rng = np.random.default_rng(19)
    spec = rng.standard_normal((g.NXH, g.NYAA, g.NZ)) + 1j * rng.standard_normal((g.NXH, g.NYAA, g.NZ))
    p_ref = co.spec_to_phys(spec, g)
    assert np.abs(pl.spec_to_phys(spec) - p_ref).max() <= 1e-13 * np.abs(p_ref).max()
    s_ref = co.phys_to_spec(p_ref, g)
    assert np.abs(pl.phys_to_spec(p_ref) - s_ref).max() <= 1e-13 * np.abs(s_ref).max()
    pl.close()


def test_steps_nz128_match_oracle():
    """3 ARS_222 steps at 16 x 16 x 128: the fused z kernel at NZAA = 192, as
    the closure's grids run it (captured in a CUDA graph like every step)."""
    _steps_match(_cfg("rbc_noslip_ra1e8.equations"), params(16, 16, 128, dt=1e-6), dt=1e-6, nsteps=3, seed=23,
                 amp=1e-2)
