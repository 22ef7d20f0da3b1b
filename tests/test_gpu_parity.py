"""Parity of the CUDA path (through the C-ABI) with the CPU oracle.

Tolerances: FP64 everywhere; transforms agree to 1e-13 of the field's maximum;
timesteps to a relative L2 error of 1e-10 per coupled variable (the bound the
plain FP64 path must hold against the reference after 100 steps)."""
import ctypes
import math
import os
import tempfile

import numpy as np
import pytest

from oracle import coral_oracle as co
from tests.problems import equations, params

pytestmark = pytest.mark.gpu


def _pl(eq, par, scheme=None):
    from coral_b200.solver import PlaneLayer
    return PlaneLayer(eq, par, scheme=scheme)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("N", [(16, 16, 16), (24, 32, 12), (64, 64, 48)])
def test_transforms_match_oracle(N):
    NX, NY, NZ = N
    eq, par = equations(), params(NX, NY, NZ, Lx=2.0, Ly=3.0)
    pl = _pl(eq, par)
    g = co.Geometry(NX, NY, NZ, 2.0, 3.0, 1.0, 0.5)
    rng = np.random.default_rng(1)
    spec = rng.standard_normal((g.NXH, g.NYAA, NZ)) + 1j * rng.standard_normal((g.NXH, g.NYAA, NZ))
    p_gpu = pl.spec_to_phys(spec)
    p_ref = co.spec_to_phys(spec, g)
    assert np.abs(p_gpu - p_ref).max() <= 1e-13 * np.abs(p_ref).max()
    phys = rng.standard_normal((g.NYAA, g.NXAA, g.NZAA))
    s_gpu = pl.phys_to_spec(phys)
    s_ref = co.phys_to_spec(phys, g)
    assert np.abs(s_gpu - s_ref).max() <= 1e-13 * np.abs(s_ref).max()
    pl.close()


def _random_state(solver, pl, seed, amp=1e-3):
    rng = np.random.default_rng(seed)
    for s, lay in enumerate(solver.lay):
        f = amp * (rng.standard_normal((pl.NXH, pl.NYAA, lay.T)) + 1j * rng.standard_normal((pl.NXH, pl.NYAA, lay.T)))
        solver.field[s] = f.copy()
        pl.set_field(s, f)
    for s, lay in enumerate(solver.zlay):
        z = amp * rng.standard_normal(lay.T)
        solver.zfield[s] = z.copy()
        pl.set_mean_field(s, z)


@pytest.mark.parametrize("scheme", ["ARS_222", "ARS_443", "ARS_111"])
def test_steps_match_oracle_small(scheme):
    eq = equations("rrbc_stressfree_ek1e-4_ra5e7", **{"5.d7": "2.d4", "1.d4": "1.d2"})
    par = params(16, 12, 16, dt=2e-4, scheme=scheme)
    ref = co.Solver(eq, par)
    pl = _pl(eq, par)
    assert pl.T == [l.T for l in ref.lay]
    _random_state(ref, pl, 3, amp=1e-2)
    for _ in range(4):
        ref.step(2e-4)
    pl.march_forward(2e-4, 4)
    pl.synchronize()
    for s in range(len(ref.lay)):
        assert _rel(pl.get_field(s), ref.field[s]) < 1e-11
    for s in range(len(ref.zlay)):
        assert _rel(pl.get_mean_field(s), ref.zfield[s]) < 1e-11
    d = pl.diagnostics()
    assert d["nonfinite"] is False
    pl.close()


def test_quicksave_import_export_roundtrip():
    from coral_b200 import initial_conditions as ic
    NX, NY, NZ = 16, 16, 16
    eq, par = equations(), params(NX, NY, NZ)
    with tempfile.TemporaryDirectory() as d:
        ic.white_noise_temperature(d, NX, NY, NZ, seed=5)
        ref = co.Solver(eq, par)
        ref.import_quicksave(d)
        pl = _pl(eq, par)
        pl.import_quicksave(d)
        assert _rel(pl.get_field(0), ref.field[0]) < 1e-12
        for s in range(len(ref.zlay)):
            assert np.abs(pl.get_mean_field(s) - ref.zfield[s]).max() <= 1e-12 * max(np.abs(ref.zfield[s]).max(), 1e-30) + 1e-18
        out = os.path.join(d, "out")
        os.makedirs(out)
        f0 = pl.get_field(0)
        pl.export_checkpoints(out)
        pl2 = _pl(eq, par)
        pl2.import_quicksave(out)
        # export_checkpoints re-projects the state through the fields it writes,
        # as the reference's does: the exporting handle's state is the imported
        # one, bit for bit; on the modes the dealiased transforms represent the
        # projection is the identity to round-off (the rest are zero after a step)
        f1, f2 = pl.get_field(0), pl2.get_field(0)
        assert np.array_equal(f1, f2)
        g = co.Geometry(NX, NY, NZ, 2 * math.pi, 2 * math.pi, 1.0, 0.5)
        act = g.active
        assert _rel(f1[act], f0[act]) < 1e-12
        pl.close()
        pl2.close()


def test_cfg0_100_steps_within_1e10():
    """64x64x48 no-slip Rayleigh-Benard, Ra=1e5, Pr=1, dt=1e-4, seeded white-noise
    temperature IC through the QuickSave path, 100 ARS_222 steps: every coupled
    variable and mean field within 1e-10 relative L2 of the oracle."""
    from coral_b200 import initial_conditions as ic
    from coral_b200 import CONFIG_DIR
    eq = open(os.path.join(CONFIG_DIR, "rbc_noslip_ra1e5.equations")).read()
    par = open(os.path.join(CONFIG_DIR, "rbc_noslip_ra1e5_64x64x48.parameters.in")).read()
    with tempfile.TemporaryDirectory() as d:
        ic.white_noise_temperature(d, 64, 64, 48, seed=0)
        ref = co.Solver(eq, par)
        ref.import_quicksave(d)
        pl = _pl(eq, par)
        pl.import_quicksave(d)
    nsteps = 100
    for _ in range(nsteps):
        ref.step(1e-4)
    pl.march_forward(1e-4, nsteps)
    pl.synchronize()
    f_gpu, f_ref = pl.get_field(0), ref.field[0]
    lay = ref.lay[0]
    for v in range(lay.nV):
        idx = lay.var_pos[v]
        assert _rel(f_gpu[..., idx], f_ref[..., idx]) < 1e-10, ref.recipe.kxky[0].vars[v]
    for s in range(len(ref.zlay)):
        assert _rel(pl.get_mean_field(s), ref.zfield[s]) < 1e-10
    pl.close()


@pytest.mark.parametrize("path", ["split", "unsplit", "complex"])
def test_all_factor_paths_match_oracle(path, monkeypatch):
    """The three solve paths give the same steps: real-scaled factors split into
    the two independent (Chebyshev parity) blocks of every system, real-scaled
    factors of the whole system, and the general complex factors."""
    monkeypatch.delenv("CORAL_COMPLEX_FACTORS", raising=False)
    monkeypatch.delenv("CORAL_NO_CLASS_SPLIT", raising=False)
    if path == "complex":
        monkeypatch.setenv("CORAL_COMPLEX_FACTORS", "1")
    elif path == "unsplit":
        monkeypatch.setenv("CORAL_NO_CLASS_SPLIT", "1")
    eq = equations("rrbc_stressfree_ek1e-4_ra5e7", **{"5.d7": "3.d4", "1.d4": "3.d2"})
    par = params(12, 16, 24, dt=1e-4)
    ref = co.Solver(eq, par)
    pl = _pl(eq, par)
    assert pl.query(700) == (0 if path == "complex" else 1)
    assert pl.query(800) == (2 if path == "split" else 1)
    if path == "split":
        assert 2 * pl.query(900) == pl.T[0]
    _random_state(ref, pl, 11, amp=1e-2)
    for _ in range(3):
        ref.step(1e-4)
    pl.march_forward(1e-4, 3)
    pl.synchronize()
    assert _rel(pl.get_field(0), ref.field[0]) < 1e-11
    pl.close()


@pytest.mark.parametrize("split,generic", [(True, False), (True, True), (False, False)])
def test_split_solve_rbc_noslip_matches_oracle(split, generic, monkeypatch):
    """No-slip Rayleigh-Benard (the benchmark recipe) at NZ = 48 with and without
    the block split, against the oracle over a few ARS_222 steps; generic: the
    tile kernels' run-time operator forms instead of the compiled group layouts."""
    monkeypatch.delenv("CORAL_COMPLEX_FACTORS", raising=False)
    if generic:
        monkeypatch.setenv("CORAL_GENERIC_TILES", "1")
    else:
        monkeypatch.delenv("CORAL_GENERIC_TILES", raising=False)
    if split:
        monkeypatch.delenv("CORAL_NO_CLASS_SPLIT", raising=False)
    else:
        monkeypatch.setenv("CORAL_NO_CLASS_SPLIT", "1")
    eq = equations("rbc_noslip_ra1e8", **{"1.d8": "1.d5"})
    par = params(16, 12, 48, dt=1e-5)
    ref = co.Solver(eq, par)
    pl = _pl(eq, par)
    assert pl.query(800) == (2 if split else 1)
    _random_state(ref, pl, 5, amp=1e-2)
    for _ in range(3):
        ref.step(1e-5)
    pl.march_forward(1e-5, 3)
    pl.synchronize()
    # band entries the substitution reads: within the block band, at least the diagonal
    Tc, kl, ku = pl.query(900), pl.query(1000), pl.query(1100)
    if split:
        assert Tc <= pl.query(1200) <= Tc * (2 * kl + ku + 1)
    else:
        assert pl.query(1200) == 0
    assert _rel(pl.get_field(0), ref.field[0]) < 1e-11
    for s in range(len(ref.zlay)):
        assert _rel(pl.get_mean_field(s), ref.zfield[s]) < 1e-11
    pl.close()


@pytest.mark.parametrize("scheme", ["ARS_222", "ARS_111"])
def test_diagnostics_match_oracle(scheme):
    """CFL time step (from the last stage's fields) and kinetic energy (volume
    averages of uu + vv + ww at the first stage) after a few steps, against the
    oracle's compute_cfl_based_timestep and output_global_quantities values."""
    eq = equations("rbc_noslip_ra1e8", **{"1.d8": "1.d5"})
    par = params(16, 12, 48, dt=1e-5, scheme=scheme)
    ref = co.Solver(eq, par)
    pl = _pl(eq, par)
    _random_state(ref, pl, 9, amp=1e-2)
    for _ in range(2):
        ref.step(1e-5)
    pl.march_forward(1e-5, 2)
    d = pl.diagnostics()
    assert d["nonfinite"] is False
    assert ref.cfl_dt is not None and ref.ke is not None
    assert abs(d["cfl_dt"] - ref.cfl_dt) <= 1e-11 * abs(ref.cfl_dt)
    assert abs(d["KE"] - ref.ke) <= 1e-11 * abs(ref.ke)
    pl.close()


@pytest.mark.parametrize("N", [(12, 12, 36), (36, 24, 12)])
def test_steps_with_runtime_plans_and_block_tails(N):
    """The benchmark recipe (no-slip RBC) at sizes whose grid lengths have no
    compiled FFT plan (x 18 and 54, y 18, z 54 and 18; y 36 is compiled) and
    whose Chebyshev counts leave a partial block of 4 rows in the x passes'
    8-row blocks (NZ mod 8 = 4): the run-time-plan kernels, their second
    shared buffer and the tail guards, over three ARS_222 steps against the
    oracle."""
    NX, NY, NZ = N
    eq = equations("rbc_noslip_ra1e8", **{"1.d8": "1.d5"})
    par = params(NX, NY, NZ, dt=1e-5)
    ref = co.Solver(eq, par)
    pl = _pl(eq, par)
    _random_state(ref, pl, 11, amp=1e-2)
    for _ in range(3):
        ref.step(1e-5)
    pl.march_forward(1e-5, 3)
    pl.synchronize()
    for s in range(len(ref.lay)):
        assert _rel(pl.get_field(s), ref.field[s]) < 1e-11
    for s in range(len(ref.zlay)):
        assert _rel(pl.get_mean_field(s), ref.zfield[s]) < 1e-11
    d = pl.diagnostics()
    assert d["nonfinite"] is False
    pl.close()


def test_invalid_inputs_are_refused_and_nonfinite_states_reported():
    """The C-ABI's error behaviour (the reference prints and stops; here a
    negative code and a message, the handle stays usable): sizes outside the
    build (NX not a multiple of 4; a grid length 3 NZ / 2 = 30 that is not
    2^a 3^b), unreadable parameter files, dt <= 0, a system index out of range;
    a NaN in the state is reported after a step (CORAL_ENONFINITE from
    coral_synchronize, and the diagnostics' flag)."""
    from coral_b200.solver import CoralError
    for bad, code in ((params(18, 16, 16), -8), (params(16, 16, 20), -8),
                      (params(16, 16, 16).replace("1.d0        ! gap", "one   ! gap"), -6),
                      ("\n".join(params(16, 16, 16).splitlines()[:10]), -6)):
        with pytest.raises(CoralError) as e:
            _pl(equations(), bad)
        assert e.value.code == code, (e.value.code, str(e.value))
    pl = _pl(equations(), params(16, 16, 16))
    with pytest.raises(CoralError) as e:
        pl.march_forward(0.0, 1)
    assert e.value.code == -1
    buf = np.zeros(8, dtype=np.complex128)
    rc = pl._lib.coral_get_field(pl._h, 7, buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert rc == -1 and "out of range" in pl._lib.coral_last_error(pl._h).decode()
    f = pl.get_field(0)
    pl.march_forward(1e-4, 1)  # still usable after the refusals
    pl.synchronize()
    f[1, 2, 0] = np.nan  # an entry the step reads (the oracle's step spreads it to 10,472 of 16,896 entries)
    pl.set_field(0, f)
    pl.march_forward(1e-4, 1)
    with pytest.raises(CoralError) as e:
        pl.synchronize()
    assert e.value.code == -5
    assert pl.diagnostics()["nonfinite"] is True
    pl.close()
