"""Ensembles on the GPU: members of different grids and parameters advanced
together (one graph per step, the band substitutions of all members in one
persistent launch per stage) compute exactly -- bit for bit -- what a single
handle of each member's problem computes."""
import numpy as np
import pytest

from tests.problems import equations, params

pytestmark = pytest.mark.gpu


def _members():
    spec = [((16, 16, 32), 2e4, 0.7), ((24, 24, 48), 1e5, 1.0), ((32, 32, 32), 3e5, 7.0), ((16, 12, 64), 5e4, 2.0)]
    out = []
    for (nx, ny, nz), ra, pr in spec:
        eq = equations(**{">>Param :: Rayleigh := 1.d5 <<": ">>Param :: Rayleigh := %r <<" % ra,
                          ">>Param :: Prandtl := 1.d0 <<": ">>Param :: Prandtl := %r <<" % pr})
        out.append((eq, params(nx, ny, nz, dt=1e-4)))
    return out


def _set_random(pl, seed):
    rng = np.random.default_rng(seed)
    for s in range(pl.n_kxky):
        f = 1e-2 * (rng.standard_normal((pl.NXH, pl.NYAA, pl.T[s])) + 1j * rng.standard_normal((pl.NXH, pl.NYAA, pl.T[s])))
        pl.set_field(s, f)
    for s in range(pl.n_zero):
        pl.set_mean_field(s, 1e-2 * rng.standard_normal(pl.Tz[s]))


def test_ensemble_members_match_single_runs_bitwise():
    from coral_b200.ensemble import Ensemble
    from coral_b200.solver import PlaneLayer
    spec = _members()
    ens = Ensemble([s[0] for s in spec], [s[1] for s in spec])
    singles = [PlaneLayer(*s) for s in spec]
    for i, (m, p) in enumerate(zip(ens.members, singles)):
        _set_random(m, 40 + i)
        _set_random(p, 40 + i)
    ens.march_forward(1e-4, 3)
    ens.synchronize()
    assert ens.batched
    for p in singles:
        p.march_forward(1e-4, 3)
        p.synchronize()
    for m, p in zip(ens.members, singles):
        for s in range(p.n_kxky):
            assert np.array_equal(m.get_field(s), p.get_field(s))
        for s in range(p.n_zero):
            assert np.array_equal(m.get_mean_field(s), p.get_mean_field(s))
        assert m.diagnostics() == p.diagnostics()
    for p in singles:
        p.close()
    ens.close()


def test_seeded_64_member_ensemble_steps():
    """The seeded 64-member ensemble (grids 32^2 x 32 ... 128^2 x 64, Ra in
    [1e4, 1e6], Pr in [0.7, 7]): a few steps, every member finite, and two of
    its members against single handles started from the same files."""
    import tempfile

    from coral_b200 import initial_conditions as ic
    from coral_b200.ensemble import seeded_ensemble
    from coral_b200.solver import PlaneLayer
    ens, spec = seeded_ensemble(64)
    assert ens.batched is False or True  # set by the first march
    ens.march_forward(1e-4, 3)
    ens.synchronize()
    assert ens.batched
    for m in ens.members:
        assert m.diagnostics()["nonfinite"] is False
    for i in (0, 63):
        eq, par, g, _, _ = spec[i]
        p = PlaneLayer(eq, par)
        with tempfile.TemporaryDirectory() as d:
            ic.white_noise_temperature(d, g[0], g[1], g[2], seed=1000 + i)
            p.import_quicksave(d)
        p.march_forward(1e-4, 3)
        assert np.array_equal(p.get_field(0), ens.members[i].get_field(0))
        p.close()
    ens.close()


def test_ensemble_of_penalised_sourced_and_filtered_members_bitwise():
    """Members with a penalisation field, mean-equation sources, and surface
    values / vertical decompositions (the reference's example files and the
    feature-test recipe) in one ensemble: bit for bit their single runs."""
    from coral_b200.ensemble import Ensemble
    from coral_b200.solver import PlaneLayer
    from tests.test_gpu_features import _example, _with_surface_vars
    spec = [(_example("coral.equations.RBC_penalised"), params(16, 16, 16, dt=1e-5)),
            (_example("coral.equations.radiative_heating_potentials"), params(16, 12, 24, dt=1e-5)),
            (_example("coral.equations.stratifiedChannel.velocityPressure"), params(24, 16, 24, dt=1e-5)),
            (_with_surface_vars(equations()), params(16, 12, 24, dt=1e-5))]
    ens = Ensemble([s[0] for s in spec], [s[1] for s in spec])
    singles = [PlaneLayer(*s) for s in spec]
    for i, (m, p) in enumerate(zip(ens.members, singles)):
        _set_random(m, 70 + i)
        _set_random(p, 70 + i)
    ens.march_forward(1e-5, 3)
    ens.synchronize()
    for p in singles:
        p.march_forward(1e-5, 3)
        p.synchronize()
    for m, p in zip(ens.members, singles):
        for s in range(p.n_kxky):
            assert np.array_equal(m.get_field(s), p.get_field(s))
        for s in range(p.n_zero):
            assert np.array_equal(m.get_mean_field(s), p.get_mean_field(s))
    for p in singles:
        p.close()
    ens.close()
