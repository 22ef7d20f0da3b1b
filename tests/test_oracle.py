"""CPU tests of the oracle against the reference's published numbers and
analytic results (no GPU needed)."""
import json
import math
import os

import numpy as np
import pytest
import scipy.linalg as sla

from oracle import coral_oracle as co
from tests.heat_problem import heat_equations, heat_params

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "heat_equation_published.json")))
CFG = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "coral_b200", "configs")


def _heat_error(scheme, dt):
    """Benchmark 00 protocol: restart divides dt by 50 for the first step
    (timeKeeping.f90:108), profiles are taken after 9 and 19 steps and the
    10-step decay of uMean is compared with exp(-Pr*k^2*10*dt)."""
    s = co.Solver(heat_equations(), heat_params(128, dt, scheme))
    z = s.g.zgrid()
    s.set_zero_var_from_phys(0, 0, 1.34e-4 * np.sin(9 * (z - 1) * np.pi / 2))
    s.set_zero_var_from_phys(1, 0, -2.3e-2 * np.sin(7 * z * np.pi / 2))
    s.set_zero_var_from_phys(2, 0, np.pi * 1e-3 * np.sin(5 * z * np.pi))
    s.step(dt / 50)
    for _ in range(8):
        s.step(dt)
    u1 = s.zero_var_profile(0, 0)
    for _ in range(10):
        s.step(dt)
    u2 = s.zero_var_profile(0, 0)
    rate = 0.33 * (9 * np.pi / 2) ** 2
    return math.sqrt(np.sum((u2 - u1 * np.exp(-rate * 10 * dt)) ** 2) / np.sum(u1 ** 2))


@pytest.mark.parametrize("scheme,key,idx", [(s, k, i) for s, k in (("ARS_111", "err111"), ("ARS_222", "err222"),
                                                                      ("ARS_443", "err443")) for i in range(7)])
def test_heat_equation_published_errors(scheme, key, idx):
    dt = GOLD["dt"][idx]
    err = _heat_error(scheme, dt)
    # the reference prints four significant digits
    assert err == pytest.approx(GOLD[key][idx], rel=2e-3)


def test_stressfree_growth_rate_matches_analytic():
    eq = open(os.path.join(CFG, "rrbc_stressfree_ek1e-4_ra5e7.equations")).read()
    eq = eq.replace("5.d7", "2.d3").replace("Prandtl := 1.d0", "Prandtl := 7.d0").replace("iEkman := 1.d4", "iEkman := 0.d0")
    par = heat_params(24, 1e-3, "ARS_222", NX=12, NY=12).replace("1.0d0", "10.0d0")
    s = co.Solver(eq, par)
    Ra, Pr = 2000.0, 7.0
    best = -1e9
    for ix, iy in [(3, 0), (2, 3), (3, 1)]:
        mass, stif = s.kxky_ops[0]
        cm, cs = s.coef[0]
        M = sum(c[ix, iy] * B.toarray() for (p, B), c in zip(mass, cm))
        L = sum(c[ix, iy] * B.toarray() for (p, B), c in zip(stif, cs))
        w = sla.eigvals(L, M)
        w = w[np.isfinite(w)]
        k = math.hypot(s.g.kx[ix], s.g.ky[iy])
        D2 = k * k + math.pi ** 2
        an = 0.5 * (-D2 * (Pr + 1) + math.sqrt((Pr + 1) ** 2 * D2 ** 2 - 4 * (Pr * D2 ** 2 - Ra * Pr * k * k / D2)))
        assert w.real.max() == pytest.approx(an, rel=1e-9, abs=1e-9)
        best = max(best, an)
    # the reference's quoted maximum growth rate lies just above the modes probed here
    assert best < GOLD["stressfree_rb_max_growthrate"] < best + 2.0


def test_transform_round_trip_and_single_mode():
    g = co.Geometry(16, 12, 10, 2.0, 3.0, 1.0, 0.5)
    rng = np.random.default_rng(0)
    spec = co.phys_to_spec(rng.standard_normal((g.NYAA, g.NXAA, g.NZAA)), g)
    spec[:, g.deal_y, :] = 0
    s2 = co.phys_to_spec(co.spec_to_phys(spec, g), g)
    assert np.abs(s2 - spec).max() < 1e-14 * np.abs(spec).max()
    s = np.zeros_like(spec)
    s[2, 1, 1] = 0.3 + 0.4j
    p = co.spec_to_phys(s, g)
    x = np.arange(g.NXAA) * g.Lx / g.NXAA
    y = np.arange(g.NYAA) * g.Ly / g.NYAA
    z = np.cos(np.pi * (2 * np.arange(g.NZAA) + 1) / (2 * g.NZAA))
    ref = 2 * np.real((0.3 + 0.4j) * np.exp(1j * (g.kx[2] * x[None, :, None] + g.ky[1] * y[:, None, None]))) * z
    assert np.abs(p - ref).max() < 1e-14


def test_band_lu_matches_dense_solve():
    rng = np.random.default_rng(1)
    n, kl, ku = 40, 3, 5
    A = np.zeros((n, n), dtype=complex)
    for d in range(-kl, ku + 1):
        A += np.diag(rng.standard_normal(n - abs(d)) + 1j * rng.standard_normal(n - abs(d)), d)
    dia = np.zeros((kl + ku + 1, n), dtype=complex)
    for i in range(n):
        for j in range(max(0, i - kl), min(n, i + ku + 1)):
            dia[ku + i - j, j] = A[i, j]
    lu, piv = co.zgbtrf_band(dia, kl, ku)
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    x = co.zgbtrs_band(lu, piv, kl, ku, b)
    assert np.abs(A @ x - b).max() < 1e-12 * np.abs(b).max()


def test_rbc_system_band_structure():
    """The interleaved RBC system is banded with nl=16, nu=27 (ldab=60)."""
    eq = open(os.path.join(CFG, "rbc_noslip_ra1e5.equations")).read()
    s = co.Solver(eq, heat_params(48, 1e-4, "ARS_222", NX=8, NY=8))
    assert s.lay[0].T == 6 * 48 - 8
    s.factorize(1e-4)
    assert s.kl_ku[0] == (16, 27)


def test_usr_output_parser_on_the_reference_file():
    """The oracle's coral.usrOutput reader on benchmark 02's own file: 17
    objects, grouped per full variable in the recipe's order (uFull, vFull,
    wFull, tFull) and in file order within one; the counters of
    initialise_bookkeeping_counters / output_slices_volumes_and_profiles put
    the first tFull profile (period 50, run started at step 1) at time index 50
    and the first slices (period 1000) at 1000."""
    import os
    from oracle import coral_oracle as co
    b02 = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "benchmark02")
    recipe = co.parse_equations(open(os.path.join(b02, "coral.equations.velocityPressure")).read())
    p = co.read_parameters_text(open(os.path.join(b02, "coral.parameters.in")).read())
    g = co.Geometry(p["NX"], p["NY"], p["NZ"], p["Lx"], p["Ly"], p["gap"], p["center"])
    objs = co.parse_usr_output(open(os.path.join(b02, "coral.usrOutput")).read(), recipe, g)
    assert len(objs) == 17
    assert [o[2] for o in objs] == sorted(o[2] for o in objs)  # grouped by variable
    assert objs[0] == ("volume", False, 0, 10000, 0)
    t_objs = [o for o in objs if o[2] == 3]
    assert [o[0] for o in t_objs] == ["volume", "zSlice", "zSlice", "zSlice", "zSlice", "xSlice", "ySlice", "profil"]
    assert [o[4] for o in t_objs if o[0] == "zSlice"] == [1, 24, 48, 72]
    sched = co.usr_output_schedule(objs, 1, 1000)
    first = {}
    for _, t, due in sched:
        for o in due:
            first.setdefault(o[0], t)
    assert first["profil"] == 50 and first["zSlice"] == 1000 and "volume" not in first


EXAMPLES = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "examples")


def test_example_recipes_with_sources_and_penalisation_parse():
    """The reference's example equation files read unmodified: sources with their
    parameters, a penalised variable with strength and width."""
    def rd(n):
        with open(os.path.join(EXAMPLES, n)) as f:
            return co.parse_equations(f.read())
    r = rd("coral.equations.RBC_penalised")
    assert [f[0] for f in r.full_vars] == ["uFull", "vFull", "wFull", "tFull", "GAMMA"]
    assert r.full_opts[4]["penal"] == [1e3, 1e2] and len(r.quad_vars) == 12
    r = rd("coral.equations.radiative_heating_potentials")
    assert r.source_params == [("HovEll", 41.66666)]
    assert [(t.index, t.dsca, t.Iz) for t in r.sources] == [(1, 1.0, 2), (2, 1.0, 2)]
    r = rd("coral.equations.stratifiedChannel.velocityPressure")
    assert [(t.index, t.dsca, t.Iz, t.sys) for t in r.sources] == [(2, -1.0, 2, 0)]
    r = rd("coral.equations.baroclinic_turbulence")
    assert sorted(t.index for t in r.sources) == [3, 4, 5]
    assert co.parse_equations(open(os.path.join(EXAMPLES, "coral.equations.RBC_penalised")).read(),
                              smagorinsky=True).full_vars[-1][0] == "nuSmago"


def test_surface_values_and_vertical_decompositions():
    """z_filter on Chebyshev series: surface values are the series at -1 / +1;
    baroclinic leaves zero vertical mean, barotropic leaves only the mean (the
    reference keeps coefficient NZ - 1, zero here)."""
    rng = np.random.default_rng(0)
    NZ = 16
    c = rng.standard_normal((3, NZ))
    c[:, NZ - 1] = 0.0
    bot = co.z_filter(c, "BotSurf", None)
    top = co.z_filter(c, "TopSurf", None)
    assert np.allclose(bot[:, 0], np.polynomial.chebyshev.chebval(-1.0, c.T), rtol=0, atol=1e-13)
    assert np.allclose(top[:, 0], np.polynomial.chebyshev.chebval(1.0, c.T), rtol=0, atol=1e-13)
    assert not bot[:, 1:].any() and not top[:, 1:].any()

    def mean(s):  # (1/2) integral over [-1, 1] of the series
        C = np.polynomial.chebyshev
        return np.array([C.chebval(1.0, C.chebint(x, lbnd=-1)) / 2.0 for x in s])
    bc = co.z_filter(c, "nowhere", "baroclinic")
    assert np.abs(mean(bc)).max() < 1e-13
    assert np.array_equal(bc[:, 1:], c[:, 1:])
    bt = co.z_filter(c, "nowhere", "barotropic")
    assert np.allclose(bt[:, 0], mean(c), rtol=0, atol=1e-13)
    assert not bt[:, 1:].any()


def test_sources_and_penalisation_fields():
    """Compute_1dCheby_transform of a constant; the default sources; the default
    penalisation mask's two surfaces at the reference's grid labels."""
    c = co.source_spectrum(-np.ones(24))
    assert abs(c[0] + 1.0) < 1e-15 and np.abs(c[1:]).max() < 1e-15
    g = co.Geometry(8, 8, 16, 2.0, 2.0, 1.0, 0.5)
    z = g.zgrid()
    assert abs(co.source_spectrum(z)[1] - 0.5) < 1e-14  # z = 0.5 + T_1 / 2
    r = co.parse_equations(open(os.path.join(EXAMPLES, "coral.equations.radiative_heating_potentials")).read())
    s = co.default_sources(r, g)
    h = 41.66666
    assert np.allclose(s[1], h * np.exp(-z * h) / (1 - np.exp(-h)) - 1.0, rtol=1e-15)
    assert np.array_equal(s[2], -np.ones(g.NZAA))
    m = co.default_penalisation_mask(g)
    assert m.shape == (g.NYAA, g.NXAA, g.NZAA)
    pi = float(np.float32(math.pi))
    x = (np.arange(g.NXAA) + 2) * g.Lx / g.NXAA
    y = (np.arange(g.NYAA) + 2) * g.Ly / g.NYAA
    m1 = z[None, None, :] - (float(np.float32(0.9)) + float(np.float32(0.1)) *
                             np.cos(5 * (x[None, :, None] + y[:, None, None]) * 2 * pi / g.Lx))
    assert np.all(m >= m1)
    f = co.penalisation_field(m, 1e3, 1e2)
    assert f.min() >= 0.0 and f.max() <= 1e3


def test_dynamo_toroidal_poloidal_file_is_refused():
    """The convective-dynamo example's toroidal-poloidal file names bxFull where
    its full variable is BxFull: the reference's parser stops on it with 'bad NL
    var definition', and so does the oracle's."""
    with open(os.path.join(EXAMPLES, "coral.equations.convective_dynamo.toroidalPoloidal")) as f:
        t = f.read()
    with pytest.raises(ValueError, match="bad NL var definition"):
        co.parse_equations(t)
