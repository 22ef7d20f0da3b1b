"""Full variables that are not plain transforms, and the mean equations'
sources, on the GPU against the oracle (marching.f90:398-415, 505-575,
778-866): penalisation fields, surface values, vertical decompositions, the
Smagorinsky viscosity, user sources and the reference's command-line switches.
The equation files of the reference's examples are read unmodified
(tests/golden/examples/, copied by tests/golden/extract_published.py)."""
import os

import numpy as np
import pytest

from oracle import coral_oracle as co
from tests.problems import equations, params

pytestmark = pytest.mark.gpu

EXAMPLES = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "examples")


def _example(name):
    with open(os.path.join(EXAMPLES, name)) as f:
        return f.read()


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _random_state(ref, pl, seed, amp):
    rng = np.random.default_rng(seed)
    for s, lay in enumerate(ref.lay):
        f = amp * (rng.standard_normal((pl.NXH, pl.NYAA, lay.T)) + 1j * rng.standard_normal((pl.NXH, pl.NYAA, lay.T)))
        ref.field[s] = f.copy()
        pl.set_field(s, f)
    for s, lay in enumerate(ref.zlay):
        z = amp * rng.standard_normal(lay.T)
        ref.zfield[s] = z.copy()
        pl.set_mean_field(s, z)


def _compare_state(ref, pl, tol):
    errs = []
    for s in range(len(ref.lay)):
        errs.append(_rel(pl.get_field(s), ref.field[s]))
    for s in range(len(ref.zlay)):
        errs.append(_rel(pl.get_mean_field(s), ref.zfield[s]))
    assert max(errs) < tol, errs
    return errs


def _run_both(eq, par, nsteps, dt, seed=3, amp=1e-3, args=None, oracle_kw=None, setup=None, tol=1e-10):
    from coral_b200.solver import PlaneLayer
    ref = co.Solver(eq, par, **(oracle_kw or {}))
    pl = PlaneLayer(eq, par, args=args)
    try:
        _random_state(ref, pl, seed, amp)
        if setup:
            setup(ref, pl)
        for _ in range(nsteps):
            ref.step(dt)
        pl.march_forward(dt, nsteps=nsteps)
        pl.synchronize()
        errs = _compare_state(ref, pl, tol)
        return ref, pl, errs
    except BaseException:
        pl.close()
        raise


def test_penalised_rbc_example_matches_oracle():
    """coral.equations.RBC_penalised: GAMMA = 1e3 (1 + tanh(1e2 mask)) / 2 of the
    reference's default mask, in the products Gu, Gv, Gw."""
    eq = _example("coral.equations.RBC_penalised")
    par = params(16, 16, 16, dt=1e-5)
    ref, pl, errs = _run_both(eq, par, 3, 1e-5)
    try:
        # the penalisation field itself (full variable 4)
        g = pl.full_phys(4)
        assert _rel(g, ref.penal_phys[4]) < 1e-13
        assert g.max() > 900.0 and g.min() < 1.0
    finally:
        pl.close()


def test_user_penalisation_mask_matches_oracle():
    eq = _example("coral.equations.RBC_penalised")
    par = params(16, 12, 24, dt=1e-5)

    def setup(ref, pl):
        rng = np.random.default_rng(11)
        m = rng.standard_normal((pl.NYAA, pl.NXAA, pl.NZAA)) * 0.01
        ref.set_penalisation_mask(m)
        pl.set_penalisation_mask(m)

    ref, pl, errs = _run_both(eq, par, 2, 1e-5, setup=setup)
    try:
        assert _rel(pl.full_phys(4), ref.penal_phys[4]) < 1e-13
    finally:
        pl.close()


def test_sources_of_the_examples_match_oracle():
    """Mean-equation sources: radiative heating (source01 from sourceParam HovEll
    and source02, the reference's default definitions) and the stratified
    channel (- Iz.Iz.source02), both example files unmodified."""
    for name, bc_ok in (("coral.equations.radiative_heating_potentials", True),
                        ("coral.equations.stratifiedChannel.velocityPressure", True)):
        eq = _example(name)
        par = params(16, 12, 24, dt=1e-4)
        ref, pl, errs = _run_both(eq, par, 3, 1e-4)
        pl.close()


def test_user_sources_match_oracle():
    """A source the reference's default PL_user_sources_definitions.f90 does not
    define (the stratified channel's source02 renamed source07, given
    exp(-(1 - z) / 0.5) as the baroclinic-turbulence example's own definitions
    file gives source03): a step fails until coral_set_source gives it, then
    matches the oracle."""
    from coral_b200.solver import CoralError, PlaneLayer
    eq = _example("coral.equations.stratifiedChannel.velocityPressure").replace("source02", "source07")
    par = params(16, 12, 24, dt=1e-4)
    pl = PlaneLayer(eq, par)
    try:
        with pytest.raises(CoralError) as e:
            pl.march_forward(1e-4, nsteps=1)
        assert e.value.code == -1 and "source07" in str(e.value)
    finally:
        pl.close()

    def setup(ref, pl):
        prof = np.exp(-(1.0 - ref.g.zgrid()) / 0.5)
        ref.set_source(7, prof)
        pl.set_source(7, prof)

    ref, pl, errs = _run_both(eq, par, 3, 1e-4, setup=setup)
    pl.close()


def test_baroclinic_turbulence_example_matches_oracle():
    """The baroclinic-turbulence example unmodified: five coupled variables with
    fourth-order operators (band kl = 35, ku = 49: the wide complex factor and
    solve), eight mean systems and sources 3-5 of its own definitions file
    (exp(-(1 - z) / shearL), the same / shearL and / shearL^2, shearL = 0.5)."""
    eq = _example("coral.equations.baroclinic_turbulence")
    par = params(16, 16, 24, dt=1e-5)

    def setup(ref, pl):
        z = ref.g.zgrid()
        L = 0.5
        for k, prof in ((3, np.exp(-(1.0 - z) / L)), (4, np.exp(-(1.0 - z) / L) / L),
                        (5, np.exp(-(1.0 - z) / L) / L ** 2)):
            ref.set_source(k, prof)
            pl.set_source(k, prof)

    ref, pl, errs = _run_both(eq, par, 2, 1e-5, setup=setup)
    try:
        ref.factorize(1e-5)
        assert ref.kl_ku[0] == (35, 49)
    finally:
        pl.close()


SURF = """>>linear_variable_bottom_boundary_value :: pBot <<
>>linear_variable_full_build :: + p <<
>>linear_variable_full_build :: + tMean <<
>>linear_variable_top_boundary_value :: chiTop <<
>>linear_variable_full_build :: + dx.chi <<
>>linear_variable_full_build :: + uMean <<
>>linear_variable_full       :: tBaroclinic <<
>>vertical_decomposition :: baroclinic <<
>>linear_variable_full_build :: + tMean <<
>>linear_variable_full_build :: + t <<
>>linear_variable_full       :: wBarotropic <<
>>vertical_decomposition :: barotropic <<
>>linear_variable_full_build :: + dz.w <<
>>linear_variable_full_build :: + t <<
"""
SURF_QUADS = """>>quadratic_variable :: sA := pBot.wFull <<
>>quadratic_variable :: sB := chiTop.tBaroclinic <<
>>quadratic_variable :: sC := wBarotropic.tFull <<
"""


def _with_surface_vars(eq):
    """rbc_noslip_ra1e5 with four more full variables (bottom and top surface
    values of p and dx chi, which are not zero at the walls, plus mean
    variables, which are; a baroclinic and a barotropic one) feeding three
    products that enter the temperature equations."""
    i = eq.index(">>quadratic_variable")
    eq = eq[:i] + SURF + eq[i:]
    i = eq.index(">>add_set_of_coupled_kxky_equations")
    eq = eq[:i] + SURF_QUADS + eq[i:]
    line = ">>add_rhs_NL     :: - Iz.Iz.dx.tu - Iz.Iz.dy.tv - Iz.tw <<"
    assert eq.count(line) == 1
    eq = eq.replace(line, line + "\n>>add_rhs_NL     :: + Iz.Iz.sA <<\n"
                    ">>add_rhs_NL     :: - Iz.Iz.dx.sB <<\n>>add_rhs_NL     :: + Iz.Iz.sC <<")
    return eq


def test_surface_values_and_vertical_decompositions_match_oracle():
    eq = _with_surface_vars(equations("rbc_noslip_ra1e5"))
    par = params(16, 12, 24, dt=1e-4)
    from coral_b200.solver import PlaneLayer
    ref = co.Solver(eq, par)
    assert [o["extract"] for o in ref.recipe.full_opts[4:]] == ["BotSurf", "TopSurf", "nowhere", "nowhere"]
    pl = PlaneLayer(eq, par)
    try:
        _random_state(ref, pl, 5, 1e-2)
        fphys, _, _ = ref.compute_phys(ref.field, ref.zfield)
        for f in range(4, 8):
            assert np.abs(fphys[f]).max() > 1e-3, f
            assert _rel(pl.full_phys(f), fphys[f]) < 1e-12, f
        # surface values are constant along z
        for f in (4, 5):
            assert np.ptp(pl.full_phys(f), axis=2).max() < 1e-12 * np.abs(fphys[f]).max(), f
        for _ in range(3):
            ref.step(1e-4)
        pl.march_forward(1e-4, nsteps=3)
        pl.synchronize()
        _compare_state(ref, pl, 1e-10)
    finally:
        pl.close()


SMAGO_VARS = """>>linear_variable_full       :: dxUfull <<
>>linear_variable_full_build :: + dx.u <<
>>linear_variable_full       :: dyUfull <<
>>linear_variable_full_build :: + dy.u <<
>>linear_variable_full       :: dxVfull <<
>>linear_variable_full_build :: + dx.v <<
>>linear_variable_full       :: dyVfull <<
>>linear_variable_full_build :: + dy.v <<
"""
SMAGO_QUADS = """>>quadratic_variable :: nuU := nuSmago.uFull <<
>>quadratic_variable :: nuT := nuSmago.tFull <<
"""


def _with_smagorinsky_vars(eq):
    i = eq.index(">>quadratic_variable")
    eq = eq[:i] + SMAGO_VARS + eq[i:]
    i = eq.index(">>add_set_of_coupled_kxky_equations")
    eq = eq[:i] + SMAGO_QUADS + eq[i:]
    line = ">>add_rhs_NL     :: - Iz.Iz.dx.tu - Iz.Iz.dy.tv - Iz.tw <<"
    assert eq.count(line) == 1
    eq = eq.replace(line, line + "\n>>add_rhs_NL     :: - Iz.Iz.dx.dx.nuT - Iz.Iz.dy.dy.nuT <<")
    return eq


def test_smagorinsky_matches_oracle():
    """--withHorizontalSmagorinsky: nuSmago = c sqrt(havg(previous + dxU^2 + dyU^2
    + dxV^2 + dyV^2)), carried from stage to stage as the reference does; its
    CFL limit; --cflFactor-along-z."""
    eq = _with_smagorinsky_vars(equations("rbc_noslip_ra1e5"))
    par = params(16, 12, 24, dt=1e-4)
    args = "--withHorizontalSmagorinsky --smagorinsky-prefactor 3.d0 --cflFactor-along-z 0.5"
    kw = dict(smagorinsky=True, smagorinsky_prefactor=3.0, cfl_factor_z=0.5)
    ref, pl, errs = _run_both(eq, par, 3, 1e-4, amp=1e-1, args=args, oracle_kw=kw)
    try:
        names = [f[0] for f in ref.recipe.full_vars]
        assert names[-1] == "nuSmago" and pl.n_full == len(names)
        nu = pl.full_phys(len(names) - 1)
        assert _rel(nu[0, 0, :], ref.smago_profile) < 1e-12
        assert np.ptp(nu, axis=(0, 1)).max() == 0.0
        d = pl.diagnostics()
        assert abs(d["cfl_dt"] / ref.cfl_dt - 1.0) < 1e-11, (d["cfl_dt"], ref.cfl_dt)
    finally:
        pl.close()


def test_bad_arguments_are_refused():
    from coral_b200.solver import CoralError, PlaneLayer
    eq = equations("rbc_noslip_ra1e5")
    par = params(16, 12, 24)
    for args in ("--no-such-switch", "--smagorinsky-prefactor", "--cflFactor-along-z x"):
        with pytest.raises(CoralError) as e:
            PlaneLayer(eq, par, args=args)
        assert e.value.code == -1, str(e.value)


@pytest.mark.parametrize("name", [
    "coral.equations.RBC_potentials", "coral.equations.RBC_primitiveVars_Vanilla",
    "coral.equations.RBC_primitiveVars_variant1", "coral.equations.RBC_primitiveVars_variant2",
    "coral.equations.stratifiedChannel.toroidalPoloidal", "coral.equations.convective_dynamo"])
def test_reference_example_recipes_match_oracle(name):
    """Every other equation file the reference ships, read unmodified: the RBC
    examples (potentials; primitive variables with up to 11 full and 18
    quadratic variables), the stratified channel in toroidal-poloidal form and
    the convective dynamo (three coupled systems, 23 quadratic variables)."""
    eq = _example(name)
    par = params(16, 12, 24, dt=1e-5)
    ref, pl, errs = _run_both(eq, par, 2, 1e-5)
    pl.close()


def test_dynamo_toroidal_poloidal_file_is_refused():
    """bxFull where the full variable is BxFull: CORAL_EPARSE, as the reference stops."""
    from coral_b200.solver import CoralError, PlaneLayer
    with pytest.raises(CoralError) as e:
        PlaneLayer(_example("coral.equations.convective_dynamo.toroidalPoloidal"), params(16, 12, 24))
    assert e.value.code == -6 and "bad NL var definition" in str(e.value)


def test_feature_recipes_under_every_kernel_variant():
    """The autotuner's kernel variants on recipes with a penalisation field,
    surface values and vertical decompositions, and the Smagorinsky viscosity, at
    384 x 384 x 32 (x passes of length 576; the y-chunked pipeline runs its
    per-band z operations and the fused z pass its given fields): bit for bit
    the default step where the variant keeps the arithmetic, to 1e-10 (the
    tolerance of the other feature tests: the penalisation term of strength 1e3
    amplifies round-off) where it changes an FFT plan, band or tile form."""
    from coral_b200.solver import PlaneLayer
    from tests.test_gpu_timeloop import _variants_match
    cases = [(_example("coral.equations.RBC_penalised"), None),
             (_with_surface_vars(equations("rbc_noslip_ra1e5")), None),
             (_with_smagorinsky_vars(equations("rbc_noslip_ra1e5")),
              "--withHorizontalSmagorinsky --smagorinsky-prefactor 3.d0")]
    par = params(384, 384, 32, dt=1e-6)
    for eq, args in cases:
        rng = np.random.default_rng(41)
        state = {}

        def make():
            pl = PlaneLayer(eq, par, args=args)
            if not state:
                state["f"] = [1e-3 * (rng.standard_normal((pl.NXH, pl.NYAA, t)) +
                                      1j * rng.standard_normal((pl.NXH, pl.NYAA, t))) for t in pl.T]
                state["z"] = [1e-3 * rng.standard_normal(t) for t in pl.Tz]
            for s, f in enumerate(state["f"]):
                pl.set_field(s, f)
            for s, z in enumerate(state["z"]):
                pl.set_mean_field(s, z)
            return pl
        _variants_match(make, 2, 1e-6, tol=1e-10).close()


@pytest.mark.parametrize("name,args,kw", [
    ("rbc_penalised_ra1e8", None, {}),
    ("rbc_smagorinsky_ra1e8", "--withHorizontalSmagorinsky --smagorinsky-prefactor 0.1",
     dict(smagorinsky=True, smagorinsky_prefactor=0.1))])
def test_feature_bench_recipes_match_oracle(name, args, kw):
    """The recipes of the bench's penalised and Smagorinsky configurations
    (their NL operators take the compiled tile forms of group widths 3, 3, 5
    and 6, 6, 2) at 16 x 12 x 24: three steps against the oracle."""
    eq = equations(name)
    par = params(16, 12, 24, dt=1e-6)
    ref, pl, errs = _run_both(eq, par, 3, 1e-6, args=args, oracle_kw=kw)
    pl.close()
