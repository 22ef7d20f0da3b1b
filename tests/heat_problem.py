"""Builds the heat-equation problem of the reference's benchmark 00 in the
coral.equations grammar: three mean fields diffusing with boundary codes 22
(top Dirichlet, bottom Neumann), 23 (top Neumann, bottom Dirichlet) and 20
(both Dirichlet), Prandtl = 0.33, and one decoupled kxky field."""

HEAT_PARAMS_TEMPLATE = """0
{NX}
{NY}
{NZ}
0
1.0d0
1.0d0
1.d0
0.5d0
0
{dt}
0.3d0
0.2d0
'{scheme}'
0
.True.
0
13.d0
"""


def heat_equations() -> str:
    L = [">>Param :: Prandtl := 3.3d-1 <<",
         ">>linear_variable_kxky :: w <<"]
    for v in ("uMean", "vMean", "wMean"):
        L.append(">>linear_variable_mean :: %s <<" % v)
    L += [">>linear_variable_full :: wFull <<",
          ">>linear_variable_full_build :: + w <<",
          ">>quadratic_variable :: ww := wFull.wFull <<",
          ">>add_set_of_coupled_kxky_equations <<",
          ">>linearly_coupled_var :: w <<", ">>add_BC_for_this_var :: 20 <<",
          ">>new_equation :: 2 <<", ">>add_d/dt_term :: + Iz.Iz.w <<",
          ">>add_rhs_linear :: + Prandtl.Iz.Iz.dx.dx.w + Prandtl.Iz.Iz.dy.dy.w + Prandtl.w <<"]
    for v, bc in (("uMean", 22), ("vMean", 23), ("wMean", 20)):
        L += [">>add_set_of_coupled_zero_equations <<",
              ">>linearly_coupled_var :: %s <<" % v, ">>add_BC_for_this_var :: %d <<" % bc,
              ">>new_equation :: 2 <<", ">>add_d/dt_term :: + Iz.Iz.%s <<" % v,
              ">>add_rhs_linear :: + Prandtl.%s <<" % v]
    L.append(">>EOF<<")
    return "\n".join(L) + "\n"


def heat_params(NZ, dt, scheme, NX=4, NY=4) -> str:
    return HEAT_PARAMS_TEMPLATE.format(NX=NX, NY=NY, NZ=NZ, dt=repr(dt), scheme=scheme)
