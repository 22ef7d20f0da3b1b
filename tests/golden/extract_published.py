"""Writes heat_equation_published.json from the reference's own benchmark report.

The reference publishes, for its heat-equation benchmark, the relative L2 error
after 10 steps for three ARS schemes at seven timesteps, as literal lists in
etc/benchmarks/00_heat_equation/error_report.py:4-15.  This script reads that
file as text (it does not execute it) and stores the numbers, so the tests can
run where the reference tree is absent.  The analytic stress-free
Rayleigh-Benard growth rate quoted by benchmark 01
(etc/benchmarks/01_Rayleigh_Benard_stressFree/benchmark_01_stressfree_rayleigh_benard.ipynb:68)
is stored beside them, with benchmark 02's published mean Nusselt number and
its standard deviation (velocity-pressure form) and a verbatim copy of that
benchmark's input files (tests/golden/benchmark02/: both equation forms),
benchmark 01's (tests/golden/benchmark01/) and the equation files of the
reference's equation examples, the stratified channel, the convective dynamo
and the baroclinic-turbulence case (tests/golden/examples/), and the names of the procedures of the marching
include (tests/golden/marching_procedures.txt).

usage: python tests/golden/extract_published.py <path-to-coral-tree>
"""
import ast
import json
import os
import re
import sys


def main(root):
    src = open(os.path.join(root, "etc/benchmarks/00_heat_equation/error_report.py")).read()
    out = {"source": "etc/benchmarks/00_heat_equation/error_report.py:4-15"}
    for name in ("err111", "err222", "err443", "dt"):
        m = re.search(name + r"\s*=\s*(\[[^\]]*\])", src, re.S)
        out[name] = ast.literal_eval(m.group(1))
    nb = open(os.path.join(root, "etc/benchmarks/01_Rayleigh_Benard_stressFree/"
                                 "benchmark_01_stressfree_rayleigh_benard.ipynb")).read()
    m = re.search(r"maximum growthrate s = ([0-9.]+)", nb)
    out["stressfree_rb_max_growthrate"] = float(m.group(1))
    out["stressfree_rb_source"] = ("etc/benchmarks/01_Rayleigh_Benard_stressFree/"
                                   "benchmark_01_stressfree_rayleigh_benard.ipynb:68")
    # benchmark 02's published mean Nusselt number (notebook cell output) and its
    # input files, copied verbatim so that the parser and the long run read the
    # reference's own files where the reference tree is absent
    # (the notebook reports the velocity-pressure run first, :97-98, then the
    # toroidal-poloidal run, :114-115)
    found = re.findall(r"the mean Nusselt number is: ([0-9.]+).*?the standard deviation: ([0-9.]+)", open(
        os.path.join(root, "etc/benchmarks/02_RRBC_julien_JFM96/benchmark_02_RRBC_julien96.ipynb")).read(), re.S)
    out["rrbc_julien96_nusselt_velocity_pressure"] = [float(found[0][0]), float(found[0][1])]
    out["rrbc_julien96_source"] = "etc/benchmarks/02_RRBC_julien_JFM96/benchmark_02_RRBC_julien96.ipynb:97-98"
    out["rrbc_julien96_nusselt_toroidal_poloidal"] = [float(found[1][0]), float(found[1][1])]
    out["rrbc_julien96_tp_source"] = "etc/benchmarks/02_RRBC_julien_JFM96/benchmark_02_RRBC_julien96.ipynb:114-115"
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "heat_equation_published.json"), "w") as f:
        json.dump(out, f, indent=1)
    dst = os.path.join(here, "benchmark02")
    os.makedirs(dst, exist_ok=True)
    for name in ("coral.equations.velocityPressure", "coral.equations.toroidalPoloidal", "coral.parameters.in",
                 "coral.timeseries", "coral.usrOutput"):
        with open(os.path.join(root, "etc/benchmarks/02_RRBC_julien_JFM96", name), "rb") as f:
            data = f.read()
        with open(os.path.join(dst, name), "wb") as f:
            f.write(data)
    # equation files of the reference's examples that use sources, penalisation and
    # the stratified channel (tests/golden/examples/, names kept)
    dst = os.path.join(here, "examples")
    os.makedirs(dst, exist_ok=True)
    ex = "etc/coral_equations_examples/coral.equations."
    for rel, name in ((ex + "RBC_penalised", None), (ex + "radiative_heating_potentials", None),
                      (ex + "RBC_potentials", None), (ex + "RBC_primitiveVars_Vanilla", None),
                      (ex + "RBC_primitiveVars_variant1", None), (ex + "RBC_primitiveVars_variant2", None),
                      ("etc/benchmarks/coral.equations.stratifiedChannel.velocityPressure", None),
                      ("etc/benchmarks/coral.equations.stratifiedChannel.toroidalPoloidal", None),
                      ("etc/benchmarks/03_convective_dynamo/coral.equations", "coral.equations.convective_dynamo"),
                      ("etc/benchmarks/03_convective_dynamo/coral.equations.toroidalPoloidal",
                       "coral.equations.convective_dynamo.toroidalPoloidal"),
                      ("etc/baroclinic_turbulence/coral.equations", "coral.equations.baroclinic_turbulence")):
        with open(os.path.join(root, rel), "rb") as f:
            data = f.read()
        with open(os.path.join(dst, name or os.path.basename(rel)), "wb") as f:
            f.write(data)
    # names of the procedures in the marching include (the ones a replacement
    # include has to define)
    with open(os.path.join(root, "src/plane_layer/PL_IMEX_timestepping_marching.f90")) as f:
        src = f.read()
    names = re.findall(r"^\s*(?:real\(kind=dp\)\s+)?(?:subroutine|function)\s+(\w+)", src, re.I | re.M)
    with open(os.path.join(here, "marching_procedures.txt"), "w") as f:
        f.write("\n".join(names) + "\n")
    # benchmark 01's input files (stress-free Rayleigh-Benard, linear growth)
    dst = os.path.join(here, "benchmark01")
    os.makedirs(dst, exist_ok=True)
    for name in ("coral.equations", "coral.parameters.in", "coral.timeseries"):
        with open(os.path.join(root, "etc/benchmarks/01_Rayleigh_Benard_stressFree", name), "rb") as f:
            data = f.read()
        with open(os.path.join(dst, name), "wb") as f:
            f.write(data)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/extract_published.py <path of the Coral source tree>")
    main(sys.argv[1])
