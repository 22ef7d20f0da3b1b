"""Long run of the reference's benchmark 02 (rotating Rayleigh-Benard, Julien
et al. 1996 no-slip case: Ra = 2.81e5, E^-1 = 707.1, Pr = 1, 96 x 96 x 48 modes,
box 2 x 2 x 1, ARS_222, CFL-adaptive dt with CFL_C = 0.2, dt_max = 1e-3,
tolerance 0.3) from its own input files (read unmodified), on the GPU, with
the mean Nusselt number computed by the benchmark's rule
(coral_b200.nusselt).  The reference publishes 4.76905 +- 0.00993 for its
velocity-pressure form and 4.77566 +- 0.00919 for its toroidal-poloidal form
(--form tp: coral.equations.toroidalPoloidal, with z derivatives in its full
variables; etc/benchmarks/02_RRBC_julien_JFM96/benchmark_02_RRBC_julien96.ipynb:97-98,114-115).

The reference starts this case from its default random initial condition
(noisy_initial_conditions, amplitude 1e-16, unseeded); here the start is the
seeded form of it (coral_b200.initial_conditions.noisy_modes).  A spin-up phase of
--spinup simulated time units is run without output; then the step index is
reset to 1 and --record time units are recorded into <out>/Timeseries.

usage: python -m coral_b200.benchmark02 --out DIR [--form vp|tp] [--inputs DIR] [--spinup T] [--record T] [--seed S]
"""
import argparse
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--form", choices=["vp", "tp"], default="vp", help="velocity-pressure or toroidal-poloidal recipe")
    ap.add_argument("--inputs", default=os.path.join(ROOT, "tests", "golden", "benchmark02"))
    ap.add_argument("--spinup", type=float, default=0.5)
    ap.add_argument("--record", type=float, default=1.0)
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--chunk", type=int, default=2000)
    ap.add_argument("--max-seconds", type=float, default=1e9, help="wall-clock limit of the recorded phase")
    ap.add_argument("--amp", type=float, default=1e-16,
                    help="amplitude of the seeded form of the reference's default initial condition")
    ap.add_argument("--white-noise", action="store_true",
                    help="start from a white-noise temperature of amplitude --amp instead")
    ap.add_argument("--cfl", type=float, default=None, help="override CFL_C of the parameter file")
    ap.add_argument("--no-projection", action="store_true", help="keep the anti-Hermitian part of the kx = 0 line")
    a = ap.parse_args(argv)

    from coral_b200 import initial_conditions as ic
    from coral_b200 import nusselt
    from coral_b200.solver import PlaneLayer

    eq = os.path.join(a.inputs, "coral.equations.velocityPressure" if a.form == "vp" else
                      "coral.equations.toroidalPoloidal")
    par = os.path.join(a.inputs, "coral.parameters.in")
    if a.cfl is None:
        pl = PlaneLayer.from_files(eq, par)
    else:
        lines = open(par).read().splitlines(True)
        lines[12] = "%r ! CFL_C (overridden)\n" % a.cfl
        pl = PlaneLayer(open(eq).read(), "".join(lines))
    pl._check(pl._lib.coral_set_timeseries_from_file(pl._h, os.fsencode(os.path.join(a.inputs, "coral.timeseries"))))
    # the invisible anti-Hermitian part of the kx = 0 line is removed after every
    # step (coral_set_hermitian_kx0); without it this case blows up near t = 0.2
    if not a.no_projection:
        pl.set_hermitian_kx0(True)
    os.makedirs(a.out, exist_ok=True)
    if a.white_noise:
        qs = os.path.join(a.out, "Restart")
        ic.white_noise_temperature(qs, pl.NX, pl.NY, pl.NZ, amplitude=a.amp, seed=a.seed)
        pl.import_quicksave(qs)
    else:
        ic.noisy_modes(pl, 2.0, 2.0, amp=a.amp, amp0=a.amp, seed=a.seed)

    def advance(t_end, outdir, wall_limit=1e9):
        t0 = time.time()
        steps = 0
        while pl.get_time()["time"] < t_end and time.time() - t0 < wall_limit:
            pl.run(a.chunk, outdir)
            steps += a.chunk
            st = pl.get_time()
            dg = pl.diagnostics()
            print("t = %.5f  dt = %.3e  steps %d  refactorisations %d  KE %.4e  cfl_dt %.3e  %.0f steps/s" % (
                st["time"], st["dt"], st["i_timestep"] - 1, st["refactorizations"], dg["KE"], dg["cfl_dt"],
                steps / (time.time() - t0)), flush=True)
        return steps, time.time() - t0

    s1, w1 = advance(a.spinup, None)
    st = pl.get_time()
    if a.record <= 0:
        pl.close()
        return
    pl.set_time(st["time"], st["dt"], 1)
    s2, w2 = advance(st["time"] + a.record, a.out, a.max_seconds)
    pl.synchronize()
    m, s, q = nusselt.mean_nusselt(a.out, pl.NZAA)
    published = {"vp": [4.76905366624831, 0.009934859274015244], "tp": [4.775658148380188, 0.009187540842645432]}
    res = dict(case="benchmark02 %s 96x96x48" % ("velocity-pressure" if a.form == "vp" else "toroidal-poloidal"),
               spinup_time=a.spinup, record_time=pl.get_time()["time"] - st["time"],
               spinup_steps=s1, record_steps=s2, steps_per_s=(s1 + s2) / (w1 + w2), seed=a.seed,
               nusselt_mean=m, nusselt_spread=s, quarters=q, published=published[a.form],
               refactorizations=pl.get_time()["refactorizations"])
    print(json.dumps(res))
    with open(os.path.join(a.out, "nusselt.json"), "w") as f:
        json.dump(res, f, indent=1)
    pl.close()


if __name__ == "__main__":
    main()
