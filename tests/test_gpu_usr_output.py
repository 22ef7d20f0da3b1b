"""User outputs (coral.usrOutput): volumes, x/y/z slices, vertically summed
slices and profiles of full and quadratic variables, written by the time loop
at their periods, against the oracle's restatement of the reference's parser,
counters and file formats (oracle.coral_oracle.parse_usr_output,
usr_output_schedule, usr_output_files)."""
import os
import tempfile

import numpy as np
import pytest

from oracle import coral_oracle as co
from tests.problems import equations, params

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
B02 = os.path.join(ROOT, "tests", "golden", "benchmark02")

TEXT = """>>Volume :: tFull ;; Period= 2 <<
>>ZSlice :: uFull ;; Period= 1 ;; Position= 5 <<
>>YSlice :: wFull ;; Period= 3 ;; Position= 2 <<
>>XSlice :: tFull ;; Period= 2 ;; Position= 7 <<
>>XSlice :: tFull ;; Period= 2 ;; Position= 700 <<
>>Zsummed:: tFull ;; Period= 2 <<
>>Profile:: tFull ;; Period= 1 <<
>>Profile:: tw ;; Period= 2 <<
>>Volume :: uw ;; Period= 3 <<
>>ZSlice :: tw ;; Period= 1 ;; Position= 3 <<
>>EOF<<
"""


def _files(d):
    out = set()
    for sub in ("Volumes", "Slices", "Profiles"):
        p = os.path.join(d, sub)
        if os.path.isdir(p):
            out |= {sub + "/" + f for f in os.listdir(p)}
    return out


def test_usr_output_files_match_oracle():
    """Four steps of the no-slip recipe (tw with its vertical mean removed)
    through coral_run: the files written, their names and their contents
    (1e-12 of each field's maximum) against the oracle stepped alongside."""
    from coral_b200.solver import PlaneLayer
    eq = equations("rbc_noslip_ra1e8", **{"1.d8": "1.d5"}).replace(
        ">>quadratic_variable :: tw := tFull.wFull <<", ">>zFiltered_quadratic_variable :: tw := tFull.wFull <<")
    par = params(16, 12, 48, dt=1e-5)
    ref = co.Solver(eq, par)
    pl = PlaneLayer(eq, par)
    rng = np.random.default_rng(21)
    for s, lay in enumerate(ref.lay):
        f = 1e-2 * (rng.standard_normal((pl.NXH, pl.NYAA, lay.T)) + 1j * rng.standard_normal((pl.NXH, pl.NYAA, lay.T)))
        ref.field[s] = f.copy()
        pl.set_field(s, f)
    objs = co.parse_usr_output(TEXT, ref.recipe, ref.g)
    assert len(objs) == 9  # the x slice at 700 > NXAA is dropped
    pl.set_usr_output(TEXT)
    with tempfile.TemporaryDirectory() as d:
        pl.run(4, d)
        want = {}
        for s, itime, due in co.usr_output_schedule(objs, 1, 4):
            ref.step(1e-5)
            fphys, qphys = ref.stage0_phys
            want.update(co.usr_output_files(due, fphys, qphys, ref.g, itime))
        assert _files(d) == set(want), sorted(_files(d) ^ set(want))
        for name, arr in want.items():
            got = np.fromfile(os.path.join(d, name))
            assert got.shape == arr.shape, name
            assert np.abs(got - arr).max() <= 1e-12 * max(np.abs(arr).max(), 1e-300), name
    pl.close()


def test_usr_output_reads_the_reference_file_and_exports_on_demand():
    """Benchmark 02's coral.usrOutput, read unmodified (17 objects at 96^2 x 48),
    exported at once with a given time index: every file named as the reference
    names it, a volume equal to coral_get_full_phys in file order, the profile
    equal to the horizontal mean of the volume."""
    from coral_b200.solver import PlaneLayer
    eq = open(os.path.join(B02, "coral.equations.velocityPressure")).read()
    par = open(os.path.join(B02, "coral.parameters.in")).read()
    recipe = co.parse_equations(eq)
    p = co.read_parameters_text(par)
    g = co.Geometry(p["NX"], p["NY"], p["NZ"], p["Lx"], p["Ly"], p["gap"], p["center"])
    text = open(os.path.join(B02, "coral.usrOutput")).read()
    objs = co.parse_usr_output(text, recipe, g)
    assert len(objs) == 17
    pl = PlaneLayer(eq, par)
    rng = np.random.default_rng(5)
    f = 1e-2 * (rng.standard_normal((pl.NXH, pl.NYAA, pl.T[0])) + 1j * rng.standard_normal((pl.NXH, pl.NYAA, pl.T[0])))
    pl.set_field(0, f)
    rc = pl._lib.coral_set_usr_output_from_file(pl._h, os.path.join(B02, "coral.usrOutput").encode())
    assert rc == 0, pl._lib.coral_last_error(pl._h).decode()
    with tempfile.TemporaryDirectory() as d:
        pl.export_usr_output(d, 7)
        want = set()
        for kind, is_q, iv, _, pos in objs:
            tag = "linear_var%02d" % (iv + 1)
            want.add({"volume": "Volumes/%s_time00000007_full.dat" % tag,
                      "zSlice": "Slices/%s_z%05d_time00000007_full.dat" % (tag, pos),
                      "ySlice": "Slices/%s_y%05d_time00000007_full.dat" % (tag, pos),
                      "xSlice": "Slices/%s_x%05d_time00000007_full.dat" % (tag, pos),
                      "profil": "Profiles/%s_time00000007_full.dat" % tag}[kind])
        assert _files(d) == want
        t_phys = pl.full_phys(3)  # tFull, [y][x][z]
        vol = np.fromfile(os.path.join(d, "Volumes/linear_var04_time00000007_full.dat"))
        assert np.array_equal(vol, t_phys.transpose(1, 0, 2).ravel())
        prof = np.fromfile(os.path.join(d, "Profiles/linear_var04_time00000007_full.dat"))
        assert np.allclose(prof, t_phys.mean(axis=(0, 1)), rtol=0, atol=1e-14 * np.abs(t_phys).max())
        zs = np.fromfile(os.path.join(d, "Slices/linear_var04_z00024_time00000007_full.dat"))
        assert np.array_equal(zs, t_phys.transpose(1, 0, 2)[:, :, 23].ravel())
    pl.close()


def test_zsummed_quadratic_variable_is_refused():
    from coral_b200.solver import CoralError, PlaneLayer
    pl = PlaneLayer(equations(), params(16, 16, 16))
    with pytest.raises(CoralError) as e:
        pl.set_usr_output(">>Zsummed:: uu ;; Period= 3 <<\n>>EOF<<\n")
    assert e.value.code == -8
    with pytest.raises(CoralError) as e:
        pl.set_usr_output(">>Slab :: uu ;; Period= 3 <<\n>>EOF<<\n")
    assert e.value.code == -6
    pl.close()


def test_usr_output_write_failure_is_reported():
    """The files are written by a host thread behind the step: a directory
    that cannot be made (a plain file in its path) comes back from coral_run
    as CORAL_EIO, and the handle keeps working (the next run into a good
    directory writes its files)."""
    from coral_b200.solver import CoralError, PlaneLayer
    eq = equations("rbc_noslip_ra1e8", **{"1.d8": "1.d5"})
    pl = PlaneLayer(eq, params(16, 12, 48, dt=1e-5))
    pl.set_usr_output(">>Profile:: tFull ;; Period= 1 <<\n>>Volume :: tFull ;; Period= 1 <<\n>>EOF<<\n")
    with tempfile.TemporaryDirectory() as d:
        blocked = os.path.join(d, "blocked")
        open(blocked, "w").close()
        with pytest.raises(CoralError) as e:
            pl.run(2, blocked)
        assert e.value.code == -7, str(e.value)
        good = os.path.join(d, "good")
        pl.run(2, good)
        assert len(_files(good)) == 4
    pl.close()
