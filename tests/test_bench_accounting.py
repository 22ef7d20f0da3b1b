"""CPU checks of bench.py's roofline accounting: launches per step, the
algorithmic bytes of the solve kernels and the traffic file lookup."""
import bench


def test_phase_launches():
    n = bench.phase_launches(2, 2)
    assert n["kstd_out"] == 1 and all(v == 2 for k, v in n.items() if k != "kstd_out")
    assert bench.phase_launches(2, 1)["kstd_out"] == 2
    assert bench.phase_launches(1, 2)["kstd_out"] == 1


def test_solve_bytes_follow_the_masked_factor_entries():
    g = {"NXH": 8, "NYA": 12, "NXA": 12, "NZ": 16, "NZA": 24, "nF": 4, "nQ": 9}
    nsys, nact, T, ncls, Tc, kl, ku = 96, 60, 88, 2, 44, 5, 9
    full = bench.phase_bytes(g, nsys, nact, T, ncls, Tc, kl, ku, 2, 8)
    masked = bench.phase_bytes(g, nsys, nact, T, ncls, Tc, kl, ku, 2, 8, factor_entries=Tc * 10)
    cols = nact * ncls * Tc
    assert full["substitution"] == cols * (2 * kl + ku + 1) * 8 + cols + 64 * cols
    assert masked["substitution"] == nact * ncls * Tc * 10 * 8 + cols + 64 * cols
    # split systems: K_std reads the solution and writes K_std once per launch
    assert full["kstd_out"] == 2 * nact * 16 * T
    # the last stage writes no K_hat: stage 0 moves 3 state-sized arrays, stage 1
    # (two K arrays more, no K_hat) 4, plus the quadratic coefficients and the
    # inactive systems' output in stage 0
    st = nsys * 16 * T
    q = nact * 16 * g["nQ"] * g["NZ"]
    assert full["rhs_nl"] == ((3 * st + q + (nsys - nact) * 16 * T) + (4 * st + q)) / 2


def test_traffic_lookup():
    v = bench.read_traffic("k_z_fused")
    assert v is not None and v > 1e9
    assert bench.read_traffic("no_such_kernel") is None
