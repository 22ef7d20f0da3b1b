"""The learned subgrid closure on the GPU: its forward, backward and Adam
kernels against the CPU restatement (oracle/closure_oracle.py), training on
subgrid data the solver generates, what the trained network gains over the
plain coarse products, and the coupling into the time step."""
import numpy as np
import pytest

from oracle import closure_oracle as clo
from tests.problems import equations, params

pytestmark = pytest.mark.gpu


def _data(rng, nsnap, NYA, NXA, NZA):
    x = rng.standard_normal((nsnap, 4, NYA, NXA, NZA)).astype(np.float32)
    y = rng.standard_normal((nsnap, 9, NYA, NXA, NZA)).astype(np.float32)
    return x, y


def test_closure_gradient_and_inference_match_oracle():
    import torch
    from coral_b200.closure import Closure
    rng = np.random.default_rng(7)
    NYA, NXA, NZA = 12, 18, 9
    x, y = _data(rng, 2, NYA, NXA, NZA)
    net = Closure(seed=3)
    ins, outs = [0.5, 0.7, 0.9, 1.3], [1.0, 2.0, 0.5, 1.5, 1.0, 0.8, 1.2, 0.9, 1.1]
    net.set_scales(ins, outs)
    npoint = NYA * NXA * NZA
    pts = rng.choice(2 * npoint, size=300, replace=False).astype(np.int64)
    dx, dy, dp = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda(), torch.from_numpy(pts).cuda()
    net.zero_gradient()
    loss = net.train(dx, dy, dp, apply=False)
    g = net.gradient()
    p = net.params().astype(np.float64)
    X = np.concatenate([clo.gather(x[s].astype(np.float64), pts[pts // npoint == s] % npoint, ins) for s in range(2)])
    T = np.concatenate([y[s].reshape(9, -1)[:, pts[pts // npoint == s] % npoint].T for s in range(2)]) / np.array(outs)
    l_ref, g_ref = clo.loss_and_grad(p, X, T)
    assert abs(loss - l_ref) <= 1e-5 * l_ref
    assert np.linalg.norm(g - g_ref) <= 1e-4 * np.linalg.norm(g_ref)
    # inference on a whole grid (double fields)
    f = rng.standard_normal((4, NYA, NXA, NZA))
    tau = torch.zeros((9, NYA, NXA, NZA), dtype=torch.float64, device="cuda")
    net.infer(torch.from_numpy(f).cuda(), tau)
    torch.cuda.synchronize()
    yr = clo.forward(p, clo.gather(f, np.arange(npoint), ins))[-1] * np.array(outs)
    got = tau.cpu().numpy().reshape(9, -1).T
    assert np.abs(got - yr).max() <= 1e-4 * np.abs(yr).max()
    net.close()


def test_closure_training_learns_a_stencil_function():
    import torch
    from coral_b200.closure import Closure
    rng = np.random.default_rng(8)
    NYA, NXA, NZA = 16, 16, 12
    x = rng.standard_normal((4, 4, NYA, NXA, NZA)).astype(np.float32)
    # targets: smooth functions of the point and its x-neighbours
    y = np.zeros((4, 9, NYA, NXA, NZA), dtype=np.float32)
    for q in range(9):
        a, b = q % 4, (q + 1) % 4
        y[:, q] = np.tanh(x[:, a] * np.roll(x[:, b], 1, axis=3))
    net = Closure(seed=1)
    net.set_scales([1, 1, 1, 1], [1] * 9)
    dx, dy = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    npoint = NYA * NXA * NZA
    g = torch.Generator(device="cpu").manual_seed(0)
    losses = []
    for it in range(300):
        pts = torch.randint(0, 4 * npoint, (2048,), generator=g).cuda()
        losses.append(net.train(dx, dy, pts, lr=3e-3))
    assert np.mean(losses[-20:]) < 0.3 * np.mean(losses[:5]), (losses[:5], losses[-20:])
    net.close()


def test_closure_in_the_time_step():
    """A network with all parameters zero adds nothing: the attached step equals
    the plain step (the unfused z passes differ only by round-off); a trained-
    looking nonzero network changes the state and keeps it finite."""
    from coral_b200.closure import Closure, detach
    from coral_b200.solver import PlaneLayer
    eq, par = equations(), params(16, 16, 24, dt=1e-4)
    rng = np.random.default_rng(9)
    a, b = PlaneLayer(eq, par), PlaneLayer(eq, par)
    f = 1e-2 * (rng.standard_normal((a.NXH, a.NYAA, a.T[0])) + 1j * rng.standard_normal((a.NXH, a.NYAA, a.T[0])))
    for pl in (a, b):
        pl.set_field(0, f)
    net = Closure(seed=2)
    net.set_params(np.zeros(net.nparam, dtype=np.float32))
    net.attach(b)
    a.march_forward(1e-4, 3)
    b.march_forward(1e-4, 3)
    fa, fb = a.get_field(0), b.get_field(0)
    assert np.linalg.norm(fb - fa) <= 1e-12 * np.linalg.norm(fa)
    net.set_params(0.05 * np.random.default_rng(1).standard_normal(net.nparam).astype(np.float32))
    detach(b)
    net.attach(b)
    b.march_forward(1e-4, 2)
    a.march_forward(1e-4, 2)
    fb2 = b.get_field(0)
    assert np.all(np.isfinite(fb2.view(np.float64)))
    assert np.linalg.norm(fb2 - a.get_field(0)) > 1e-8 * np.linalg.norm(a.get_field(0))
    for x in (a, b):
        x.close()
    net.close()


def test_trained_closure_gains_over_plain_coarse_products():
    """Subgrid data from the solver itself: a fine 48 x 48 x 24 no-slip run
    (Ra 1e6, CFL-adaptive) truncated to 16 x 16 x 12; the network trained on 6 snapshots cuts
    the error of the coarse quadratic variables against the filtered fine ones
    on 2 held-out snapshots (a-priori gain = 1 - error with / error without)."""
    import torch
    from coral_b200.closure import Closure, subgrid_snapshot
    from coral_b200.solver import PlaneLayer
    from coral_b200.closure_demo import texts
    from coral_b200.initial_conditions import noisy_modes
    eqf, parf = texts(1e6, (48, 48, 24), dt_max=1e-4, cfl=0.3)
    _, parc = texts(1e6, (16, 16, 12), dt_max=1e-4, cfl=0.3)
    fine = PlaneLayer(eqf, parf)
    coarse = PlaneLayer(eqf, parc)
    noisy_modes(fine, 2 * np.pi, 2 * np.pi, amp=1e-6, amp0=0.0, seed=10)
    fine.set_hermitian_kx0(True)
    fine.run(800)  # CFL-adaptive time loop: growth from the small perturbation, then saturation
    xs, ys = [], []
    for _ in range(8):
        fine.run(10)
        x, y = subgrid_snapshot(fine, coarse)
        xs.append(x)
        ys.append(y)
    x = np.stack(xs).astype(np.float32)
    y = np.stack(ys).astype(np.float32)
    assert np.all(np.isfinite(x)) and np.all(np.isfinite(y))
    ins = 1.0 / (x[:6].std(axis=(0, 2, 3, 4)) + 1e-30)
    outs = y[:6].std(axis=(0, 2, 3, 4)) + 1e-30
    net = Closure(seed=4)
    net.set_scales(ins, outs)
    dx, dy = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    npoint = int(np.prod(x.shape[2:]))
    g = torch.Generator(device="cpu").manual_seed(0)
    for it in range(600):
        pts = torch.randint(0, 6 * npoint, (4096,), generator=g).cuda()
        net.train(dx, dy, pts, lr=2e-3)
    err_with = err_without = 0.0
    for s in (6, 7):
        tau = torch.zeros((9,) + x.shape[2:], dtype=torch.float64, device="cuda")
        net.infer(torch.from_numpy(x[s].astype(np.float64)).cuda(), tau)
        torch.cuda.synchronize()
        pred = tau.cpu().numpy()
        err_with += float(np.sum((y[s] - pred) ** 2))
        err_without += float(np.sum(y[s].astype(np.float64) ** 2))
    gain = 1.0 - err_with / err_without
    print("a-priori gain on held-out snapshots: %.3f" % gain)
    assert gain > 0.2
    for h in (fine, coarse):
        h.close()
    net.close()
