"""CPU restatement of the learned subgrid closure's network (test infrastructure).

TEST INFRASTRUCTURE ONLY: the checker of the GPU kernels in
coral_b200/csrc/closure.cu, not product code.  The reference has no learned
closure; this restates the network the product defines: 5 input channels
(u, v, w, T times in_scale, and z' = the Gauss-Chebyshev coordinate in [-1, 1])
at the 27 points of a 3 x 3 x 3 stencil (periodic in x and y, zero beyond the
walls), three tanh layers of 64 and a linear layer of 9; weights rounded to
BF16 (round to nearest even) as the kernels use them, everything else in FP64
here (FP32 on the GPU).  Loss = mean over points of
sum_q (y_q - target_q / out_scale_q)^2; gradients by backpropagation.
"""
import numpy as np

CIN, TAPS, HID, OUT = 5, 27, 64, 9
NIN = CIN * TAPS
SIZES = [(HID, NIN), (HID, HID), (HID, HID), (OUT, HID)]


def param_count():
    return sum(o * i + o for o, i in SIZES)


def unpack(p):
    """flat parameters -> [(W, b)] in the kernels' layout (W0, b0, W1, b1, ...)."""
    out, k = [], 0
    for o, i in SIZES:
        W = p[k:k + o * i].reshape(o, i)
        k += o * i
        b = p[k:k + o]
        k += o
        out.append((W, b))
    return out


def bf16(x):
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    u = (u + (0x7FFF + ((u >> 16) & 1))) & np.uint32(0xFFFF0000)
    return u.view(np.float32).astype(np.float64)


def zeta(NZA):
    i = np.arange(1, NZA + 1)
    return np.cos(np.pi * (2 * i - 1) / (2 * NZA))


def gather(fields, points, in_scale):
    """fields: (4, NYA, NXA, NZA); points: linear indices [y][x][z] -> (npts, 135),
    column c * 27 + tap, tap = ((dy + 1) * 3 + dx + 1) * 3 + dz + 1."""
    _, NYA, NXA, NZA = fields.shape
    z = points % NZA
    x = (points // NZA) % NXA
    y = points // (NZA * NXA)
    zt = zeta(NZA)
    X = np.zeros((len(points), NIN))
    tap = 0
    for dy in (-1, 0, 1):
        for dx in (-1, 0, 1):
            for dz in (-1, 0, 1):
                yy, xx, zz = (y + dy) % NYA, (x + dx) % NXA, z + dz
                inside = (zz >= 0) & (zz < NZA)
                zc = np.where(inside, zz, 0)
                for c in range(4):
                    X[:, c * TAPS + tap] = np.where(inside, fields[c, yy, xx, zc] * in_scale[c], 0.0)
                X[:, 4 * TAPS + tap] = np.where(inside, zt[zc], 0.0)
                tap += 1
    return X


def forward(p, X):
    L = unpack(p)
    acts = [X]
    h = X
    for li, (W, b) in enumerate(L):
        a = h @ bf16(W).T + b
        h = np.tanh(a) if li < 3 else a
        acts.append(h)
    return acts


def loss_and_grad(p, X, T):
    """T: targets already divided by out_scale, (npts, 9)."""
    L = unpack(p)
    acts = forward(p, X)
    y = acts[-1]
    n = X.shape[0]
    d = y - T
    loss = float((d * d).sum() / n)
    g = [None] * 4
    delta = 2.0 * d / n
    for li in (3, 2, 1, 0):
        W, b = L[li]
        hin = acts[li]
        g[li] = (delta.T @ hin, delta.sum(axis=0))
        if li > 0:
            delta = (delta @ bf16(W)) * (1.0 - hin * hin)
    flat = np.concatenate([np.concatenate([gw.ravel(), gb]) for gw, gb in g])
    return loss, flat
