"""Python mirror of the learned-closure C-ABI (coral_closure_* in include/coral_b200.h),
plus the training-data pipeline: a fine-grid run of the GPU solver, truncated to
the coarse modes, gives the coarse resolved fields and the subgrid parts
tau_q = P(q_fine) - q(P(fields)) of the quadratic variables."""
import ctypes

import numpy as np

from . import _lib
from .solver import CoralError


class Closure:
    def __init__(self, device=0, seed=0):
        self._lib = _lib.load()
        c = ctypes.c_void_p()
        rc = self._lib.coral_closure_create(int(device), ctypes.c_ulonglong(seed), ctypes.byref(c))
        if rc != 0:
            raise CoralError(rc, self._lib.coral_closure_last_error(None).decode())
        self._c = c
        self.nparam = self._lib.coral_closure_param_count()

    def _check(self, rc):
        if rc != 0:
            raise CoralError(rc, self._lib.coral_closure_last_error(self._c).decode())

    def set_scales(self, in_scale, out_scale):
        a = (ctypes.c_float * 4)(*[float(v) for v in in_scale])
        b = (ctypes.c_float * 9)(*[float(v) for v in out_scale])
        self._check(self._lib.coral_closure_set_scales(self._c, a, b))

    def params(self):
        out = np.zeros(self.nparam, dtype=np.float32)
        self._check(self._lib.coral_closure_get_params(self._c, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                                       self.nparam))
        return out

    def set_params(self, p):
        a = np.ascontiguousarray(p, dtype=np.float32)
        self._check(self._lib.coral_closure_set_params(self._c, a.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                                       self.nparam))

    def gradient(self):
        out = np.zeros(self.nparam, dtype=np.float32)
        self._check(self._lib.coral_closure_get_gradient(self._c, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                                         self.nparam))
        return out

    def zero_gradient(self):
        self._check(self._lib.coral_closure_zero_gradient(self._c))

    def train(self, inputs, targets, points, lr=1e-3, apply=True):
        """inputs (nsnap, 4, NYAA, NXAA, NZAA) and targets (nsnap, 9, ...) float32
        device tensors, points int64 device tensor; returns the loss."""
        nsnap, _, NYA, NXA, NZA = inputs.shape
        loss = ctypes.c_double()
        self._check(self._lib.coral_closure_train(self._c, ctypes.c_void_p(inputs.data_ptr()),
                                                  ctypes.c_void_p(targets.data_ptr()), nsnap, NXA, NYA, NZA,
                                                  ctypes.c_void_p(points.data_ptr()), points.numel(), float(lr),
                                                  1 if apply else 0, ctypes.byref(loss)))
        return loss.value

    def infer(self, fields, tau, stream=0):
        """fields (4, NYAA, NXAA, NZAA) and tau (9, ...) float64 device tensors."""
        _, NYA, NXA, NZA = fields.shape
        self._check(self._lib.coral_closure_infer(self._c, ctypes.c_void_p(fields.data_ptr()), NXA, NYA, NZA,
                                                  ctypes.c_void_p(tau.data_ptr()), ctypes.c_void_p(stream)))

    def attach(self, pl):
        pl._check(self._lib.coral_closure_attach(pl._h, self._c))

    def close(self):
        if getattr(self, "_c", None):
            self._lib.coral_closure_destroy(self._c)
            self._c = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def detach(pl):
    pl._check(pl._lib.coral_closure_attach(pl._h, None))


# quadratic variables of the Rayleigh-Benard recipes, as products of the full
# variables (uFull, vFull, wFull, tFull) = (0, 1, 2, 3): uu uv uw vv vw ww tu tv tw
RBC_QUADS = ((0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2), (3, 0), (3, 1), (3, 2))


def truncate(spec_f, coarse):
    """Spectral coefficients of a fine grid (NX/2, NYAA, NZ) restricted to the
    coarse handle's active modes: kx < NXc/2, |ky| < NYc/2, n < NZc (the coarse
    grid's dealiased ky rows stay zero)."""
    NXHc, NYAc, NZc, NYc = coarse.NXH, coarse.NYAA, coarse.NZ, coarse.NY
    NYAf = spec_f.shape[1]
    out = np.zeros((NXHc, NYAc, NZc), dtype=np.complex128)
    for iy in range(NYAc):
        ky = iy if iy <= NYAc // 2 else iy - NYAc
        if abs(ky) >= NYc / 2:
            continue
        out[:, iy, :] = spec_f[:NXHc, ky % NYAf, :NZc]
    return out


def coarse_project(phys, coarse):
    """C(P(.)) of a coarse physical field: its coarse spectrum with the dealiased
    ky rows cleared, transformed back (what the coarse step's K_hat sees of it)."""
    s = coarse.phys_to_spec(phys)
    NYAc, NYc = coarse.NYAA, coarse.NY
    for iy in range(NYAc):
        ky = iy if iy <= NYAc // 2 else iy - NYAc
        if abs(ky) >= NYc / 2:
            s[:, iy, :] = 0.0
    return coarse.spec_to_phys(s)


def subgrid_snapshot(fine, coarse, quads=RBC_QUADS):
    """Coarse inputs (4, NYAA, NXAA, NZAA) and subgrid targets (9, ...) of the
    fine handle's current state, all through the library's own transforms:
    f_c = C(P(f)) for each full variable (P: truncation to the coarse active
    modes, C: the coarse inverse transform) and, for each quadratic variable,
    tau_q = C(P(q_fine)) - C(P(f_c1 f_c2)) -- the part of the filtered fine
    product that the coarse product misses, in the modes the coarse NL
    assembly uses."""
    fphys = [fine.full_phys(f) for f in range(4)]
    fc = np.stack([coarse.spec_to_phys(truncate(fine.phys_to_spec(p), coarse)) for p in fphys])
    tau = []
    for a, b in quads:
        pq = coarse.spec_to_phys(truncate(fine.phys_to_spec(fphys[a] * fphys[b]), coarse))
        tau.append(pq - coarse_project(fc[a] * fc[b], coarse))
    return fc, np.stack(tau)
