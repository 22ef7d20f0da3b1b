"""Python mirror of the ensemble C-ABI (coral_ensemble_* in include/coral_b200.h):
many independent plane-layer runs advanced together, one CUDA graph per step,
the band substitutions of all members in one persistent launch per stage."""
import ctypes

from . import _lib
from .solver import CoralError, PlaneLayer


class Ensemble:
    def __init__(self, equations_texts, parameters_texts, scheme=None, device=0):
        if len(equations_texts) != len(parameters_texts) or not equations_texts:
            raise ValueError("one equations text and one parameters text per member")
        self._lib = _lib.load()
        n = len(equations_texts)
        eqs = (ctypes.c_char_p * n)(*[t.encode() for t in equations_texts])
        pars = (ctypes.c_char_p * n)(*[t.encode() for t in parameters_texts])
        e = ctypes.c_void_p()
        rc = self._lib.coral_ensemble_create(n, eqs, pars, scheme.encode() if scheme else None, int(device),
                                             ctypes.byref(e))
        if rc != 0:
            raise CoralError(rc, self._lib.coral_ensemble_last_error(None).decode())
        self._e = e
        self.members = []
        for i in range(n):
            h = ctypes.c_void_p()
            self._check(self._lib.coral_ensemble_member(self._e, i, ctypes.byref(h)))
            self.members.append(PlaneLayer._wrap(h, self))

    def _check(self, rc):
        if rc != 0:
            raise CoralError(rc, self._lib.coral_ensemble_last_error(self._e).decode())

    def query(self, what):
        v = ctypes.c_longlong()
        self._check(self._lib.coral_ensemble_query(self._e, int(what), ctypes.byref(v)))
        return v.value

    @property
    def batched(self):
        return bool(self.query(2))

    def march_forward(self, dt, nsteps=1):
        self._check(self._lib.coral_ensemble_march(self._e, float(dt), int(nsteps)))

    def synchronize(self):
        self._check(self._lib.coral_ensemble_synchronize(self._e))

    def close(self):
        if getattr(self, "_e", None):
            for m in self.members:
                m._h = None
            self._lib.coral_ensemble_destroy(self._e)
            self._e = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# The seeded 64-member ensemble: grids uniform in {32^2 x 32, 64^2 x 48,
# 96^2 x 64, 128^2 x 64}, log10 Ra ~ U[4, 6], Pr ~ U[0.7, 7] (PCG64 seed 3, drawn
# per member in the order grid, Ra, Pr), no-slip Rayleigh-Benard, Lx = Ly = 2 pi,
# ARS_222, dt = 1e-4; member i starts from the white-noise temperature initial
# condition with seed 1000 + i.
ENSEMBLE_GRIDS = ((32, 32, 32), (64, 64, 48), (96, 96, 64), (128, 128, 64))


def seeded_members(n=64, seed=3, dt=1e-4):
    """[(equations text, parameters text, (NX, NY, NZ), Ra, Pr)] of the seeded ensemble."""
    import math
    import os

    import numpy as np

    from . import CONFIG_DIR
    with open(os.path.join(CONFIG_DIR, "rbc_noslip_ra1e5.equations")) as f:
        eq0 = f.read()
    with open(os.path.join(CONFIG_DIR, "rbc_noslip_ra1e5_64x64x48.parameters.in")) as f:
        par0 = f.read().splitlines(True)
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for _ in range(n):
        g = ENSEMBLE_GRIDS[int(rng.integers(0, len(ENSEMBLE_GRIDS)))]
        ra = 10.0 ** rng.uniform(4.0, 6.0)
        pr = rng.uniform(0.7, 7.0)
        eq = eq0.replace(">>Param :: Prandtl := 1.d0 <<", ">>Param :: Prandtl := %r <<" % pr)
        eq = eq.replace(">>Param :: Rayleigh := 1.d5 <<", ">>Param :: Rayleigh := %r <<" % ra)
        par = list(par0)
        par[1], par[2], par[3] = "%d\n" % g[0], "%d\n" % g[1], "%d\n" % g[2]
        par[5] = par[6] = "%r\n" % (2 * math.pi)
        par[10] = "%r\n" % dt
        out.append((eq, "".join(par), g, ra, pr))
    return out


def seeded_ensemble(n=64, seed=3, dt=1e-4, device=0, workdir=None):
    """The seeded ensemble with every member's initial condition imported."""
    import tempfile

    from . import initial_conditions as ic
    spec = seeded_members(n, seed, dt)
    ens = Ensemble([s[0] for s in spec], [s[1] for s in spec], device=device)
    with tempfile.TemporaryDirectory(dir=workdir) as d:
        for i, (_, _, g, _, _) in enumerate(spec):
            ic.white_noise_temperature(d, g[0], g[1], g[2], seed=1000 + i)
            ens.members[i].import_quicksave(d)
    return ens, spec
