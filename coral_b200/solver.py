"""Python mirror of the reference's plane-layer data structure
(full_problem_data_structure_T, src/plane_layer/PL_IMEX_timestepping.f90:143-219)
on top of the C-ABI.  Same procedure names and argument meaning:

    init                  -> PlaneLayer(...)            (PL_IMEX_timestepping.f90:510)
    factorize_operators   -> factorize_operators(dt)    (:351-422)
    march_forward         -> march_forward(dt)          (PL_IMEX_timestepping_marching.f90:3)
    import_quickSave      -> import_quicksave(dir)      (PL_IMEX_timestepping_output.f90:309)
    export_checkpoints    -> export_checkpoints(dir)    (PL_IMEX_timestepping_output.f90:385)
    PS_fields_T%spec_to_phys / phys_to_spec             (slabs.fftw3mpi/transforms.f90:155-301)

Errors raise CoralError (the reference prints and stops).
Arrays use C order with the reference's Fortran shapes reversed:
    field (NX/2, NYAA, T) complex128, spec (NX/2, NYAA, NZ) complex128,
    phys (NYAA, NXAA, NZAA) float64.
"""
import ctypes
import os

import numpy as np

from . import _lib


class CoralError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (_lib.ERRORS.get(code, "?"), code, msg))
        self.code = code


Q = dict(NX=0, NY=1, NZ=2, NXAA=3, NYAA=4, NZAA=5, N_KXKY=6, N_ZERO=7, N_FULL=8, N_QUAD=9, STAGES=10,
         DEVICE_BYTES=11, LAUNCHES=12)


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class PlaneLayer:
    def __init__(self, equations_text, parameters_text, scheme=None, device=0, args=None):
        """args: the reference's command-line switches, e.g.
        "--withHorizontalSmagorinsky --smagorinsky-prefactor 0.1" (coral_create_with_args)."""
        self._lib = _lib.load()
        h = ctypes.c_void_p()
        rc = self._lib.coral_create_with_args(equations_text.encode(), parameters_text.encode(),
                                              scheme.encode() if scheme else None, int(device),
                                              args.encode() if args else None, ctypes.byref(h))
        if rc != 0:
            raise CoralError(rc, self._lib.coral_last_error(None).decode())
        self._h = h
        self._owner = None
        self._init_sizes()

    def _init_sizes(self):
        q = self.query
        self.NX, self.NY, self.NZ = q(Q["NX"]), q(Q["NY"]), q(Q["NZ"])
        self.NXAA, self.NYAA, self.NZAA = q(Q["NXAA"]), q(Q["NYAA"]), q(Q["NZAA"])
        self.NXH = self.NX // 2
        self.n_kxky = q(Q["N_KXKY"])
        self.n_zero = q(Q["N_ZERO"])
        self.n_full = q(Q["N_FULL"])
        self.n_quad = q(Q["N_QUAD"])
        self.stages = q(Q["STAGES"])
        self.T = [q(100 + i) for i in range(self.n_kxky)]
        self.Tz = [q(200 + i) for i in range(self.n_zero)]

    @classmethod
    def _wrap(cls, handle, owner):
        """A view of a handle owned by someone else (an ensemble member): same
        procedures, but close() leaves the handle alone."""
        self = cls.__new__(cls)
        self._lib = _lib.load()
        self._h = handle
        self._owner = owner
        self._init_sizes()
        return self

    @classmethod
    def from_files(cls, equations_path, parameters_path, scheme=None, device=0, args=None):
        with open(equations_path) as f:
            e = f.read()
        with open(parameters_path) as f:
            p = f.read()
        return cls(e, p, scheme, device, args)

    # --- plumbing
    def _check(self, rc):
        if rc != 0:
            raise CoralError(rc, self._lib.coral_last_error(self._h).decode())

    def query(self, what):
        v = ctypes.c_longlong()
        self._check(self._lib.coral_query(self._h, int(what), ctypes.byref(v)))
        return v.value

    def close(self):
        if getattr(self, "_h", None):
            if getattr(self, "_owner", None) is None:
                self._lib.coral_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def device_bytes(self):
        return self.query(Q["DEVICE_BYTES"])

    @property
    def kernel_launches(self):
        return self.query(Q["LAUNCHES"])

    # --- reference procedures
    def factorize_operators(self, dt):
        self._check(self._lib.coral_factorize(self._h, float(dt)))

    def march_forward(self, dt, nsteps=1):
        self._check(self._lib.coral_march(self._h, float(dt), int(nsteps)))

    def synchronize(self):
        self._check(self._lib.coral_synchronize(self._h))

    def get_field(self, isys=0, out=None):
        """State of kxky system isys, (NX/2, NYAA, T) complex.  out: an existing
        C-contiguous complex128 array of that shape to copy into (page-locked
        memory makes the copy a DMA at full link speed)."""
        shape = (self.NXH, self.NYAA, self.T[isys])
        if out is None:
            out = np.empty(shape, dtype=np.complex128)
        elif out.shape != shape or out.dtype != np.complex128 or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous complex128 array of shape %s" % (shape,))
        self._check(self._lib.coral_get_field(self._h, isys, _dptr(out)))
        return out

    def set_field(self, isys, field):
        a = np.ascontiguousarray(field, dtype=np.complex128)
        if a.shape != (self.NXH, self.NYAA, self.T[isys]):
            raise ValueError("field shape %s != %s" % (a.shape, (self.NXH, self.NYAA, self.T[isys])))
        self._check(self._lib.coral_set_field(self._h, isys, _dptr(a)))

    def get_mean_field(self, isys=0):
        a = np.empty(self.Tz[isys], dtype=np.float64)
        self._check(self._lib.coral_get_mean_field(self._h, isys, _dptr(a)))
        return a

    def set_mean_field(self, isys, field):
        a = np.ascontiguousarray(field, dtype=np.float64)
        if a.shape != (self.Tz[isys],):
            raise ValueError("mean field shape")
        self._check(self._lib.coral_set_mean_field(self._h, isys, _dptr(a)))

    def spec_to_phys(self, spec):
        s = np.ascontiguousarray(spec, dtype=np.complex128)
        if s.shape != (self.NXH, self.NYAA, self.NZ):
            raise ValueError("spec shape")
        p = np.empty((self.NYAA, self.NXAA, self.NZAA))
        self._check(self._lib.coral_spec_to_phys(self._h, _dptr(s), _dptr(p)))
        return p

    def phys_to_spec(self, phys):
        p = np.ascontiguousarray(phys, dtype=np.float64)
        if p.shape != (self.NYAA, self.NXAA, self.NZAA):
            raise ValueError("phys shape")
        s = np.empty((self.NXH, self.NYAA, self.NZ), dtype=np.complex128)
        self._check(self._lib.coral_phys_to_spec(self._h, _dptr(p), _dptr(s)))
        return s

    def full_phys(self, ivar):
        p = np.empty((self.NYAA, self.NXAA, self.NZAA))
        self._check(self._lib.coral_get_full_phys(self._h, int(ivar), _dptr(p)))
        return p

    def import_quicksave(self, directory, rolling=1):
        self._check(self._lib.coral_import_quicksave(self._h, os.fsencode(directory), int(rolling)))

    def export_checkpoints(self, directory, rolling=1):
        self._check(self._lib.coral_export_checkpoint(self._h, os.fsencode(directory), int(rolling)))

    def set_var_phys(self, isys, ivar, phys):
        p = np.ascontiguousarray(phys, dtype=np.float64)
        if p.shape != (self.NYAA, self.NXAA, self.NZAA):
            raise ValueError("phys shape")
        self._check(self._lib.coral_set_var_phys(self._h, int(isys), int(ivar), _dptr(p)))

    def set_mean_var_profile(self, isys, ivar, prof):
        p = np.ascontiguousarray(prof, dtype=np.float64)
        if p.shape != (self.NZAA,):
            raise ValueError("profile shape")
        self._check(self._lib.coral_set_mean_var_profile(self._h, int(isys), int(ivar), _dptr(p)))

    @property
    def stream(self):
        """The cudaStream_t of the handle, as an integer."""
        v = ctypes.c_void_p()
        self._check(self._lib.coral_stream(self._h, ctypes.byref(v)))
        return v.value or 0

    PHASES = ("inv_y", "inv_x", "inv_z", "z_products", "fwd_x", "fwd_y", "nl_assembly", "rhs_nl", "mean_systems",
              "substitution", "kstd_out")

    def profile_step(self, dt):
        """One eager step with CUDA events per kernel class; returns {phase: ms}."""
        ms = np.zeros(len(self.PHASES))
        self._check(self._lib.coral_profile_step(self._h, float(dt), _dptr(ms), len(ms)))
        return dict(zip(self.PHASES, ms.tolist()))

    # --- timeseries and the time loop (plane_layer_main.f90:138-205)
    def set_timeseries(self, text):
        """coral.timeseries text (master_recipe%add_timeseries)."""
        self._check(self._lib.coral_set_timeseries(self._h, text.encode()))
        self.n_timeseries = text.count(">>Volume_average") + text.count(">>Horizontal_avg")

    def set_usr_output(self, text):
        """coral.usrOutput text (master_recipe%add_outputs): volumes, slices,
        vertically summed slices and profiles that run() writes at their periods."""
        self._check(self._lib.coral_set_usr_output(self._h, text.encode()))

    def export_usr_output(self, directory, time_integer):
        """Write every user-output object now from the current state."""
        self._check(self._lib.coral_export_usr_output(self._h, str(directory).encode(), int(time_integer)))

    def timeseries(self):
        """Values of the timeseries objects at the last step's first stage."""
        out = np.zeros(16)
        self._check(self._lib.coral_timeseries(self._h, _dptr(out), 16))
        return out

    def set_time(self, time, dt, i_timestep=1):
        self._check(self._lib.coral_set_time(self._h, float(time), float(dt), int(i_timestep)))

    def get_time(self):
        out = np.zeros(4)
        self._check(self._lib.coral_get_time(self._h, _dptr(out)))
        return dict(time=float(out[0]), dt=float(out[1]), i_timestep=int(out[2]), refactorizations=int(out[3]))

    def run(self, nsteps, output_directory=None):
        """nsteps of the driver loop with CFL-adaptive dt; timeseries files under
        output_directory/Timeseries when given."""
        d = os.fsencode(output_directory) if output_directory else None
        self._check(self._lib.coral_run(self._h, int(nsteps), d))

    def var_positions(self, isys, ivar):
        """Positions within T of the Galerkin coefficients of coupled variable
        ivar of kxky system isys (the interleaved layout)."""
        n = ctypes.c_int()
        self._check(self._lib.coral_var_positions(self._h, int(isys), int(ivar), None, 0, ctypes.byref(n)))
        buf = (ctypes.c_int * max(n.value, 1))()
        self._check(self._lib.coral_var_positions(self._h, int(isys), int(ivar), buf, n.value, ctypes.byref(n)))
        return np.frombuffer(buf, dtype=np.int32)[:n.value].copy()

    def autotune(self, dt, repeats=2):
        """Time the kernel variants of the step and keep the fastest; returns the report."""
        buf = ctypes.create_string_buffer(2048)
        self._check(self._lib.coral_autotune(self._h, float(dt), int(repeats), buf, 2048))
        return buf.value.decode()

    def set_variant(self, knob, value):
        """Pin one kernel variant of the autotuner (0 default, 1 alternative)."""
        self._check(self._lib.coral_set_variant(self._h, knob.encode(), int(value)))

    def set_hermitian_kx0(self, on=True):
        """Project the kx = 0 line onto its Hermitian part after every step
        (removes the invisible anti-Hermitian part; off by default)."""
        self._check(self._lib.coral_set_hermitian_kx0(self._h, 1 if on else 0))

    def set_source(self, index, profile):
        """sourceNN's physical values on the Gauss-Chebyshev grid (NZAA)."""
        a = np.ascontiguousarray(profile, dtype=np.float64)
        if a.shape != (self.NZAA,):
            raise ValueError("profile must have NZAA values")
        self._check(self._lib.coral_set_source(self._h, int(index), _dptr(a)))

    def set_penalisation_mask(self, mask):
        """the penalisation mask on the grid, (NYAA, NXAA, NZAA)."""
        a = np.ascontiguousarray(mask, dtype=np.float64)
        if a.shape != (self.NYAA, self.NXAA, self.NZAA):
            raise ValueError("mask must be (NYAA, NXAA, NZAA)")
        self._check(self._lib.coral_set_penalisation_mask(self._h, _dptr(a)))

    def set_z_transform(self, form):
        """0: FP64 FFT z transforms; 1: int8-digit tensor-core contractions."""
        self._check(self._lib.coral_set_z_transform(self._h, int(form)))

    def diagnostics(self):
        out = np.zeros(3)
        self._check(self._lib.coral_diagnostics(self._h, _dptr(out)))
        return dict(cfl_dt=float(out[0]), KE=float(out[1]), nonfinite=bool(out[2]))
