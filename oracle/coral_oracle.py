"""CPU restatement of Coral's plane-layer IMEX timestep (the oracle).

TEST INFRASTRUCTURE ONLY.  This module is the checker against which the CUDA
path is compared.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import it.  The
product (``coral_b200``) never imports, calls or links anything in ``oracle/``.

What it restates (file:line citations are into the Coral v1.3 sources):

* parameter file reader ............ src/plane_layer/PL_geometry.f90:269-305
* equation-file grammar ............ src/plane_layer/PL_equations.f90:435-593,
                                     1089-1754, 1758-2043 and
                                     src/plane_layer/PL_string_to_data.f90:53-118,387-465
* wavenumbers / dealias masks ...... src/plane_layer/PL_geometry.f90:80-236
* Chebyshev I (integration) and M (multiplication by z) matrices
                                     src/cheby_tools/chebyshev_elementary.f90:28-151
* Galerkin boundary stencils ....... src/cheby_tools/chebyshev_galerkin_2.f90:7-409
* system shapes, shuffles, blocks .. src/plane_layer/PL_IMEX_timestepping.f90:664-1635
* evolution operator + band LU ..... src/plane_layer/PL_IMEX_timestepping.f90:351-422,
                                     src/plane_layer/PL_algebra_z_3D.f90:218-276,
                                     src/sparse_tools/sparse_formats_z.f90:812-847
* ARS IMEX tableaux ................ src/timesteppers/IMEX_schemes.f90:21-402
* transforms (slab build, 1 rank) .. src/slabs.fftw3mpi/transforms.f90:155-301,583-625
* one timestep ..................... src/plane_layer/PL_IMEX_timestepping_marching.f90:3-588
* QuickSave import / export ........ src/plane_layer/PL_IMEX_timestepping_output.f90:309-456
* Gauss-Chebyshev grid and weights . src/plane_layer/PL_cheby_misc.f90:8-55
* sources, penalisation, Smagorinsky, surface values, vertical decompositions
                                     src/plane_layer/PL_IMEX_timestepping_marching.f90:
                                     398-415,505-575,711-866,
                                     PL_IMEX_timestepping.f90:238-274 and the shipped
                                     PL_user_sources_definitions.f90 /
                                     PL_user_penalisation_mask.f90

Third-party arithmetic the reference delegates to libraries is restated with
the same published algorithms: FFTW's unnormalised c2c / c2r / r2c and
REDFT01 / REDFT10 (scipy.fft's pocketfft computes the same transforms; the
DCT-II/III conventions of scipy.fft with norm=None equal FFTW's REDFT10/REDFT01),
and LAPACK's ZGBTRF / ZGBTRS / DGBTRF / DGBTRS band LU with partial pivoting
(scipy.linalg.lapack calls the reference LAPACK routines of the same name).
"""
from __future__ import annotations

import dataclasses
import math
import os
import re
from typing import Dict, List, Optional, Tuple

import numpy as np
import scipy.fft as sfft
import scipy.linalg.lapack as lapack
import scipy.sparse as sp

# --------------------------------------------------------------------------------------
# parameter file  (src/plane_layer/PL_geometry.f90:269-305)
# --------------------------------------------------------------------------------------


def _fortran_float(tok: str) -> float:
    return float(tok.strip().replace("d", "e").replace("D", "e"))


def read_parameters_text(text: str) -> dict:
    """Reads coral.parameters.in: 17 fixed lines, first token of each is the value."""
    lines = [l for l in text.splitlines()]
    tok = [l.split()[0] if l.split() else "" for l in lines]
    p = dict(
        NX=int(tok[1]), NY=int(tok[2]), NZ=int(tok[3]),
        Lx=_fortran_float(tok[5]), Ly=_fortran_float(tok[6]),
        gap=_fortran_float(tok[7]), center=_fortran_float(tok[8]),
        dt_max=_fortran_float(tok[10]), tolerance=_fortran_float(tok[11]),
        CFL_C=_fortran_float(tok[12]),
        scheme=tok[13].strip("'\""),
        qsave_restart=tok[15].lower().strip(".") in ("true", "t"),
        time_limit=_fortran_float(tok[17]),
    )
    return p


# --------------------------------------------------------------------------------------
# equation file  (src/plane_layer/PL_equations.f90, PL_string_to_data.f90)
# --------------------------------------------------------------------------------------


@dataclasses.dataclass
class Piece:
    """One linear operator piece: dsca * dx^kx * dy^ky * Iz^Iz * mz^mz applied to var jVar
    in equation iEqn (linear_operator_recipe_T, PL_equations.f90:57-66)."""
    dsca: float
    kx: int
    ky: int
    Iz: int
    mz: int
    jVar: int
    iEqn: int


@dataclasses.dataclass
class NLTerm:
    """atom_NL_term_T (PL_equations.f90:22-30)."""
    dsca: float
    dx: int
    dy: int
    Iz: int
    mz: int
    quad: int
    eqn: int


@dataclasses.dataclass
class FullTerm:
    """a_linear_contribution_T (PL_equations.f90:69-77)."""
    kind: str  # 'kxky' | 'zero'
    var: int
    dsca: float
    dx: int
    dy: int
    dz: int
    mz: int


@dataclasses.dataclass
class SourceTerm:
    """source_term_T (PL_equations.f90:37-45): dsca * Iz^Iz * sourceNN in equation
    eqn of mean system sys."""
    dsca: float
    Iz: int
    index: int
    sys: int
    eqn: int


@dataclasses.dataclass
class CoupledSystem:
    vars: List[str]
    bcs: List[int]
    orders: List[int]
    mass: List[Piece]
    stif: List[Piece]
    nl: List[NLTerm]


@dataclasses.dataclass
class Recipe:
    params: List[Tuple[str, float]]
    kxky_vars: List[str]
    zero_vars: List[str]
    full_vars: List[Tuple[str, str, List[FullTerm]]]  # (name, extract_at, terms)
    quad_vars: List[Tuple[str, int, int, bool]]      # (name, ivar1, ivar2, remove_mean)
    kxky: List[CoupledSystem]
    zero: List[CoupledSystem]
    kxky_loc: Dict[str, Tuple[int, int]]
    zero_loc: Dict[str, Tuple[int, int]]
    # per full variable: extract ('nowhere' | 'BotSurf' | 'TopSurf'), decomp (None |
    # 'barotropic' | 'baroclinic'), penal (None | [strength, width]), smago (bool)
    full_opts: List[dict] = dataclasses.field(default_factory=list)
    source_params: List[Tuple[str, float]] = dataclasses.field(default_factory=list)
    sources: List[SourceTerm] = dataclasses.field(default_factory=list)
    smagorinsky: bool = False


def _clean(s: str) -> str:
    return s.replace(" ", "").replace("\0", "")


def _break_pieces(line: str) -> List[Tuple[float, str]]:
    """break_linear_operators_in_pieces (PL_string_to_data.f90:387-439): every '+'
    piece of the line in order, then every '-' piece in order."""
    out = []
    for sign_char, sgn in (("+", 1.0), ("-", -1.0)):
        aux = line
        while sign_char in aux:
            aux = aux[aux.index(sign_char) + 1:]
            ends = [aux.index(c) for c in "+-<" if c in aux]
            end = min(ends) if ends else len(aux)
            out.append((sgn, aux[:end].rstrip()))
    return out


def _atoms(line: str, dz_str: str):
    """interpret_full_variable_definition (PL_string_to_data.f90:53-118)."""
    res = []
    for sgn, s in _break_pieces(line):
        a = dict(sgn=sgn, dsca=sgn, dx=0, dy=0, Iz=0, mz=0, unsorted=[])
        for chunk in s.split("."):
            c = _clean(chunk)
            if c == "dx":
                a["dx"] += 1
            elif c == "dy":
                a["dy"] += 1
            elif c == dz_str:
                a["Iz"] += 1
            elif c == "mz":
                a["mz"] += 1
            else:
                a["unsorted"].append(c)
        res.append(a)
    return res


def _payload(line: str) -> str:
    i = line.index("::") + 2
    j = line.index("<<")
    return line[i:j]


def parse_equations(text: str, smagorinsky: bool = False) -> Recipe:
    """build_full_recipe_from_text_file (PL_equations.f90:435-593).  smagorinsky:
    the --withHorizontalSmagorinsky switch, which adds the full variable nuSmago
    before the first quadratic variable (:519-526)."""
    params: List[Tuple[str, float]] = []
    source_params: List[Tuple[str, float]] = []
    sources: List[SourceTerm] = []
    full_opts: List[dict] = []
    smago_pending = smagorinsky

    def new_full(name, extract="nowhere", penal=None, smago=False):
        full_vars.append((name, extract, []))
        full_opts.append(dict(extract=extract, decomp=None, penal=penal, smago=smago))
    kxky_vars: List[str] = []
    zero_vars: List[str] = []
    full_vars: List[Tuple[str, str, List[FullTerm]]] = []
    quad_vars: List[Tuple[str, int, int, bool]] = []
    kxky: List[CoupledSystem] = []
    zero: List[CoupledSystem] = []
    kxky_loc: Dict[str, Tuple[int, int]] = {}
    zero_loc: Dict[str, Tuple[int, int]] = {}

    current = "kxky"   # which kind of coupled set the lines below the last header belong to

    def param_value(name):
        for n, v in params:
            if n == name:
                return v
        return None

    for raw in text.splitlines():
        line = raw
        if line.startswith(">>="):
            continue
        if not line.startswith(">>"):
            continue
        key = line[2:]
        if key.startswith("EOF"):
            break
        if key.startswith("Param"):
            body = line[line.index("::") + 2: line.index("<<")]
            name, val = body.split(":=")
            params.append((_clean(name), _fortran_float(val)))
        elif key.startswith("sourceParam"):   # add_source_parameter (:985-996)
            body = line[line.index("::") + 2: line.index("<<")]
            name, val = body.split(":=")
            source_params.append((_clean(name), _fortran_float(val)))
        elif key.startswith("linear_variable_kxky"):
            kxky_vars.append(_clean(_payload(line)))
        elif key.startswith("linear_variable_mean"):
            zero_vars.append(_clean(_payload(line)))
        elif key.startswith("linear_variable_full_build"):
            name, ext, terms = full_vars[-1]
            for a in _atoms(line, "dz"):
                t = FullTerm(kind="null", var=-1, dsca=a["dsca"], dx=a["dx"], dy=a["dy"],
                             dz=a["Iz"], mz=a["mz"])
                for s in a["unsorted"]:
                    if s in zero_vars:
                        t.kind, t.var = "zero", zero_vars.index(s)
                    elif s in kxky_vars:
                        t.kind, t.var = "kxky", kxky_vars.index(s)
                    else:
                        v = param_value(s)
                        if v is None:
                            raise ValueError("unknown string in equations: " + s)
                        t.dsca = t.dsca * v
                if t.kind == "null":
                    raise ValueError("invalid full variable def.")
                terms.append(t)
        elif key.startswith("linear_variable_full"):
            new_full(_clean(_payload(line)))
        elif key.startswith("linear_variable_bottom_boundary_value"):
            new_full(_clean(_payload(line)), "BotSurf")
        elif key.startswith("linear_variable_top_boundary_value"):
            new_full(_clean(_payload(line)), "TopSurf")
        elif key.startswith("vertical_decomposition"):  # filter_linear_variable_full (:1052-1067)
            kind = _payload(line).strip()
            if kind not in ("baroclinic", "barotropic"):
                raise ValueError("vertical_decomposition should be baroclinic or barotropic")
            full_opts[-1]["decomp"] = kind
        elif key.startswith("enable_penalisation"):     # :508-511, 1035-1050
            new_full(_clean(_payload(line)), penal=[0.0, 0.0])
        elif key.startswith("penalisation_strength"):
            full_opts[-1]["penal"][0] = _fortran_float(_payload(line))
        elif key.startswith("penalisation_width"):
            full_opts[-1]["penal"][1] = _fortran_float(_payload(line))
        elif key.startswith("quadratic_variable") or key.startswith("zFiltered_quadratic_variable"):
            if smago_pending:
                new_full("nuSmago", smago=True)
            smago_pending = False
            body = line[line.index("::") + 2: line.index("<<")]
            qname, rhs = body.split(":=")
            v1, v2 = [_clean(x) for x in rhs.split(".", 1)]
            names = [f[0] for f in full_vars]

            def idx(v):
                if v == "ONE":
                    return -1
                if v not in names:
                    raise ValueError("bad NL var definition (wrong reference to linear var.)")
                return names.index(v)
            quad_vars.append((_clean(qname), idx(v1), idx(v2), key.startswith("zFiltered")))
        elif key.startswith("add_set_of_coupled_kxky_equations"):
            kxky.append(CoupledSystem([], [], [], [], [], []))
            current = "kxky"
        elif key.startswith("add_set_of_coupled_zero_equations"):
            zero.append(CoupledSystem([], [], [], [], [], []))
            current = "zero"
        elif key.startswith("linearly_coupled_var"):
            name = _clean(_payload(line))
            loc, sysl = (zero_loc, zero) if current == "zero" else (kxky_loc, kxky)
            sysl[-1].vars.append(name)
            sysl[-1].bcs.append(0)
            loc[name] = (len(sysl) - 1, len(sysl[-1].vars) - 1)
        elif key.startswith("add_BC_for_this_var"):
            sysl = zero if current == "zero" else kxky
            sysl[-1].bcs[-1] = int(_payload(line).strip())
        elif key.startswith("new_equation"):
            sysl = zero if current == "zero" else kxky
            sysl[-1].orders.append(int(_payload(line).strip()))
        elif key.startswith("add_d/dt_term") or key.startswith("add_rhs_linear"):
            sysl = zero if current == "zero" else kxky
            s = sysl[-1]
            dest = s.mass if key.startswith("add_d/dt_term") else s.stif
            for a in _atoms(line, "Iz"):
                dsca = a["dsca"]
                jvar = -1
                for st in a["unsorted"]:
                    if st in s.vars:
                        jvar = s.vars.index(st)
                    else:
                        v = param_value(st)
                        if v is None:
                            raise ValueError("unknown string in equations: " + st)
                        dsca = v * dsca
                if jvar < 0:
                    raise ValueError("invalid stif/mass matrix definition")
                dest.append(Piece(dsca, a["dx"], a["dy"], a["Iz"], a["mz"], jvar, len(s.orders) - 1))
        elif key.startswith("add_rhs_NL"):
            sysl = zero if current == "zero" else kxky
            s = sysl[-1]
            qnames = [q[0] for q in quad_vars]
            for a in _atoms(line, "Iz"):
                dsca = a["dsca"]
                q = -1
                for st in a["unsorted"]:
                    if st in qnames:
                        q = qnames.index(st)
                    else:
                        v = param_value(st)
                        if v is None:
                            raise ValueError("unknown string in equations: " + st)
                        dsca = v * dsca
                if q < 0:
                    raise ValueError("invalid quad_var_index")
                s.nl.append(NLTerm(dsca, a["dx"], a["dy"], a["Iz"], a["mz"], q, len(s.orders) - 1))
        elif key.startswith("add_rhs_source"):
            # build_zero_sources_in_full_recipe (PL_equations.f90:1156-1230): mean systems only
            if current != "zero":
                raise ValueError("add_rhs_source outside a set of mean equations")
            for a in _atoms(line, "Iz"):
                if a["dx"] or a["dy"]:
                    raise ValueError("x/y-derivative in a source term")
                t = SourceTerm(a["dsca"], a["Iz"], 0, len(zero) - 1, len(zero[-1].orders) - 1)
                for st in a["unsorted"]:
                    if len(st) == 8 and st.startswith("source"):
                        if not st[6:].isdigit():
                            raise ValueError("Source terms must be of the form sourceNN")
                        t.index = int(st[6:])
                        break
                    v = param_value(st)
                    if v is None:
                        raise ValueError("unknown string in equations: " + st)
                    t.dsca = v * t.dsca
                if t.index == 0:
                    raise ValueError("invalid source_index")
                sources.append(t)
        else:
            raise ValueError("the line could not be read: " + line[:78])
    return Recipe(params, kxky_vars, zero_vars, full_vars, quad_vars, kxky, zero, kxky_loc, zero_loc,
                  full_opts, source_params, sources, smagorinsky)


# --------------------------------------------------------------------------------------
# geometry (PL_geometry.f90:80-236) and Gauss-Chebyshev grid (PL_cheby_misc.f90:8-55)
# --------------------------------------------------------------------------------------


@dataclasses.dataclass
class Geometry:
    NX: int
    NY: int
    NZ: int
    Lx: float
    Ly: float
    gap: float
    center: float

    def __post_init__(self):
        self.NXAA = 3 * self.NX // 2
        self.NYAA = 3 * self.NY // 2
        self.NZAA = 3 * self.NZ // 2
        self.NXH = self.NX // 2
        pi = 4.0 * math.atan(1.0)
        self.ky_box = 2.0 * pi / self.Ly
        self.kx_box = 2.0 * pi / self.Lx
        ky = np.empty(self.NYAA)
        for iy in range(self.NYAA):
            k_index = iy + 1
            if k_index >= self.NYAA // 2 + 1:
                ky[iy] = -float((self.NYAA + 1 - k_index) * self.ky_box)
            else:
                ky[iy] = float((k_index - 1) * self.ky_box)
        kx = np.array([ix * self.kx_box for ix in range(self.NXH)], dtype=np.float64)
        self.ky = ky
        self.kx = kx
        self.deal_y = np.abs(ky) >= self.ky_box * self.NY / 2.0
        self.deal_x = np.abs(kx) >= self.kx_box * self.NX / 2.0
        self.px = 1j * kx
        self.py = 1j * ky

    @property
    def active(self) -> np.ndarray:
        """(NXH, NYAA) mask of systems that are neither dealiased nor the (0,0) mode."""
        m = ~(self.deal_x[:, None] | self.deal_y[None, :])
        m[0, 0] = False
        return m

    def zgrid(self) -> np.ndarray:
        pi = 4.0 * math.atan(1.0)
        i = np.arange(1, self.NZAA + 1)
        return self.center + np.cos(pi * (2 * i - 1) / (2 * self.NZAA)) * 0.5 * self.gap

    def zweights(self) -> np.ndarray:
        pi = 4.0 * math.atan(1.0)
        i = np.arange(1, self.NZAA + 1)
        g = np.cos(pi * (2 * i - 1) / (2 * self.NZAA))
        mid = np.empty(self.NZAA + 1)
        mid[0] = 1.0
        mid[-1] = -1.0
        mid[1:-1] = 0.5 * (g[1:] + g[:-1])
        return (mid[:-1] - mid[1:]) / 2.0 * self.gap


def complex_pow(z: complex, n: int) -> complex:
    """Fortran complex**integer by repeated multiplication."""
    r = complex(1.0, 0.0)
    for _ in range(n):
        r = r * z
    return r


# --------------------------------------------------------------------------------------
# ARS tableaux (src/timesteppers/IMEX_schemes.f90)
# --------------------------------------------------------------------------------------


def _f32(x: float) -> float:
    """A Fortran default-real literal: rounded to single precision, then widened."""
    return float(np.float32(x))


def ars_tableau(name: str):
    """Returns (imp_stages, A (imp x imp), A_hat (imp+1 x imp+1)) as float64 arrays."""
    if name == "ARS_111":
        A = np.array([[1.0]])
        Ah = np.zeros((2, 2)); Ah[1, 0] = 1.0
    elif name == "ARS_122":
        A = np.array([[0.5]])
        Ah = np.zeros((2, 2)); Ah[1, 0] = 0.5
    elif name == "ARS_233":
        g = (3.0 + math.sqrt(3.0)) / 6.0
        A = np.array([[g, 0.0], [1.0 - 2.0 * g, g]])
        Ah = np.zeros((3, 3)); Ah[1, 0] = g; Ah[2, 0] = g - 1.0; Ah[2, 1] = 2.0 * (1.0 - g)
    elif name == "ARS_232":
        d = -2.0 * math.sqrt(2.0) / 3.0
        g = 1.0 - 1.0 / math.sqrt(2.0)
        A = np.array([[g, 0.0], [1.0 - g, g]])
        Ah = np.zeros((3, 3)); Ah[1, 0] = g; Ah[2, 0] = d; Ah[2, 1] = 1.0 - d
    elif name == "ARS_222":
        g = 1.0 - 1.0 / math.sqrt(2.0)
        d = 1.0 - 1.0 / (2.0 * g)
        A = np.array([[g, 0.0], [1.0 - g, g]])
        Ah = np.zeros((3, 3)); Ah[1, 0] = g; Ah[2, 0] = d; Ah[2, 1] = 1.0 - d
    elif name == "ARS_343":
        g = _f32(0.43586652150845895)
        umg = _f32(0.28206673924577053)
        b1 = _f32(1.2084966491760099)
        b2 = _f32(-0.64436317068446880)
        a42 = 0.5529291479
        A = np.array([[g, 0, 0], [umg, g, 0], [b1, b2, g]], dtype=np.float64)
        Ah = np.zeros((4, 4))
        Ah[1, 0] = g
        Ah[2, 0] = (15.0 / 4.0 - 15.0 * g + 21.0 / 4.0 * g ** 2) * a42 - 7.0 / 2.0 + 13.0 * g - 4.5 * g ** 2
        Ah[2, 1] = -(15.0 / 4.0 - 15.0 * g + 21.0 / 4.0 * g ** 2) * a42 + 4.0 - 12.5 * g + 4.5 * g ** 2
        Ah[3, 0] = 1.0 - a42 - a42
        Ah[3, 1] = a42
        Ah[3, 2] = a42
    elif name == "ARS_443":
        A = np.array([[0.5, 0, 0, 0], [1 / 6.0, 0.5, 0, 0], [-0.5, 0.5, 0.5, 0], [1.5, -1.5, 0.5, 0.5]])
        Ah = np.zeros((5, 5))
        Ah[1, 0] = 0.5
        Ah[2, 0] = 11.0 / 18.0; Ah[2, 1] = 1.0 / 18.0
        Ah[3, 0] = 5.0 / 6.0; Ah[3, 1] = -5.0 / 6.0; Ah[3, 2] = 0.5
        Ah[4, 0] = 0.25; Ah[4, 1] = 7.0 / 4.0; Ah[4, 2] = 0.75; Ah[4, 3] = -7.0 / 4.0
    else:
        raise ValueError("Invalid time-stepping scheme code: " + name)
    return A.shape[0], np.asarray(A, dtype=np.float64), Ah


# --------------------------------------------------------------------------------------
# Chebyshev tools (chebyshev_elementary.f90:28-151, chebyshev_galerkin_2.f90:7-409)
# --------------------------------------------------------------------------------------


def cheb_elementary(N: int, center: float, gap: float, padding: int):
    """Dense (Npad x Npad) integration matrix I and multiplication-by-z matrix M."""
    Np = N + padding
    M = np.zeros((Np, Np))
    M[1, 0] = gap / 2.0
    for i in range(Np - 1):
        M[i, i + 1] = gap / 4.0
    for i in range(1, Np - 1):
        M[i + 1, i] = gap / 4.0
    for i in range(Np):
        M[i, i] = center
    I = np.zeros((Np, Np))
    I[1, 0] = 2.0
    for fi in range(2, Np):         # Fortran i = 2..Npad-1
        I[fi, fi - 1] = 1.0 / float(fi)          # row fi+1, col fi (1-based) -> [fi, fi-1]
    for fi in range(2, Np):         # super diagonal: row fi, col fi+1, -1/(fi-1)
        I[fi - 1, fi] = -1.0 / float(fi - 1)
    I *= gap / 4.0
    return I, M


def cheb_IM(N: int, center: float, gap: float, a: int, b: int, padding: int = 15) -> np.ndarray:
    """trunc(I^a M^b) to (N x N) (PL_IMEX_timestepping.f90:735-762, sparse_formats_d.f90:152-218)."""
    I, M = cheb_elementary(N, center, gap, padding)
    Np = I.shape[0]
    R = np.eye(Np)
    for _ in range(a):
        R = R @ I
    for _ in range(b):
        R = R @ M
    return R[:N, :N].copy()


def stencil(N: int, bc: int) -> np.ndarray:
    """Dense Galerkin stencil S (N x ncol): Chebyshev coefs = S @ Galerkin coefs."""
    if bc == 0:
        return np.eye(N)
    if bc in (10, 11, 12, 13):
        S = np.zeros((N, N - 1))
        for j in range(1, N):
            if bc == 10:
                d0, d1 = -1.0, 1.0
            elif bc == 11:
                d0, d1 = 1.0, 1.0
            elif bc == 12:
                d0, d1 = -(j + 1.0) ** 2, float(j) ** 2
            else:
                d0, d1 = (j + 1.0) ** 2, float(j) ** 2
            S[j - 1, j - 1] = d0
            S[j, j - 1] = d1
        return S
    if bc in (20, 21, 22, 23, 24):
        S = np.zeros((N, N - 2))
        if bc == 24:
            S[0, 0] = 1.0
            S[1, 1] = 1.0
            for j in range(3, N - 1):
                S[j + 1, j - 1] = 1.0
                n = float(j + 1)
                S[j - 1, j - 1] = -n ** 2 * (n ** 2 + 1.0) / ((n ** 2 - 3.0 * n + 2.0) * (n ** 2 - 5.0 * n + 6.0))
            return S
        for j in range(1, N - 1):
            if bc == 20:
                S[j - 1, j - 1] = -1.0
                S[j + 1, j - 1] = 1.0
            elif bc == 21:
                S[j - 1, j - 1] = -1.0
                n = float(j + 1)
                S[j + 1, j - 1] = (n - 2.0) ** 2 / n ** 2
            else:
                n = float(j - 1)
                sgn = -1.0 if bc == 22 else 1.0
                S[j - 1, j - 1] = 1.0
                S[j, j - 1] = sgn * (4.0 * n + 4.0) / (2.0 * n ** 2 + 6.0 * n + 5.0)
                S[j + 1, j - 1] = -(n ** 2 + (n + 1.0) ** 2) / ((n + 1.0) ** 2 + (n + 2.0) ** 2)
        return S
    if bc in (40, 41, 42, 43):
        S = np.zeros((N, N - 4))
        for j in range(1, N - 3):
            if bc == 40:
                n = float(j + 3)
                S[j - 1, j - 1] = -1.0
                S[j + 1, j - 1] = (2.0 * n - 4.0) / (n - 1.0)
                S[j + 3, j - 1] = -(n - 3.0) / (n - 1.0)
            elif bc == 41:
                n = float(j + 3)
                m = 24.0 * n / (2.0 * n ** 2 - 4.0 * n + 3.0)
                m = m - 18.0 / (n - 1.0)
                S[j - 1, j - 1] = -1.0
                S[j + 1, j - 1] = m + 2.0
                S[j + 3, j - 1] = -m - 1.0
            else:
                n = float(j - 1)
                s = -1.0 if bc == 42 else 1.0
                S[j - 1, j - 1] = 1.0
                S[j, j - 1] = s * (2.0 * n + 2.0) / (n ** 2 + 5.0 * n + 7.0)
                S[j + 1, j - 1] = -(2.0 * n ** 3 + 12.0 * n ** 2 + 28.0 * n + 24.0) / (n ** 3 + 8.0 * n ** 2 + 22.0 * n + 21.0)
                S[j + 2, j - 1] = -s * (2.0 * n + 2.0) / (n ** 2 + 5.0 * n + 7.0)
                S[j + 3, j - 1] = (n ** 3 + 4.0 * n ** 2 + 6.0 * n + 3.0) / (n ** 3 + 8.0 * n ** 2 + 22.0 * n + 21.0)
        return S
    raise ValueError("unknown boundary-condition code %d" % bc)


# --------------------------------------------------------------------------------------
# coupled-system layout (PL_IMEX_timestepping.f90:858-1033, 1086-1488)
# --------------------------------------------------------------------------------------


class SystemLayout:
    """Sizes and the polynomial-degree interleaving of one coupled system."""

    def __init__(self, NZ: int, sysrec: CoupledSystem):
        nV = len(sysrec.vars)
        if len(sysrec.orders) != nV:
            raise ValueError("Incompatible number of coupled equations and variables")
        self.nV = nV
        self.var_size = [NZ - bc // 10 for bc in sysrec.bcs]
        self.eq_size = [NZ - o for o in sysrec.orders]
        T1 = sum(self.eq_size)
        T2 = sum(self.var_size)
        if T1 != T2:
            raise ValueError("Incompatible number of boundary conditions")
        self.T = T1
        self.var_pos = self._interleave(self.var_size)
        self.eq_pos = self._interleave(self.eq_size)

    def _interleave(self, sizes):
        """pos[v][c] = position in the polynomial-degree ordering (0-based)."""
        nV = len(sizes)
        nmin = min(sizes)
        pos = []
        rem = 0
        for v in range(nV):
            p = []
            for c in range(sizes[v]):
                if c < nmin:
                    p.append(v + c * nV)
                else:
                    p.append(nmin * nV + rem + (c - nmin))
            rem += sizes[v] - nmin
            pos.append(np.array(p, dtype=np.int64))
        return pos


def build_piece_matrix(NZ, center, gap, lay: SystemLayout, sysrec: CoupledSystem, pc: Piece,
                       cache) -> sp.csr_matrix:
    """Real T x T matrix of one recipe piece in polynomial ordering (without dsca and
    Fourier factors): Q * insert(trunc(I^Iz M^mz)[order:,:] @ S_var) * P."""
    key = (pc.Iz, pc.mz)
    if key not in cache:
        cache[key] = cheb_IM(NZ, center, gap, pc.Iz, pc.mz)
    o = sysrec.orders[pc.iEqn]
    block = cache[key][o:, :] @ stencil(NZ, sysrec.bcs[pc.jVar])
    rows = lay.eq_pos[pc.iEqn]
    cols = lay.var_pos[pc.jVar]
    R, C = np.nonzero(block)
    return sp.csr_matrix((block[R, C], (rows[R], cols[C])), shape=(lay.T, lay.T))


# --------------------------------------------------------------------------------------
# transforms (slabs.fftw3mpi/transforms.f90:155-301, 583-625)
# --------------------------------------------------------------------------------------


def spec_to_phys(spec: np.ndarray, g: Geometry) -> np.ndarray:
    """c2r_transform.  spec[kx][ky][n] (NXH, NYAA, NZ) -> phys[y][x][z] (NYAA, NXAA, NZAA)."""
    b = sfft.ifft(spec, axis=1, norm="forward")          # FFTW_BACKWARD, unnormalised
    b[:, :, 0] *= 2.0
    X = np.zeros((g.NYAA, g.NXAA // 2 + 1, g.NZ), dtype=np.complex128)
    X[:, :g.NXH, :] = b.transpose(1, 0, 2) * 0.5
    r = sfft.irfft(X, n=g.NXAA, axis=1, norm="forward")  # c2r, unnormalised
    pad = np.zeros((g.NYAA, g.NXAA, g.NZAA))
    pad[:, :, :g.NZ] = r
    return sfft.dct(pad, type=3, axis=2)                 # REDFT01


def phys_to_spec(phys: np.ndarray, g: Geometry) -> np.ndarray:
    """r2c_transform.  phys[y][x][z] -> spec[kx][ky][n]."""
    a = sfft.dct(phys, type=2, axis=2)[:, :, :g.NZ]      # REDFT10, truncate
    c = sfft.rfft(a, axis=1)[:, :g.NXH, :]                # r2c, keep kx < NX/2
    c = np.ascontiguousarray(c.transpose(1, 0, 2))
    c[:, :, 0] *= 0.5
    s = sfft.fft(c, axis=1)
    return s * (1.0 / (g.NXAA * g.NYAA * g.NZAA))


def r2r_forward(arr: np.ndarray, NZAA: int) -> np.ndarray:
    """1-D mean-field Chebyshev transform (transforms.f90:605-625)."""
    s = sfft.dct(arr, type=2)
    s[0] *= 0.5
    return s / NZAA


def r2r_backward(arr: np.ndarray) -> np.ndarray:
    """transforms.f90:583-603."""
    s = arr.copy()
    s[0] *= 2.0
    return sfft.dct(s, type=3) / 2.0


# --------------------------------------------------------------------------------------
# sources, penalisation, surface values and vertical decompositions
# --------------------------------------------------------------------------------------


def z_filter(spec: np.ndarray, extract: str, decomp: Optional[str]) -> np.ndarray:
    """The z operations on a full variable's Chebyshev coefficients (last axis, NZ)
    before its inverse transform (marching.f90:543-575): the value at the bottom
    or top surface (T_n(-1) = (-1)^n, T_n(1) = 1) in coefficient 0, the rest
    zeroed; then the vertical mean removed (baroclinic,
    PL_IMEX_timestepping.f90:238-250) or the vertical fluctuations removed
    (barotropic, :252-274), sequentially as the reference loops."""
    spec = spec.copy()
    NZ = spec.shape[-1]
    if extract == "BotSurf":
        for iz in range(2, NZ + 1):
            spec[..., 0] = spec[..., 0] - spec[..., iz - 1] * (-1) ** iz
            spec[..., iz - 1] = 0.0
    elif extract == "TopSurf":
        for iz in range(2, NZ + 1):
            spec[..., 0] = spec[..., 0] + spec[..., iz - 1]
            spec[..., iz - 1] = 0.0
    if decomp == "baroclinic":
        spec[..., 0] = 0.0
        for q in range(1, NZ // 2):
            spec[..., 0] = spec[..., 0] - spec[..., 2 * q] * (0.5 / (2.0 * q + 1.0) - 0.5 / (2.0 * q - 1.0))
    elif decomp == "barotropic":
        for q in range(1, NZ // 2):
            spec[..., 0] = spec[..., 0] + spec[..., 2 * q] * (0.5 / (2.0 * q + 1.0) - 0.5 / (2.0 * q - 1.0))
            spec[..., 2 * q - 1] = 0.0
            spec[..., 2 * q] = 0.0
    return spec


def source_spectrum(phys: np.ndarray) -> np.ndarray:
    """Compute_1dCheby_transform (marching.f90:845-866): REDFT10 / N, coefficient 0
    halved."""
    c = sfft.dct(np.asarray(phys, dtype=np.float64), type=2) / len(phys)
    c[0] = c[0] * 0.5
    return c


def default_sources(r: Recipe, g: Geometry) -> Dict[int, np.ndarray]:
    """The two sources of the reference's default PL_user_sources_definitions.f90:
    source01 = HovEll exp(-z HovEll) / (1 - exp(-HovEll)) - 1 (HovEll a
    sourceParam; 0 when the file has none, as sourceParams returns, which makes it
    NaN), source02 = -1, on the Gauss-Chebyshev grid."""
    z = g.zgrid()
    hov = None
    for n, v in r.source_params:
        if n == "HovEll":
            hov = v
            break
    out = {2: -np.ones(g.NZAA)}
    if hov is None and r.source_params:
        return out   # the reference stops here (an unknown sourceParams name)
    h = 0.0 if hov is None else hov
    with np.errstate(invalid="ignore", divide="ignore"):
        out[1] = h * np.exp(-z * h) / (1.0 - np.exp(-h)) - 1.0
    return out


def default_penalisation_mask(g: Geometry) -> np.ndarray:
    """max of the two masks of the reference's default PL_user_penalisation_mask.f90
    on the grid, (NYAA, NXAA, NZAA): z - (0.9 + 0.1 cos(5 (x + y) 2 pi / Lx)) and
    0.4 exp(-(6 + cos(2 pi x / Lx))^2) / exp(-25) - z, at the reference's grid
    labels x = (i + 2) Lx / NXAA, y = (j + 2) Ly / NYAA (PL_geometry.f90:138-145,
    phys_iStart = 1), with its single-precision literals pi, 0.9 and 0.1."""
    pi = float(np.float32(3.14159265358979311599796346854))
    c09, c01 = float(np.float32(0.9)), float(np.float32(0.1))
    x = (np.arange(g.NXAA) + 2) * 1.0 * g.Lx / g.NXAA
    y = (np.arange(g.NYAA) + 2) * 1.0 * g.Ly / g.NYAA
    z = g.zgrid()
    X = x[None, :, None]
    Y = y[:, None, None]
    Z = z[None, None, :]
    m1 = Z - (c09 + c01 * np.cos(5 * (X + Y) * 2 * pi / g.Lx))
    m2 = (0.4 * np.exp(-((6.0 + np.cos(2 * pi * X / g.Lx)) ** 2)) / np.exp(-25.0)) - Z
    return np.maximum(m1, m2)


def penalisation_field(mask: np.ndarray, strength: float, width: float) -> np.ndarray:
    """init_penalisation (marching.f90:778-822): strength (1 + tanh(width mask)) / 2."""
    pm = np.tanh(width * mask)
    pm = (1.0 + pm) / 2.0
    return strength * pm


# --------------------------------------------------------------------------------------
# the solver
# --------------------------------------------------------------------------------------


class Solver:
    """State and operators of one plane-layer problem on one rank (world_size = 1)."""

    def __init__(self, equations_text: str, parameters_text: str, scheme: Optional[str] = None,
                 smagorinsky: bool = False, smagorinsky_prefactor: float = 1.0, cfl_factor_z: float = 1.0):
        self.recipe = parse_equations(equations_text, smagorinsky)
        p = read_parameters_text(parameters_text)
        self.params = p
        self.g = Geometry(p["NX"], p["NY"], p["NZ"], p["Lx"], p["Ly"], p["gap"], p["center"])
        self.scheme = scheme or p["scheme"]
        self.nstages, self.A, self.Ah = ars_tableau(self.scheme)
        self._build()
        self.dt_factored = None
        self.smagorinsky_prefactor = smagorinsky_prefactor
        self.cfl_factor_z = cfl_factor_z
        self.smago_profile = np.zeros(self.g.NZAA)   # nuSmago's physical values (one per z)
        self.sources = default_sources(self.recipe, self.g)
        self.penal_mask = default_penalisation_mask(self.g)
        self.penal_phys = {}
        for i, o in enumerate(self.recipe.full_opts):
            if o["penal"] is not None:
                self.penal_phys[i] = penalisation_field(self.penal_mask, *o["penal"])

    def set_source(self, index: int, profile: np.ndarray):
        """A user source sourceNN from its values on the Gauss-Chebyshev grid (the
        reference's PL_user_sources_definitions.f90 include)."""
        self.sources[index] = np.asarray(profile, dtype=np.float64).copy()

    def set_penalisation_mask(self, mask: np.ndarray):
        """max over the user's masks on the grid, (NYAA, NXAA, NZAA) (the reference's
        PL_user_penalisation_mask.f90 include); every penalised variable's field is
        remade from it."""
        self.penal_mask = np.asarray(mask, dtype=np.float64).copy()
        for i, o in enumerate(self.recipe.full_opts):
            if o["penal"] is not None:
                self.penal_phys[i] = penalisation_field(self.penal_mask, *o["penal"])

    # ---------------- setup ----------------
    def _build(self):
        g, r = self.g, self.recipe
        NZ = g.NZ
        cache: Dict = {}
        self.lay = []
        self.kxky_ops = []
        for s in r.kxky:
            lay = SystemLayout(NZ, s)
            self.lay.append(lay)
            mass = [(pc, build_piece_matrix(NZ, g.center, g.gap, lay, s, pc, cache)) for pc in s.mass]
            stif = [(pc, build_piece_matrix(NZ, g.center, g.gap, lay, s, pc, cache)) for pc in s.stif]
            self.kxky_ops.append((mass, stif))
        self.zlay = []
        self.zero_ops = []
        for s in r.zero:
            lay = SystemLayout(NZ, s)
            self.zlay.append(lay)
            M = sp.csr_matrix((lay.T, lay.T))
            L = sp.csr_matrix((lay.T, lay.T))
            for pc in s.mass:
                M = M + pc.dsca * build_piece_matrix(NZ, g.center, g.gap, lay, s, pc, cache)
            for pc in s.stif:
                L = L + pc.dsca * build_piece_matrix(NZ, g.center, g.gap, lay, s, pc, cache)
            self.zero_ops.append((M.tocsr(), L.tocsr()))
        # Fourier prefactor of every piece, per (kx, ky): dsca * py^b * px^a
        self.coef = []
        for mass, stif in self.kxky_ops:
            cm = [self._prefactor(pc) for pc, _ in mass]
            cs = [self._prefactor(pc) for pc, _ in stif]
            self.coef.append((cm, cs))
        # state
        self.field = [np.zeros((g.NXH, g.NYAA, l.T), dtype=np.complex128) for l in self.lay]
        self.zfield = [np.zeros(l.T) for l in self.zlay]
        # Cheb_IM cache for NL assembly
        self._im_cache = cache
        self.cfl_dt = None
        self.ke = None

    def _prefactor(self, pc) -> np.ndarray:
        g = self.g
        out = np.empty((g.NXH, g.NYAA), dtype=np.complex128)
        for ix in range(g.NXH):
            pxa = complex_pow(complex(g.px[ix]), pc.kx)
            for iy in range(g.NYAA):
                out[ix, iy] = (pc.dsca * complex_pow(complex(g.py[iy]), pc.ky)) * pxa
        return out

    def _apply(self, ops, coefs, x: np.ndarray) -> np.ndarray:
        """y[kx,ky,:] = sum_p coef_p[kx,ky] * (B_p @ x[kx,ky,:])."""
        sh = x.shape
        X = x.reshape(-1, sh[-1])
        y = np.zeros_like(X)
        for (pc, B), c in zip(ops, coefs):
            y += c.reshape(-1)[:, None] * (B @ X.T).T
        return y.reshape(sh)

    def band_of_system(self, isys: int, dt: float, ix: int, iy: int):
        """Evolution operator E = M - dt*a11*L of one (kx,ky) system as a dense matrix."""
        mass, stif = self.kxky_ops[isys]
        cm, cs = self.coef[isys]
        T = self.lay[isys].T
        M = np.zeros((T, T), dtype=np.complex128)
        L = np.zeros((T, T), dtype=np.complex128)
        for (pc, B), c in zip(mass, cm):
            M += c[ix, iy] * B.toarray()
        for (pc, B), c in zip(stif, cs):
            L += c[ix, iy] * B.toarray()
        zsca = complex(-dt * self.A[0, 0], 0.0)
        return M + zsca * L

    def factorize(self, dt: float):
        """factorize_operators (PL_IMEX_timestepping.f90:351-422) with zgbtrf per system."""
        g = self.g
        act = g.active
        self.lu = []
        self.kl_ku = []
        for isys, lay in enumerate(self.lay):
            mass, stif = self.kxky_ops[isys]
            # union band structure over pieces
            kl = ku = 0
            for _, B in mass + stif:
                Bc = B.tocoo()
                if Bc.nnz:
                    kl = max(kl, int((Bc.row - Bc.col).max()))
                    ku = max(ku, int((Bc.col - Bc.row).max()))
            self.kl_ku.append((kl, ku))
            T = lay.T
            # band form (kl+ku+1, T) of each piece: dia[ku + r - c, c]
            def toband(B):
                Bc = B.tocoo()
                out = np.zeros((kl + ku + 1, T))
                out[ku + Bc.row - Bc.col, Bc.col] = Bc.data
                return out
            mb = [toband(B) for _, B in mass]
            sb = [toband(B) for _, B in stif]
            cm, cs = self.coef[isys]
            zsca = complex(-dt * self.A[0, 0], 0.0)
            facs = {}
            for ix in range(g.NXH):
                for iy in range(g.NYAA):
                    if not act[ix, iy]:
                        continue
                    Mb = np.zeros((kl + ku + 1, T), dtype=np.complex128)
                    Lb = np.zeros((kl + ku + 1, T), dtype=np.complex128)
                    for b, c in zip(mb, cm):
                        Mb += c[ix, iy] * b
                    for b, c in zip(sb, cs):
                        Lb += c[ix, iy] * b
                    ab = np.zeros((2 * kl + ku + 1, T), dtype=np.complex128)
                    ab[kl:, :] = Mb + zsca * Lb
                    lu, piv, info = lapack.zgbtrf(ab, kl, ku)
                    if info != 0:
                        raise RuntimeError("zgbtrf failed (info=%d) at kx=%d ky=%d" % (info, ix, iy))
                    facs[(ix, iy)] = (lu, piv)
            self.lu.append(facs)
        self.zlu = []
        for (M, L), lay in zip(self.zero_ops, self.zlay):
            E = (M + (-dt * self.A[0, 0]) * L).tocoo()
            kl = int(max(0, (E.row - E.col).max())) if E.nnz else 0
            ku = int(max(0, (E.col - E.row).max())) if E.nnz else 0
            ab = np.zeros((2 * kl + ku + 1, lay.T))
            ab[kl + ku + E.row - E.col, E.col] = E.data
            lu, piv, info = lapack.dgbtrf(ab, kl, ku)
            if info != 0:
                raise RuntimeError("dgbtrf failed (info=%d)" % info)
            self.zlu.append((lu, piv, kl, ku))
        self.dt_factored = dt

    # ---------------- spectral assembly ----------------
    def _stencil_extract(self, isys: int, v: int, aux: np.ndarray) -> np.ndarray:
        """padStencilExtractShuffle: Chebyshev coefficients (NZ) of var v from the state."""
        lay = self.lay[isys]
        S = stencil(self.g.NZ, self.recipe.kxky[isys].bcs[v])
        return aux[..., lay.var_pos[v]] @ S.T

    def full_var_spec(self, src_kxky, src_zero) -> List[np.ndarray]:
        """compute_full_variables_in_physical_space, spectral part (marching.f90:436-503)."""
        g, r = self.g, self.recipe
        out = []
        for name, ext, terms in r.full_vars:
            spec = np.zeros((g.NXH, g.NYAA, g.NZ), dtype=np.complex128)
            for t in terms:
                if t.kind == "kxky":
                    isys, pos = r.kxky_loc[r.kxky_vars[t.var]]
                    buf = self._stencil_extract(isys, pos, src_kxky[isys])
                    buf = t.dsca * buf
                    if t.dz:
                        buf = self.differentiate(buf, t.dz)
                    if t.dx == 0 and t.dy == 0 and t.dz == 0:
                        spec = spec + buf
                    else:
                        fx = np.array([complex_pow(complex(p), t.dx) for p in g.px])
                        fy = np.array([complex_pow(complex(p), t.dy) for p in g.py])
                        spec = spec + buf * fx[:, None, None] * fy[None, :, None]
                else:
                    isys, pos = r.zero_loc[r.zero_vars[t.var]]
                    lay = self.zlay[isys]
                    S = stencil(g.NZ, r.zero[isys].bcs[pos])
                    buf = S @ src_zero[isys][lay.var_pos[pos]]
                    if t.dz:  # differentiate_zero, then dsca (marching.f90:488-494)
                        buf = self.differentiate(buf, t.dz)
                    spec[0, 0, :] = spec[0, 0, :] + buf * t.dsca
            o = r.full_opts[len(out)] if r.full_opts else None
            if o is not None and o["penal"] is None and not o["smago"]:
                spec = z_filter(spec, o["extract"], o["decomp"])
            out.append(spec)
        return out

    def differentiate(self, c: np.ndarray, order: int) -> np.ndarray:
        """differentiate_kxky / differentiate_zero (PL_IMEX_timestepping.f90:276-360)
        along the last axis (Chebyshev coefficients 0..NZ-1), `order` times: the
        coefficients shifted down by one (deriv(n) = c(n + 1)) solved against the
        Chebyshev integration operator trunc(I)[rows 2..NZ, cols 1..NZ-1]
        (prepare_chebyshev_integration, :488-505; padding 10), the last
        coefficient set to zero."""
        g = self.g
        NZ = g.NZ
        I, _ = cheb_elementary(NZ, g.center, g.gap, 10)
        A = I[1:NZ, 0:NZ - 1]  # upper triangular: diagonal and second super-diagonal
        out = np.array(c, dtype=np.result_type(c, np.float64), copy=True)
        for _ in range(order):
            rhs = out[..., 1:NZ].copy()
            d = np.zeros_like(rhs)
            # back substitution (the band LU of an upper-triangular band has no pivots)
            for n in range(NZ - 2, -1, -1):
                v = rhs[..., n]
                if n + 2 <= NZ - 2:
                    v = v - A[n, n + 2] * d[..., n + 2]
                d[..., n] = v / A[n, n]
            out[..., :NZ - 1] = d
            out[..., NZ - 1] = 0.0
        return out

    def nl_terms(self, qspec: List[np.ndarray]):
        """K_hat assembly (marching.f90:319-397)."""
        g, r = self.g, self.recipe
        act = g.active
        khat = []
        for isys, s in enumerate(r.kxky):
            lay = self.lay[isys]
            K = np.zeros((g.NXH, g.NYAA, lay.T), dtype=np.complex128)
            for t in s.nl:
                fx = np.array([complex_pow(complex(p), t.dx) for p in g.px])
                fy = np.array([complex_pow(complex(p), t.dy) for p in g.py])
                buf = (t.dsca * fx[:, None] * fy[None, :])[:, :, None] * qspec[t.quad]
                key = (t.Iz, t.mz)
                if key not in self._im_cache:
                    self._im_cache[key] = cheb_IM(g.NZ, g.center, g.gap, t.Iz, t.mz)
                trunc = self._im_cache[key][s.orders[t.eqn]:, :]
                K[:, :, lay.eq_pos[t.eqn]] += buf @ trunc.T
            K[~act] = 0.0
            khat.append(K)
        zk = []
        for isys, s in enumerate(r.zero):
            lay = self.zlay[isys]
            K = np.zeros(lay.T)
            for t in s.nl:
                buf = t.dsca * qspec[t.quad][0, 0, :].real
                key = (t.Iz, t.mz)
                if key not in self._im_cache:
                    self._im_cache[key] = cheb_IM(g.NZ, g.center, g.gap, t.Iz, t.mz)
                trunc = self._im_cache[key][s.orders[t.eqn]:, :]
                K[lay.eq_pos[t.eqn]] += trunc @ buf
            # sources (marching.f90:398-415): constant terms of the mean equations
            for t in r.sources:
                if t.sys != isys:
                    continue
                if t.index not in self.sources:
                    raise ValueError("source%02d is not defined" % t.index)
                buf = source_spectrum(self.sources[t.index])[:g.NZ] * t.dsca
                key = (t.Iz, 0)
                if key not in self._im_cache:
                    self._im_cache[key] = cheb_IM(g.NZ, g.center, g.gap, t.Iz, 0)
                trunc = self._im_cache[key][s.orders[t.eqn]:, :]
                K[lay.eq_pos[t.eqn]] += trunc @ buf
            zk.append(K)
        return khat, zk

    def compute_phys(self, src_kxky, src_zero):
        """Full variables in physical space plus the quadratic variables' spectra."""
        g, r = self.g, self.recipe
        fspec = self.full_var_spec(src_kxky, src_zero)
        fphys = []
        for i, sp_ in enumerate(fspec):
            o = r.full_opts[i] if r.full_opts else None
            if o is not None and o["penal"] is not None:
                # a penalised variable is its mask field, never transformed (marching.f90:515)
                fphys.append(self.penal_phys[i])
            elif o is not None and o["smago"]:
                # nuSmago (marching.f90:516-541): the previous values plus the squares of
                # dxUfull, dyUfull, dxVfull, dyVfull, averaged horizontally, prefactor * sqrt
                acc = np.broadcast_to(self.smago_profile, (g.NYAA, g.NXAA, g.NZAA)).copy()
                for j, (nm, _, _) in enumerate(r.full_vars[:i]):
                    if nm in ("dxUfull", "dyUfull", "dxVfull", "dyVfull"):
                        acc = acc + fphys[j] ** 2
                prof = acc.sum(axis=0).sum(axis=0) / g.NXAA / g.NYAA
                self.smago_profile = self.smagorinsky_prefactor * np.sqrt(prof)
                fphys.append(np.broadcast_to(self.smago_profile, (g.NYAA, g.NXAA, g.NZAA)).copy())
            else:
                fphys.append(spec_to_phys(sp_, g))
        self._cfl(fphys)
        qphys, qspec = [], []
        for name, i1, i2, rm in r.quad_vars:
            if i1 == -1:
                ph = fphys[i2].copy()
            elif i2 == -1:
                ph = fphys[i1].copy()
            else:
                ph = fphys[i1] * fphys[i2]
            s = phys_to_spec(ph, g)
            if rm:
                s[:, :, 0] = 0.0
                for q in range(1, g.NZ // 2):
                    s[:, :, 0] = s[:, :, 0] - s[:, :, 2 * q] * (0.5 / (2.0 * q + 1.0) - 0.5 / (2.0 * q - 1.0))
                ph = spec_to_phys(s, g)
            qphys.append(ph)
            qspec.append(s)
        return fphys, qphys, qspec

    def _cfl(self, fphys):
        """compute_cfl_based_timestep (marching.f90:200-254): the w term scaled by
        cflFactor_along_z and left out at or below 1e-10."""
        g = self.g
        if len(fphys) < 3:
            self.cfl_dt = None
            return
        w = g.zweights()
        u = np.abs(fphys[0]).max() * g.NXAA / g.Lx
        v = np.abs(fphys[1]).max() * g.NYAA / g.Ly
        f = getattr(self, "cfl_factor_z", 1.0)
        wz = max(v, (np.abs(fphys[2]) / w[None, None, :] * f).max()) if f > 1e-10 else v
        m = max(u, v, wz)
        self.cfl_dt = 1.0 / m if m > 0 else float('inf')
        if self.recipe.smagorinsky:
            # marching.f90:241-251, with the single-precision literals 0.95 and 3.141592
            c = float(np.float32(np.float32(2) * np.float32(3.141592)) ** np.float32(2))
            den = c * float(np.max(fphys[-1])) * ((g.NXAA / g.Lx) ** 2 + (g.NYAA / g.Ly) ** 2)
            self.cfl_dt = min(self.cfl_dt, float(np.float32(0.95)) / den if den > 0 else float('inf'))

    def volume_average(self, phys: np.ndarray) -> float:
        """output_global_quantities 'volume' object (PL_IMEX_timestepping_output.f90:38-52)."""
        w = self.g.zweights()
        return float((phys * w[None, None, :]).sum() / self.g.NXAA / self.g.NYAA)

    # ---------------- the timestep ----------------
    def step(self, dt: float):
        """one_step_beyond (marching.f90:3-48)."""
        g, r = self.g, self.recipe
        if self.dt_factored is None or self.dt_factored != dt:
            self.factorize(dt)
        act = g.active
        deal = ~act
        deal[0, 0] = False
        aux = [f.copy() for f in self.field]
        zaux = [f.copy() for f in self.zfield]
        Kstd, Khat, zKstd, zKhat = [], [], [], []
        for i in range(self.nstages):
            fphys, qphys, qspec = self.compute_phys(aux, zaux)
            if i == 0:
                self.stage0_phys = (fphys, qphys)
                self.ke = None
                names = [q[0] for q in r.quad_vars]
                if all(n in names for n in ("uu", "vv", "ww")):
                    self.ke = sum(self.volume_average(qphys[names.index(n)]) for n in ("uu", "vv", "ww"))
            kh, zkh = self.nl_terms(qspec)
            Khat.append(kh)
            zKhat.append(zkh)
            Ks_i, zKs_i = [], []
            for isys, lay in enumerate(self.lay):
                mass, stif = self.kxky_ops[isys]
                cm, cs = self.coef[isys]
                rhs = self._apply(mass, cm, self.field[isys])
                if g.NXH > 0:
                    rhs[0, 0, :] = 0.0      # mass(1,1) is the empty matrix
                for j in range(i):
                    rhs = rhs + (dt * self.A[i, j]) * Kstd[j][isys]
                    rhs = rhs + (dt * self.Ah[i + 1, j]) * Khat[j][isys]
                rhs = rhs + (dt * self.Ah[i + 1, i]) * Khat[i][isys]
                # backsolve: identity for dealiased modes and (0,0)
                newaux = rhs.copy()
                kl, ku = self.kl_ku[isys]
                for (ix, iy), (lu, piv) in self.lu[isys].items():
                    x, info = lapack.zgbtrs(lu, kl, ku, rhs[ix, iy, :], piv)
                    if info != 0:
                        raise RuntimeError("zgbtrs failed")
                    newaux[ix, iy, :] = x
                aux[isys] = newaux
                ks = self._apply(stif, cs, newaux)
                ks[~act] = 0.0
                Ks_i.append(ks)
            for isys, lay in enumerate(self.zlay):
                M, L = self.zero_ops[isys]
                rhs = M @ self.zfield[isys]
                for j in range(i):
                    rhs = rhs + (dt * self.A[i, j]) * zKstd[j][isys]
                    rhs = rhs + (dt * self.Ah[i + 1, j]) * zKhat[j][isys]
                rhs = rhs + (dt * self.Ah[i + 1, i]) * zKhat[i][isys]
                lu, piv, kl, ku = self.zlu[isys]
                x, info = lapack.dgbtrs(lu, kl, ku, rhs, piv)
                if info != 0:
                    raise RuntimeError("dgbtrs failed")
                zaux[isys] = x
                zKs_i.append(L @ x)
            Kstd.append(Ks_i)
            zKstd.append(zKs_i)
        for isys in range(len(self.lay)):
            f = aux[isys].copy()
            f[~act] = 0.0
            self.field[isys] = f
        self.zfield = [z.copy() for z in zaux]

    # ---------------- timeseries and the time loop ----------------
    def timeseries_values(self, objects):
        """output_global_quantities (PL_IMEX_timestepping_output.f90:5-127) on the
        first stage's fields of the last step.  objects: [(name, zpos)] with zpos
        None for a volume average, else the 1-based grid level of a horizontal
        average; name a full or quadratic variable."""
        fphys, qphys = self.stage0_phys
        fnames = [f[0] for f in self.recipe.full_vars]
        qnames = [q[0] for q in self.recipe.quad_vars]
        out = []
        for name, zpos in objects:
            ph = fphys[fnames.index(name)] if name in fnames else qphys[qnames.index(name)]
            if zpos is None:
                out.append(self.volume_average(ph))
            else:
                out.append(float(ph[:, :, zpos - 1].sum() / self.g.NXAA / self.g.NYAA))
        return out

    def run(self, nsteps, objects=()):
        """The time loop of plane_layer_main.f90:138-205 with the dt rules of
        timeKeeping.f90:78-89,171-183 (parameters dt_max, tolerance, CFL_C of the
        parameter file).  Returns [(step index, time, dt used, timeseries values)]."""
        p = self.params
        if not hasattr(self, "t_time"):
            self.t_time, self.t_dt_current, self.t_dt, self.t_step = 0.0, p["dt_max"], p["dt_max"], 1
        rows = []
        for _ in range(nsteps):
            if abs(self.t_dt - self.t_dt_current) > p["tolerance"] * self.t_dt_current:
                self.t_dt_current = self.t_dt
            self.step(self.t_dt_current)
            rows.append((self.t_step, self.t_time, self.t_dt_current, self.timeseries_values(objects)))
            dt = self.cfl_dt * p["CFL_C"]
            if dt > p["dt_max"]:
                dt = p["dt_max"]
            if dt < 1e-9:
                raise RuntimeError("minimal timestep reached")
            self.t_dt = dt
            self.t_time += self.t_dt_current
            self.t_step += 1
        return rows

    # ---------------- state in physical space (checkpoint / quicksave) ----------------
    def var_cheb(self, isys: int, v: int) -> np.ndarray:
        """Chebyshev coefficients spec[kx][ky][n] of coupled var v of kxky system isys."""
        return self._stencil_extract(isys, v, self.field[isys])

    def set_var_from_phys(self, isys: int, v: int, phys: np.ndarray):
        """import_quicksave for one kxky var (PL_IMEX_timestepping_output.f90:338-356):
        phys -> spec -> square-stencil backsolve -> truncate/shuffle/insert (cumulative)."""
        g = self.g
        lay = self.lay[isys]
        spec = phys_to_spec(phys, g)
        S = stencil(g.NZ, self.recipe.kxky[isys].bcs[v])
        n = S.shape[1]
        Ssq = S[:n, :n]
        gal = np.linalg.solve(Ssq, spec[..., :n].reshape(-1, n).T).T.reshape(g.NXH, g.NYAA, n)
        self.field[isys][..., lay.var_pos[v]] += gal

    def set_zero_var_from_phys(self, isys: int, v: int, prof: np.ndarray):
        g = self.g
        lay = self.zlay[isys]
        c = r2r_forward(prof, g.NZAA)[:g.NZ]
        S = stencil(g.NZ, self.recipe.zero[isys].bcs[v])
        n = S.shape[1]
        gal = np.linalg.solve(S[:n, :n], c[:n])
        self.zfield[isys][lay.var_pos[v]] += gal

    def zero_var_profile(self, isys: int, v: int) -> np.ndarray:
        g = self.g
        lay = self.zlay[isys]
        S = stencil(g.NZ, self.recipe.zero[isys].bcs[v])
        c = np.zeros(g.NZAA)
        c[:g.NZ] = S @ self.zfield[isys][lay.var_pos[v]]
        return r2r_backward(c)

    def import_quicksave(self, directory: str, rolling: int = 1):
        """import_quicksave (PL_IMEX_timestepping_output.f90:309-383): files hold the field
        in z-fastest, then y, then x order."""
        g, r = self.g, self.recipe
        for isys, s in enumerate(r.kxky):
            self.field[isys][:] = 0.0
            for v in range(len(s.vars)):
                fn = os.path.join(directory, "QuickSave.kxky.sys%03d.var%03d.rolling%d" % (isys + 1, v + 1, rolling))
                a = np.fromfile(fn, dtype=np.float64).reshape(g.NXAA, g.NYAA, g.NZAA)
                self.set_var_from_phys(isys, v, np.ascontiguousarray(a.transpose(1, 0, 2)))
        for isys, s in enumerate(r.zero):
            self.zfield[isys][:] = 0.0
            for v in range(len(s.vars)):
                fn = os.path.join(directory, "QuickSave.zero.sys%03d.var%03d.rolling%d" % (isys + 1, v + 1, rolling))
                self.set_zero_var_from_phys(isys, v, np.fromfile(fn, dtype=np.float64))


# --------------------------------------------------------------------------------------
# banded-solve helpers used by the tests (zgbtrf / zgbtrs semantics)
# --------------------------------------------------------------------------------------


def zgbtrf_band(ab_dia: np.ndarray, kl: int, ku: int):
    """Factor a matrix given in DIA rows (kl+ku+1, n); returns (lu, ipiv) in LAPACK band layout."""
    n = ab_dia.shape[1]
    ab = np.zeros((2 * kl + ku + 1, n), dtype=np.complex128)
    ab[kl:, :] = ab_dia
    lu, piv, info = lapack.zgbtrf(ab, kl, ku)
    if info != 0:
        raise RuntimeError("zgbtrf info=%d" % info)
    return lu, piv


def zgbtrs_band(lu, piv, kl, ku, b):
    x, info = lapack.zgbtrs(lu, kl, ku, b, piv)
    if info != 0:
        raise RuntimeError("zgbtrs info=%d" % info)
    return x


# --------------------------------------------------------------------------------------
# user outputs (coral.usrOutput): the parser of PL_equations.f90:322-427 with the line
# readers of PL_string_to_data.f90:244-300, the counters of
# PL_IMEX_timestepping_marching.f90:620-697, and the files of
# PL_IMEX_timestepping_output.f90:250-307,489-581,685-715 and
# slabs.fftw3mpi/transforms.f90:53-105,772-866 (P = 1)
# --------------------------------------------------------------------------------------

USR_KINDS = {">>Volume ::": "volume", ">>ZSlice ::": "zSlice", ">>YSlice ::": "ySlice",
             ">>XSlice ::": "xSlice", ">>Zsummed::": "zAvged", ">>Profile::": "profil"}


def parse_usr_output(text: str, recipe: Recipe, g: Geometry):
    """Objects [(kind, is_quad, var_index0, period, position)] in output order:
    the full variables' objects first (variable order, then file order), then the
    quadratic variables'.  Positions beyond the grid are dropped, as the reference
    does (with a message); position is 1-based (0 for kinds without one)."""
    fnames = [f[0] for f in recipe.full_vars]
    qnames = [q[0] for q in recipe.quad_vars]
    per_f = [[] for _ in fnames]
    per_q = [[] for _ in qnames]
    limit = {"zSlice": g.NZAA, "ySlice": g.NYAA, "xSlice": g.NXAA}
    for line in text.splitlines():
        if line[2:5] == "EOF":
            break
        if not line.strip():
            continue
        kind = USR_KINDS.get(line[:11])
        if kind is None:
            raise ValueError("coral.usrOutput: bad line %r" % line)
        dc, pp, end = line.index("::") + 2, line.index(";; Period="), line.index("<<")
        name = line[dc:pp].strip()
        if kind in limit:
            ps = line.index(";; Position=")
            period = int(line[pp + 10:ps])
            pos = int(line[ps + 12:end])
            if pos > limit[kind]:
                continue
        else:
            period, pos = int(line[pp + 10:end]), 0
        if name in fnames:
            per_f[fnames.index(name)].append((kind, False, fnames.index(name), period, pos))
        if name in qnames:
            per_q[qnames.index(name)].append((kind, True, qnames.index(name), period, pos))
    return [o for v in per_f for o in v] + [o for v in per_q for o in v]


def usr_output_files(objs, fphys, qphys, g: Geometry, itime: int):
    """{relative file name: float64 array in file order} of the objects, from the
    full and quadratic variables' physical fields (phys[y][x][z])."""
    out = {}
    w = g.zweights()
    for kind, is_q, iv, _, pos in objs:
        ph = qphys[iv] if is_q else fphys[iv]
        pre = "quadra" if is_q else "linear"
        tag = "%s_var%02d" % (pre, iv + 1)
        tr = ph.transpose(1, 0, 2)  # transposed_phys(z, y, x) in C order [x][y][z]
        if kind == "volume":
            out["Volumes/%s_time%08d_full.dat" % (tag, itime)] = tr.ravel()
        elif kind == "zSlice":
            out["Slices/%s_z%05d_time%08d_full.dat" % (tag, pos, itime)] = tr[:, :, pos - 1].ravel()
        elif kind == "ySlice":
            out["Slices/%s_y%05d_time%08d_full.dat" % (tag, pos, itime)] = tr[:, pos - 1, :].ravel()
        elif kind == "xSlice":
            out["Slices/%s_x%05d_time%08d_full.dat" % (tag, pos, itime)] = tr[pos - 1, :, :].ravel()
        elif kind == "zAvged":
            out["Slices/%s_zAvged_time%08d_full.dat" % (tag, itime)] = (tr * w[None, None, :]).sum(axis=2).ravel()
        else:
            out["Profiles/%s_time%08d_full.dat" % (tag, itime)] = ph.sum(axis=(0, 1)) / g.NXAA / g.NYAA
    return out


def usr_output_schedule(objs, i_timestep: int, nsteps: int):
    """[(step number within the run, time_integer, [objects due])]: counters start
    at i_timestep mod period and time_integer at i_timestep; every step's first
    stage advances both and writes the objects whose counter reaches the period."""
    counters = [i_timestep % o[3] for o in objs]
    t = i_timestep
    sched = []
    for s in range(nsteps):
        t += 1
        due = []
        for k, o in enumerate(objs):
            counters[k] += 1
            if counters[k] == o[3]:
                counters[k] = 0
                due.append(o)
        sched.append((s, t, due))
    return sched
