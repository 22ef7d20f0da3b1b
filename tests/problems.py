"""Small problem definitions shared by the tests."""
import math
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CFG = os.path.join(ROOT, "coral_b200", "configs")

PARAMS = """0           ! resolution
{NX}          ! NX
{NY}          ! NY
{NZ}          ! NZ
0           ! geometry
{Lx!r}  ! Lx
{Ly!r}  ! Ly
1.d0        ! gap
0.5d0       ! center
0           ! timestepping
{dt!r}  ! dt_max
0.3d0       ! tolerance
1.d30       ! CFL
'{scheme}'   ! scheme
0           ! quicksave
.True.      ! restart
0           ! timer
1.d9        ! time limit
"""


def params(NX, NY, NZ, dt=1e-4, Lx=2 * math.pi, Ly=2 * math.pi, scheme="ARS_222"):
    return PARAMS.format(NX=NX, NY=NY, NZ=NZ, Lx=Lx, Ly=Ly, dt=dt, scheme=scheme)


def equations(name="rbc_noslip_ra1e5", **replace):
    with open(os.path.join(CFG, name + ".equations")) as f:
        t = f.read()
    for k, v in replace.items():
        t = t.replace(k, v)
    return t
