"""Run parameters for the quasi-linear shearing-box step.

Mirrors the fields of the reference's ``Inputs`` struct that the time step
reads (QL_DNS/Auxiliary/Input_parameters.cpp:68-138) and the derived model
dimensions (QL_DNS/Models/Model.h:27-38).
"""
from __future__ import annotations

import dataclasses
import math

MODEL_BQLIN = 0      # MHD_BQlin     (QL_DNS/Models/MHD_BQlin.cpp)
MODEL_FULLQLIN = 1   # MHD_FullQlin  (QL_DNS/Models/MHD_FullQlin.cpp)
INTEGRATOR_RK3_EXP = 0  # RK3CN_Elin  (QL_DNS/Integrators/RK3CN_Elin.cpp)
INTEGRATOR_RK3_CN = 1   # RK3CN       (QL_DNS/Integrators/RK3CN.cpp)

MODEL_NAMES = {"MHD_BQlin": MODEL_BQLIN, "MHD_FullQlin": MODEL_FULLQLIN}


@dataclasses.dataclass
class QLParams:
    model: int = MODEL_BQLIN
    integrator: int = INTEGRATOR_RK3_EXP
    nx: int = 16                 # nx_  (Input_parameters.cpp:68)
    ny: int = 16                 # ny_
    NZ: int = 32                 # nz_  (real z grid; dealiased length is nz)
    L: tuple = (1.0, math.pi, 1.0)
    q: float = 1.5
    omega: float = 1.0           # used by MHD_FullQlin; MHD_BQlin hardwires 2q/3
    nu: float = 1.0 / 2000
    eta: float = 1.0 / 2000
    B0z: float = 0.0
    viscosity_order: int = 2
    dt: float = 0.01
    remap: int = 1               # Remap?
    quasilinear: int = 1         # QuasiLinear?

    # Derived dimensions (Model.h:31-36)
    @property
    def nz(self) -> int:
        return 1 + 2 * int(self.NZ / 3.0)

    @property
    def nxy(self) -> int:
        return (self.nx - 1) * (self.ny // 2)

    @property
    def nmf(self) -> int:
        return 2 if self.model == MODEL_BQLIN else 4

    @property
    def nlin(self) -> int:
        return 4

    def replace(self, **kw) -> "QLParams":
        return dataclasses.replace(self, **kw)


def mri_16x16_nz32(**kw) -> QLParams:
    """QL MRI 16x16 modes x NZ=32, Re=Rm=2000, dt=0.01 (500 steps)."""
    p = QLParams(nx=16, ny=16, NZ=32, nu=1 / 2000, eta=1 / 2000, dt=0.01)
    return p.replace(**kw)


def mri_64x64_nz128(**kw) -> QLParams:
    """QL MRI production size: 64x64 modes x NZ=128, Re=Rm=8000, dt=0.005 (2000 steps)."""
    p = QLParams(nx=64, ny=64, NZ=128, nu=1 / 8000, eta=1 / 8000, dt=0.005)
    return p.replace(**kw)


def adjoint_32x32_nz64(**kw) -> QLParams:
    """Adjoint case: 32x32 modes x NZ=64, Re=Rm=4000, dt=0.01."""
    p = QLParams(nx=32, ny=32, NZ=64, nu=1 / 4000, eta=1 / 4000, dt=0.01)
    return p.replace(**kw)


@dataclasses.dataclass
class DNSParams:
    """Full 3-D shearing-box MHD on an Mx x My x NZ grid (2/3 dealiased in x, y
    and z), in the shearing-wave frame of the QL models: the same box, shear q,
    rotation omega, vertical field B0z, dissipation (nu, eta, viscosity_order),
    integrators and remap rule.  The spectral mode set is the QL layout of
    ``ql()`` (nx = 2 floor(Mx/3) + 2, ny = 2 floor(My/3) + 2), each mode column
    carrying the three components of u and of b instead of (u, zeta, b, eta);
    the kx = ky = 0 column holds the mean fields (Ux, Uy, 0, Bx, By, 0)."""
    integrator: int = INTEGRATOR_RK3_EXP
    Mx: int = 64
    My: int = 128
    NZ: int = 64
    L: tuple = (1.0, math.pi, 1.0)
    q: float = 1.5
    omega: float = 1.0
    nu: float = 1.0 / 4000
    eta: float = 1.0 / 4000
    B0z: float = 0.0
    viscosity_order: int = 2
    dt: float = 0.005
    remap: int = 1
    dealias_xy: int = 1          # zero modes with |kx(t)| > Mx/3 (2 pi/Lx) at each stage

    @property
    def nx(self) -> int:
        return 2 * (self.Mx // 3) + 2

    @property
    def ny(self) -> int:
        return 2 * (self.My // 3) + 2

    @property
    def nz(self) -> int:
        return 1 + 2 * int(self.NZ / 3.0)

    @property
    def nxy(self) -> int:
        return (self.nx - 1) * (self.ny // 2)

    def ql(self) -> QLParams:
        """The MHD_FullQlin parameters on the same mode set."""
        return QLParams(model=MODEL_FULLQLIN, integrator=self.integrator, nx=self.nx, ny=self.ny, NZ=self.NZ,
                        L=tuple(self.L), q=self.q, omega=self.omega, nu=self.nu, eta=self.eta, B0z=self.B0z,
                        viscosity_order=self.viscosity_order, dt=self.dt, remap=self.remap, quasilinear=1)

    def replace(self, **kw) -> "DNSParams":
        return dataclasses.replace(self, **kw)


def dns_64x128x64(**kw) -> DNSParams:
    """Full DNS MRI: 64 x 128 x 64 grid, Re=Rm=4000, dt=0.005 (1000 steps)."""
    p = DNSParams(Mx=64, My=128, NZ=64, nu=1 / 4000, eta=1 / 4000, dt=0.005)
    return p.replace(**kw)
