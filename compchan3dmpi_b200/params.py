"""Run parameters of the channel solver (the reference's comdata + param.dat).

Reference: v1.9/codes/comdata.f90:4-68 (compile-time constants and the
fixed-column ``param.dat`` reader).  Axis convention is the reference's:
``nP = (nP1, nP2, nP3)`` = (streamwise x, spanwise, wall-normal).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, replace

RK2 = 2   # reference midpoint scheme, comdata.f90:8 (maxiter = 2)
RK3 = 3   # SSP-RK3, no reference counterpart

FORCE_WALLSHEAR = 0   # reference lagged wall-shear forcing, main_v1.9.f90:547-553
FORCE_NONE = 1


@dataclass
class ChanParams:
    nP: tuple = (64, 48, 65)
    Re: float = 3000.0            # param.dat (Re)
    Mac: float = 1.5              # param.dat (Mac)
    dt: float = 1.0e-4            # param.dat (dt); v1.8 hardcodes 1e-4
    Pr: float = 0.71              # comdata.f90:12  invPr = 1/0.71
    gama: float = 1.4             # comdata.f90:11
    Pe: tuple = (2.0, 2.0, 0.2)   # PexVal, PeyVal, PezVal (v1.8_validation/codes/comData.f90:12-14)
    Lx: float = 4.0 * math.pi     # comdata.f90:81
    Ly: float = 4.0 * math.pi / 3.0  # comdata.f90:82
    Tw: tuple = (1.0, 1.0)        # main_v1.9.f90:628, 635
    istat: int = 10               # param.dat (istat)
    rk_scheme: int = RK2
    forcing: int = FORCE_WALLSHEAR
    device: int = 0
    mixed: bool = False           # float stage storage and fluxes, double accumulation (CHAN_MIXED)

    def with_(self, **kw) -> "ChanParams":
        return replace(self, **kw)

    @property
    def n_interior(self) -> int:
        n1, n2, n3 = self.nP
        return (n1 - 2) * (n2 - 2) * (n3 - 2)

    @property
    def stages(self) -> int:
        return 3 if self.rk_scheme == RK3 else 2

    @property
    def ggM(self) -> float:
        return self.gama * (self.gama - 1) * (self.Mac * self.Mac)

    @property
    def dx(self) -> float:
        return self.Lx / (self.nP[0] - 1)

    @property
    def dy(self) -> float:
        return self.Ly / (self.nP[1] - 1)

    @property
    def dXi(self) -> float:
        return 2.0 / (self.nP[2] - 1)


def reference_params(nP=(64, 48, 65), **kw) -> ChanParams:
    """The reference's own physics (parity mode): RK2, Pr = 0.71, wall-shear forcing."""
    return ChanParams(nP=tuple(nP), **kw)


def production_params(nP=(256, 192, 193), **kw) -> ChanParams:
    """Production workload physics: SSP-RK3, Pr = 0.72 (dt is set from CFL by the caller)."""
    base = dict(Pr=0.72, rk_scheme=RK3)
    base.update(kw)
    return ChanParams(nP=tuple(nP), **base)
