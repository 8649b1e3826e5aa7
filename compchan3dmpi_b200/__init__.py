"""B200-native time-step hot path of the compressible channel DNS
theparvezahmad/compChan3Dmpi.

The compute path is ``lib/libchanrhs.so`` (CUDA, sm_100a, C ABI in
include/chanrhs.h).  This package holds the host-side mirror of the
reference's interface (``Channel``), its deck formats, mesh and the seeded
initial condition.
"""
from .params import ChanParams, reference_params, production_params, RK2, RK3, FORCE_WALLSHEAR, FORCE_NONE  # noqa
from .mesh import mesh_cosine, mesh_tanh, make_mesh, wall_coeffs, cfl_dt, periodic_coords  # noqa
from .ic import laminar_noise  # noqa
from .channel import Channel, ChanError, BlowUpError  # noqa

__all__ = ["ChanParams", "reference_params", "production_params", "RK2", "RK3", "FORCE_WALLSHEAR",
           "FORCE_NONE", "mesh_cosine", "mesh_tanh", "make_mesh", "wall_coeffs", "cfl_dt",
           "periodic_coords", "laminar_noise", "Channel", "ChanError", "BlowUpError"]
