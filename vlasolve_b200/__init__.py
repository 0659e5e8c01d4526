"""vlasolve_b200: the split semi-Lagrangian step of the spherical (r, v_r, J)
Vlasov-Poisson system on one NVIDIA B200 (sm_100a).

The compute path is the CUDA C-ABI library libvlasolve_b200.so (see
include/vlasolve_b200.h); this package is its host-side mirror of the
reference solver interface.
"""
from .params import ParamsParser
from .solver import (Config, VlasovSolver21Spline, config_from_dict,
                     config_from_params, default_grid, default_init, default_solver)

__all__ = ["ParamsParser", "Config", "VlasovSolver21Spline", "config_from_dict",
           "config_from_params", "default_grid", "default_init", "default_solver"]
