"""Solver parameters with the reference's defaults.

Defaults follow create_param_main (src/general/mod_sim_param.f90:376-452):
rankine_rad 0.1, vortex_rad 0.1, cutoff_rad 0.001, far_field_ratio_doublet
10, vortstretch T, divergence_filtering T, diffusion T, turbulent_viscosity
F, mu_inf 1.8e-5 / rho_inf 1.225.
"""
from dataclasses import dataclass, field

from . import abi


@dataclass
class FmmParams:
    box_length: float = 1.0
    n_box: tuple = (1, 1, 1)
    origin: tuple = (0.0, 0.0, 0.0)
    n_octree_levels: int = 5
    min_octree_part: int = 5
    multipole_degree: int = 4
    rankine_rad: float = 0.1
    cutoff_rad: float = 0.001
    far_field_ratio_doublet: float = 10.0
    vortstretch: bool = True
    divergence_filtering: bool = True
    diffusion: bool = True
    turbulent_viscosity: bool = False
    nu_inf: float = 1.8e-5 / 1.225
    u_inf: tuple = (0.0, 0.0, 0.0)
    precision: int = abi.DUST_PREC_FP64

    def struct(self):
        s = abi.FmmParams()
        s.box_length = float(self.box_length)
        for d in range(3):
            s.n_box[d] = int(self.n_box[d])
            s.origin[d] = float(self.origin[d])
            s.u_inf[d] = float(self.u_inf[d])
        s.n_octree_levels = int(self.n_octree_levels)
        s.min_octree_part = int(self.min_octree_part)
        s.multipole_degree = int(self.multipole_degree)
        s.rankine_rad = float(self.rankine_rad)
        s.cutoff_rad = float(self.cutoff_rad)
        s.far_field_ratio_doublet = float(self.far_field_ratio_doublet)
        s.vortstretch = int(bool(self.vortstretch))
        s.divergence_filtering = int(bool(self.divergence_filtering))
        s.diffusion = int(bool(self.diffusion))
        s.turbulent_viscosity = int(bool(self.turbulent_viscosity))
        s.nu_inf = float(self.nu_inf)
        s.precision = int(self.precision)
        return s

    def replace(self, **kw):
        d = dict(self.__dict__)
        d.update(kw)
        return FmmParams(**d)
