"""femtools_b200 — sm_100a backend for FEMTools.jl's dynamic-relaxation solvers.

Host-side mirror of the reference's Stokes/thermal DR API (solve!, solve_coupled!,
the assemble_* kernels) over the C ABI of libfemtools_b200 (include/femtools_b200.h).
The directory name is not an importable identifier; load it by path (see
tests/conftest.py) under the module name `femtools_b200`.
"""
from . import _abi  # noqa: F401
from . import mesh  # noqa: F401
from . import problem  # noqa: F401
from . import configs  # noqa: F401
from . import coloring  # noqa: F401
from .coloring import color_mesh, generate_element_groups  # noqa: F401
from .mesh import structured_mixed_mesh, element_tables, MixedMesh  # noqa: F401
from .problem import StokesMaterial, DruckerPrager, DirichletBoundaryCondition  # noqa: F401

__all__ = ["structured_mixed_mesh", "element_tables", "MixedMesh", "StokesMaterial", "DruckerPrager",
           "DirichletBoundaryCondition", "color_mesh", "generate_element_groups"]

from . import solver  # noqa: E402,F401
from .solver import (StokesDR, ThermalDiffusionDR, solve, solve_stokes_dyrel, solve_coupled,  # noqa: E402,F401
                     solve_thermal, assemble_pressure_residual, assemble_momentum_residual,
                     assemble_stokes_residuals, assemble_augmented_momentum_jacobian,
                     assemble_viscosity_weighted_pressure_scaling, update_stokes_current_stress,
                     assemble_shear_heating, assemble_thermal_residual, assemble_diffusion_matrices_colored,
                     assemble_adjoint_residual, viscosity_sensitivity, solve_adjoint, precompute_geometry,
                     update_geometry)
from . import autodiff  # noqa: E402,F401
from .autodiff import DRCheckpoint, solve_log_viscosity  # noqa: E402,F401
from . import warmstart  # noqa: E402,F401
from . import postprocess  # noqa: E402,F401
from .postprocess import (compute_strain_rate_stress_postprocess, update_old_stress_from_cells,  # noqa: E402,F401
                          write_vtk, write_stokes_vtk, VtkMesh)
from . import cellpressure  # noqa: E402,F401
from .cellpressure import (CellPressureStokesDR, stokes_preconditioner_3d,  # noqa: E402,F401
                           assemble_stokes_pressure_residual_3d, assemble_stokes_momentum_residual_3d,
                           solve_cell_pressure, solve_adjoint_cell_pressure, stokes_material_gradient_3d)
from . import lithostatic  # noqa: E402,F401
from .lithostatic import LithostaticPressureDR, assemble_lithostatic_pressure, solve_lithostatic  # noqa: E402,F401
from . import cap  # noqa: E402,F401
from .cap import (DruckerPragerCap, cap_geometry, cap_yield_function, cap_invariants,  # noqa: E402,F401
                  cap_invariants_phase, softened_cohesion, cap_return_map, cap_local_update)
