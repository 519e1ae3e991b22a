"""marinehydro_b200 -- B200 (sm_100a) implementation of MarineHydro.jl's
boundary-element hot path: Green-function influence-matrix assembly, the
dense complex solve and the outputs built on it (added mass, radiation
damping, diffraction force).

The compute runs in ``lib/libmarinehydro_b200.so`` (hand-written CUDA for
sm_100a behind the C ABI in ``include/marinehydro_b200.h``).  This package is
the host-side mirror of the reference's public API for that path.
"""
from .meshes import (Mesh, combine_meshes, mesh_hemisphere, mesh_two_hemispheres, panel_geometry,
                     wavebot_profile, axisymmetric_mesh, polygon_geometry, wavebot_mesh)
from .api import (SETTINGS, set_g, set_rho, GreensFunction, Rankine, RankineReflected,
                  RankineReflectedNegative, GFWu, ExactGuevelDelhommeau, gf_mask,
                  DEFAULT_GREEN_FUNCTIONS, DeviceMesh, device_mesh, assemble_matrices,
                  assemble_matrix_wu, solve, calculate_radiation_forces, DiffractionForce,
                  radiation_bc, AiryBC, airy_waves_potential, airy_waves_velocity,
                  airy_waves_pressure, integrate_pressure, FroudeKrylovForce)
from .bodies import (FloatingBody, combine_floatingbodies, make_body_name_list_unique,
                     translational_dofs, rotational_dofs, hydro_batch, BatchInfo,
                     compute_hydrodynamic_coefficients)
from .gradients import (MeshTangent, VjpResult, JvpResult, hydro_batch_vjp, hydro_batch_jvp,
                        hydro_batch_rrule,
                        hemisphere_tangents, two_hemispheres_tangents, polygon_geometry_jvp,
                        wavebot_tangents)
from .meshgen import (GeneratedMesh, generate_hemisphere, generate_two_hemispheres, generate_wavebot,
                      generate_combined, generated_tangents, generated_tangent, generated_param_grad)
from .power import two_body_power, optimize_two_body_power
from .design import SplitMix64, Design, designs, design_batch
from ._native import (Context, MarineHydroError, ArgumentError, NotConvergedError,
                      SingularMatrixError, device_count, default_context)
from . import _native as native

__all__ = [n for n in dir() if not n.startswith("_")]
