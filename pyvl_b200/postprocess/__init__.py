"""Post-processing on the GPU kernels (python/pyvl/postprocess): forces, velocities, pressure."""

from .forces import circulatory_forces as circulatory_forces
from .forces import lift_coefficient as lift_coefficient
from .pressure import compute_dynamic_pressure_variable as compute_dynamic_pressure_variable
from .pressure import compute_surface_dynamic_pressure as compute_surface_dynamic_pressure
from .velocity import compute_velocities as compute_velocities
from .velocity import compute_velocities_variable as compute_velocities_variable
