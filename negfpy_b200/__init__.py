"""negfpy_b200: the per-(omega, k) phonon NEGF path of negfpy on NVIDIA B200.

Drop-in replacements for negfpy's hot-path API (same signatures, errors and
results) run on hand-written sm_100a CUDA kernels behind the C ABI in
``include/negf_b200.h``; the batched entry points in ``spectrum`` evaluate
whole (omega x k) grids in one pass.  There is no CPU fallback.
"""

from .types import Device1D, DeviceKSpace, LeadBlocks, LeadKSpace
from .surface_gf import (
    surface_gf,
    surface_gf_generalized_eigen,
    surface_gf_generalized_eigen_svd,
    surface_gf_legacy_eigen_svd,
    surface_gf_sancho_rubio,
)
from .negf import (
    device_green_function,
    transmission,
    transmission_kavg,
    transmission_kavg_adaptive,
    transmission_kavg_adaptive_global_eta,
)
from .dos import (
    lead_surface_dos,
    lead_surface_dos_kavg,
    lead_surface_dos_kavg_adaptive,
    lead_surface_dos_spectrum,
    leads_surface_dos_spectrum,
)
from .spectrum import kappa_from_grid, thermal_conductance_from_spectrum, transmission_grid
from .thermal_current import (
    heat_current_1d,
    heat_current_density_3d,
    heat_current_from_spectrum,
    heat_current_per_length_2d,
    transverse_length_from_vector,
)
from .models import (
    ChainParams,
    MaterialKspaceParams,
    analytic_band_max,
    device_mass_defect,
    device_perfect_chain,
    lead_blocks,
    interface_contacts,
    material_kspace_device,
    material_kspace_lead,
)

__version__ = "0.1.0"
