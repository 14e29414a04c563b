"""oscars_b200 -- the OSCARS radiation hot path on NVIDIA B200 (sm_100a).

``oscars_b200.sr.sr`` mirrors the ``oscars.sr.sr`` calls add_bfield_undulator, add_bfield_epu,
set_particle_beam, set_ctstartstop, calculate_trajectory, calculate_spectrum,
calculate_flux_rectangle and calculate_power_density_rectangle; the numerical work runs in
liboscars_b200.so behind the C ABI of include/oscars_b200.h.
"""
from . import sr  # noqa: F401

__all__ = ["sr"]
