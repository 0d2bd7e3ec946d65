"""ising_b200: B200 (sm_100a) Heisenberg Metropolis / parallel-tempering hot path.

A drop-in for the Monte Carlo path of SamuelJosephs/ISING: local field and dE, the
colour-class sweep, replica exchange and the winding-number reduction, behind the C-ABI
of include/ising_gpu.h (libisinggpu.so).  Importing this package loads the CUDA library;
there is no CPU fallback.
"""
from . import _lib
from ._lib import IsingError, Params, load
from .api import (ChainMesh, Ensembles, ParallelTempering, ProposalNet, bcc_unit_cell, calculate_heisenberg_energy,
                  calculate_skyrmion_number, calculate_winding_density_interpolated, calculate_winding_number2,
                  calculate_winding_number_density, chain_mesh_statistics, chain_mesh_statistics_full,
                  compute_skyrmion_distribution, demag_field, write_demagnetisation_field_to_file, frame_filename, gaussian_filter_2d, interpolation_scale,
                  set_interpolation_scale, write_frame_info, write_winding_number_density_interpolated,
                  skyrmion_number_from_density,
                  hyper_kagome_unit_cell, local_energy_batch, make_chain_mesh, metropolis_mcs, observables,
                  params, pt_file_tag, reference_params, sc_unit_cell, temperature_ladder,
                  total_heisenberg_energy, unit_cell, winding_all_slices, winding_density_all_slices,
                  write_pt_data_csv, write_spins_to_file, write_winding_number_density)

__all__ = ["ChainMesh", "Ensembles", "ParallelTempering", "ProposalNet", "IsingError", "Params", "load", "bcc_unit_cell",
           "calculate_skyrmion_number", "calculate_winding_density_interpolated", "chain_mesh_statistics_full",
           "compute_skyrmion_distribution", "demag_field", "write_demagnetisation_field_to_file", "frame_filename", "gaussian_filter_2d", "interpolation_scale",
           "set_interpolation_scale", "write_frame_info", "write_winding_number_density_interpolated",
           "skyrmion_number_from_density",
           "calculate_heisenberg_energy", "calculate_winding_number2", "calculate_winding_number_density",
           "chain_mesh_statistics", "hyper_kagome_unit_cell", "local_energy_batch", "make_chain_mesh",
           "metropolis_mcs", "observables", "params", "pt_file_tag", "reference_params", "sc_unit_cell",
           "temperature_ladder", "total_heisenberg_energy", "unit_cell", "winding_all_slices",
           "winding_density_all_slices", "write_pt_data_csv", "write_spins_to_file", "write_winding_number_density"]

load()
