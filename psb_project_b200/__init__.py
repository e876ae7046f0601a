"""B200-native particle-simulation hot path of PSB_Project.

Uniform-grid neighbour search, SPH density and forces, the PCISPH
predictor-corrector loop and box walls, as hand-written sm_100a CUDA
kernels behind a C ABI (include/psb.h, lib/libpsb.so). This package is the
Python host side: the scene description and a ctypes binding.
"""
from .scene import (DEM, PCISPH, PROFILE_CONFIG, PROFILE_REF, WARM_LEARNED, WARM_PREVIOUS, WARM_ZERO, WCSPH, Block,
                    Scene, batch_scenes, c1_scenes, config_scene, dam_break, dashpot_from_restitution, dem_block, ref_scene,
                    sphere_shell)
from . import colliders, emitters
from .runtime import (CORRECTOR_LAUNCHES, CORRECTOR_PERSISTENT, BatchSimulation, FluidDemCoupling, IsoGrid, PsbError, Simulation, batch_positions, iso_grid, lattice, lib,
                      mlp_init_weights, mlp_unpack, scene_positions, write_obj, write_txt, write_vol, write_xml)

__all__ = ["Scene", "Block", "Simulation", "PsbError", "config_scene", "dam_break", "ref_scene", "lattice",
           "scene_positions", "lib", "PCISPH", "WCSPH", "PROFILE_REF", "PROFILE_CONFIG", "WARM_ZERO",
           "WARM_PREVIOUS", "WARM_LEARNED", "mlp_init_weights", "mlp_unpack", "DEM", "dem_block",
           "dashpot_from_restitution", "IsoGrid", "iso_grid", "BatchSimulation", "batch_positions", "batch_scenes", "sphere_shell",
           "write_txt", "write_xml", "write_vol", "write_obj", "c1_scenes", "FluidDemCoupling", "colliders", "emitters",
           "CORRECTOR_LAUNCHES", "CORRECTOR_PERSISTENT"]
