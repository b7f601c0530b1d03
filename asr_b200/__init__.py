"""asr_b200: B200-native (sm_100a) augmented-space recursion hot path of mavensgroup/asr.

The operator, chains and continued fractions run in the compiled library asr_b200/_lib/libasr_b200.so through its C ABI
(include/asr_b200.h); this package is the host-side mirror of the reference's operator interface.
"""
from . import crystal, lattices, synthetic
from ._lib import AsrError, LIB_PATH, lib
from .augcls import AugclsOp, Context, build_augcls_operator, default_context
from .chains import (ChainSpec, autotune, cf_species, chains_adjoint, chains_adjoint_ext, chains_proj, chains_run,
                     chains_run_device, chains_run_lanes, chains_run_lanes_device, dos_final, edc_green_blk, edc_green_proj,
                     lanczos, set_tuning, tuning)
from .contour import contour_moment, contour_nodes, contour_nodes_closed, contour_nodes_fermi, fermi_npole, gauss_legendre

__all__ = ["crystal", "lattices", "synthetic", "AsrError", "LIB_PATH", "lib", "AugclsOp", "Context", "build_augcls_operator",
           "default_context", "ChainSpec", "autotune", "cf_species", "chains_adjoint", "chains_adjoint_ext", "chains_proj",
           "edc_green_proj", "chains_run", "chains_run_device", "chains_run_lanes", "chains_run_lanes_device", "dos_final",
           "edc_green_blk", "lanczos", "set_tuning", "tuning", "contour_moment", "contour_nodes", "contour_nodes_closed",
           "contour_nodes_fermi", "fermi_npole", "gauss_legendre"]
