"""Loader of the compiled C-ABI library (asr_b200/_lib/libasr_b200.so) with its ctypes signatures.

The library is built in place by ``python -c 'import __graft_entry__; __graft_entry__.build()'`` (or ``make -C
asr_b200/csrc``).  There is no fallback: every call of the package goes through this library, and importing a function
that needs it raises if it is missing.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libasr_b200.so")
_LIB = None

d_p = C.POINTER(C.c_double)
i_p = C.POINTER(C.c_int)
i64_p = C.POINTER(C.c_int64)
vp = C.c_void_p

ASR_OK, ASR_EINVAL, ASR_ENOMEM, ASR_ECUDA, ASR_ETIMEOUT, ASR_EEDGE, ASR_ESTATE = range(7)
MODE_PLAIN, MODE_EDC = 0, 1
TAILS = {"none": 0, "hull": 1, "bp": 2, "avg2": 3}
FP64, FP32 = 0, 1

# names of every exported entry point declared in include/asr_b200.h
EXPORTS = ["asr_version", "asr_last_error", "asr_ctx_create", "asr_ctx_destroy", "asr_ctx_sync", "asr_ctx_stats",
           "asr_ctx_set_stream", "asr_ctx_profile", "asr_ctx_hold_workspace", "asr_ctx_kernel_stats", "asr_ctx_kernel_stats_kind",
           "asr_ctx_launches", "asr_op_build", "asr_op_free", "asr_op_dims", "asr_op_export_tables",
           "asr_op_set_params", "asr_op_freeze_site", "asr_op_freeze_any", "asr_op_unfreeze", "asr_op_set_start",
           "asr_op_set_chi", "asr_op_set_class_conc", "asr_op_apply", "asr_op_rand_c", "asr_op_project_c",
           "asr_chains_run", "asr_chains_run_dev", "asr_cf_eval", "asr_cf_adjoint", "asr_chains_adjoint",
           "asr_cf_eval_noalloc", "asr_ed3_blocks", "asr_supercell_build", "asr_supercell_free",
           "asr_supercell_apply", "asr_kpm_moments", "asr_kpm_dos", "asr_sro_layout", "asr_gauss_legendre",
           "asr_contour_nodes", "asr_contour_nodes_closed", "asr_contour_nodes_fermi", "asr_contour_moment",
           "asr_op_build_targets", "asr_chains_proj", "asr_epi_blocks", "asr_autotune", "asr_op_tuning",
           "asr_op_set_tuning", "asr_op_hp_c", "asr_dos_final", "asr_chains_run_lanes", "asr_chains_run_lanes_dev",
           "asr_chains_adjoint_ext"]


class ChainGroup(C.Structure):
    """asr_chain_group of include/asr_b200.h."""
    _fields_ = [("c", d_p), ("d", d_p), ("o", d_p), ("e", d_p), ("pa", d_p), ("pb", d_p), ("frozen_sp", C.c_int),
                ("start_orb", C.c_int), ("nlev", C.c_int), ("reserved", C.c_int)]


class Ed3Group(C.Structure):
    """asr_ed3_group of include/asr_b200.h."""
    _fields_ = [("g", d_p), ("d", d_p), ("dc", d_p), ("dl", d_p), ("enu", d_p), ("o", d_p), ("p", d_p), ("central", C.c_int),
                ("start_orb", C.c_int), ("nlev", C.c_int), ("reserved", C.c_int)]


class AsrError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"asr_b200 error {code}: {msg}")
        self.code = code


def lib():
    """The loaded library; raises if it was not built (no CPU fallback exists)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"asr_b200: compiled library missing at {LIB_PATH}; run __graft_entry__.build()")
    L = C.CDLL(LIB_PATH)
    L.asr_version.restype = C.c_int
    L.asr_last_error.argtypes = [C.c_char_p, C.c_size_t]
    L.asr_ctx_create.argtypes = [C.c_int, C.POINTER(vp)]
    L.asr_ctx_destroy.argtypes = [vp]
    L.asr_ctx_sync.argtypes = [vp]
    L.asr_ctx_stats.argtypes = [vp, i64_p, i64_p, i64_p]
    L.asr_ctx_set_stream.argtypes = [vp, vp]
    L.asr_ctx_profile.argtypes = [vp, C.c_int]
    L.asr_ctx_hold_workspace.argtypes = [vp, C.c_int]
    L.asr_ctx_kernel_stats.argtypes = [vp, d_p, i64_p, d_p, d_p]
    L.asr_ctx_kernel_stats_kind.argtypes = [vp, C.c_int, d_p, i64_p, d_p, d_p]
    L.asr_ctx_launches.argtypes = [vp, i64_p]
    L.asr_op_build.argtypes = [vp, C.c_int, i_p, i_p, C.c_int, i_p, i_p, C.c_int, d_p, C.c_int, i_p, i_p, C.c_int, d_p, C.c_int,
                               C.c_int, C.c_int, i_p, i_p, d_p, C.c_int, C.c_int, d_p, C.POINTER(vp)]
    L.asr_op_build_targets.argtypes = L.asr_op_build.argtypes[:-1] + [i_p, C.c_int, i_p, i_p, C.POINTER(vp)]
    L.asr_op_free.argtypes = [vp]
    L.asr_op_dims.argtypes = [vp, i_p]
    L.asr_op_export_tables.argtypes = [vp] + [i_p] * 8 + [d_p, d_p, i_p, i_p]
    L.asr_op_set_params.argtypes = [vp, d_p, d_p, d_p, d_p]
    L.asr_op_freeze_site.argtypes = [vp, C.c_int, C.c_int]
    L.asr_op_freeze_any.argtypes = [vp, C.c_int, C.c_int, i_p]
    L.asr_op_hp_c.argtypes = [vp, d_p, d_p, C.c_int]
    L.asr_chains_adjoint_ext.argtypes = [vp, vp, C.POINTER(ChainGroup), C.c_int, d_p, C.c_int, d_p, C.c_double, C.c_int,
                                         C.c_int, C.c_int, C.c_int, d_p, i_p, d_p]
    L.asr_chains_run_lanes.argtypes = [vp, vp, C.POINTER(ChainGroup), C.c_int, i_p, d_p, C.c_int, C.c_double, C.c_int, C.c_int,
                                       C.c_int, d_p, i_p]
    L.asr_chains_run_lanes_dev.argtypes = [vp, vp, C.POINTER(ChainGroup), C.c_int, i_p, vp, C.c_int, C.c_double, C.c_int,
                                           C.c_int, C.c_int, vp]
    L.asr_dos_final.argtypes = [vp, vp, C.POINTER(ChainGroup), C.c_int, i_p, i_p, i_p, d_p, C.c_int, C.c_int, C.c_double,
                                C.c_double, C.c_double, C.c_int, C.c_double, C.c_int, C.c_int, d_p, d_p]
    L.asr_op_unfreeze.argtypes = [vp]
    L.asr_op_set_start.argtypes = [vp, C.c_int]
    L.asr_op_set_chi.argtypes = [vp, d_p]
    L.asr_op_set_class_conc.argtypes = [vp, C.c_int, d_p]
    L.asr_op_apply.argtypes = [vp, d_p, d_p, C.c_int]
    L.asr_op_rand_c.argtypes = [vp, d_p, d_p, d_p, C.c_int]
    L.asr_op_project_c.argtypes = [vp, d_p, C.c_int]
    L.asr_chains_run.argtypes = [vp, vp, C.POINTER(ChainGroup), C.c_int, d_p, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int,
                                 C.c_int, d_p, d_p, d_p, i_p]
    L.asr_chains_run_dev.argtypes = [vp, vp, C.POINTER(ChainGroup), C.c_int, vp, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int,
                                     C.c_int, vp, d_p, d_p, i_p]
    L.asr_cf_eval.argtypes = [vp, d_p, d_p, i_p, C.c_int, C.c_int, d_p, C.c_int, C.c_int, d_p, d_p, i64_p]
    L.asr_cf_adjoint.argtypes = [d_p, d_p, C.c_int, C.c_double, C.c_double, C.c_int, C.c_double, C.c_double, d_p, d_p, d_p]
    L.asr_cf_eval_noalloc.argtypes = [vp, d_p, d_p, i_p, C.c_int, C.c_int, d_p, C.c_int, C.c_int, d_p, i64_p]
    L.asr_chains_adjoint.argtypes = [vp, vp, C.POINTER(ChainGroup), C.c_int, d_p, C.c_int, d_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                     d_p, d_p]
    L.asr_chains_proj.argtypes = [vp, vp, C.POINTER(ChainGroup), C.c_int, d_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, i_p,
                                  i_p, d_p, d_p, d_p, d_p, i_p]
    L.asr_epi_blocks.argtypes = [vp, vp, C.POINTER(ChainGroup), d_p, d_p, C.c_int, d_p, C.c_int, C.c_int, C.c_int, C.c_int, d_p,
                                 i_p]
    L.asr_autotune.argtypes = [vp, vp, C.POINTER(ChainGroup), C.c_int, d_p, C.c_int, C.c_int, C.c_int, i_p, i_p, d_p]
    L.asr_op_tuning.argtypes = [vp, C.c_int, i_p, i_p, i_p, d_p]
    L.asr_op_set_tuning.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int]
    L.asr_ed3_blocks.argtypes = [vp, vp, C.POINTER(Ed3Group), C.c_int, d_p, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, d_p,
                                 i_p, d_p, d_p, d_p]
    L.asr_supercell_build.argtypes = [vp, C.c_int, C.c_int, i_p, i_p, C.c_int, d_p, d_p, d_p, d_p, d_p, d_p, C.POINTER(vp)]
    L.asr_supercell_free.argtypes = [vp]
    L.asr_supercell_apply.argtypes = [vp, d_p, d_p, C.c_int]
    L.asr_kpm_moments.argtypes = [vp, vp, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_int, C.c_int, d_p]
    L.asr_kpm_dos.argtypes = [d_p, C.c_int, C.c_double, C.c_double, d_p, C.c_int, d_p]
    L.asr_sro_layout.argtypes = [C.c_int, C.c_int, i_p, C.c_int, C.c_int, d_p, d_p, C.c_uint64, C.c_int, i_p, d_p]
    L.asr_gauss_legendre.argtypes = [C.c_int, d_p, d_p]
    L.asr_contour_nodes.argtypes = [C.c_double, C.c_double, C.c_int, C.c_double, d_p, d_p]
    L.asr_contour_nodes_closed.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, d_p, d_p]
    L.asr_contour_nodes_fermi.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, d_p, d_p]
    L.asr_contour_moment.argtypes = [d_p, d_p, d_p, C.c_int, C.c_double, C.c_int, d_p]
    _LIB = L
    return L


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    lib().asr_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(rc: int):
    if rc != ASR_OK:
        raise AsrError(rc, last_error())
