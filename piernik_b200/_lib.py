"""ctypes binding of libpiernik_b200.so (declarations in include/piernik_b200.h).

The shared library is built in-tree by ``piernik_b200.build`` and is required:
there is no CPU fallback, and loading fails with an explicit error when the
library is missing or cannot be opened.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libpiernik_b200.so")

PK_OK = 0
PK_CFL = {"none": 0, "warn": 1, "redo": 2, "repeat": 2, "flex": 3, "flexible": 3, "auto": 4, "adaptive": 4}
ERRORS = {-1: "PK_E_ARG", -2: "PK_E_CUDA", -3: "PK_E_NOMEM", -4: "PK_E_UNSUPPORTED", -5: "PK_E_STATE",
          -6: "PK_E_DTMIN"}
PK_FLUID = {"ion": 0, "neu": 1, "dst": 2}
PK_LIM = {"vanleer": 0, "minmod": 1, "moncen": 2, "superbee": 3}
PK_LAYOUT_FORTRAN, PK_LAYOUT_SOA = 0, 1
PK_EULER, PK_RK2_1, PK_RK2_2 = 10000, 10001, 10002
PK_ST_DN_NEGATIVE, PK_ST_EI_NEGATIVE, PK_ST_TIMEOUT = 1, 2, 4
PK_VARIANT_STAGED = 7
PK_ARITH = {"bitexact": 0, "fma": 1}

# every symbol include/piernik_b200.h declares
EXPORTS = (
    "pk_config_default", "pk_create", "pk_destroy", "pk_last_error", "pk_abi_version", "pk_block_add",
    "pk_upload", "pk_download", "pk_solve_cg", "pk_fill_guards", "pk_sweep", "pk_glm_damp",
    "pk_timestep_raw", "pk_time_step", "pk_fluid_update", "pk_run", "pk_get_time_state",
    "pk_set_time_state", "pk_status", "pk_sync", "pk_set_tile", "pk_stream", "pk_profile_enable",
    "pk_profile_read", "pk_tile_variants", "pk_set_batch", "pk_set_refined_launch", "pk_use_graph", "pk_set_arithmetic",
    "pk_upload_device", "pk_download_device", "pk_adjoint_set", "pk_adjoint_get", "pk_adjoint_sweep",
    "pk_grad_forward", "pk_grad_backward", "pk_grad_release",
    "pk_timestep_raw_noalloc", "pk_set_adjoint_tile", "pk_set_domain", "pk_block_place",
    "pk_block_remote", "pk_halo_peers", "pk_halo_sizes", "pk_halo_pack", "pk_halo_unpack", "pk_set_comm",
    "pk_halo_sizes_dir", "pk_halo_pack_dir", "pk_halo_unpack_dir",
    "pk_set_instances", "pk_get_instance_state", "pk_set_instance_state", "pk_block_place_level",
    "pk_set_stage_variant", "pk_fp64_peak", "pk_restrict",
    "pk_prolong_block",
    "pk_block_remove",
    "pk_mark_refinement",
    "pk_refine_map",
    "pk_refine_candidates",
)

HALO_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_int32)
REDUCE_FN = C.CFUNCTYPE(C.c_double, C.c_void_p, C.c_double, C.c_int32)


class PkConfig(C.Structure):
    _fields_ = [
        ("nfluids", C.c_int32),
        ("fluid_kind", C.c_int32 * 3),
        ("gamma", C.c_double * 3),
        ("magnetic", C.c_int32),
        ("limiter", C.c_int32),
        ("limiter_b", C.c_int32),
        ("use_smalld", C.c_int32),
        ("use_smallei", C.c_int32),
        ("disallow_negatives", C.c_int32),
        ("smalld", C.c_double),
        ("smallei", C.c_double),
        ("cfl", C.c_double),
        ("cfl_glm", C.c_double),
        ("glm_alpha", C.c_double),
        ("integration_order", C.c_int32),
        ("nb", C.c_int32),
        ("dt_initial", C.c_double),
        ("dt_max_grow", C.c_double),
        ("dt_min", C.c_double),
        ("dt_max", C.c_double),
        ("tend", C.c_double),
        ("skip_sweep", C.c_int32 * 3),
        ("cflcontrol", C.c_int32),
        ("cfl_max", C.c_double),
        ("dt_shrink", C.c_double),
        ("max_redostep_attempts", C.c_int32),
        ("interpolation", C.c_int32),
        ("w_epsilon", C.c_double),
        ("solver", C.c_int32),
        ("ord_fluid_prolong", C.c_int32),
        ("ord_mag_prolong", C.c_int32),
        ("ch_grid", C.c_int32),
        ("use_eglm", C.c_int32),
    ]


URC_THRESHOLD, URC_GRAD, URC_RELGRAD, URC_LOECHNER = 0, 1, 2, 3
URC_METHODS = {"threshold": URC_THRESHOLD, "grad": URC_GRAD, "relgrad": URC_RELGRAD, "Loechner": URC_LOECHNER,
               "second_order": URC_LOECHNER, "d2": URC_LOECHNER}


class PkUrc(C.Structure):
    _fields_ = [("method", C.c_int32), ("field", C.c_int32), ("thr", C.c_double), ("aux", C.c_double)]


class PkTimeState(C.Structure):
    _fields_ = [
        ("t", C.c_double),
        ("dt", C.c_double),
        ("dt_old", C.c_double),
        ("c_all", C.c_double),
        ("chspeed", C.c_double),
        ("nstep", C.c_int32),
        ("dt_full", C.c_double),
        ("c_all_old", C.c_double),
        ("dt_cur_shrink", C.c_double),
        ("stepcfl", C.c_double),
        ("t_saved", C.c_double),
        ("nstep_saved", C.c_int32),
        ("tstep_attempt", C.c_int32),
        ("repeat_step", C.c_int32),
        ("redone", C.c_int32),
        ("cfl_c", C.c_double),
    ]


class PkError(RuntimeError):
    pass


_lib = None


def load(path: str = LIBPATH):
    """Open the CUDA library; raises PkError when it is absent (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise PkError(f"{path} is missing: build it with piernik_b200.build.build() "
                      "(the sweep has no CPU implementation)")
    L = C.CDLL(path)
    for name in EXPORTS:
        getattr(L, name)
    H = C.c_void_p
    dp = C.POINTER(C.c_double)
    L.pk_config_default.argtypes = [C.POINTER(PkConfig)]
    L.pk_config_default.restype = None
    L.pk_create.argtypes = [C.POINTER(PkConfig), C.POINTER(H)]
    L.pk_destroy.argtypes = [H]
    L.pk_last_error.argtypes = [H]
    L.pk_last_error.restype = C.c_char_p
    L.pk_block_add.argtypes = [H, C.POINTER(C.c_int32), dp, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
    L.pk_upload.argtypes = [H, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32]
    L.pk_download.argtypes = [H, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32]
    L.pk_solve_cg.argtypes = [H, C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_double]
    L.pk_fill_guards.argtypes = [H]
    L.pk_sweep.argtypes = [H, C.c_int32, C.c_double, C.c_double]
    L.pk_glm_damp.argtypes = [H, C.c_double]
    L.pk_timestep_raw.argtypes = [H, dp, dp]
    L.pk_time_step.argtypes = [H, dp]
    L.pk_fluid_update.argtypes = [H]
    L.pk_run.argtypes = [H, C.c_int32]
    L.pk_get_time_state.argtypes = [H, C.POINTER(PkTimeState)]
    L.pk_set_time_state.argtypes = [H, C.POINTER(PkTimeState)]
    L.pk_status.argtypes = [H, C.POINTER(C.c_uint32)]
    L.pk_sync.argtypes = [H]
    L.pk_set_tile.argtypes = [H, C.c_int32, C.c_int32, C.c_int32, C.c_int32]
    L.pk_tile_variants.argtypes = [C.POINTER(C.c_int32)] * 3
    L.pk_set_batch.argtypes = [H, C.c_int32, C.c_int32, C.c_int32]
    L.pk_set_refined_launch.argtypes = [H, C.c_int32]
    L.pk_use_graph.argtypes = [H, C.c_int32]
    L.pk_set_arithmetic.argtypes = [H, C.c_int32]
    L.pk_set_instances.argtypes = [H, C.c_int32]
    L.pk_block_place_level.argtypes = [H, C.c_int32, C.c_int32, C.POINTER(C.c_int64)]
    L.pk_set_stage_variant.argtypes = [H, C.c_int32]
    L.pk_fp64_peak.argtypes = [C.POINTER(C.c_double)]
    L.pk_restrict.argtypes = [H]
    L.pk_prolong_block.argtypes = [H, C.c_int32]
    L.pk_block_remove.argtypes = [H, C.c_int32]
    L.pk_mark_refinement.argtypes = [H, C.POINTER(PkUrc), C.c_int32, C.POINTER(C.c_int32)]
    L.pk_refine_map.argtypes = [H, C.c_int32, C.c_void_p]
    L.pk_refine_candidates.argtypes = [H, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int64), C.c_int32,
                                       C.POINTER(C.c_int32)]
    L.pk_get_instance_state.argtypes = [H, C.c_int32, C.POINTER(PkTimeState)]
    L.pk_set_instance_state.argtypes = [H, C.c_int32, C.POINTER(PkTimeState)]
    L.pk_upload_device.argtypes = [H, C.c_int32, C.c_void_p]
    L.pk_download_device.argtypes = [H, C.c_int32, C.c_void_p]
    L.pk_adjoint_set.argtypes = [H, C.c_int32, C.c_void_p, C.c_int32]
    L.pk_adjoint_get.argtypes = [H, C.c_int32, C.c_void_p, C.c_int32]
    L.pk_adjoint_sweep.argtypes = [H, C.c_int32, C.c_double, C.c_double]
    L.pk_grad_forward.argtypes = [H, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p]
    L.pk_grad_backward.argtypes = [H]
    L.pk_grad_release.argtypes = [H]
    L.pk_set_adjoint_tile.argtypes = [H, C.c_int32, C.c_int32, C.c_int32]
    L.pk_set_domain.argtypes = [H, C.POINTER(C.c_int64), C.POINTER(C.c_int32)]
    L.pk_block_place.argtypes = [H, C.c_int32, C.POINTER(C.c_int64)]
    L.pk_block_remote.argtypes = [H, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int64)]
    L.pk_halo_peers.argtypes = [H, C.POINTER(C.c_int32), C.c_int32, C.POINTER(C.c_int32)]
    L.pk_halo_sizes.argtypes = [H, C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    L.pk_halo_pack.argtypes = [H, C.c_int32, C.c_void_p]
    L.pk_halo_sizes_dir.argtypes = [H, C.c_int32, C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    L.pk_halo_pack_dir.argtypes = [H, C.c_int32, C.c_int32, C.c_void_p]
    L.pk_halo_unpack_dir.argtypes = [H, C.c_int32, C.c_int32, C.c_void_p]
    L.pk_halo_unpack.argtypes = [H, C.c_int32, C.c_void_p]
    L.pk_set_comm.argtypes = [H, C.c_void_p, C.c_void_p, C.c_void_p]
    L.pk_timestep_raw_noalloc.argtypes = [C.POINTER(PkConfig), C.c_int32, C.POINTER(C.c_int32),
                                          C.POINTER(C.c_double), C.POINTER(C.c_void_p), C.c_void_p,
                                          C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_char_p, C.c_int32]
    L.pk_stream.argtypes = [H]
    L.pk_stream.restype = C.c_void_p
    L.pk_profile_enable.argtypes = [H, C.c_int32]
    L.pk_profile_read.argtypes = [H, C.POINTER(C.c_int64), C.POINTER(C.c_int64), dp]
    _lib = L
    return L
