"""ctypes binding of the METHOD-B200 C ABI (include/method_b200.h).

The library is built in-tree (``python -m method_b200.build``) and loaded from
this package directory.  There is no fallback: if the library or a CUDA device
is missing, the calls fail with an exception.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmethod_b200.so")

STATUS = {0: "MTH_OK", 1: "MTH_ERR_C2P", 2: "MTH_ERR_IMPLICIT", 3: "MTH_ERR_INVALID",
          4: "MTH_ERR_CUDA"}

# Exported symbols of include/method_b200.h, in declaration order.
SYMBOLS = [
    "mth_create", "mth_destroy", "mth_last_error", "mth_get_dims", "mth_set_prims",
    "mth_upload", "mth_download", "mth_apply_bcs", "mth_prims_to_all", "mth_c2p",
    "mth_flux_F", "mth_source", "mth_flux_vector", "mth_c2p_cells", "mth_step", "mth_update_time", "mth_evolve",
    "mth_step_parts", "mth_step_part", "mth_next_dt", "mth_advance_time", "mth_halo_bytes",
    "mth_halo_pack", "mth_halo_unpack", "mth_halo_outflow", "mth_sync",
    "mth_get_stats", "mth_reset_stats", "mth_step_host", "mth_step_host_bytes", "mth_pin_host",
    "mth_unpin_host",
    "mth_set_stream", "mth_profile_step", "mth_mlp_train", "mth_mlp_grad", "mth_mlp_forward",
    "mth_mlp_forward_tc",
    "mth_mlp_make_pairs", "mth_mlp_make_pairs_srrmhd", "mth_set_mlp", "mth_c2p_batch", "mth_c2p_ctx_create", "mth_c2p_ctx_destroy",
    "mth_c2p_ctx_set_mlp", "mth_c2p_ctx_run", "mth_c2p_ctx_stats", "mth_c2p_srmhd_noalloc",
    "mth_save_text", "mth_device_state", "mth_ensemble_create", "mth_ensemble_destroy",
    "mth_ensemble_last_error", "mth_ensemble_set_prims", "mth_ensemble_download",
    "mth_ensemble_set_mlp", "mth_ensemble_set_mlp_srrmhd", "mth_ensemble_set_stream", "mth_ensemble_autotune", "mth_ensemble_tuning", "mth_ensemble_step",
    "mth_ensemble_profile", "mth_ensemble_sync", "mth_ensemble_stats", "mth_ensemble_info",
]

MLP_NPARAM = 9928
MLP_NSTAT = 20


class MlpTrainConfig(C.Structure):
    _fields_ = [("seed", C.c_ulonglong), ("n_samples", C.c_longlong), ("iterations", C.c_int),
                ("batch", C.c_int), ("lr", C.c_float), ("gamma", C.c_double), ("model", C.c_int)]


class C2PBatchStats(C.Structure):
    _fields_ = [("cells", C.c_longlong), ("iterations", C.c_longlong),
                ("unconverged", C.c_longlong), ("fallbacks", C.c_longlong)]


class Config(C.Structure):
    _fields_ = [
        ("model", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("xmin", C.c_double), ("xmax", C.c_double), ("ymin", C.c_double),
        ("ymax", C.c_double), ("zmin", C.c_double), ("zmax", C.c_double),
        ("endTime", C.c_double), ("cfl", C.c_double), ("Ng", C.c_int),
        ("gamma", C.c_double), ("sigma", C.c_double), ("cp", C.c_double),
        ("weno_order", C.c_int), ("bcs", C.c_int), ("integrator", C.c_int),
        ("precision", C.c_int), ("guess", C.c_int), ("device", C.c_int),
        ("functional_sigma", C.c_int), ("sigma_exp", C.c_double),
        ("x_slab", C.c_int), ("x_global_nx", C.c_int), ("x_offset", C.c_int), ("regime", C.c_int),
        ("sigma_crossover", C.c_double), ("sigma_span", C.c_double),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("c2p_cells", C.c_longlong), ("c2p_evals", C.c_longlong),
        ("c2p_unconverged", C.c_longlong), ("implicit_cells", C.c_longlong),
        ("implicit_evals", C.c_longlong), ("implicit_failed", C.c_longlong),
        ("steps", C.c_longlong), ("t", C.c_double), ("dt", C.c_double), ("iters", C.c_int),
        ("c2p_fallbacks", C.c_longlong), ("implicit_fallbacks", C.c_longlong),
    ]


class EnsembleTuning(C.Structure):
    _fields_ = [("tile_height", C.c_int * 3), ("flux_ctas", C.c_int * 3), ("cell_ctas", C.c_int),
                ("default_ms", C.c_float), ("tuned_ms", C.c_float)]


class KernelTime(C.Structure):
    _fields_ = [("name", C.c_char * 40), ("launches", C.c_int), ("total_ms", C.c_double),
                ("bytes_per_launch", C.c_double)]


_LIB = None


def load():
    """Loads libmethod_b200.so and declares the prototypes."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing; build it with `python -m method_b200.build`")
    L = C.CDLL(LIB_PATH)
    H = C.c_void_p
    D = C.POINTER(C.c_double)
    L.mth_create.argtypes = [C.POINTER(Config), C.POINTER(H)]
    L.mth_destroy.argtypes = [H]
    L.mth_last_error.argtypes = [H]
    L.mth_last_error.restype = C.c_char_p
    L.mth_get_dims.argtypes = [H, C.POINTER(C.c_int)]
    L.mth_set_prims.argtypes = [H, D]
    L.mth_upload.argtypes = [H, D, D, D]
    L.mth_download.argtypes = [H, D, D, D]
    for n in ("mth_apply_bcs", "mth_prims_to_all", "mth_c2p", "mth_evolve", "mth_sync",
              "mth_reset_stats"):
        getattr(L, n).argtypes = [H]
    L.mth_flux_F.argtypes = [H, D]
    L.mth_source.argtypes = [H, D]
    L.mth_flux_vector.argtypes = [H, C.c_int, D]
    L.mth_c2p_cells.argtypes = [C.c_int, C.c_double, C.c_double, C.c_longlong, D, D, D,
                                C.c_double, C.c_int]
    L.mth_step.argtypes = [H, C.c_double]
    L.mth_update_time.argtypes = [H, C.c_int]
    L.mth_step_parts.argtypes = [H, C.POINTER(C.c_int)]
    L.mth_step_part.argtypes = [H, C.c_double, C.c_int]
    L.mth_next_dt.argtypes = [H, D]
    L.mth_advance_time.argtypes = [H, C.c_double]
    L.mth_halo_bytes.argtypes = [H, C.POINTER(C.c_ulonglong)]
    L.mth_halo_pack.argtypes = [H, C.c_int, C.c_int, C.c_void_p]
    L.mth_halo_unpack.argtypes = [H, C.c_int, C.c_int, C.c_void_p]
    L.mth_halo_outflow.argtypes = [H, C.c_int, C.c_int]
    L.mth_get_stats.argtypes = [H, C.POINTER(Stats)]
    L.mth_device_state.argtypes = [H, C.POINTER(D), C.POINTER(D), C.POINTER(D)]
    L.mth_save_text.argtypes = [H, C.c_char_p, C.c_char_p, C.c_int]
    L.mth_step_host.argtypes = [H, D, D, D, C.c_double]
    L.mth_step_host_bytes.argtypes = [H, C.POINTER(C.c_ulonglong), C.POINTER(C.c_ulonglong)]
    L.mth_pin_host.argtypes = [C.c_void_p, C.c_ulonglong]
    L.mth_unpin_host.argtypes = [C.c_void_p]
    L.mth_set_stream.argtypes = [H, C.c_void_p]
    L.mth_profile_step.argtypes = [H, C.c_double, C.c_int, C.POINTER(KernelTime), C.c_int,
                                   C.POINTER(C.c_int)]
    F = C.POINTER(C.c_float)
    L.mth_mlp_train.argtypes = [C.POINTER(MlpTrainConfig), F, F, F, C.c_int]
    L.mth_mlp_grad.argtypes = [F, C.c_int, F, F, F, F, C.c_int]
    L.mth_mlp_forward.argtypes = [F, C.c_int, F, F, C.c_int]
    L.mth_mlp_forward_tc.argtypes = [F, C.c_int, F, F, C.c_int]
    L.mth_mlp_make_pairs.argtypes = [C.c_longlong, C.c_ulonglong, C.c_double, F, F, D, D, C.c_int]
    L.mth_mlp_make_pairs_srrmhd.argtypes = [C.c_longlong, C.c_ulonglong, C.c_double, F, F, D, D,
                                            C.c_int]
    L.mth_set_mlp.argtypes = [H, F, F]
    L.mth_c2p_batch.argtypes = [C.c_double, C.c_longlong, C.c_void_p, C.c_void_p, C.c_void_p,
                                C.c_int, C.c_int, F, F, C.c_void_p, C.POINTER(C2PBatchStats)]
    L.mth_c2p_ctx_create.argtypes = [C.c_longlong, C.c_int, C.POINTER(C.c_void_p)]
    L.mth_c2p_ctx_destroy.argtypes = [C.c_void_p]
    L.mth_c2p_ctx_set_mlp.argtypes = [C.c_void_p, F, F]
    L.mth_c2p_ctx_run.argtypes = [C.c_void_p, C.c_double, C.c_longlong, C.c_void_p, C.c_void_p,
                                  C.c_void_p, C.c_int, C.c_int, C.c_void_p]
    L.mth_c2p_ctx_stats.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C2PBatchStats)]
    L.mth_c2p_srmhd_noalloc.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                         C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.POINTER(C.c_longlong)]
    E = C.c_void_p
    L.mth_ensemble_create.argtypes = [C.POINTER(Config), C.c_int, C.POINTER(E)]
    L.mth_ensemble_destroy.argtypes = [E]
    L.mth_ensemble_last_error.argtypes = [E]
    L.mth_ensemble_set_prims.argtypes = [E, C.c_int, D]
    L.mth_ensemble_download.argtypes = [E, C.c_int, D, D, D]
    L.mth_ensemble_set_mlp.argtypes = [E, F, F]
    L.mth_ensemble_set_mlp_srrmhd.argtypes = [E, F, F]
    L.mth_ensemble_set_stream.argtypes = [E, C.c_void_p]
    L.mth_ensemble_autotune.argtypes = [E, C.c_int, C.POINTER(C.c_int)]
    L.mth_ensemble_tuning.argtypes = [E, C.POINTER(EnsembleTuning)]
    L.mth_ensemble_step.argtypes = [E, C.c_int]
    L.mth_ensemble_profile.argtypes = [E, C.c_int, C.POINTER(KernelTime), C.c_int,
                                       C.POINTER(C.c_int)]
    L.mth_ensemble_sync.argtypes = [E]
    L.mth_ensemble_stats.argtypes = [E, C.c_int, C.POINTER(Stats)]
    L.mth_ensemble_info.argtypes = [E, C.POINTER(C.c_longlong), C.POINTER(C.c_int)]
    for n in SYMBOLS:
        if n not in ("mth_last_error", "mth_ensemble_last_error"):
            getattr(L, n).restype = C.c_int
    L.mth_ensemble_last_error.restype = C.c_char_p
    _LIB = L
    return L
