"""Loader for libaw_b200.so, the C ABI declared in include/aw_b200.h.

The library is built in-tree (``atlaswerks_b200/csrc/Makefile``) for sm_100a.
There is no fallback: if the library is missing or fails to load, every
entry point raises.
"""
from __future__ import annotations

import ctypes
import os
import re
import subprocess
from typing import List

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
LIB_PATH = os.path.join(PKG, "libaw_b200.so")
HEADER_DIR = os.path.join(ROOT, "include")

_lib = None


class AwError(RuntimeError):
    """A C-ABI call returned non-zero; the message is aw_last_error()."""


def build(force: bool = False) -> str:
    """Compile the CUDA library for sm_100a (nvcc cross-compiles without a GPU)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-j8", "-C", os.path.join(PKG, "csrc")], check=True)
    return LIB_PATH


_c = ctypes
_fp = ctypes.c_void_p
_i = ctypes.c_int
_f = ctypes.c_float
_d = ctypes.c_double

# argument types of every entry point, in header order
SIGNATURES = {
    "aw_last_error": ([], ctypes.c_char_p),
    "aw_version": ([], ctypes.c_char_p),
    "aw_apply": ([_fp] * 5 + [_i] * 3 + [_f, _fp], _i),
    "aw_gradient": ([_fp] * 4 + [_i] * 3 + [_d] * 3 + [_i, _fp], _i),
    "aw_compose_hv": ([_fp] * 9 + [_i] * 3 + [_d] * 3 + [_f, _i, _i, _fp], _i),
    "aw_compose_vh": ([_fp] * 9 + [_i] * 3 + [_d] * 3 + [_f, _i, _i, _fp], _i),
    "aw_splat": ([_fp] * 5 + [_i] * 3 + [_f, _fp], _i),
    "aw_splat_static_fits": ([_i, _i, _i], _i),
    "aw_splat_static": ([_fp] * 5 + [_i] * 3 + [_f, _fp], _i),
    "aw_downsample": ([_fp, _i, _i, _i, _d, _d, _d, _fp, _i, _i, _i, _fp], _i),
    "aw_resample_image": ([_fp, _i, _i, _i, _d, _d, _d, _fp, _i, _i, _i, _d, _d, _d, _fp], _i),
    "aw_upsample_hfield": ([_fp] * 3 + [_i] * 3 + [_fp] * 3 + [_i] * 4 + [_fp], _i),
    "aw_fluid_create": ([_i] * 3 + [_d] * 3 + [_f] * 3 + [_fp], _i),
    "aw_fluid_apply": ([_fp] * 4 + [_i, _fp], _i),
    "aw_fluid_destroy": ([_fp], _i),
    "aw_fluid_get_shapes": ([_fp, _fp], _i),
    "aw_fluid_set_shapes": ([_fp, _i, _i, _i], _i),
    "aw_fluid_autotune": ([_fp, _fp], _i),
    "aw_fluid_status": ([_fp, _fp, _fp], _i),
    "aw_fluid_wait_selftest": ([_fp, _i, _fp], _i),
    "aw_greedy_status": ([_fp, _fp, _fp], _i),
    "aw_ldmm_status": ([_fp, _fp, _fp], _i),
    "aw_greedy_create": ([_i] * 3 + [_d] * 3 + [_f] * 4 + [_fp], _i),
    "aw_greedy_destroy": ([_fp], _i),
    "aw_greedy_set_step": ([_fp, _f], _i),
    "aw_greedy_get_step": ([_fp, _fp], _i),
    "aw_greedy_set_auto_step_reduce": ([_fp, _i], _i),
    "aw_greedy_set_staged_update": ([_fp, _i], _i),
    "aw_greedy_last_energy": ([_fp, _fp], _i),
    "aw_identity": ([_fp, _fp, _fp, _i, _i, _i, _fp], _i),
    "aw_warmstart_param_floats": ([], ctypes.c_size_t),
    "aw_warmstart_create": ([_i] * 6 + [_fp, ctypes.c_size_t, ctypes.c_float, _fp], _i),
    "aw_warmstart_destroy": ([_fp], _i),
    "aw_warmstart_predict": ([_fp] * 7, _i),
    "aw_warmstart_register": ([_fp, _fp, _fp, ctypes.c_double, _i, _i, _i] + [_fp] * 6, _i),
    "aw_greedy_set_fast_interpolation": ([_fp, _i], _i),
    "aw_greedy_set_fused_update": ([_fp, _i], _i),
    "aw_greedy_update_tile": ([_fp, _i, _fp], _i),
    "aw_greedy_iterate": ([_fp] * 15 + [_i, _fp], _i),
    "aw_greedy_run": ([_fp] * 15 + [_i, _i, _fp], _i),
    "aw_greedy_profile": ([_fp] * 15 + [_i, _fp, _fp], _i),
    "aw_greedy_get_energies": ([_fp, _fp, _i, _fp], _i),
    "aw_atlas_create": ([_i] * 3 + [_d] * 3 + [_f] * 4 + [_i, _fp], _i),
    "aw_atlas_destroy": ([_fp], _i),
    "aw_atlas_set_subject": ([_fp, _i, _fp, _i, _i, _i, _f], _i),
    "aw_atlas_field": ([_fp, _i, _fp, _fp, _fp], _i),
    "aw_atlas_mean_buffer": ([_fp, _fp], _i),
    "aw_atlas_compute_mean": ([_fp, _fp], _i),
    "aw_atlas_iterate": ([_fp, _i, _i, _fp], _i),
    "aw_atlas_get_step": ([_fp, _i, _fp], _i),
    "aw_atlas_get_energies": ([_fp, _i, _fp, _i, _fp], _i),
    "aw_ldmm_use_orig_gradient_calc": ([_fp, _i], _i),
    "aw_ldmm_create": ([_i] * 3 + [_d] * 3 + [_f] * 3 + [_i, _f, _f, _fp], _i),
    "aw_ldmm_destroy": ([_fp], _i),
    "aw_ldmm_set_step": ([_fp, _f], _i),
    "aw_ldmm_get_step": ([_fp, _fp], _i),
    "aw_ldmm_iterate": ([_fp] * 4 + [_i, _fp], _i),
    "aw_ldmm_alphas": ([_fp, _fp, _fp, _fp, _fp, _fp], _i),
    "aw_ldmm_run": ([_fp] * 4 + [_i, _i, _fp], _i),
    "aw_ldmm_get_energies": ([_fp, _fp, _i, _fp], _i),
    "aw_ldmm_i1_at_0": ([_fp] * 6, _i),
    "aw_ldmm_shoot_iterate": ([_fp] * 7, _i),
    "aw_ldmm_adshoot_iterate": ([_fp] * 7, _i),
    "aw_ldmm_adshoot_final_maps": ([_fp] * 4, _i),
    "aw_ldmm_get_vec_energies": ([_fp, _fp, _i, _fp], _i),
    "aw_ldmm_atlas_accumulate": ([_fp] * 4 + [ctypes.c_float, ctypes.c_long, _fp], _i),
    "aw_ldmm_set_vector_energy": ([_fp, _i], _i),
    "aw_ldmm_geodesic_shoot": ([_fp] * 7, _i),
    "aw_ldmm_velshoot_iterate": ([_fp] * 6 + [_i, _fp], _i),
    "aw_ldmm_get_vec_step_energies": ([_fp, _fp, _i], _i),
    "aw_ldmm_atlas_voxel_median": ([_fp, _i, _i, _i, _i, _i, _fp, _fp], _i),
    "aw_ldmm_atlas_normalize": ([_fp, _fp, ctypes.c_long, _fp], _i),
    "aw_nn_conv3d_scratch_floats": ([_i] * 7, ctypes.c_size_t),
    "aw_nn_conv3d_direct_planes": ([_i] * 7, _i),
    "aw_nn_set_gemm_only": ([_i], None),
    "aw_nn_conv3d_fwd": ([_fp] + [_i] * 5 + [_fp, _fp, _i, _i, _i, _fp, _fp, _fp,
                                           ctypes.c_size_t, _fp], _i),
    "aw_nn_conv3d_dgrad": ([_fp] + [_i] * 5 + [_fp, _i, _i, _fp, _fp, _fp, ctypes.c_size_t,
                                             _fp], _i),
    "aw_nn_wgrad_scratch_floats": ([_i, _i, _i, _i], ctypes.c_size_t),
    "aw_nn_conv3d_wgrad": ([_fp, _fp] + [_i] * 8 + [_fp, _fp, _fp], _i),
    "aw_nn_bias_scratch_floats": ([ctypes.c_long, _i], ctypes.c_size_t),
    "aw_nn_bias_grad": ([_fp, ctypes.c_long, _i, _fp, _fp, _fp], _i),
    "aw_nn_pool": ([_fp] + [_i] * 5 + [_fp, _i, _fp, _fp, _fp], _i),
    "aw_nn_upsample": ([_fp] + [_i] * 5 + [_fp, _i, _i, _i, _fp], _i),
    "aw_nn_slice": ([_fp, _i, _i, _fp, _i, _i, _i, ctypes.c_long, _i, _fp], _i),
    "aw_nn_pack_pair": ([_fp, _fp, ctypes.c_long, _fp, _fp], _i),
    "aw_nn_mse_scratch_doubles": ([ctypes.c_long], ctypes.c_size_t),
    "aw_nn_mse": ([_fp, _fp, ctypes.c_long, _fp, _fp, _fp, _fp], _i),
    "aw_nn_adam": ([_fp, _fp, _fp, _fp, ctypes.c_long, _f, _f, _f, _f, _i, _fp], _i),
    "aw_nn_weights_bf16": ([_fp, _i, _i, _i, _fp, _fp, _fp], _i),
    "aw_nn_displacement_to_h": ([_fp, _i, _i, _i, _fp, _fp, _fp, _fp], _i),
    "aw_nn_status": ([_fp], _i),
}


def header_symbols() -> List[str]:
    """Every function name declared in include/*.h."""
    names = []
    for fn in sorted(os.listdir(HEADER_DIR)):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(HEADER_DIR, fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(aw_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def lib() -> ctypes.CDLL:
    """The loaded library (raises if it cannot be loaded)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise AwError(f"{LIB_PATH} is missing: build it with `make -C atlaswerks_b200/csrc` "
                          "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != 0:
        raise AwError(lib().aw_last_error().decode())
