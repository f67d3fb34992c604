"""ctypes bindings of the C ABI in include/bfvm.h (libbfvm.so).

The library is built in-tree (``make -C biofvm_b200/csrc``); importing this
module without it raises, so no caller can silently fall back to anything.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_int, c_int64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbfvm.so")

BFVM_OK = 0
BFVM_ERR_ARG = 1
BFVM_ERR_CUDA = 2
BFVM_ERR_STATE = 3
BFVM_ERR_NOMEM = 4
BFVM_ERR_MESH = 5

STEP_BULK = 1
STEP_CELLS = 2
STEP_DIFFUSION = 4
STEP_ALL = 7

PATH_AUTO = 0
PATH_GENERIC = 1
PATH_TMA = 2
PATH_DIRECT = 3

FP64 = 64
FP32 = 32
FP32_FP64MATH = 3264

BATCH_FUSED = 0
BATCH_BRANCHES = 1
BATCH_PERSISTENT = 2
BATCH_PLANES = 3

_P = c_void_p  # opaque solver handle
_DP = POINTER(c_double)
_LP = POINTER(c_int64)
_IP = POINTER(c_int)

# name -> (restype, argtypes); the order follows include/bfvm.h
SIGNATURES = {
    "bfvm_last_error": (c_char_p, []),
    "bfvm_version": (c_int, []),
    "bfvm_create": (c_int, [POINTER(c_void_p), c_int]),
    "bfvm_destroy": (c_int, [_P]),
    "bfvm_resize_space": (c_int, [_P] + [c_double] * 9),
    "bfvm_resize_space_nodes": (c_int, [_P] + [c_double] * 6 + [c_int] * 3),
    "bfvm_set_mesh": (c_int, [_P, _IP, _DP, c_int]),
    "bfvm_get_mesh": (c_int, [_P, _IP, _DP, _IP]),
    "bfvm_resize_densities": (c_int, [_P, c_int]),
    "bfvm_add_density": (c_int, [_P, c_double, c_double]),
    "bfvm_set_density_coefficients": (c_int, [_P, c_int, c_double, c_double]),
    "bfvm_get_num_densities": (c_int, [_P, _IP]),
    "bfvm_set_densities": (c_int, [_P, _DP]),
    "bfvm_get_densities": (c_int, [_P, _DP]),
    "bfvm_get_voxel_densities": (c_int, [_P, c_int64, _LP, _DP]),
    "bfvm_set_voxel_densities": (c_int, [_P, c_int64, _LP, _DP]),
    "bfvm_get_voxel_densities_noalloc": (c_int, [_P, c_int64, _LP, _DP]),
    "bfvm_device_densities": (c_int, [_P, POINTER(c_void_p)]),
    "bfvm_set_bulk_rates": (c_int, [_P, _DP, _DP, _DP]),
    "bfvm_set_bulk_rates_sparse": (c_int, [_P, c_int64, _LP, _DP, _DP, _DP]),
    "bfvm_add_dirichlet_node": (c_int, [_P, c_int64, _DP]),
    "bfvm_update_dirichlet_node": (c_int, [_P, c_int64, _DP]),
    "bfvm_remove_dirichlet_node": (c_int, [_P, c_int64]),
    "bfvm_clear_dirichlet_nodes": (c_int, [_P]),
    "bfvm_get_num_dirichlet_nodes": (c_int, [_P, _LP]),
    "bfvm_set_agents": (c_int, [_P, c_int64, _LP, _DP, _DP]),
    "bfvm_get_agent_densities": (c_int, [_P, _DP]),
    "bfvm_set_agents_async": (c_int, [_P, c_int64, _LP, _DP, _DP]),
    "bfvm_get_agent_densities_async": (c_int, [_P, _DP]),
    "bfvm_wait_transfers": (c_int, [_P]),
    "bfvm_simulate_bulk_sources_and_sinks": (c_int, [_P, c_double]),
    "bfvm_simulate_cell_sources_and_sinks": (c_int, [_P, c_double]),
    "bfvm_simulate_diffusion_decay": (c_int, [_P, c_double]),
    "bfvm_simulate_diffusion_decay_2d": (c_int, [_P, c_double]),
    "bfvm_apply_dirichlet_conditions": (c_int, [_P]),
    "bfvm_step": (c_int, [_P, c_double, c_int, c_int]),
    "bfvm_reset_diffusion_setup": (c_int, [_P]),
    "bfvm_set_precision": (c_int, [_P, c_int]),
    "bfvm_set_sweep_config": (c_int, [_P, c_int, c_int, c_int, c_int]),
    "bfvm_get_sweep_config": (c_int, [_P, c_int, _IP]),
    "bfvm_set_row_stages": (c_int, [_P, c_int]),
    "bfvm_set_row_build": (c_int, [_P, c_int]),
    "bfvm_get_row_build": (c_int, [_P, _IP, _IP]),
    "bfvm_set_kernel_path": (c_int, [_P, c_int]),
    "bfvm_set_fuse_sources": (c_int, [_P, c_int]),
    "bfvm_get_fuse_sources": (c_int, [_P, _IP]),
    "bfvm_synchronize": (c_int, [_P]),
    "bfvm_get_stream": (c_int, [_P, POINTER(c_void_p)]),
    "bfvm_get_launch_count": (c_int, [_P, _LP]),
    "bfvm_set_slab_planes": (c_int, [_P, c_int]),
    "bfvm_get_slab_planes": (c_int, [_P, _IP]),
    "bfvm_selftest_bounded_wait": (c_int, [c_int, c_int64, _IP, _DP]),
    "bfvm_set_cluster_steps": (c_int, [_P, c_int]),
    "bfvm_get_cluster_steps": (c_int, [_P, _IP]),
    "bfvm_set_grid_steps": (c_int, [_P, c_int]),
    "bfvm_get_grid_steps": (c_int, [_P, _IP]),
    "bfvm_profile_step": (c_int, [_P, c_double, c_int, c_int, _DP]),
    "bfvm_tune_sweeps": (c_int, [_P, c_double, c_int]),
    "bfvm_get_sweep_kernel": (c_int, [_P, c_int, _IP]),
    "bfvm_compute_all_gradient_vectors": (c_int, [_P]),
    "bfvm_get_gradient_vectors": (c_int, [_P, _DP]),
    "bfvm_device_gradients": (c_int, [_P, POINTER(c_void_p)]),
    "bfvm_adjoint_forward": (c_int, [_P, c_double, c_int, c_int, c_int]),
    "bfvm_adjoint_backward": (c_int, [_P, c_void_p, c_int, _DP, _DP, _DP, _DP, _DP]),
    "bfvm_adjoint_release": (c_int, [_P]),
    "bfvm_set_z_slab": (c_int, [_P, c_int, _IP, c_int]),
    "bfvm_zslab_fixup": (c_int, [_P, c_void_p]),
    "bfvm_batch_create": (c_int, [POINTER(c_void_p), c_int]),
    "bfvm_batch_destroy": (c_int, [_P]),
    "bfvm_batch_add": (c_int, [_P, _P]),
    "bfvm_batch_clear": (c_int, [_P]),
    "bfvm_batch_size": (c_int, [_P, _IP]),
    "bfvm_batch_step": (c_int, [_P, c_double, c_int, c_int]),
    "bfvm_batch_tune": (c_int, [_P, c_double, c_int, c_int]),
    "bfvm_batch_set_config": (c_int, [_P, _IP, _IP, c_int64]),
    "bfvm_batch_get_config": (c_int, [_P, _IP, _IP, _LP]),
    "bfvm_batch_set_mode": (c_int, [_P, c_int]),
    "bfvm_batch_get_mode": (c_int, [_P, _IP]),
    "bfvm_batch_set_persistent_chunk": (c_int, [_P, c_int]),
    "bfvm_batch_get_persistent_chunk": (c_int, [_P, _IP]),
    "bfvm_batch_get_plan": (c_int, [_P, _IP, _LP]),
    "bfvm_batch_synchronize": (c_int, [_P]),
}

_lib = None


class BfvmError(RuntimeError):
    def __init__(self, code: int, func: str, msg: str):
        super().__init__(f"{func} failed (code {code}): {msg}")
        self.code = code


def load_library(path: str | None = None) -> ctypes.CDLL:
    """Loads libbfvm.so once and declares every entry point of bfvm.h."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise ImportError(
            f"{p} is missing: build it with `make -C biofvm_b200/csrc` "
            "(there is no CPU fallback for the transport path)"
        )
    lib = ctypes.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    if path is None:
        _lib = lib
    return lib


def check(code: int, func: str) -> None:
    if code != BFVM_OK:
        msg = load_library().bfvm_last_error().decode("utf-8", "replace")
        raise BfvmError(code, func, msg)


def call(name: str, *args) -> None:
    check(getattr(load_library(), name)(*args), name)


def dptr(a: np.ndarray | None):
    """double* of a C-contiguous float64 array (None -> NULL)."""
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous, "need C-contiguous float64"
    return a.ctypes.data_as(_DP)


def lptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.int64 and a.flags.c_contiguous, "need C-contiguous int64"
    return a.ctypes.data_as(_LP)
