"""ctypes binding of libkrigecuda.so (the krige_* C-ABI, include/krigekit_b200.h).

The library is the only compute path: there is no CPU fallback.  Importing
this module fails loudly when the shared library is missing or when no CUDA
device is visible.
"""
from __future__ import annotations

import atexit
import ctypes
import os
import weakref

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libkrigecuda.so")

_c_int = ctypes.c_int
_c_double = ctypes.c_double
_c_char_p = ctypes.c_char_p
_c_i64 = ctypes.c_int64
_p_int = ctypes.POINTER(ctypes.c_int)
_p_dbl = ctypes.POINTER(ctypes.c_double)
_p_i64 = ctypes.POINTER(ctypes.c_int64)

ALLOC_FN = ctypes.CFUNCTYPE(ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p)
FREE_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_void_p)

# name -> (argtypes, restype)
SIGNATURES = {
    "krige_create": ([_p_i64], _c_int),
    "krige_destroy": ([_p_i64], _c_int),
    "krige_ind_create": ([_p_i64], _c_int),
    "krige_ind_set_ncat": ([_c_i64, _c_int], _c_int),
    "krige_initialize": ([_c_i64, _c_int, _c_int, _c_int, _c_int, _c_int,
                          _c_int, _c_int, _c_int, _c_int, _c_int, _c_int, _c_int, _c_int, _c_int, _c_int,
                          _c_int, _c_char_p, _p_dbl, _c_int], _c_int),
    "krige_set_obs": ([_c_i64, _c_int, _c_int, _c_int, _p_dbl, _p_dbl, _p_dbl, _c_int, _c_double, _c_double],
                      _c_int),
    "krige_update_obs_value": ([_c_i64, _c_int, _c_int, _p_dbl], _c_int),
    "krige_set_obs_drift": ([_c_i64, _c_int, _c_int, _c_int, _p_dbl], _c_int),
    "krige_reset_vgm": ([_c_i64, _c_int, _c_int], _c_int),
    "krige_set_vgm": ([_c_i64, _c_int, _c_int, _c_char_p, _c_double, _c_double, _c_double, _c_double, _c_double,
                       _c_double, _c_double, _c_double, _c_int], _c_int),
    "krige_set_grid": ([_c_i64, _c_int, _c_int, _p_dbl, _p_dbl, _p_dbl], _c_int),
    "krige_set_grid_block": ([_c_i64, _c_int, _c_int, _c_int, _p_dbl, _c_int, _p_int, _p_dbl, _p_dbl, _p_dbl,
                              _p_dbl], _c_int),
    "krige_set_grid_cv": ([_c_i64], _c_int),
    "krige_set_grid_drift": ([_c_i64, _c_int, _c_int, _c_int, _p_dbl], _c_int),
    "krige_set_search": ([_c_i64, _c_int, _c_double, _c_double, _c_double, _c_double, _c_double, _c_int], _c_int),
    "krige_solve": ([_c_i64, _c_int, _c_int], _c_int),
    "krige_solver_stats": ([_c_i64, _p_int], None),
    "krige_get_last_error": ([ctypes.c_char_p, _c_int], _c_int),
    "krige_get_nblocks": ([_c_i64, _p_int], _c_int),
    "krige_get_nsim": ([_c_i64, _p_int], _c_int),
    "krige_get_block_coord": ([_c_i64, _c_int, _c_int, _p_dbl], _c_int),
    "krige_get_estimate": ([_c_i64, _c_int, _c_int, _p_dbl], _c_int),
    "krige_get_estimate_all": ([_c_i64, _c_int, _c_int, _c_int, _p_dbl], _c_int),
    "krige_get_variance": ([_c_i64, _c_int, _p_dbl], _c_int),
    "krige_get_variance_all": ([_c_i64, _c_int, _c_int, _p_dbl], _c_int),
    # space-time entry points (kriging_st_capi.f90)
    "krige_st_create": ([_p_i64], _c_int),
    "krige_st_destroy": ([_p_i64], _c_int),
    "krige_st_initialize": ([_c_i64, _c_int, _c_int, _c_int, _c_int, _c_int, _c_int, _c_int, _c_int, _c_int,
                             _c_int, _c_int, _c_int, _c_char_p, _p_dbl, _c_int], _c_int),
    "krige_st_set_st_model": ([_c_i64, _c_char_p, _c_char_p, _c_double, _c_double, _c_double, _c_double], _c_int),
    "krige_st_set_obs": ([_c_i64, _c_int, _c_int, _c_int, _p_dbl, _p_dbl, _p_dbl, _c_int, _c_double, _c_double],
                         _c_int),
    "krige_st_reset_vgm": ([_c_i64, _c_int, _c_int], _c_int),
    "krige_st_set_vgm": ([_c_i64, _c_int, _c_int, _c_char_p, _c_double, _c_double, _c_double, _c_double,
                          _c_double, _c_double, _c_double, _c_double], _c_int),
    "krige_st_set_vgm_temporal": ([_c_i64, _c_int, _c_int, _c_char_p, _c_double, _c_double, _c_double], _c_int),
    "krige_st_set_vgm_joint_sills": ([_c_i64, _c_int, _c_int, _c_int, _p_dbl], _c_int),
    "krige_st_set_grid": ([_c_i64, _c_int, _p_dbl, _p_dbl, _p_dbl, _p_dbl], _c_int),
    "krige_st_set_grid_block": ([_c_i64, _c_int, _p_dbl, _p_dbl, _p_int, _c_int, _p_dbl, _p_dbl, _p_dbl, _p_dbl,
                                 _p_dbl], _c_int),
    "krige_st_set_grid_drift": ([_c_i64, _c_int, _c_int, _p_dbl], _c_int),
    "krige_st_set_search": ([_c_i64, _c_int, _c_double, _c_double, _c_double, _c_double, _c_double, _c_double,
                             _c_int], _c_int),
    # extensions of the GPU library
    "krige_set_precision": ([_c_i64, _c_int], _c_int),
    "krige_set_nmin": ([_c_i64, _c_int], _c_int),
    "krige_set_device": ([_c_i64, _c_int, ctypes.c_void_p], _c_int),
    "krige_set_allocator": ([ALLOC_FN, FREE_FN, ctypes.c_void_p], None),
    "krige_get_neighbours": ([_c_i64, _c_int, _c_int, _c_int, _p_int, _p_int], _c_int),
    "krige_get_mmax": ([_c_i64, _c_int, _p_int], _c_int),
    "krige_get_status": ([_c_i64, _c_int, _p_int], _c_int),
    "krige_gpu_stats": ([_c_i64, _p_int, _p_dbl], _c_int),
    "krige_gpu_counters": ([_c_i64, _c_int, _p_int], _c_int),
    "krige_gpu_profile": ([_c_i64, _c_int], _c_int),
    "krige_set_autotune": ([_c_i64, _c_int], _c_int),
    "krige_set_sim": ([_c_i64, _c_int, ctypes.c_void_p, _c_int, _c_int, ctypes.c_void_p], _c_int),
    "krige_get_sim_neighbours": ([_c_i64, _c_int, _c_int, _p_int, _p_int], _c_int),
    "krige_set_sim_draw": ([_c_i64, _c_int], _c_int),
    "krige_get_kernel_plan": ([_c_i64, _p_int, _p_dbl], _c_int),
    "krige_autotune_clear": ([], _c_int),
    "krige_gpu_phases": ([_c_i64, _p_dbl, _p_int], _c_int),
    "krige_gpu_kernel_ms": ([_c_i64, _p_dbl], _c_int),
    "krige_resolve_static": ([_c_i64, _c_int, _c_int, _p_dbl], _c_int),
    # in-memory weight store (reference layouts, kriging.py:259-274)
    "krige_get_weight_dims": ([_c_i64, _p_int, _p_int, _p_int], _c_int),
    "krige_get_weight_nnear": ([_c_i64, _c_int, _c_int, _p_int], _c_int),
    "krige_get_weight_inear": ([_c_i64, _c_int, _c_int, _c_int, _p_int], _c_int),
    "krige_get_weight_data": ([_c_i64, _c_int, _c_int, _c_int, _c_int, _p_dbl], _c_int),
    "krige_get_weight_var": ([_c_i64, _c_int, _c_int, _p_dbl], _c_int),
    "krige_set_weights": ([_c_i64, _c_int, _c_int, _c_int, _c_int, _p_int, _p_int, _p_dbl, _p_int, _p_dbl],
                          _c_int),
    "krige_free_weight_store": ([_c_i64], _c_int),
    "krige_to_str": ([_c_i64], ctypes.c_void_p),
}

_lib = None


def load():
    """Load libkrigecuda.so; raise if it is missing (no fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m krigekit_b200.build` "
            "(the GPU kriging path has no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (args, res) in SIGNATURES.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def last_error() -> str:
    buf = ctypes.create_string_buffer(4096)
    load().krige_get_last_error(buf, len(buf))
    return buf.value.decode("utf-8", errors="replace").strip()


def check(ierr: int, name: str) -> None:
    if int(ierr) != 0:
        raise RuntimeError(last_error() or f"{name} failed with ierr={int(ierr)}")


def call(name: str, *args) -> None:
    check(getattr(load(), name)(*args), name)


# -- torch-backed device allocator ------------------------------------------
_torch_blocks = {}
_alloc_cb = None
_free_cb = None


def use_torch_allocator() -> None:
    """Route the library's device buffers through torch's caching allocator."""
    global _alloc_cb, _free_cb
    if _alloc_cb is not None:
        return
    import torch

    def _alloc(nbytes, _ctx):
        t = torch.empty(int(nbytes), dtype=torch.uint8, device="cuda")
        ptr = t.data_ptr()
        _torch_blocks[ptr] = t
        return ptr

    def _free(ptr, _ctx):
        _torch_blocks.pop(ptr, None)

    _alloc_cb = ALLOC_FN(_alloc)
    _free_cb = FREE_FN(_free)
    load().krige_set_allocator(_alloc_cb, _free_cb, None)


# -- handles alive at interpreter exit ----------------------------------------
_live = weakref.WeakSet()


def register(obj) -> None:
    """Track an object owning a handle; its ``close()`` runs at interpreter exit."""
    _live.add(obj)


@atexit.register
def _close_all() -> None:
    # Destroy engines while torch and the allocator callbacks still exist.
    for obj in list(_live):
        try:
            obj.close()
        except Exception:
            pass
