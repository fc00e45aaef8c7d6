"""Loader of the in-tree CUDA library (ariel_b200/_lib/libariel_b200.so).

There is no CPU fallback: if the library is missing this module raises, and every compute
entry point of the library returns ARIEL_ERR_NO_DEVICE when no sm_100 device is present.
"""
import ctypes as C
import os

from . import _abi as A

_HERE = os.path.dirname(os.path.abspath(__file__))
SO_PATH = os.path.join(_HERE, "_lib", "libariel_b200.so")
_lib = None

# Every symbol include/ariel.h declares, with its ctypes signature.
_vp = C.c_void_p
SIGNATURES = {
    "ariel_abi_version": ([], C.c_int32),
    "ariel_params_default": ([C.POINTER(A.AsimParams)], None),
    "ariel_scene_dambreak": ([C.POINTER(A.AsimSceneDesc), C.c_int32], None),
    "ariel_mesh_create": ([_vp, C.c_int32, _vp, C.c_int32, _vp, C.c_float, C.POINTER(C.c_int32)], C.c_int),
    "ariel_mesh_destroy": ([C.c_int32], C.c_int),
    "ariel_mesh_info": ([C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32), _vp, C.POINTER(C.c_float)], C.c_int),
    "ariel_scene_load": ([C.c_char_p, C.c_float, C.c_uint64, C.POINTER(A.AsimSceneDesc), C.POINTER(A.AsimSceneInfo),
                          C.c_char_p, C.c_int32], C.c_int),
    "ariel_scene_parse": ([C.c_char_p, C.c_char_p, C.c_float, C.c_uint64, C.POINTER(A.AsimSceneDesc),
                           C.POINTER(A.AsimSceneInfo), C.c_char_p, C.c_int32], C.c_int),
    "ariel_get_level_set": ([_vp, C.c_int32, _vp, C.c_int64], C.c_int),
    "ariel_surface_mesh": ([_vp, C.c_int32, _vp, C.c_int64, _vp, C.c_int64, C.POINTER(C.c_int64),
                            C.POINTER(C.c_int64)], C.c_int),
    "ariel_export_surface": ([_vp, C.c_int32, C.c_char_p, C.c_int32], C.c_int),
    "ariel_status_string": ([C.c_int], C.c_char_p),
    "ariel_create": ([C.POINTER(A.AsimSceneDesc), C.POINTER(A.AsimParams), C.POINTER(_vp)], C.c_int),
    "ariel_create_batch": ([C.POINTER(A.AsimSceneDesc), C.c_int32, C.POINTER(A.AsimParams), C.POINTER(_vp)], C.c_int),
    "ariel_destroy": ([_vp], C.c_int),
    "ariel_scene_count": ([_vp, C.POINTER(C.c_int32)], C.c_int),
    "ariel_init": ([_vp], C.c_int),
    "ariel_step": ([_vp, C.c_int32], C.c_int),
    "ariel_stage": ([_vp, C.c_int32], C.c_int),
    "ariel_synchronize": ([_vp], C.c_int),
    "ariel_particle_count": ([_vp, C.c_int32, C.POINTER(C.c_int64)], C.c_int),
    "ariel_get_particles": ([_vp, C.c_int32, _vp, _vp, _vp, _vp, _vp], C.c_int),
    "ariel_set_particles": ([_vp, C.c_int32, C.c_int64, _vp, _vp, _vp, _vp], C.c_int),
    "ariel_get_cells": ([_vp, C.c_int32, _vp, _vp], C.c_int),
    "ariel_get_grid": ([_vp, C.c_int32, C.c_int32, _vp, C.c_int64], C.c_int),
    "ariel_set_grid": ([_vp, C.c_int32, C.c_int32, _vp, C.c_int64], C.c_int),
    "ariel_get_dimensions": ([_vp, C.c_int32, C.POINTER(C.c_int32)], C.c_int),
    "ariel_stats": ([_vp, C.c_int32, C.POINTER(A.AsimStats)], C.c_int),
    "ariel_get_max_density": ([_vp, C.c_int32, C.POINTER(C.c_float)], C.c_int),
    "ariel_timer_begin": ([_vp], C.c_int),
    "ariel_timer_end": ([_vp, C.POINTER(C.c_double)], C.c_int),
    "ariel_upload_state": ([_vp, C.c_int32, _vp, _vp], C.c_int),
    "ariel_download_state": ([_vp, C.c_int32, _vp, _vp], C.c_int),
    "ariel_timing_reset": ([_vp], C.c_int),
    "ariel_timing_get": ([_vp, _vp, C.POINTER(C.c_double), _vp, C.c_int32, C.POINTER(C.c_int32)], C.c_int),
    "ariel_solver_totals": ([_vp, C.c_int32, C.POINTER(A.AsimSolverTotals)], C.c_int),
    "ariel_selftest_barrier_timeout": ([C.c_double], C.c_int),
    "ariel_kernel_launches": ([], C.c_int64),
    "ariel_last_error": ([], C.c_char_p),
    "ariel_sort_by_cell_noalloc": ([_vp, C.c_int64, C.c_int32, _vp, _vp, _vp, _vp], C.c_int),
    "ariel_checkpoint_save": ([_vp, C.c_char_p], C.c_int),
    "ariel_checkpoint_load": ([_vp, C.c_char_p], C.c_int),
    "ariel_export_particles": ([_vp, C.c_int32, C.c_char_p, C.c_int32], C.c_int),
    "ariel_server_config_default": ([C.POINTER(A.AsimServerConfig)], None),
    "ariel_server_create": ([C.POINTER(A.AsimParams), C.POINTER(A.AsimServerConfig), C.POINTER(_vp)], C.c_int),
    "ariel_server_submit": ([_vp, C.POINTER(A.AsimSceneDesc), C.c_int32, C.POINTER(C.c_int64)], C.c_int),
    "ariel_server_poll": ([_vp, C.c_int64, C.POINTER(A.AsimRequestInfo)], C.c_int),
    "ariel_server_wait": ([_vp, C.c_int64, C.c_double], C.c_int),
    "ariel_server_drain": ([_vp, C.c_double], C.c_int),
    "ariel_server_fetch": ([_vp, C.c_int64, _vp, _vp], C.c_int),
    "ariel_server_release": ([_vp, C.c_int64], C.c_int),
    "ariel_server_stats": ([_vp, C.POINTER(A.AsimServerStats)], C.c_int),
    "ariel_server_shutdown": ([_vp], C.c_int),
    "ariel_state_bytes": ([C.POINTER(A.AsimSceneDesc), C.c_int32, C.POINTER(A.AsimParams),
                           C.POINTER(C.c_int64)], C.c_int),
}


class ArielError(RuntimeError):
    def __init__(self, code, what):
        detail = ""
        if code == A.ARIEL_ERR_CUDA and _lib is not None:
            detail = " [%s]" % _lib.ariel_last_error().decode(errors="replace")
        super().__init__("%s failed: %s%s" % (what, A.status_name(code), detail))
        self.code = code


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(SO_PATH):
            raise ImportError("ariel_b200: CUDA library not built (%s missing); run "
                              "`python ariel_b200/build.py` or __graft_entry__.build()" % SO_PATH)
        L = C.CDLL(SO_PATH)
        for name, (args, res) in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def check(code, what):
    if code != A.ARIEL_OK:
        raise ArielError(code, what)
