"""ctypes binding of ``libhydrob200.so`` (the C ABI in ``include/hydrob200.h``
and ``include/hydrob200_refview.h``). No torch types cross the boundary."""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhydrob200.so")

HB_OK = 0
STATUS = {0: "HB_OK", 1: "HB_E_INVALID", 2: "HB_E_BADMESH", 3: "HB_E_CUDA", 4: "HB_E_NONFINITE",
          5: "HB_E_BARRIER_TIMEOUT", 6: "HB_E_IO", 7: "HB_E_UNDEFINED_REF", 8: "HB_E_NOMEM", 9: "HB_E_TOO_LARGE"}
VARIANT_H, VARIANT_F = 0, 1
REF_STEP_STATIC_MAX_CELLS = 65536   # HB_REF_STEP_STATIC_MAX_CELLS
FP64, FP32, SPLIT = 0, 1, 2
LAYOUT_EDGE, LAYOUT_TILE = 0, 1

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int32)


class HydroError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


class MeshDesc(C.Structure):
    _fields_ = [("cells", C.c_int32), ("ndays", C.c_int32), ("nhq", C.c_int32), ("steps_per_day", C.c_int32),
                ("dt", C.c_double), ("hm1", C.c_double), ("hm2", C.c_double), ("jl", C.c_double),
                ("nac", _dp), ("klas", _dp), ("side", _dp), ("cosf", _dp), ("sinf", _dp), ("slcos", _dp),
                ("slsin", _dp), ("zbc", _dp), ("zb1", _dp), ("area", _dp), ("fnc", _dp), ("bfeat", _dp),
                ("nhq1", _ip), ("zw", _dp), ("qw", _dp), ("qt", _dp), ("dqt", _dp), ("zt", _dp), ("dzt", _dp)]


class Options(C.Structure):
    _fields_ = [("variant", C.c_int32), ("precision", C.c_int32), ("device", C.c_int32), ("renumber", C.c_int32),
                ("tile_config", C.c_int32), ("layout", C.c_int32), ("tile_cells", C.c_int32),
                ("persistent", C.c_int32)]


def _view_types(real):
    rp = C.POINTER(real)

    class CellView(C.Structure):
        _fields_ = [(n, rp) for n in ("H", "U", "V", "W", "Z")] + [("NHQ1", _ip)] + \
                   [(n, rp) for n in ("ZBC", "ZB1", "AREA", "FNC", "BoundaryFeature", "ZW", "QW", "QT", "DQT", "ZT", "DZT")]

    class SideView(C.Structure):
        _fields_ = [(n, rp) for n in ("KLAS", "NAC", "SIDE", "COSF", "SINF", "SLCOS", "SLSIN",
                                      "FLUX0", "FLUX1", "FLUX2", "FLUX3")]

    class MeshView(C.Structure):
        _fields_ = [(n, C.c_int32) for n in ("NHQ", "NQ", "NZ", "NWE", "NDAYS", "CELL")] + \
                   [(n, real) for n in ("DT", "HM1", "HM2", "JL")] + [("cells", CellView), ("sides", SideView)]

    return MeshView


RefMeshView = _view_types(C.c_double)
RefMeshViewF32 = _view_types(C.c_float)

_lib = None


def lib():
    """Load the library (building it first when the sources are newer)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        import importlib.util
        spec = importlib.util.spec_from_file_location("_hb_build", os.path.join(os.path.dirname(HERE), "build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build(verbose=False)
    l = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    sig = {
        "hb_options_default": (None, [C.POINTER(Options)]),
        "hb_tile_configs": (C.c_int, [_ip, _ip, C.c_int32]),
        "hb_launch_shapes": (C.c_int, [_ip, _ip, _ip, C.c_int32]),
        "hb_create": (C.c_int, [C.POINTER(MeshDesc), C.POINTER(Options), C.POINTER(vp)]),
        "hb_destroy": (C.c_int, [vp]),
        "hb_create_batch": (C.c_int, [C.POINTER(MeshDesc), C.c_int32, C.POINTER(Options), C.POINTER(vp)]),
        "hb_batch_size": (C.c_int, [vp, C.POINTER(C.c_int32)]),
        "hb_scenario_cells": (C.c_int, [vp, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
        "hb_set_state_at": (C.c_int, [vp, C.c_int32, _dp, _dp, _dp, _dp, _dp]),
        "hb_get_state_at": (C.c_int, [vp, C.c_int32, _dp, _dp, _dp, _dp, _dp]),
        "hb_get_flux_at": (C.c_int, [vp, C.c_int32, _dp, _dp, _dp, _dp]),
        "hb_get_klas_at": (C.c_int, [vp, C.c_int32, _dp]),
        "hb_get_permutation_at": (C.c_int, [vp, C.c_int32, _ip]),
        "hb_set_tile_config": (C.c_int, [vp, C.c_int32]),
        "hb_get_tile_config": (C.c_int, [vp, C.POINTER(C.c_int32)]),
        "hb_autotune": (C.c_int, [vp, C.c_int32, vp, C.POINTER(C.c_float), C.c_int32, C.POINTER(C.c_int32)]),
        "hb_set_state": (C.c_int, [vp, _dp, _dp, _dp, _dp, _dp]),
        "hb_get_state": (C.c_int, [vp, _dp, _dp, _dp, _dp, _dp]),
        "hb_get_flux": (C.c_int, [vp, _dp, _dp, _dp, _dp]),
        "hb_get_klas": (C.c_int, [vp, _dp]),
        "hb_step": (C.c_int, [vp, C.c_int32, vp]),
        "hb_sync": (C.c_int, [vp, vp]),
        "hb_position": (C.c_int, [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
        "hb_set_position": (C.c_int, [vp, C.c_int64]),
        "hb_step_host": (C.c_int, [vp, _dp, _dp, _dp, _dp, _dp, C.c_int32, vp]),
        "hb_capture_graph": (C.c_int, [vp, C.c_int32, vp]),
        "hb_graph_launch": (C.c_int, [vp, vp]),
        "hb_device_state": (C.c_int, [vp] + [C.POINTER(vp)] * 5 + [C.POINTER(C.c_int32)]),
        "hb_get_permutation": (C.c_int, [vp, _ip]),
        "hb_device_errors": (C.c_int, [vp, C.POINTER(C.c_uint32)]),
        "hb_set_barrier_limit": (C.c_int, [vp, C.c_int64, C.c_int32]),
        "hb_last_error": (C.c_int, []),
        "hb_last_error_string": (C.c_char_p, []),
        "hb_status_string": (C.c_char_p, [C.c_int]),
        "hb_deck_load": (C.c_int, [C.c_char_p, C.POINTER(vp)]),
        "hb_deck_mesh": (C.c_int, [vp, C.POINTER(MeshDesc)]),
        "hb_deck_state": (C.c_int, [vp] + [C.POINTER(_dp)] * 5),
        "hb_deck_free": (C.c_int, [vp]),
        "hb_ref_calculate_flux": (C.c_int, [C.POINTER(RefMeshView), C.c_int32, C.c_int32, C.c_int32, vp]),
        "hb_ref_update_cell": (C.c_int, [C.POINTER(RefMeshView), C.c_int32, vp]),
        "hb_ref_calculate_flux_f32": (C.c_int, [C.POINTER(RefMeshViewF32), C.c_int32, C.c_int32, C.c_int32, vp]),
        "hb_ref_update_cell_f32": (C.c_int, [C.POINTER(RefMeshViewF32), C.c_int32, vp]),
        "hb_ref_take_device_errors": (C.c_int, [C.POINTER(C.c_uint32)]),
        "hb_ref_step_static": (C.c_int, [C.POINTER(RefMeshView), C.c_int32, C.c_int32, C.c_int32, vp]),
        "hb_output_open": (C.c_int, [vp, C.c_char_p, C.POINTER(vp)]),
        "hb_output_frame": (C.c_int, [vp, C.c_int32, C.c_int32, _dp, _dp, _dp, _dp]),
        "hb_output_close": (C.c_int, [vp]),
        "hb_deck_ntoutput": (C.c_int, [vp, C.POINTER(C.c_int32)]),
        "hb_checkpoint_size": (C.c_int, [vp, C.POINTER(C.c_size_t)]),
        "hb_checkpoint_save": (C.c_int, [vp, C.c_void_p, C.c_size_t]),
        "hb_checkpoint_load": (C.c_int, [vp, C.c_void_p, C.c_size_t]),
        "hb_state_record_bytes": (C.c_int, [vp, C.POINTER(C.c_int32)]),
        "hb_halo_define": (C.c_int, [vp, _ip, C.c_int32, C.POINTER(C.c_int32)]),
        "hb_halo_pack": (C.c_int, [vp, C.c_int32, C.c_void_p, vp]),
        "hb_halo_unpack": (C.c_int, [vp, C.c_int32, C.c_void_p, vp]),
        "hb_write_dump": (C.c_int, [vp, C.c_int32, C.POINTER(MeshDesc), C.c_char_p]),
        "hb_adjoint_create": (C.c_int, [vp, _ip, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.POINTER(vp)]),
        "hb_adjoint_destroy": (C.c_int, [vp]),
        "hb_adjoint_set_parameters": (C.c_int, [vp, _dp, _dp]),
        "hb_adjoint_set_initial": (C.c_int, [vp, _dp, _dp, _dp]),
        "hb_adjoint_set_observations": (C.c_int, [vp, _dp]),
        "hb_adjoint_forward": (C.c_int, [vp, C.POINTER(C.c_double), _dp, vp]),
        "hb_adjoint_backward": (C.c_int, [vp, _dp, _dp, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(l, name)
        f.restype = res
        f.argtypes = args
    _lib = l
    return l


def check(status: int) -> None:
    if status != HB_OK:
        msg = lib().hb_last_error_string()
        raise HydroError(status, msg.decode() if msg else "")


# every symbol the C headers declare (checked by the CPU tests)
EXPORTED = ["hb_options_default", "hb_tile_configs", "hb_launch_shapes", "hb_create", "hb_destroy", "hb_set_state", "hb_get_state", "hb_get_flux",
            "hb_get_klas", "hb_step", "hb_sync", "hb_position", "hb_set_position", "hb_step_host", "hb_capture_graph",
            "hb_graph_launch", "hb_device_state", "hb_get_permutation", "hb_device_errors", "hb_set_barrier_limit", "hb_last_error",
            "hb_last_error_string", "hb_status_string", "hb_deck_load", "hb_deck_mesh", "hb_deck_state",
            "hb_deck_free", "hb_ref_calculate_flux", "hb_ref_update_cell", "hb_ref_calculate_flux_f32",
            "hb_ref_update_cell_f32", "hb_ref_take_device_errors", "hb_ref_step_static",
            "hb_create_batch", "hb_batch_size", "hb_scenario_cells", "hb_set_state_at", "hb_get_state_at",
            "hb_get_flux_at", "hb_get_klas_at", "hb_get_permutation_at", "hb_set_tile_config", "hb_get_tile_config",
            "hb_autotune", "hb_checkpoint_size", "hb_checkpoint_save", "hb_checkpoint_load", "hb_write_dump", "hb_output_open", "hb_output_frame", "hb_output_close",
            "hb_deck_ntoutput", "hb_adjoint_create", "hb_adjoint_destroy", "hb_adjoint_set_parameters",
            "hb_adjoint_set_initial", "hb_adjoint_set_observations", "hb_adjoint_forward", "hb_adjoint_backward",
            "hb_state_record_bytes", "hb_halo_define", "hb_halo_pack", "hb_halo_unpack"]
