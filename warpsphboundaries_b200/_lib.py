"""ctypes binding of libwsb.so (include/wsb.h).

The library is the only compute path of this package: there is no CPU
fallback.  If it is missing, importing this module raises with the command
that builds it.
"""
import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_int, c_int32, c_int64, c_size_t, c_void_p
from pathlib import Path

LIB_PATH = Path(os.environ.get("WSB_LIB", Path(__file__).resolve().parent / "_build" / "libwsb.so"))

WSB_OK, WSB_ERR_ARG, WSB_ERR_CUDA, WSB_ERR_UNSUPPORTED, WSB_ERR_SIZE, WSB_ERR_DEVICE = 0, -1, -2, -3, -4, -5
PREC_FP64, PREC_MIXED, PREC_FP32 = 0, 1, 2
RADIAL_PLANE, RADIAL_SPHERE = 0, 1
OUT_LAM, OUT_G, OUT_COV, OUT_M1, OUT_M2, OUT_ALL, OUT_ASSIGN = 1, 2, 4, 8, 16, 31, 32

EXPORTS = ["wsb_last_error", "wsb_version", "wsb_surface_create", "wsb_surface_destroy", "wsb_surface_info_get",
           "wsb_surface_cells", "wsb_fixed_topology", "wsb_slot_channels_plain", "wsb_contract",
           "wsb_aggregate_workspace_size", "wsb_aggregate_staging_size", "wsb_set_pair_events", "wsb_aggregate", "wsb_aggregate_prepare", "wsb_aggregate_evaluate",
           "wsb_aggregate_evaluate_groups", "wsb_aggregate_groups", "wsb_aggregate_noalloc",
           "wsb_aggregate_backward", "wsb_cone_area", "wsb_dir_extreme", "wsb_signed_distance",
           "wsb_kinematics", "wsb_radial_channels", "wsb_mesh_create", "wsb_mesh_destroy",
           "wsb_mesh_workspace_size", "wsb_mesh_inside", "wsb_mesh_channels", "wsb_triangle_channels",
           "wsb_triangle_combine", "wsb_disks_create", "wsb_disks_destroy", "wsb_disk_workspace_size",
           "wsb_disk_aggregate", "wsb_disk_cone_area", "wsb_disk_dir_extreme", "wsb_pair_weights",
           "wsb_pair_channels", "wsb_scene_create", "wsb_scene_destroy", "wsb_scene_add_body", "wsb_scene_add_surface",
           "wsb_scene_set_pose", "wsb_scene_info", "wsb_scene_workspace_size", "wsb_scene_aggregate",
           "wsb_server_create", "wsb_server_destroy", "wsb_serve_submit", "wsb_serve_poll", "wsb_serve_wait",
           "wsb_serve_release", "wsb_server_stats"]


class SurfaceInfo(ctypes.Structure):
    _fields_ = [("n_verts", c_int64), ("n_edges", c_int64), ("nx", c_int32), ("ny", c_int32),
                ("lo_x", c_double), ("lo_y", c_double), ("cell", c_double), ("K", c_int32), ("n_items", c_int64),
                ("n_bins", c_int32), ("bbox_lo_x", c_double), ("bbox_lo_y", c_double), ("bbox_hi_x", c_double),
                ("bbox_hi_y", c_double), ("background", c_int), ("support_max", c_double)]


def _load():
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is not built: run `python -m warpsphboundaries_b200.build` "
                           "(this package has no CPU fallback)")
    lib = ctypes.CDLL(str(LIB_PATH))
    P, D, I32P, PP = c_void_p, POINTER(c_double), POINTER(c_int32), POINTER(c_void_p)
    sig = {
        "wsb_last_error": (c_char_p, []),
        "wsb_version": (c_int, []),
        "wsb_surface_create": (c_int, [D, c_int64, I32P, c_int64, c_int, c_double, c_int, POINTER(c_void_p)]),
        "wsb_surface_destroy": (c_int, [P]),
        "wsb_surface_info_get": (c_int, [P, POINTER(SurfaceInfo)]),
        "wsb_surface_cells": (c_int, [P, I32P, I32P]),
        "wsb_fixed_topology": (c_int, [P, P, P, P, c_int64, P, P, P]),
        "wsb_slot_channels_plain": (c_int, [P, c_int, P, P, P, c_int64, P, P]),
        "wsb_contract": (c_int, [P, c_int, P, P, P, P, c_int64, P, P, P, P, P, P, P]),
        "wsb_aggregate_workspace_size": (c_size_t, [P, c_int64]),
        "wsb_aggregate_staging_size": (c_size_t, [P, c_int64]),
        "wsb_set_pair_events": (c_int, [P, P]),
        "wsb_aggregate": (c_int, [P, c_int, c_int, P, P, P, c_int64, P, D, c_int, c_int, P, P, P, P, P, P, c_size_t,
                                  P, P]),
        "wsb_aggregate_prepare": (c_int, [P, P, P, P, c_int64, P, D, c_int, P, c_size_t, P]),
        "wsb_aggregate_evaluate": (c_int, [P, c_int, c_int, P, c_int64, P, c_int, P, P, P, P, P, P, c_size_t, P]),
        "wsb_aggregate_evaluate_groups": (c_int, [P, c_int, I32P, c_int, P, c_int64, P, c_int, PP, PP, PP, PP, PP, P,
                                                  c_size_t, P]),
        "wsb_aggregate_groups": (c_int, [P, c_int, I32P, c_int, P, P, P, c_int64, P, D, c_int, c_int, PP, PP, PP, PP,
                                         PP, P, c_size_t, P]),
        "wsb_aggregate_noalloc": (c_int, [P, c_int, c_int, P, P, P, c_int64, P, D, c_int, c_int, P, P, P, P, P, P,
                                          P]),
        "wsb_aggregate_backward": (c_int, [P, c_int, P, P, P, c_int64, P, D, c_int, P, P, P, P, P, P, c_size_t, P]),
        "wsb_cone_area": (c_int, [P, P, c_int64, P, P, c_double, P, P, c_size_t, P]),
        "wsb_dir_extreme": (c_int, [P, c_int64, P, P, P, P, c_size_t, P]),
        "wsb_signed_distance": (c_int, [P, P, c_int64, c_double, P, P, P, P, P]),
        "wsb_kinematics": (c_int, [P, c_int32, P, c_int64, P, P, P, P, P]),
        "wsb_radial_channels": (c_int, [c_int, c_int, c_int, P, P, P, P, c_int64, I32P, c_int, P, P, P, P]),
        "wsb_mesh_create": (c_int, [D, c_int64, I32P, c_int64, c_double, c_int, POINTER(c_void_p)]),
        "wsb_mesh_destroy": (c_int, [P]),
        "wsb_mesh_workspace_size": (c_size_t, [P, c_int64]),
        "wsb_mesh_inside": (c_int, [P, P, c_int64, P, P]),
        "wsb_mesh_channels": (c_int, [P, c_int, P, P, c_int64, P, P, P, c_size_t, P]),
        "wsb_triangle_channels": (c_int, [D, c_double, c_double, c_int, c_int, P, P, P, c_int64, c_double, c_int, P, P,
                                          P, P]),
        "wsb_triangle_combine": (c_int, [P, P, P, P, c_int64, c_int, P, P, P, P, P, P, P, P, P, P, P]),
        "wsb_disks_create": (c_int, [D, D, c_int64, c_double, c_int, POINTER(c_void_p)]),
        "wsb_disks_destroy": (c_int, [P]),
        "wsb_disk_workspace_size": (c_size_t, [P, c_int64]),
        "wsb_disk_aggregate": (c_int, [P, c_int, P, P, P, c_int64, P, c_int, P, P, P, P, P, P, c_size_t, P]),
        "wsb_disk_cone_area": (c_int, [P, P, P, P, c_int64, P, P, c_double, P, P]),
        "wsb_disk_dir_extreme": (c_int, [P, P, P, P, c_int64, P, P, P, P]),
        "wsb_pair_channels": (c_int, [P, c_int, c_int, P, P, c_int64, P, P, c_int64, P, P, P]),
        "wsb_pair_weights": (c_int, [c_int, P, P, c_int64, P, P, c_int64, P, c_int64, P, c_int64, P, P, P, P]),
        "wsb_scene_create": (c_int, [c_int, POINTER(c_void_p)]),
        "wsb_scene_destroy": (c_int, [P]),
        "wsb_scene_add_body": (c_int, [P, D, POINTER(c_int)]),
        "wsb_scene_add_surface": (c_int, [P, c_int, P]),
        "wsb_scene_set_pose": (c_int, [P, c_int, D, P]),
        "wsb_scene_info": (c_int, [P, POINTER(c_int), POINTER(c_int)]),
        "wsb_scene_workspace_size": (c_size_t, [P, c_int64]),
        "wsb_scene_aggregate": (c_int, [P, c_int, I32P, c_int, P, P, P, c_int64, c_int64, PP, PP, PP, PP, PP, P,
                                        c_size_t, P]),
        "wsb_server_create": (c_int, [c_int, c_int, c_int64, c_size_t, POINTER(c_void_p)]),
        "wsb_server_destroy": (c_int, [P]),
        "wsb_serve_submit": (c_int, [P, P, c_int, c_int, c_int, P, P, c_int64, P, P, P, P, P, P, P,
                                     POINTER(c_int64)]),
        "wsb_serve_poll": (c_int, [P, c_int64, POINTER(c_int)]),
        "wsb_serve_wait": (c_int, [P, c_int64]),
        "wsb_serve_release": (c_int, [P, c_int64]),
        "wsb_server_stats": (c_int, [P, POINTER(c_int64), D, D, POINTER(c_size_t)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


lib = _load()


def last_error():
    msg = lib.wsb_last_error()
    return msg.decode() if msg else ""


def check(rc, what=""):
    """raise the Python exception of a WSB_ERR_* code (ValueError, NotImplementedError, RuntimeError)."""
    if rc == WSB_OK:
        return
    msg = f"{what}: {last_error()}" if what else last_error()
    if rc in (WSB_ERR_ARG, WSB_ERR_SIZE):
        raise ValueError(msg)
    if rc == WSB_ERR_UNSUPPORTED:
        raise NotImplementedError(msg)
    raise RuntimeError(msg)


def ptr(t):
    """device (or host) address of a tensor, None -> NULL."""
    return None if t is None else c_void_p(t.data_ptr())


def ptrs(tensors):
    """a host array of device addresses (None -> NULL), for the per-group output arguments."""
    return (c_void_p * len(tensors))(*[None if t is None else t.data_ptr() for t in tensors])


def int32s(values):
    """a host int32 array."""
    return (c_int32 * len(values))(*values)


def dptr(a):
    """ctypes double* of a host numpy float64 array."""
    return a.ctypes.data_as(POINTER(c_double))
