"""libwsb.so loads on a machine without a GPU and exports every entry point include/wsb.h declares."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "wsb.h"
LIB = ROOT / "warpsphboundaries_b200" / "_build" / "libwsb.so"


def declared():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(wsb_[a-z_0-9]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared()
    for must in ("wsb_surface_create", "wsb_fixed_topology", "wsb_aggregate", "wsb_aggregate_backward",
                 "wsb_signed_distance", "wsb_kinematics", "wsb_slot_channels_plain", "wsb_contract"):
        assert must in names


def test_library_exports_every_declared_symbol():
    if not LIB.exists():
        from warpsphboundaries_b200 import build
        build.build()
    lib = ctypes.CDLL(str(LIB))
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    from warpsphboundaries_b200 import _lib
    assert sorted(_lib.EXPORTS) == declared()


def test_errors_without_device_are_raised_not_silent():
    """a compute call with invalid arguments returns an error code (no CPU fallback answers instead)."""
    from warpsphboundaries_b200 import _lib
    rc = _lib.lib.wsb_fixed_topology(None, None, None, None, 4, None, None, None)
    assert rc == _lib.WSB_ERR_ARG
    with pytest.raises(ValueError):
        _lib.check(rc, "wsb_fixed_topology")
    assert _lib.lib.wsb_version() >= 100


def test_grouped_aggregate_checks_its_arguments_without_a_device():
    """the grouped entry points refuse a NULL surface before touching a device."""
    from warpsphboundaries_b200 import _lib
    none5 = [_lib.ptrs([None]) for _ in range(5)]
    rc = _lib.lib.wsb_aggregate_evaluate_groups(None, 1, _lib.int32s([2]), _lib.PREC_FP64, None, 4, None,
                                                _lib.OUT_ALL, *none5, None, 0, None)
    assert rc == _lib.WSB_ERR_ARG
    rc = _lib.lib.wsb_aggregate_groups(None, 1, _lib.int32s([2]), _lib.PREC_FP64, None, None, None, 4, None, None, 0,
                                       _lib.OUT_ALL, *none5, None, 0, None)
    assert rc == _lib.WSB_ERR_ARG


def test_detector_inputs_check_their_arguments_without_a_device():
    """wsb_cone_area / wsb_dir_extreme refuse a NULL surface before touching a device."""
    from warpsphboundaries_b200 import _lib
    assert _lib.lib.wsb_cone_area(None, None, 4, None, None, 0.5, None, None, 0, None) == _lib.WSB_ERR_ARG
    assert _lib.lib.wsb_dir_extreme(None, 4, None, None, None, None, 0, None) == _lib.WSB_ERR_ARG


def test_disk_entry_points_check_their_arguments_without_a_device():
    """the disk element refuses bad inputs before touching a device: NULL handles, a non-positive radius, a
    non-finite centre, a bad support, an unknown kernel id."""
    import math
    from warpsphboundaries_b200 import _lib
    L = _lib.lib
    D = ctypes.c_double
    h = ctypes.c_void_p()
    c = (D * 4)(0.0, 0.0, 1.0, 1.0)
    for radii, sup in (((D * 2)(0.5, -1.0), 0.1), ((D * 2)(0.5, 0.5), 0.0), ((D * 2)(0.5, 0.5), math.inf)):
        assert L.wsb_disks_create(c, radii, 2, sup, 0, ctypes.byref(h)) == _lib.WSB_ERR_ARG
    bad = (D * 4)(0.0, math.nan, 1.0, 1.0)
    assert L.wsb_disks_create(bad, (D * 2)(0.5, 0.5), 2, 0.1, 0, ctypes.byref(h)) == _lib.WSB_ERR_ARG
    assert L.wsb_disks_create(c, (D * 2)(0.5, 0.5), 2, 0.1, 0, None) == _lib.WSB_ERR_ARG
    assert L.wsb_disk_aggregate(None, 1, None, None, None, 4, None, _lib.OUT_ALL, None, None, None, None, None, None,
                                0, None) == _lib.WSB_ERR_ARG
    assert L.wsb_disk_cone_area(None, None, None, None, 4, None, None, 0.5, None, None) == _lib.WSB_ERR_ARG
    assert L.wsb_disk_dir_extreme(None, None, None, None, 4, None, None, None, None) == _lib.WSB_ERR_ARG
    assert L.wsb_disk_workspace_size(None, 4) == 0
    assert L.wsb_disks_destroy(None) == _lib.WSB_OK
