"""Host logic of the closed-surface family (no GPU): surface validation in the C ABI, request mapping, argument
checks."""
import ctypes

import numpy as np
import pytest

from warpsphboundaries_b200 import _lib, workloads
from warpsphboundaries_b200.mesh3d import Evaluator, Geometry, _column
from warpsphboundaries_b200.radial import Request, baseline


def _tet():
    V = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], float)
    F = np.array([[0, 2, 1], [0, 1, 3], [0, 3, 2], [1, 2, 3]], np.int32)
    return V, F


def _create(V, F, smax=0.1):
    V = np.ascontiguousarray(V, np.float64)
    F = np.ascontiguousarray(F, np.int32)
    h = ctypes.c_void_p()
    rc = _lib.lib.wsb_mesh_create(V.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(V),
                                  F.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), len(F), smax, 0, ctypes.byref(h))
    return rc, h


def test_surface_checks_run_before_any_device_work():
    V, F = _tet()
    assert _create(V, F[:3])[0] == _lib.WSB_ERR_ARG                   # open (3 faces)
    assert _create(V, F[:, ::-1])[0] == _lib.WSB_ERR_ARG              # inward normals: negative volume
    bad = F.copy()
    bad[0] = bad[0][::-1]
    assert _create(V, bad)[0] == _lib.WSB_ERR_ARG                     # one face flipped: inconsistent orientation
    bad = F.copy()
    bad[1, 2] = 7
    assert _create(V, bad)[0] == _lib.WSB_ERR_ARG                     # index out of range
    assert _create(V, F, smax=0.0)[0] == _lib.WSB_ERR_ARG
    Vd = V.copy()
    Vd[3] = [0.5, 0.5, 0.0]                                           # flat: zero volume, degenerate faces
    assert _create(Vd, F)[0] == _lib.WSB_ERR_ARG
    assert "mesh_create" in _lib.last_error()


def test_channel_abi_argument_errors():
    f = _lib.lib.wsb_mesh_channels
    assert f(None, 2, None, None, 4, None, None, None, 0, None) == _lib.WSB_ERR_ARG
    assert _lib.lib.wsb_mesh_workspace_size(None, 10) == 0
    assert _lib.lib.wsb_mesh_inside(None, None, 3, None, None) == _lib.WSB_ERR_ARG


def test_request_columns():
    b = baseline(3)
    assert [_column(r) for r in b] == list(range(28))
    assert _column(Request((0, 0, 0), (2, 0))) == _column(Request((0, 0, 0), (0, 2)))
    assert _column(Request((1, 1, 0), (0,))) is None


def test_evaluator_arguments():
    V, F = _tet()
    g = Geometry.closed_surface(V, F)
    with pytest.raises(ValueError):
        Evaluator(g, kernel="quintic")
    with pytest.raises(NotImplementedError):
        Evaluator(g, precision="float32")
    with pytest.raises(NotImplementedError):
        Evaluator(g, [Request((1, 1, 0), (0,))])
    with pytest.raises(RuntimeError):
        Evaluator(g, device="cpu")
    ev = Evaluator(g)
    with pytest.raises(ValueError):
        ev.prepare([[0.1, 0.1, 0.1]], 0.0)
    with pytest.raises(ValueError):
        ev.prepare([[np.nan, 0.1, 0.1]], 0.1)
    with pytest.raises(ValueError):                                    # element < 1e-4 of the support
        Evaluator(Geometry.closed_surface(V * 1e-5, F)).prepare([[0.1, 0.1, 0.1]], 1.0)


def _cube_tets():
    C = np.array([[x, y, z] for x in (0, 1) for y in (0, 1) for z in (0, 1)], float)
    i = lambda x, y, z: x * 4 + y * 2 + z
    tets = [[i(0, 0, 0), i(1, 0, 0), i(0, 1, 0), i(0, 0, 1)], [i(1, 1, 0), i(1, 0, 0), i(0, 1, 0), i(1, 1, 1)],
            [i(1, 0, 1), i(1, 0, 0), i(1, 1, 1), i(0, 0, 1)], [i(0, 1, 1), i(0, 1, 0), i(0, 0, 1), i(1, 1, 1)],
            [i(1, 0, 0), i(0, 1, 0), i(0, 0, 1), i(1, 1, 1)]]
    return [C[t] for t in tets]


def test_tetrahedral_mesh_boundary():
    """Geometry.from_elements (fluxbridge geometry.py:20-63): a conforming tetrahedral mesh becomes the closed
    surface of its union -- the shared faces cancel, every boundary face is outward -- for a cube of five tetrahedra
    (12 faces, volume 1) and a fan of an icosphere from its centre (the icosphere's own 320 faces, same volume);
    overlapping and degenerate elements and 2-D / surface elements are refused."""
    from warpsphboundaries_b200.mesh3d import Geometry
    g = Geometry.from_elements(_cube_tets())
    vol = lambda V, F: sum(float(np.dot(V[a], np.cross(V[b], V[c]))) for a, b, c in F) / 6
    assert len(g.faces) == 12 and len(g.vertices) == 8 and abs(vol(g.vertices, g.faces) - 1.0) < 1e-15
    assert g.from_tets
    Vs, Fs = workloads.icosphere(2, 0.6, 0.02, seed=3)
    fan = Geometry.from_elements([np.stack([np.zeros(3), Vs[a], Vs[b], Vs[c]]) for a, b, c in Fs])
    assert len(fan.faces) == len(Fs) and abs(vol(fan.vertices, fan.faces) - vol(Vs, Fs)) < 1e-14
    assert {tuple(sorted(map(tuple, fan.vertices[f]))) for f in fan.faces} == \
        {tuple(sorted(map(tuple, Vs[f]))) for f in Fs}
    t0 = _cube_tets()[0]
    with pytest.raises(ValueError):
        Geometry.from_elements([t0, t0])
    with pytest.raises(ValueError):
        Geometry.from_elements([np.array([[0, 0, 0], [1, 0, 0], [2, 0, 0], [0, 1, 0]], float)])
    with pytest.raises(NotImplementedError):
        Geometry.from_elements([np.eye(3)], dimension=2)
