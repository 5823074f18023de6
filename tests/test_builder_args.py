"""Argument checks of the GPU builders' entry points, which run on the host
before anything reaches a device (no GPU needed): empty inputs succeed with
nothing built, bad sizes and null pointers are refused, and an index past a
mesh's vertices is refused without appending anything to the library."""
import ctypes

import numpy as np

from aviatorengine2_b200 import _lib, scenes
from aviatorengine2_b200._lib import lib

P = ctypes.c_void_p


def test_empty_builds_succeed_without_a_device():
    cnt = ctypes.c_uint32(7)
    assert lib().ae_build_bvh_device(None, 0, 256, None, ctypes.byref(cnt), None, None) == 0
    assert cnt.value == 0
    assert lib().ae_mesh_blas_device(None, 0, None, 0, None, ctypes.byref(cnt), None, None) == 0
    assert lib().ae_mesh_blas_device_many(0, None, None, None, None, None, None, None, None) == 0
    m = scenes.MeshLibrary(gpu=True)
    assert m.add_many([]) == []


def test_bad_arguments_refused():
    cnt = ctypes.c_uint32()
    # a box count with no buffers, no count pointer, indices not a multiple of 3
    assert lib().ae_build_bvh_device(None, 5, 256, None, ctypes.byref(cnt), None, None) == -1
    assert lib().ae_build_bvh_device(None, 0, 256, None, None, None, None) == -1
    assert lib().ae_mesh_blas_device(None, 3, None, 4, None, ctypes.byref(cnt), None, None) == -1
    assert lib().ae_mesh_blas_device_many(2, None, None, None, None, None, None, None, None) == -1


def test_library_many_refuses_bad_index_and_appends_nothing():
    v, i = scenes.box_mesh((1.0, 1.0, 1.0))
    bad = np.array(i, np.uint32).copy()
    bad[5] = len(v)
    m = scenes.MeshLibrary(gpu=True)
    h = scenes.MeshLibrary()
    h.add(v, i)
    k = 2
    vs = [np.ascontiguousarray(v, _lib.VERTEX)] * k
    ix = [np.ascontiguousarray(i, np.uint32), bad]
    out = np.zeros(k, np.int32)
    # The size arrays are kept in names: ctypes only holds their addresses.
    nv = np.array([len(a) for a in vs], np.uint32)
    ni = np.array([len(a) for a in ix], np.uint32)
    rc = lib().ae_mesh_library_add_many_gpu(m.handle, k, (P * k)(*[a.ctypes.data for a in vs]), _lib.ptr(nv),
                                            (P * k)(*[a.ctypes.data for a in ix]), _lib.ptr(ni), None, _lib.ptr(out))
    assert rc == -4  # AE_ERR_LAYOUT
    assert all(len(a) == 0 for a in m.arrays())
    # ragged index count
    ragged = np.ascontiguousarray(i, np.uint32)[:-1].copy()
    nv1 = np.array([len(v)], np.uint32)
    ni1 = np.array([len(ragged)], np.uint32)
    rc = lib().ae_mesh_library_add_many_gpu(m.handle, 1, (P * 1)(vs[0].ctypes.data), _lib.ptr(nv1),
                                            (P * 1)(ragged.ctypes.data), _lib.ptr(ni1), None, _lib.ptr(out))
    assert rc == -1
