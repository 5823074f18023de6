"""The closest-hit workload's scene packed by the reference's own scene code
(oracle/ref_scene.py over oracle/_ref: MeshLibrary::Add's steps, MeshBounds,
BuildBVH, MeshToGPU) equals the library's packing byte for byte, so the
benchmark's reference arm and our arm trace the same scene; and the oracle's
byte layouts (oracle/layouts.py, which the oracle side uses instead of the
library's) equal the library's dtypes field by field."""
import os
import sys

import numpy as np
import pytest

import _oracle as O
from aviatorengine2_b200 import _lib, scenes, synth

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import ref_scene as R  # noqa: E402

needs_ref = pytest.mark.skipif(not R.available(), reason="reference build (oracle/_ref) not present")

ARRAYS = ("objects", "tlas", "lights", "vertices", "indices", "blas", "instances")


def test_oracle_layouts_equal_library_dtypes():
    L = O._lib
    for name in ("VERTEX", "NODE", "OBJECT", "INSTANCE", "RAY", "HIT", "CONFIG"):
        assert getattr(L, name) == getattr(_lib, name), name
    assert (L.SHAPE_MESH, L.MAT_LAMBERTIAN, L.MAT_DIFFUSE_LIGHT, L.NO_TEXTURE, L.MISS) == \
           (_lib.SHAPE_MESH, _lib.MAT_LAMBERTIAN, _lib.MAT_DIFFUSE_LIGHT, _lib.NO_TEXTURE, _lib.MISS)


def test_oracle_binding_imports_no_library_module():
    assert "aviatorengine2_b200" not in O.__dict__
    src = open(O.__file__).read()
    assert "import aviatorengine2_b200" not in src and "from aviatorengine2_b200" not in src
    assert "aviatorengine2_b200" not in open(R.__file__).read().split('"""')[2]


def _same(a, b):
    for f in ARRAYS:
        x, y = np.ascontiguousarray(getattr(a, f)), np.ascontiguousarray(getattr(b, f))
        assert x.shape == y.shape and np.array_equal(x.view(np.uint8), y.view(np.uint8)), f
    assert np.array_equal(np.array(a.config).reshape(1).view(np.uint8), np.array(b.config).reshape(1).view(np.uint8))


@needs_ref
@pytest.mark.parametrize("seed", [2, 11])
def test_reference_packing_equals_library_small(seed):
    kw = dict(seed=seed, width=240, height=135, levels=(4, 3, 3, 2, 2), grid=64)
    _same(R.build_instanced(synth.instanced_meshes_spec(**kw)), scenes.instanced_meshes(**kw))


@needs_ref
def test_reference_packing_equals_library_full_size():
    """The benchmark's 2,099,206-triangle scene (scaled instances)."""
    a = R.build_instanced(synth.instanced_meshes_spec())
    b = scenes.instanced_meshes()
    _same(a, b)
    assert a.triangles == 2099206 and R.scene_digest(a) == R.scene_digest(b)
