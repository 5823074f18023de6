"""Primary-ray IDs of the precision form's closest hit (4-wide BVH with 8-bit
child bounds rounded outward, watertight triangle test; AE_VARIANT_QUANT).

* Against the FP32-node form with the same triangle test (AE_VARIANT_PLAIN_WT:
  the reference's binary FP32 BVH, walked in the reference's order): every
  instance and triangle ID, t and barycentric is identical - the 8-bit bounds
  lose no hit.  Tolerance zero, on the full 1920x1080 camera rays of the
  10M-triangle wavefront scene and on the 960x540 camera rays of the
  2.1M-triangle instanced scene.
* Against the reference's own triangle test (AE_VARIANT_PLAIN): the two tests
  may only disagree where the reference's test (hybrid:564-598) has cracks
  or leaks at shared edges, or where two surfaces lie at the same depth
  within rounding.  Every disagreement must be explained
  (bench.classify_ids: crack, leak, depth tie); none may be left over.
"""
import numpy as np
import pytest

from aviatorengine2_b200 import Context, _lib, scenes
from bench import classify_ids

pytestmark = pytest.mark.gpu


def check(ctx, rays, label):
    plain = ctx.closest_hit(rays, _lib.VARIANT_PLAIN)
    fp32_wt = ctx.closest_hit(rays, _lib.VARIANT_PLAIN_WT)
    quant = ctx.closest_hit(rays, _lib.VARIANT_QUANT)
    # 8-bit nodes against FP32 nodes, same triangle test: identical.
    assert np.array_equal(quant.view(np.uint8), fp32_wt.view(np.uint8)), label
    c = classify_ids(plain, quant)
    print(f"{label}: {c}")
    assert c["unexplained"] == 0, c
    assert c["agreement_excluding_explained"] == 1.0
    assert (quant["object"] != _lib.MISS).mean() > 0.3
    return c


def test_precision_ids_wavefront_scene_1080p():
    s = scenes.wavefront_scene(gpu_build=True)
    with Context(1920, 1080) as ctx:
        ctx.upload(s)
        ctx.prepare_fast()
        check(ctx, ctx.camera_rays(), "wavefront_scene 1920x1080")


def test_precision_ids_instanced_meshes_960x540():
    s = scenes.instanced_meshes(width=960, height=540, gpu_build=True)
    with Context(960, 540) as ctx:
        ctx.upload(s)
        ctx.prepare_fast()
        check(ctx, ctx.camera_rays(), "instanced_meshes 960x540")


def test_plain_wt_equals_quant_on_random_rays():
    """Rays from anywhere in the instanced scene in every direction: the
    FP32-node and 8-bit-node walks agree bit for bit, ties included."""
    s = scenes.instanced_meshes(width=256, height=256, levels=(5, 4, 4, 3, 3), grid=128)
    rng = np.random.default_rng(21)
    n = 200000
    r = np.zeros(n, _lib.RAY)
    o = rng.uniform(0, 100, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r["ox"], r["oy"], r["oz"] = o.T
    r["dx"], r["dy"], r["dz"] = d.T
    r["tnear"] = 0.001
    with Context(256, 256) as ctx:
        ctx.upload(s)
        ctx.prepare_fast()
        a = ctx.closest_hit(r, _lib.VARIANT_PLAIN_WT)
        b = ctx.closest_hit(r, _lib.VARIANT_QUANT)
    assert np.array_equal(a.view(np.uint8), b.view(np.uint8))
    assert (a["object"] != _lib.MISS).mean() > 0.2
