"""The precision form (AE_MODE_WAVEFRONT_PRECISION: watertight triangle test,
FP16 shading normals and UVs, compensated accumulation) scored against the
FP64 CPU oracle with the GPU's FP64 image-error reduction, next to the plain
FP32 megakernel; and the reduction itself against numpy."""
import numpy as np
import pytest

import _oracle as O
from aviatorengine2_b200 import Context, _lib, scenes

pytestmark = pytest.mark.gpu

# The precision form may add at most one percentage point of mean relative
# error (against the FP64 oracle) to the plain FP32 form's.
MRE_SLACK = 0.01
EPS = 1e-3


def _numpy_error(img, ref, eps):
    x = img[..., :3].astype(np.float64)
    r = np.asarray(ref, np.float64)[..., :3]
    d = np.abs(x - r)
    return {"mre": float((d / (np.abs(r) + eps)).mean()), "mae": float(d.mean()), "max": float(d.max()),
            "rmse": float(np.sqrt((d * d).mean()))}


def test_image_error_reduction_matches_numpy():
    s = scenes.cornell_box(width=80, height=60, depth=4)
    with Context(80, 60) as ctx:
        ctx.upload(s)
        ctx.render_frame(_lib.MODE_COMPUTE_ONLY)
        acc = ctx.read_image(_lib.IMAGE_ACCUM)
        rng = np.random.default_rng(0)
        ref = acc.astype(np.float64) * (1.0 + rng.normal(0.0, 0.01, acc.shape)) + rng.normal(0.0, 1e-4, acc.shape)
        got = ctx.image_error(ref, eps=EPS)
        want = _numpy_error(acc, ref, EPS)
        for k in want:
            assert got[k] == pytest.approx(want[k], rel=1e-12, abs=1e-300), k
        # Fixed reduction order: identical on a second call.
        assert ctx.image_error(ref, eps=EPS) == got


def _frames(scene, mode, frames):
    w, h = int(scene.config["width"]), int(scene.config["height"])
    with Context(w, h) as ctx:
        ctx.upload(scene)
        c = scene.config.copy()
        for b in range(frames):
            c["batch"] = b
            ctx.set_config(c)
            ctx.render_frame(mode)
        return ctx.read_image(_lib.IMAGE_ACCUM)


def _oracle64(scene, frames):
    c = scene.config.copy()
    acc = None
    for b in range(frames):
        c["batch"] = b
        acc, _, _ = O.render_frame(scene, c, acc, precision=64)
    return acc


SCENES = {
    "cornell": lambda: scenes.cornell_box(width=96, height=64, depth=6),
    "materials": lambda: scenes.hybrid_box(width=80, height=60, depth=5),
    "smooth_meshes": lambda: scenes.wavefront_scene(seed=21, width=64, height=48, depth=4, n_meshes=4, n_instances=24,
                                                    n_lights=4, target_tris=20_000),
}


@pytest.mark.parametrize("name", sorted(SCENES))
def test_precision_mre_against_fp64_oracle(name):
    s = SCENES[name]()
    frames = 8
    ref = _oracle64(s, frames)
    w, h = int(s.config["width"]), int(s.config["height"])
    errs = {}
    for label, mode in (("plain", _lib.MODE_COMPUTE_ONLY), ("wavefront", _lib.MODE_WAVEFRONT),
                        ("precision", _lib.MODE_WAVEFRONT_PRECISION)):
        with Context(w, h) as ctx:
            ctx.upload(s)
            c = s.config.copy()
            for b in range(frames):
                c["batch"] = b
                ctx.set_config(c)
                ctx.render_frame(mode)
            errs[label] = ctx.image_error(ref, eps=EPS)
            if mode == _lib.MODE_WAVEFRONT_PRECISION:
                assert ctx.wavefront_info()["errors"] == 0
    print(f"{name}: MRE vs FP64 oracle plain {errs['plain']['mre']:.3e} wavefront {errs['wavefront']['mre']:.3e} "
          f"precision {errs['precision']['mre']:.3e}")
    # The wavefront form reproduces the plain frames exactly.
    assert errs["wavefront"] == errs["plain"]
    assert errs["precision"]["mre"] <= errs["plain"]["mre"] + MRE_SLACK


def test_precision_primary_ids():
    """Primary-ray instance and triangle IDs of the precision form's
    closest hit (watertight test over 8-bit bounds) against the plain
    reference-order kernel."""
    s = scenes.wavefront_scene(seed=4, width=480, height=270, n_instances=256, target_tris=1_000_000)
    with Context(480, 270) as ctx:
        ctx.upload(s)
        rays = ctx.camera_rays()
        a = ctx.closest_hit(rays, _lib.VARIANT_PLAIN)
        b = ctx.closest_hit(rays, _lib.VARIANT_QUANT)
    same = (a["object"] == b["object"]) & (a["prim"] == b["prim"])
    frac = float(same.mean())
    print(f"primary-ray ID agreement (precision vs plain): {frac:.6f} of {len(rays)}")
    assert frac >= 0.9999


def test_compensated_accumulation_over_many_frames():
    """The precision form keeps the accumulation as a Kahan-compensated sum of
    frame colours.  Over 1024 frames its image stays within a few ulps of the
    FP64 mean of its own frames, while the reference's running lerp
    (accum += (frame - accum) / (n + 1)) drifts by more."""
    s = scenes.cornell_box(width=48, height=32, depth=3)
    frames = 1024
    out = {}
    for label, mode in (("lerp", _lib.MODE_WAVEFRONT), ("kahan", _lib.MODE_WAVEFRONT_PRECISION)):
        with Context(48, 32) as ctx:
            ctx.upload(s)
            c = s.config.copy()
            total = np.zeros((32, 48, 3), np.float64)
            for b in range(frames):
                c["batch"] = b
                ctx.set_config(c)
                ctx.render_frame(mode)
                total += ctx.read_image(_lib.IMAGE_FRAME)[..., :3].astype(np.float64)
            acc = ctx.read_image(_lib.IMAGE_ACCUM)[..., :3].astype(np.float64)
        mean = total / frames
        rel = np.abs(acc - mean) / np.maximum(np.abs(mean), 1e-6)
        out[label] = (float(rel.mean()), float(rel.max()))
    print(f"accumulation vs FP64 mean of 1024 frames: lerp mean/max rel {out['lerp']}, kahan {out['kahan']}")
    assert out["kahan"][1] < 1e-6
    assert out["kahan"][0] < out["lerp"][0]
