"""The wavefront path tracer against the plain megakernel and the oracle:
frames bit for bit (same RNG order, same arithmetic, closest hits from the
optimised walk), over several frames of accumulation, with metal, glass and
analytic primitives, and with several samples per frame."""
import numpy as np
import pytest

import _oracle as O
from aviatorengine2_b200 import Context, _lib, scenes

pytestmark = pytest.mark.gpu


def same(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint32), np.ascontiguousarray(b).view(np.uint32))


def render(scene, mode, frames, samples=1):
    c = scene.config.copy()
    c["samples"] = samples
    out = []
    with Context(int(c["width"]), int(c["height"]), samples=samples) as ctx:
        ctx.upload(scene)
        for b in range(frames):
            c["batch"] = b
            ctx.set_config(c)
            ctx.render_frame(mode)
            out.append((ctx.read_image(_lib.IMAGE_FRAME), ctx.read_image(_lib.IMAGE_ACCUM),
                        ctx.read_image(_lib.IMAGE_DISPLAY)))
        if mode == _lib.MODE_WAVEFRONT:
            info = ctx.wavefront_info()
            assert info["errors"] == 0
            assert info["threads"] in (64, 128, 256) and info["stack"] in (16, 24, 32)
    return out


def test_wavefront_equals_plain_cornell():
    s = scenes.cornell_box()
    a = render(s, _lib.MODE_WAVEFRONT, 3)
    b = render(s, _lib.MODE_COMPUTE_ONLY, 3)
    for k in range(3):
        assert same(a[k][0], b[k][0]), f"frame {k}"
        assert same(a[k][1], b[k][1])
        assert np.array_equal(a[k][2], b[k][2])


def test_wavefront_equals_oracle_materials_and_analytic():
    s = scenes.hybrid_box(width=160, height=120, depth=6)
    a = render(s, _lib.MODE_WAVEFRONT, 2)
    cfg = s.config.copy()
    acc = None
    for k in range(2):
        cfg["batch"] = k
        acc, _, frame = O.render_frame(s, cfg, acc)
        assert same(a[k][0], frame), f"frame {k}"
        assert same(a[k][1], acc)


def test_wavefront_samples_per_frame():
    s = scenes.cornell_box(width=96, height=64)
    a = render(s, _lib.MODE_WAVEFRONT, 2, samples=3)
    b = render(s, _lib.MODE_COMPUTE_ONLY, 2, samples=3)
    for k in range(2):
        assert same(a[k][1], b[k][1])
