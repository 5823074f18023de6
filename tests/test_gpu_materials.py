"""Textured materials and participating media on the GPU against the oracle
through the C ABI.  Textures (ae_upload_textures + every render form):
compute-only frames bit for bit, the wavefront form equal to them, the
ray-cast G-buffer's albedo plane and the deferred resolve bit for bit, and a
served request equal to frames rendered alone.  Media (isotropic volumes, an
analytic triangle, a moving sphere): the megakernel and the deferred resolve
bit for bit; the optimised forms refuse such scenes."""
import numpy as np
import pytest

import _oracle as O
from aviatorengine2_b200 import Context, Server, _lib, scenes

pytestmark = pytest.mark.gpu


def same(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint32), np.ascontiguousarray(b).view(np.uint32))


def render(s, mode, frames):
    c = s.config.copy()
    out = []
    with Context(int(c["width"]), int(c["height"])) as ctx:
        ctx.upload(s)
        for b in range(frames):
            c["batch"] = b
            ctx.set_config(c)
            ctx.render_frame(mode)
            out.append((ctx.read_image(_lib.IMAGE_ACCUM), ctx.read_image(_lib.IMAGE_DISPLAY)))
    return out


def test_textured_frames_equal_oracle():
    s = scenes.textured_box()
    gpu = render(s, _lib.MODE_COMPUTE_ONLY, 3)
    cfg = s.config.copy()
    acc = None
    for b in range(3):
        cfg["batch"] = b
        acc, disp, _ = O.render_frame(s, cfg, acc)
        assert same(gpu[b][0], acc), f"frame {b}"
        want = np.rint(np.clip(disp[..., :3], 0, 1) * 255).astype(np.int32)
        assert np.abs(gpu[b][1][..., :3].astype(np.int32) - want).max() <= 1


def test_textured_wavefront_equals_plain():
    s = scenes.textured_box()
    a = render(s, _lib.MODE_WAVEFRONT, 2)
    b = render(s, _lib.MODE_COMPUTE_ONLY, 2)
    for k in range(2):
        assert same(a[k][0], b[k][0]) and np.array_equal(a[k][1], b[k][1]), f"frame {k}"


def test_textured_gbuffer_and_deferred_equal_oracle():
    s = scenes.textured_box(width=96, height=72, depth=4)
    c = s.config.copy()
    c["traceScale"], c["historyCap"] = 1.0, 32.0
    w, h = int(c["width"]), int(c["height"])
    st = O.HybridState(w, h)
    with Context(w, h, hybrid=True) as ctx:
        ctx.upload(s)
        for f in range(2):
            c["frameIndex"] = f
            c["historyReset"] = 1 if f == 0 else 0
            ctx.set_config(c)
            ctx.build_gbuffer()
            gb = ctx.read_planes()
            ogb = O.gbuffer(s, c)
            assert np.array_equal(gb[2], ogb[2]), "albedo plane"
            ctx.render_frame(_lib.MODE_DEFERRED)
            O.hybrid_frame(s, c, gb, st, "oracle")
            assert same(ctx.read_deferred_accum(), st.img[st.history]), f"frame {f}"


def test_textured_served_request_equals_frames():
    s = scenes.textured_box(width=64, height=48)
    ref = render(s, _lib.MODE_COMPUTE_ONLY, 2)[-1]
    with Context(64, 48) as ctx:
        ctx.upload(s)
        with Server(slots=2048, max_requests=4, arena_bytes=1 << 24) as srv:
            sid = srv.add_scene(ctx)
            res, acc, dsp = srv.wait(srv.submit(sid, 64, 48, 2, s.config), 60000)
    assert res["status"] == 0
    assert same(acc, ref[0]) and np.array_equal(dsp, ref[1])


def test_media_frames_equal_oracle():
    """Participating media in the plain megakernel: the RNG draws HitVolume
    makes inside the walk follow the reference's visit order exactly."""
    s = scenes.media_box()
    gpu = render(s, _lib.MODE_COMPUTE_ONLY, 3)
    cfg = s.config.copy()
    acc = None
    for b in range(3):
        cfg["batch"] = b
        acc, _, _ = O.render_frame(s, cfg, acc)
        assert same(gpu[b][0], acc), f"frame {b}"


def test_media_deferred_equals_oracle():
    s = scenes.media_box(width=96, height=72, depth=4)
    c = s.config.copy()
    c["traceScale"], c["historyCap"] = 1.0, 32.0
    w, h = int(c["width"]), int(c["height"])
    st = O.HybridState(w, h)
    with Context(w, h, hybrid=True) as ctx:
        ctx.upload(s)
        for f in range(2):
            c["frameIndex"] = f
            c["historyReset"] = 1 if f == 0 else 0
            ctx.set_config(c)
            ctx.build_gbuffer()
            gb = ctx.read_planes()
            ctx.render_frame(_lib.MODE_DEFERRED)
            O.hybrid_frame(s, c, gb, st, "oracle")
            assert same(ctx.read_deferred_accum(), st.img[st.history]), f"frame {f}"


def test_media_refused_by_optimised_forms():
    """Media consume RNG draws in the reference's visit order, which the
    nearest-first walk does not keep: the wavefront form and the server
    refuse such scenes with a clear error instead of rendering differently."""
    from aviatorengine2_b200 import AeError
    s = scenes.media_box(width=32, height=24)
    with Context(32, 24) as ctx:
        ctx.upload(s)
        with pytest.raises(AeError) as e:
            ctx.render_frame(_lib.MODE_WAVEFRONT)
        assert e.value.code == -7
        with Server(slots=1024, max_requests=2, arena_bytes=1 << 22) as srv:
            with pytest.raises(AeError):
                srv.add_scene(ctx)
