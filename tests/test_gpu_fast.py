"""The optimised closest-hit kernels against the oracle.

FAST (4-wide quantised BLAS, nearest-first, reference triangle test): hit IDs,
t and barycentrics bit-exact - the tie rule reproduces the reference's
"later visit wins" answer in any visit order.
QUANT (watertight triangle test): t and barycentrics come from a different
formula, so they agree within tolerance; IDs must agree on primary rays.
"""
import numpy as np
import pytest

import _oracle as O
from aviatorengine2_b200 import AeError, Context, _lib, scenes

pytestmark = pytest.mark.gpu


def ctx_for(scene):
    c = Context(int(scene.config["width"]), int(scene.config["height"]))
    c.upload(scene)
    c.prepare_fast()
    return c


def same(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint8), np.ascontiguousarray(b).view(np.uint8))


@pytest.fixture(scope="module")
def instanced():
    return scenes.instanced_meshes(width=640, height=360)


def random_rays(n, lo, hi, seed):
    rng = np.random.default_rng(seed)
    r = np.zeros(n, _lib.RAY)
    o = rng.uniform(lo, hi, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r["ox"], r["oy"], r["oz"] = o.T
    r["dx"], r["dy"], r["dz"] = d.T
    r["tnear"] = 0.001
    return r


def coplanar_only(got, want):
    """Rows where got and want differ must be hits on two surfaces that meet
    the ray within a few ulps of each other (coincident geometry, where the
    reference's own answer depends on its slab rounding and visit order)."""
    diff = (got.view(np.uint8).reshape(-1, 20) != want.view(np.uint8).reshape(-1, 20)).any(1)
    if not diff.any():
        return 0
    g, w = got[diff], want[diff]
    assert np.all(g["object"] != _lib.MISS) and np.all(w["object"] != _lib.MISS)
    ulp = np.spacing(np.abs(w["t"]).astype(np.float32))
    assert np.all(np.abs(g["t"] - w["t"]) <= 16 * ulp), "a mismatch is not a coplanar tie"
    return int(diff.sum())


def test_fast_cornell_bit_exact():
    s = scenes.cornell_box()
    with ctx_for(s) as c:
        rays = c.camera_rays()
        assert same(c.closest_hit(rays, _lib.VARIANT_FAST), O.closest_hit(s, rays))
        r = random_rays(200000, -2, 12, 3)
        r["dx"][:2000], r["dy"][:2000], r["dz"][:2000] = 0.0, -1.0, 0.0  # axis-parallel
        got, want = c.closest_hit(r, _lib.VARIANT_FAST), O.closest_hit(s, r)
    # The tall cube's bottom face lies in the floor's plane: rays from below
    # meet both within an ulp or two, the only place the answers may differ.
    n = coplanar_only(got, want)
    assert n <= 200


def test_fast_instanced_primary_and_bounce_bit_exact(instanced):
    s = instanced
    with ctx_for(s) as c:
        prim = c.camera_rays()
        want = O.closest_hit(s, prim)
        got = c.closest_hit(prim, _lib.VARIANT_FAST)
        assert same(got, want)
        bounce, valid = c.bounce_rays(prim, want)
        b = bounce[valid]
        assert same(c.closest_hit(b, _lib.VARIANT_FAST), O.closest_hit(s, b))


@pytest.mark.parametrize("variant", [_lib.VARIANT_FAST_WALK])
def test_walk_variant_equals_fast(instanced, variant):
    """FAST_WALK (the same walk one step at a time per thread, persistent
    grid) returns FAST's hits byte for byte - coherent camera rays, bounce
    rays, random rays, ragged sizes."""
    s = instanced
    with ctx_for(s) as c:
        prim = c.camera_rays()
        fast = c.closest_hit(prim, _lib.VARIANT_FAST)
        assert same(c.closest_hit(prim, variant), fast)
        bounce, valid = c.bounce_rays(prim, fast)
        b = bounce[valid]
        assert same(c.closest_hit(b, variant), O.closest_hit(s, b))
        r = random_rays(300000, 0, 100, 6)
        assert same(c.closest_hit(r, variant), c.closest_hit(r, _lib.VARIANT_FAST))
        for n in (1, 31, 33, 1000):
            assert same(c.closest_hit(r[:n], variant), c.closest_hit(r[:n], _lib.VARIANT_FAST))


def test_walk_variant_large_device_batch(instanced):
    """A device-resident batch above 512K rays takes the walker's chunked
    assignment (warps claim runs of consecutive rays); its hits equal FAST's
    byte for byte, twice in a row (fresh and reused counters)."""
    import torch
    s = instanced
    with ctx_for(s) as c:
        prim = c.camera_rays()
        fast = c.closest_hit(prim, _lib.VARIANT_FAST)
        bounce, valid = c.bounce_rays(prim, fast)
        r = np.concatenate([bounce[valid], random_rays(600000, 0, 100, 9)])
        assert len(r) > (1 << 19)
        want = c.closest_hit(r, _lib.VARIANT_FAST)
        dev = torch.device("cuda", 0)
        d_r = torch.from_numpy(r.view(np.uint8)).to(dev)
        for _ in range(2):
            d_h = torch.zeros(len(r) * 20, dtype=torch.uint8, device=dev)
            torch.cuda.synchronize(dev)  # the library works on its own stream
            c.closest_hit_device(d_r.data_ptr(), len(r), d_h.data_ptr(), _lib.VARIANT_FAST_WALK)
            c.synchronize()
            got = d_h.cpu().numpy().view(_lib.HIT)
            assert same(got, want)


@pytest.mark.parametrize("variant", [_lib.VARIANT_FAST_WALK])
def test_walk_variant_cornell(variant):
    s = scenes.cornell_box()
    with ctx_for(s) as c:
        rays = c.camera_rays()
        assert same(c.closest_hit(rays, variant), O.closest_hit(s, rays))
        r = random_rays(100000, -2, 12, 7)
        assert same(c.closest_hit(r, variant), c.closest_hit(r, _lib.VARIANT_FAST))


def test_fast_random_rays_inside_scene(instanced):
    s = instanced
    with ctx_for(s) as c:
        r = random_rays(300000, 0, 100, 5)
        assert same(c.closest_hit(r, _lib.VARIANT_FAST), O.closest_hit(s, r))


def test_fast_ties_between_coincident_objects():
    """Two instances of one flat grid at the same place: every hit is hit
    twice at the same t, and the reference's visit order picks which; rays
    through grid vertices and diagonals add triangle-level ties.  Directions
    are tilted off the axes so no slab test multiplies zero by infinity."""
    rng = np.random.default_rng(8)
    lib = scenes.MeshLibrary()
    v, i = scenes.heightfield(33, 32.0, 0.0, rng)
    h = lib.add(v, i)
    ents = [scenes.entity(_lib.SHAPE_MESH, _lib.MAT_LAMBERTIAN, (0.0, 0.0, 0.0), mesh=h),
            scenes.entity(_lib.SHAPE_MESH, _lib.MAT_LAMBERTIAN, (0.0, 0.0, 0.0), mesh=h)]
    objects, tlas, lights, insts, order = scenes.pack(ents, lib)
    vv, ii, bb = lib.arrays()
    cfg = scenes.make_config(64, 64, (0.0, 10.0, 0.0), (0.0, 0.0, 0.01))
    s = scenes.PackedScene(objects, tlas, lights, vv, ii, bb, insts, cfg)
    n = 20000
    r = np.zeros(n, _lib.RAY)
    r["ox"] = rng.uniform(-15, 15, n).astype(np.float32)
    r["oz"] = rng.uniform(-15, 15, n).astype(np.float32)
    r["oy"] = 5.0
    d = np.stack([rng.uniform(-0.3, 0.3, n), -np.ones(n), rng.uniform(-0.3, 0.3, n)], 1)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r["dx"], r["dy"], r["dz"] = d.T.astype(np.float32)
    r["tnear"] = 0.001
    with Context(64, 64) as c:
        c.upload(s)
        c.prepare_fast()
        got = c.closest_hit(r, _lib.VARIANT_FAST)
        others = [c.closest_hit(r, _lib.VARIANT_FAST_WALK)]
    want = O.closest_hit(s, r)
    assert (want["object"] != _lib.MISS).mean() > 0.5
    assert same(got, want)
    for o in others:
        assert same(o, want)


def test_quant_primary_ids_and_values(instanced):
    s = instanced
    with ctx_for(s) as c:
        prim = c.camera_rays()
        want = O.closest_hit(s, prim)
        got = c.closest_hit(prim, _lib.VARIANT_QUANT)
    hit = want["object"] != _lib.MISS
    agree = (got["object"] == want["object"]) & (got["prim"] == want["prim"])
    # The watertight test and the reference's may only disagree where the ray
    # meets a shared edge: either both report a triangle of that edge, or the
    # reference falls through a crack and the watertight hit lies on an edge.
    dis = ~agree
    bary = np.stack([got["alpha"], got["beta"], 1 - got["alpha"] - got["beta"]], 1).min(1)
    bw = np.stack([want["alpha"], want["beta"], 1 - want["alpha"] - want["beta"]], 1).min(1)
    assert np.all((bary[dis] < 1e-3) | (bw[dis] < 1e-3)), "a disagreement away from every edge"
    assert agree.mean() >= 0.999
    both = agree & hit
    rel = np.abs(got["t"][both] - want["t"][both]) / np.maximum(want["t"][both], 1e-6)
    assert rel.max() < 1e-5
    # The reference's barycentrics come from a world-space difference of
    # nearly equal points (hybrid:591-594) and lose digits on small, distant
    # triangles; the sheared watertight form does not.  Agreement is close
    # everywhere and tight almost everywhere.
    da = np.abs(got["alpha"][both] - want["alpha"][both])
    db = np.abs(got["beta"][both] - want["beta"][both])
    assert max(da.max(), db.max()) < 0.05
    assert np.percentile(np.maximum(da, db), 99.9) < 1e-3


def test_fast_refuses_media():
    s = scenes.cornell_box()
    s.objects["colorType"][0] = _lib.MAT_ISOTROPIC
    with Context(64, 48) as c:
        c.upload(s)
        with pytest.raises(AeError):
            c.prepare_fast()


@pytest.mark.parametrize("variant", [_lib.VARIANT_FAST, _lib.VARIANT_QUANT, _lib.VARIANT_FAST_WALK])
def test_host_call_with_page_locked_buffers(instanced, variant):
    """ae_closest_hit over page-locked host buffers: FAST and QUANT trace them
    in place (the kernel reads rays and writes hits in host memory), the walker
    variant through its staged pipeline; the hits equal the device-pointer
    call's byte for byte, as with pageable buffers."""
    import torch
    s = instanced
    with ctx_for(s) as c:
        prim = c.camera_rays()
        r = np.concatenate([prim, random_rays(70001, 0, 100, 11)])
        h_r = torch.from_numpy(r.view(np.uint8).copy()).pin_memory()
        h_h = torch.zeros(len(r) * 20, dtype=torch.uint8).pin_memory()
        _lib.check(_lib.lib().ae_closest_hit(c.handle, h_r.data_ptr(), len(r), h_h.data_ptr(), variant), c.handle)
        dev = torch.device("cuda", 0)
        d_r = h_r.to(dev)
        d_h = torch.zeros(len(r) * 20, dtype=torch.uint8, device=dev)
        torch.cuda.synchronize(dev)
        c.closest_hit_device(d_r.data_ptr(), len(r), d_h.data_ptr(), variant)
        c.synchronize()
        assert torch.equal(h_h, d_h.cpu())
        assert same(h_h.numpy().view(_lib.HIT), c.closest_hit(r, variant))


def test_misaligned_rays(instanced):
    """Rays that do not start on a 16-byte boundary: the device-pointer call
    refuses them (AE_ERR_INVALID, nothing launched); the host-buffer call
    traces them through its aligned staging, page-locked or not."""
    import torch
    s = instanced
    with ctx_for(s) as c:
        r = random_rays(5000, 0, 100, 12)
        want = c.closest_hit(r, _lib.VARIANT_FAST)
        dev = torch.device("cuda", 0)
        d_r = torch.zeros(len(r) * 32 + 16, dtype=torch.uint8, device=dev)
        d_h = torch.zeros(len(r) * 20, dtype=torch.uint8, device=dev)
        with pytest.raises(AeError) as e:
            c.closest_hit_device(d_r.data_ptr() + 4, len(r), d_h.data_ptr(), _lib.VARIANT_FAST)
        assert e.value.code == -1
        h_buf = torch.zeros(len(r) * 32 + 16, dtype=torch.uint8).pin_memory()
        h_buf[8:8 + len(r) * 32].copy_(torch.from_numpy(r.view(np.uint8)))
        for variant in (_lib.VARIANT_FAST, _lib.VARIANT_QUANT):
            h_h = torch.zeros(len(r) * 20, dtype=torch.uint8).pin_memory()
            _lib.check(_lib.lib().ae_closest_hit(c.handle, h_buf.data_ptr() + 8, len(r), h_h.data_ptr(), variant),
                       c.handle)
            assert same(h_h.numpy().view(_lib.HIT), c.closest_hit(r, variant))
        assert same(c.closest_hit(r, _lib.VARIANT_FAST), want)
