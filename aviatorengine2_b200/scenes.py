"""Scene authoring and the seeded synthetic scenes of the measured workloads.

Mirrors the reference's authoring split: meshes go into a MeshLibrary (one BLAS
each, scene/mesh_library.h:91-159), renderable entities carry a transform and
a material (scene/components.h), and packing builds the TLAS and the byte
arrays the device reads (renderer/renderer.cpp:1087-1130).  Emissive surfaces
are analytic quads, as Scene::MeshEligible routes them (scene/scene.h:543-546).

Workloads (all inputs seeded; no dataset is involved):
  cornell_box      320x240 closed box: 5 mesh-quad walls, 2 rotated mesh cubes,
                   1 analytic emissive quad (radiance 15), 8 TLAS objects,
                   albedo uniform in [0.2, 0.8]^3, fov 40, black sky.
  instanced_meshes 64 instances of 8 procedural meshes (3 value-noise
                   heightfields of 512x512 vertices, icospheres at levels
                   7, 6, 6, 5, 5), 2,099,206 unique triangles; random rotation,
                   uniform scale in [0.5, 2], translation in a 100^3 box.
  wavefront_scene  1024 instances of 32 meshes (heightfields and icospheres
                   from the generators above), about 10M unique triangles;
                   materials per mesh 60% Lambertian, 25% metal (fuzz =
                   roughness in [0.05, 0.6], or GGX rough metal of that
                   roughness with ggx=True), 15% dielectric (IOR 1.5); 16
                   emissive quads above the field.
  hybrid_box       the Cornell box plus analytic spheres and boxes, for the
                   hybrid renderer's raster/analytic split.
  textured_box     the Cornell box with textured materials on every shape.
  media_box        the Cornell box with isotropic volumes (a box and a
                   sphere), an analytic triangle and a moving sphere.
  serving_scenes   8 scenes built like wavefront_scene with 50k to 5M unique
                   triangles and 512 instances each (4096 in all), whose
                   instances move along seeded random walks (random_walk).
"""
import ctypes

import numpy as np

from . import _lib, synth
from ._lib import check, lib, ptr


# ---------------------------------------------------------------------------
# Mesh library
# ---------------------------------------------------------------------------
class MeshLibrary:
    """MeshLibrary of scene/mesh_library.h over the C ABI.  With gpu=True each
    add() builds its BLAS on the GPU (ae_mesh_library_add_gpu: the same
    bytes as the host build)."""

    def __init__(self, gpu=False):
        self.gpu = bool(gpu)
        self._h = lib().ae_mesh_library_create()
        if not self._h:
            raise MemoryError("ae_mesh_library_create")

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            lib().ae_mesh_library_destroy(h)

    def add(self, vertices, indices, double_sided=False):
        v = np.ascontiguousarray(vertices, dtype=_lib.VERTEX)
        i = np.ascontiguousarray(indices, dtype=np.uint32).ravel()
        fn = "ae_mesh_library_add_gpu" if self.gpu else "ae_mesh_library_add"
        handle = getattr(lib(), fn)(self._h, ptr(v), len(v), ptr(i), len(i), int(double_sided))
        if handle < 0:
            raise _lib.AeError(handle, fn)
        return handle

    def add_many(self, meshes, double_sided=None):
        """add() for a list of (vertices, indices); with gpu=True the BLAS are
        built together (ae_mesh_library_add_many_gpu: the same bytes as k
        add() calls).  Returns the handles."""
        if not self.gpu:
            ds = double_sided or [False] * len(meshes)
            return [self.add(v, i, d) for (v, i), d in zip(meshes, ds)]
        vs = [np.ascontiguousarray(v, dtype=_lib.VERTEX) for v, _ in meshes]
        ix = [np.ascontiguousarray(i, dtype=np.uint32).ravel() for _, i in meshes]
        k = len(meshes)
        vp = (ctypes.c_void_p * k)(*[a.ctypes.data for a in vs])
        ip = (ctypes.c_void_p * k)(*[a.ctypes.data for a in ix])
        nv = np.array([len(a) for a in vs], np.uint32)
        ni = np.array([len(a) for a in ix], np.uint32)
        ds = np.array([int(bool(d)) for d in (double_sided or [False] * k)], np.int32)
        out = np.zeros(max(k, 1), np.int32)
        check(lib().ae_mesh_library_add_many_gpu(self._h, k, vp, ptr(nv), ip, ptr(ni), ptr(ds), ptr(out)),
              what="ae_mesh_library_add_many_gpu")
        return [int(h) for h in out[:k]]

    def range(self, handle):
        r = np.zeros(1, _lib.MESH_RANGE)
        check(lib().ae_mesh_library_range(self._h, handle, ptr(r)), what="ae_mesh_library_range")
        return r[0]

    def arrays(self):
        nv, ni, nb = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        L = lib()
        L.ae_mesh_library_sizes(self._h, ctypes.byref(nv), ctypes.byref(ni), ctypes.byref(nb))

        def view(p, n, dt):
            if n == 0:
                return np.zeros(0, dt)
            buf = (ctypes.c_char * (n * dt.itemsize)).from_address(p)
            return np.frombuffer(buf, dtype=dt).copy()

        return (view(L.ae_mesh_library_vertices(self._h), nv.value, _lib.VERTEX),
                view(L.ae_mesh_library_indices(self._h), ni.value, np.dtype(np.uint32)),
                view(L.ae_mesh_library_blas(self._h), nb.value, _lib.NODE))

    @property
    def handle(self):
        return self._h


def build_bvh(bounds, gpu=False, warp_subtree=None):
    """BuildBVH (scene/bvh.h:275-295) over an (n, 6) float32 array of boxes;
    gpu=True runs the device builder (ae_build_bvh_gpu, same output), with
    `warp_subtree` as its phase threshold when given."""
    b = np.ascontiguousarray(bounds, dtype=np.float32).reshape(-1, 6)
    n = len(b)
    nodes = np.zeros(max(2 * n, 1), _lib.NODE)
    order = np.zeros(max(n, 1), np.uint32)
    count = ctypes.c_uint32()
    if gpu and warp_subtree is not None:
        fn = "ae_build_bvh_gpu_ex"
        rc = lib().ae_build_bvh_gpu_ex(ptr(b), n, int(warp_subtree), ptr(nodes), ctypes.byref(count), ptr(order))
    else:
        fn = "ae_build_bvh_gpu" if gpu else "ae_build_bvh"
        rc = getattr(lib(), fn)(ptr(b), n, ptr(nodes), ctypes.byref(count), ptr(order))
    check(rc, what=fn)
    return nodes[:count.value].copy(), order[:n].copy()


# ---------------------------------------------------------------------------
# Mesh generators (local space, outward normals, counter-clockwise winding)
# ---------------------------------------------------------------------------
def _verts(p, n, uv):
    v = np.zeros(len(p), _lib.VERTEX)
    v["px"], v["py"], v["pz"] = p[:, 0], p[:, 1], p[:, 2]
    v["nx"], v["ny"], v["nz"] = n[:, 0], n[:, 1], n[:, 2]
    v["u"], v["v"] = uv[:, 0], uv[:, 1]
    return v


def quad_mesh(u, v):
    """A parallelogram spanning u and v, centred on its middle (the mesh twin of
    an analytic quad, Mesh::CreateQuad in scene/mesh.h:248-268)."""
    u = np.asarray(u, np.float32)
    v = np.asarray(v, np.float32)
    n = np.cross(u, v)
    n = (n / np.linalg.norm(n)).astype(np.float32)
    corners = np.array([0 * u, u, u + v, v], np.float32) - (u + v) * np.float32(0.5)
    uv = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32)
    return _verts(corners, np.tile(n, (4, 1)), uv), np.array([0, 1, 2, 0, 2, 3], np.uint32)


def box_mesh(half):
    """A box of 12 triangles with per-face normals (Mesh::CreateBox layout)."""
    hx, hy, hz = (np.float32(h) for h in half)
    faces = [((0, 0, 1), [(-hx, -hy, hz), (hx, -hy, hz), (hx, hy, hz), (-hx, hy, hz)]),
             ((0, 0, -1), [(hx, -hy, -hz), (-hx, -hy, -hz), (-hx, hy, -hz), (hx, hy, -hz)]),
             ((-1, 0, 0), [(-hx, -hy, -hz), (-hx, -hy, hz), (-hx, hy, hz), (-hx, hy, -hz)]),
             ((1, 0, 0), [(hx, -hy, hz), (hx, -hy, -hz), (hx, hy, -hz), (hx, hy, hz)]),
             ((0, 1, 0), [(-hx, hy, hz), (hx, hy, hz), (hx, hy, -hz), (-hx, hy, -hz)]),
             ((0, -1, 0), [(-hx, -hy, -hz), (hx, -hy, -hz), (hx, -hy, hz), (-hx, -hy, hz)])]
    p, n, uv, idx = [], [], [], []
    for k, (nrm, quad) in enumerate(faces):
        p += quad
        n += [nrm] * 4
        uv += [(0, 0), (1, 0), (1, 1), (0, 1)]
        b = 4 * k
        idx += [b, b + 1, b + 2, b, b + 2, b + 3]
    return _verts(np.array(p, np.float32), np.array(n, np.float32), np.array(uv, np.float32)), np.array(idx, np.uint32)


def _rows(mesh):
    """synth's (vertex rows, indices) as (Vertex_GPU array, indices)."""
    rows, idx = mesh
    return np.ascontiguousarray(rows, np.float32).view(_lib.VERTEX).reshape(-1), idx


def icosphere(level, radius=1.0):
    """Icosahedron subdivided `level` times, projected to a sphere:
    20 * 4^level triangles (synth.icosphere)."""
    return _rows(synth.icosphere(level, radius))


def heightfield(n, size, amplitude, rng):
    """n x n vertex grid with three octaves of value-noise height;
    2 (n-1)^2 triangles (synth.heightfield)."""
    return _rows(synth.heightfield(n, size, amplitude, rng))


# ---------------------------------------------------------------------------
# Entities and packing
# ---------------------------------------------------------------------------
def entity(shape, material, position, rotation=(0.0, 0.0, 0.0, 1.0), albedo=(1, 1, 1), **kw):
    e = np.zeros(1, _lib.ENTITY)[0]
    e["shape"], e["material"] = shape, material
    e["position"], e["rotation"] = position, rotation
    e["prev_position"], e["prev_rotation"] = position, rotation
    e["albedo"] = albedo
    e["scale"] = kw.pop("scale", 1.0)
    e["ior"] = kw.pop("ior", 1.0)
    e["texture_id"] = _lib.NO_TEXTURE
    e["texture_tint"] = 0.25
    for k, v in kw.items():
        e[k] = v
    return e


def yaw_quat(radians):
    """Rotation about +Y, x,y,z,w (QuatY, math/quat.hpp:238)."""
    h = np.float32(radians) * np.float32(0.5)
    return (0.0, float(np.sin(h)), 0.0, float(np.cos(h)))


random_quat = synth.random_quat


class PackedScene:
    """The seven device arrays of RenderFrame's bind order
    (renderer/renderer.cpp:1456-1459) plus the config they were made for."""

    def __init__(self, objects, tlas, lights, vertices, indices, blas, instances, config, order=None, name="",
                 textures=None):
        self.objects, self.tlas, self.lights = objects, tlas, lights
        self.vertices, self.indices, self.blas, self.instances = vertices, indices, blas, instances
        self.config = config
        self.order = order
        self.name = name
        self.textures = textures  # (layers, height, width, 4) RGBA8 sRGB, or None

    @property
    def triangles(self):
        return len(self.indices) // 3

    def device_bytes(self):
        return sum(a.nbytes for a in (self.objects, self.tlas, self.lights, self.vertices, self.indices, self.blas,
                                      self.instances))


def pack(entities, meshes, gpu=False):
    """RebuildAcceleration minus the upload: TLAS over the entities, objects in
    slot order, light IDs, instances (renderer/renderer.cpp:1087-1130).
    gpu=True builds and packs on the GPU (ae_pack_scene_gpu, same bytes)."""
    ents = np.ascontiguousarray(np.array(entities, dtype=_lib.ENTITY))
    n = len(ents)
    objects = np.zeros(max(n, 1), _lib.OBJECT)
    nodes = np.zeros(2 * n + 1, _lib.NODE)
    lights = np.zeros(max(n, 1), np.uint32)
    insts = np.zeros(max(n, 1), _lib.INSTANCE)
    order = np.zeros(max(n, 1), np.uint32)
    nn, nl, ni = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
    fn = "ae_pack_scene_gpu" if gpu else "ae_pack_scene"
    check(getattr(lib(), fn)(ptr(ents), n, meshes.handle if meshes else None, ptr(objects), ptr(nodes),
                             ctypes.byref(nn), ptr(lights), ctypes.byref(nl), ptr(insts), ctypes.byref(ni),
                             ptr(order)), what=fn)
    return objects[:n].copy(), nodes[:nn.value].copy(), lights[:nl.value].copy(), insts[:ni.value].copy(), order[:n]


def make_config(width, height, source, target, fov=40.0, depth=8, sky=(0, 0, 0), samples=1, exposure=1.0):
    c = np.zeros(1, _lib.CONFIG)[0]
    c["source_x"], c["source_y"], c["source_z"] = source
    c["target_x"], c["target_y"], c["target_z"] = target
    c["up_x"], c["up_y"], c["up_z"] = 0.0, 1.0, 0.0
    c["fov"], c["focus_dist"] = fov, 1.0
    c["width"], c["height"] = width, height
    c["samples"], c["batches"], c["depth"] = samples, 1, depth
    c["sky_r"], c["sky_g"], c["sky_b"] = sky
    c["exposure"] = exposure
    c["traceScale"] = 1.0
    c["historyCap"] = 32.0
    c["zNear"], c["zFar"] = 0.1, 10000.0
    return c


def _finish(entities, meshes, config, name):
    objects, tlas, lights, insts, order = pack(entities, meshes)
    v, i, b = meshes.arrays()
    config = config.copy()
    config["num_lights"] = len(lights)
    config["num_spheres"] = len(objects)
    return PackedScene(objects, tlas, lights, v, i, b, insts, config, order, name)


def cornell_box(seed=1, width=320, height=240, depth=8):
    """Closed box of 5 mesh-quad walls, 2 yawed mesh cubes and an analytic
    emissive quad (8 objects, 36 triangles counting the light as 2)."""
    rng = np.random.default_rng(seed)
    meshes = MeshLibrary()
    ents = []
    L = 10.0

    def alb():
        return tuple(float(x) for x in rng.uniform(0.2, 0.8, 3))

    # The light first: the reference gathers quads before meshes.
    ents.append(entity(_lib.SHAPE_QUAD, _lib.MAT_DIFFUSE_LIGHT, (3.5, L - 0.01, 3.5), albedo=(1, 1, 1),
                       emission=15.0, u=(3.0, 0.0, 0.0), v=(0.0, 0.0, 3.0)))
    walls = [((L / 2, 0.0, L / 2), (0, 0, L), (L, 0, 0)),       # floor, normal +y
             ((L / 2, L, L / 2), (L, 0, 0), (0, 0, L)),         # ceiling, normal -y
             ((L / 2, L / 2, 0.0), (L, 0, 0), (0, L, 0)),       # back, normal +z
             ((0.0, L / 2, L / 2), (0, L, 0), (0, 0, L)),       # left, normal +x
             ((L, L / 2, L / 2), (0, 0, L), (0, L, 0))]         # right, normal -x
    for centre, u, v in walls:
        h = meshes.add(*quad_mesh(u, v), double_sided=True)
        ents.append(entity(_lib.SHAPE_MESH, _lib.MAT_LAMBERTIAN, centre, albedo=alb(), mesh=h))
    for centre, half, yaw in (((3.3, 1.5, 3.7), (1.5, 1.5, 1.5), -0.3), ((6.6, 3.0, 6.2), (1.5, 3.0, 1.5), 0.35)):
        h = meshes.add(*box_mesh(half))
        ents.append(entity(_lib.SHAPE_MESH, _lib.MAT_LAMBERTIAN, centre, rotation=yaw_quat(yaw), albedo=alb(), mesh=h))
    cfg = make_config(width, height, (5.0, 5.0, 24.0), (5.0, 5.0, 0.0), fov=40.0, depth=depth, sky=(0, 0, 0))
    return _finish(ents, meshes, cfg, "cornell_box")


def procedural_textures(layers=4, width=64, height=48, seed=9):
    """A texture array of RGBA8 sRGB layers (the shape BuildGPUArray makes):
    checkers, stripes and value noise of seeded colours, so neighbouring
    texels differ and bilinear blends are exercised."""
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:height, 0:width]
    out = np.zeros((layers, height, width, 4), np.uint8)
    for k in range(layers):
        c0, c1 = rng.integers(0, 256, 3), rng.integers(0, 256, 3)
        kind = k % 3
        if kind == 0:
            m = ((x // (4 + k)) + (y // (3 + k))) % 2
        elif kind == 1:
            m = ((x + 2 * y) // (5 + k)) % 2
        else:
            m = rng.random((height, width)) > 0.5
        img = np.where(m[..., None] != 0, c0, c1).astype(np.int64)
        img += rng.integers(-12, 13, img.shape)
        out[k, ..., :3] = np.clip(img, 0, 255)
        out[k, ..., 3] = 255
    return out


def textured_box(seed=6, width=160, height=120, depth=6):
    """The Cornell box with textured materials on every shape the
    intersectors give UVs for: mesh walls and a mesh icosphere (vertex UVs),
    an analytic quad (alpha, beta), an analytic sphere with a UV rotation
    (get_sphere_uv) and a yawed analytic box (BoxFaceUV); tints 0, 0.25 and
    1, a textured metal, and a 4-layer procedural texture array."""
    rng = np.random.default_rng(seed)
    meshes = MeshLibrary()
    ents = []
    L = 10.0
    ents.append(entity(_lib.SHAPE_QUAD, _lib.MAT_DIFFUSE_LIGHT, (3.5, L - 0.01, 3.5), albedo=(1, 1, 1),
                       emission=15.0, u=(3.0, 0.0, 0.0), v=(0.0, 0.0, 3.0)))
    walls = [((L / 2, 0.0, L / 2), (0, 0, L), (L, 0, 0)),
             ((L / 2, L, L / 2), (L, 0, 0), (0, 0, L)),
             ((L / 2, L / 2, 0.0), (L, 0, 0), (0, L, 0)),
             ((0.0, L / 2, L / 2), (0, L, 0), (0, 0, L)),
             ((L, L / 2, L / 2), (0, 0, L), (0, L, 0))]
    tints = (0.0, 0.25, 1.0)
    for k, (centre, u, v) in enumerate(walls):
        h = meshes.add(*quad_mesh(u, v), double_sided=True)
        ents.append(entity(_lib.SHAPE_MESH, _lib.MAT_LAMBERTIAN, centre, mesh=h,
                           albedo=tuple(float(a) for a in rng.uniform(0.3, 0.9, 3)),
                           texture_id=k % 4, texture_tint=tints[k % 3]))
    ico = meshes.add(*icosphere(3, 1.4))
    ents.append(entity(_lib.SHAPE_MESH, _lib.MAT_LAMBERTIAN, (7.0, 1.4, 3.0), mesh=ico, rotation=yaw_quat(0.7),
                       albedo=(0.8, 0.6, 0.4), texture_id=2, texture_tint=0.25))
    ents.append(entity(_lib.SHAPE_SPHERE, _lib.MAT_LAMBERTIAN, (3.0, 1.2, 6.5), radius=1.2,
                       rotation=yaw_quat(1.1), albedo=(0.9, 0.9, 0.9), texture_id=1, texture_tint=0.0))
    ents.append(entity(_lib.SHAPE_BOX, _lib.MAT_LAMBERTIAN, (6.5, 1.0, 7.0), half_extent=(1.0, 1.0, 0.8),
                       rotation=yaw_quat(-0.4), albedo=(0.7, 0.8, 0.9), texture_id=3, texture_tint=1.0))
    ents.append(entity(_lib.SHAPE_QUAD, _lib.MAT_LAMBERTIAN, (5.0, 6.0, 0.05), u=(3.0, 0.0, 0.0), v=(0.0, 2.0, 0.0),
                       albedo=(1.0, 1.0, 1.0), texture_id=0, texture_tint=0.25))
    ents.append(entity(_lib.SHAPE_SPHERE, _lib.MAT_METAL, (5.0, 3.5, 4.0), radius=0.9, fuzz=0.2,
                       albedo=(0.9, 0.85, 0.8), texture_id=2, texture_tint=0.25))
    cfg = make_config(width, height, (5.0, 5.0, 24.0), (5.0, 5.0, 0.0), fov=40.0, depth=depth, sky=(0, 0, 0))
    s = _finish(ents, meshes, cfg, "textured_box")
    s.textures = procedural_textures()
    return s


def instanced_meshes(seed=2, width=1920, height=1080, levels=(7, 6, 6, 5, 5), grid=512, n_instances=64,
                     n_heightfields=3, gpu_build=False):
    """64 instances over 8 unique meshes; 2,099,206 triangles at the defaults
    (synth.instanced_meshes_spec).  gpu_build: BLAS builds on the GPU
    (identical bytes)."""
    spec = synth.instanced_meshes_spec(seed, width, height, levels, grid, n_instances, n_heightfields)
    meshes = MeshLibrary(gpu=gpu_build)
    handles = meshes.add_many([_rows(m) for m in spec["geometry"]])
    ents = [entity(_lib.SHAPE_MESH, _lib.MAT_LAMBERTIAN, i["position"], rotation=i["rotation"], scale=i["scale"],
                   albedo=i["albedo"], mesh=handles[i["mesh"]]) for i in spec["instances"]]
    cam = spec["camera"]
    cfg = make_config(cam["width"], cam["height"], cam["source"], cam["target"], fov=cam["fov"], depth=cam["depth"],
                      sky=cam["sky"])
    return _finish(ents, meshes, cfg, "instanced_meshes")


def hybrid_box(seed=3, width=160, height=120, depth=4):
    """The Cornell box with every kind of primitive the hybrid renderer sorts:
    mesh walls and a mesh cube (rasterized), an unrotated solid box (raster
    proxy), a yawed box, a metal sphere and a glass sphere (analytic), and the
    emissive quad light."""
    s = cornell_box(seed=seed, width=width, height=height, depth=depth)
    rng = np.random.default_rng(seed)
    meshes = MeshLibrary()
    ents = []
    L = 10.0
    ents.append(entity(_lib.SHAPE_QUAD, _lib.MAT_DIFFUSE_LIGHT, (3.5, L - 0.01, 3.5), emission=15.0,
                       u=(3.0, 0.0, 0.0), v=(0.0, 0.0, 3.0)))
    ents.append(entity(_lib.SHAPE_SPHERE, _lib.MAT_METAL, (7.0, 1.2, 3.0), albedo=(0.8, 0.7, 0.5), radius=1.2,
                       fuzz=0.1))
    ents.append(entity(_lib.SHAPE_SPHERE, _lib.MAT_DIELECTRIC, (2.5, 4.5, 6.5), radius=1.0, ior=1.5))
    ents.append(entity(_lib.SHAPE_BOX, _lib.MAT_LAMBERTIAN, (2.0, 0.75, 7.5), albedo=(0.6, 0.3, 0.3),
                       half_extent=(0.75, 0.75, 0.75)))
    ents.append(entity(_lib.SHAPE_BOX, _lib.MAT_LAMBERTIAN, (8.0, 4.0, 7.0), rotation=yaw_quat(0.4),
                       albedo=(0.3, 0.6, 0.3), half_extent=(0.6, 1.0, 0.6)))
    walls = [((L / 2, 0.0, L / 2), (0, 0, L), (L, 0, 0)), ((L / 2, L, L / 2), (L, 0, 0), (0, 0, L)),
             ((L / 2, L / 2, 0.0), (L, 0, 0), (0, L, 0)), ((0.0, L / 2, L / 2), (0, L, 0), (0, 0, L)),
             ((L, L / 2, L / 2), (0, 0, L), (0, L, 0))]
    for centre, u, v in walls:
        h = meshes.add(*quad_mesh(u, v), double_sided=True)
        ents.append(entity(_lib.SHAPE_MESH, _lib.MAT_LAMBERTIAN, centre,
                           albedo=tuple(float(x) for x in rng.uniform(0.2, 0.8, 3)), mesh=h))
    h = meshes.add(*box_mesh((1.2, 1.2, 1.2)))
    ents.append(entity(_lib.SHAPE_MESH, _lib.MAT_LAMBERTIAN, (5.0, 1.2, 5.0), rotation=yaw_quat(0.5),
                       albedo=(0.7, 0.7, 0.2), mesh=h))
    cfg = s.config.copy()
    return _finish(ents, meshes, cfg, "hybrid_box")


def media_box(seed=7, width=128, height=96, depth=6):
    """The Cornell box with participating media and the remaining analytic
    shapes: an isotropic fog box and an isotropic smoke sphere (HitVolume,
    hybrid:779-822: one RNG draw per volume the walk tests; ISOTROPIC
    scattering, 1020-1025), an analytic triangle, a sphere moving over the
    shutter (Position2, the ray's time draw), and a glass box."""
    rng = np.random.default_rng(seed)
    meshes = MeshLibrary()
    ents = []
    L = 10.0
    ents.append(entity(_lib.SHAPE_QUAD, _lib.MAT_DIFFUSE_LIGHT, (3.5, L - 0.01, 3.5), emission=15.0,
                       u=(3.0, 0.0, 0.0), v=(0.0, 0.0, 3.0)))
    ents.append(entity(_lib.SHAPE_BOX, _lib.MAT_ISOTROPIC, (6.5, 2.0, 5.5), half_extent=(1.5, 2.0, 1.5),
                       rotation=yaw_quat(0.3), albedo=(0.8, 0.8, 0.9), density=0.35))
    ents.append(entity(_lib.SHAPE_SPHERE, _lib.MAT_ISOTROPIC, (3.0, 5.5, 4.5), radius=1.3, albedo=(0.9, 0.6, 0.4),
                       density=0.8))
    ents.append(entity(_lib.SHAPE_TRIANGLE, _lib.MAT_LAMBERTIAN, (1.0, 0.5, 8.0), u=(3.0, 0.0, 0.0),
                       v=(0.0, 3.0, -1.0), albedo=(0.3, 0.7, 0.4)))
    mover = entity(_lib.SHAPE_SPHERE, _lib.MAT_METAL, (2.5, 1.0, 2.5), radius=0.9, albedo=(0.8, 0.8, 0.8), fuzz=0.05)
    mover["prev_position"] = (3.3, 1.2, 2.8)  # Position2: where the shutter closes
    ents.append(mover)
    ents.append(entity(_lib.SHAPE_BOX, _lib.MAT_DIELECTRIC, (7.5, 6.5, 7.0), half_extent=(0.7, 0.7, 0.7),
                       rotation=yaw_quat(-0.6), ior=1.5))
    walls = [((L / 2, 0.0, L / 2), (0, 0, L), (L, 0, 0)), ((L / 2, L, L / 2), (L, 0, 0), (0, 0, L)),
             ((L / 2, L / 2, 0.0), (L, 0, 0), (0, L, 0)), ((0.0, L / 2, L / 2), (0, L, 0), (0, 0, L)),
             ((L, L / 2, L / 2), (0, 0, L), (0, L, 0))]
    for centre, u, v in walls:
        h = meshes.add(*quad_mesh(u, v), double_sided=True)
        ents.append(entity(_lib.SHAPE_MESH, _lib.MAT_LAMBERTIAN, centre,
                           albedo=tuple(float(x) for x in rng.uniform(0.2, 0.8, 3)), mesh=h))
    cfg = make_config(width, height, (5.0, 5.0, 24.0), (5.0, 5.0, 0.0), fov=40.0, depth=depth, sky=(0, 0, 0))
    return _finish(ents, meshes, cfg, "media_box")


def wavefront_meshes(rng, n_meshes=32, target_tris=10_000_000, metal=_lib.MAT_METAL):
    """wavefront_scene's unique meshes, alternating heightfields and
    icospheres sized to share `target_tris` triangles, and a material kind
    per mesh (60 % Lambertian, 25 % metal, 15 % dielectric); `metal` is the
    metal kind: MAT_METAL (the reference's fuzzed mirror) or MAT_GGX_METAL."""
    geometry, kinds = [], []
    budget = target_tris
    for k in range(n_meshes):
        remaining = n_meshes - k
        want = budget / remaining
        if k % 2 == 0:
            n = int(max(16, min(1024, round((want / 2) ** 0.5 + 1))))
            v, i = heightfield(n, 20.0, 2.5, rng)
        else:
            lv = int(max(2, min(8, round(np.log(max(want, 80) / 20) / np.log(4)))))
            v, i = icosphere(lv, 5.0)
        budget -= len(i) // 3
        geometry.append((v, i))
        r = rng.random()
        kinds.append(_lib.MAT_LAMBERTIAN if r < 0.6 else (metal if r < 0.85 else _lib.MAT_DIELECTRIC))
    return geometry, kinds


def wavefront_scene(seed=4, width=1920, height=1080, depth=12, n_meshes=32, n_instances=1024, n_lights=16,
                    target_tris=10_000_000, gpu_build=False, ggx=False):
    """The wavefront workload: meshes drawn from the heightfield and icosphere
    generators until about `target_tris` unique triangles, instanced 1024
    times, lit by 16 emissive quads.  Metal meshes are the reference's fuzzed
    mirror (fuzz = roughness in [0.05, 0.6]) or, with ggx=True, GGX rough
    metal of that roughness (MAT_GGX_METAL; the same random draws, so the
    scene is otherwise identical).  gpu_build: BLAS builds on the GPU."""
    rng = np.random.default_rng(seed)
    meshes = MeshLibrary(gpu=gpu_build)
    geometry, kinds = wavefront_meshes(rng, n_meshes, target_tris,
                                       metal=_lib.MAT_GGX_METAL if ggx else _lib.MAT_METAL)
    handles = meshes.add_many(geometry)
    mat = []
    for k in range(n_meshes):
        mat.append(dict(albedo=tuple(float(x) for x in rng.uniform(0.2, 0.8, 3)),
                        fuzz=float(rng.uniform(0.05, 0.6)), ior=1.5))
    ents = []
    for q in range(n_lights):
        x, z = (q % 4) * 50.0 + 5.0, (q // 4) * 50.0 + 5.0
        ents.append(entity(_lib.SHAPE_QUAD, _lib.MAT_DIFFUSE_LIGHT, (x, 120.0, z), emission=15.0,
                           u=(15.0, 0.0, 0.0), v=(0.0, 0.0, 15.0)))
    for k in range(n_instances):
        m = k % n_meshes
        pos = (float(rng.uniform(0, 200)), float(rng.uniform(0, 60)), float(rng.uniform(0, 200)))
        ents.append(entity(_lib.SHAPE_MESH, kinds[m], pos, rotation=random_quat(rng),
                           scale=float(rng.uniform(0.5, 2.0)), mesh=handles[m], **mat[m]))
    cfg = make_config(width, height, (100.0, 90.0, 330.0), (100.0, 30.0, 100.0), fov=40.0, depth=depth,
                      sky=(0.0, 0.0, 0.0))
    return _finish(ents, meshes, cfg, "wavefront_scene")


SERVING_TRIANGLES = (50_000, 120_000, 250_000, 500_000, 1_000_000, 2_000_000, 3_500_000, 5_000_000)


def serving_scenes(seed=5, tri_targets=SERVING_TRIANGLES, instances_per_scene=512, depth=8, n_meshes=8,
                   gpu_build=False):
    """The serving workload's resident scenes: wavefront_scene's generators
    and material mix at each triangle budget, `instances_per_scene` instances
    each, 16 emissive quads."""
    return [wavefront_scene(seed=seed + k, width=640, height=480, depth=depth, n_meshes=n_meshes,
                            n_instances=instances_per_scene, n_lights=16, target_tris=t, gpu_build=gpu_build)
            for k, t in enumerate(tri_targets)]


def random_walk(instances, rng, step=0.5, angle=0.05):
    """One step of every instance along a seeded random walk: a normal
    translation of `step` per axis and a rotation by a small random angle
    about a random axis; meshes, bases and scale are kept."""
    out = np.array(instances, copy=True)
    n = len(out)
    d = rng.normal(0.0, step, (n, 3)).astype(np.float32)
    out["px"] += d[:, 0]
    out["py"] += d[:, 1]
    out["pz"] += d[:, 2]
    axis = rng.normal(0.0, 1.0, (n, 3))
    axis /= np.linalg.norm(axis, axis=1, keepdims=True)
    th = rng.normal(0.0, angle, n) * 0.5
    dq = np.concatenate([axis * np.sin(th)[:, None], np.cos(th)[:, None]], axis=1)
    q = np.stack([out["qx"], out["qy"], out["qz"], out["qw"]], axis=1).astype(np.float64)
    # Hamilton product dq * q (x, y, z, w order).
    x1, y1, z1, w1 = dq.T
    x2, y2, z2, w2 = q.T
    r = np.stack([w1 * x2 + x1 * w2 + y1 * z2 - z1 * y2,
                  w1 * y2 - x1 * z2 + y1 * w2 + z1 * x2,
                  w1 * z2 + x1 * y2 - y1 * x2 + z1 * w2,
                  w1 * w2 - x1 * x2 - y1 * y2 - z1 * z2], axis=1)
    r /= np.linalg.norm(r, axis=1, keepdims=True)
    out["qx"], out["qy"], out["qz"], out["qw"] = (r[:, k].astype(np.float32) for k in range(4))
    return out
