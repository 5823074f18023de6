"""TEST INFRASTRUCTURE ONLY.  Packs the closest-hit workload's scene with the
reference's own CPU scene code (oracle/_ref/libaeref_scene.so), for the
reference arm of the benchmark and for the test that the library packs the
same bytes.

Input: the workload spec of aviatorengine2_b200/synth.py (seeded meshes,
instance transforms and materials, camera), which loads no native code.  The
steps are RebuildAcceleration's (renderer/renderer.cpp:1087-1130):
  * MeshLibrary::Add per mesh (scene/mesh_library.h:91-159) through
    aeref_mesh_add_u32: the reference's own bounds helpers and BuildBVH;
  * MeshBounds per instance (scene/shapes.h:124-145) through the reference's
    own function; a scaled instance passes its local box scaled by its scale,
    which gives the scaled corners the library's instance-scale extension
    (MeshInstance_GPU::pad0) transforms;
  * BuildBVH over those boxes (scene/bvh.h:275-295) for the TLAS;
  * PackObjects (renderer/renderer.cpp:815-929): objects in slot order through
    the reference's MeshToGPU, instance records with the mesh ranges, light
    slots (LightIndices, 803-813);
  * the camera fields of Config (renderer/renderer.h:76-159) as
    Renderer::Initialize and SyncCamera fill them.
"""
import ctypes
import hashlib
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SCENE = os.path.join(HERE, "_ref", "libaeref_scene.so")


def _layouts():
    import importlib.util
    spec = importlib.util.spec_from_file_location("ae_oracle_layouts", os.path.join(HERE, "layouts.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


L = _layouts()


def available():
    return os.path.exists(REF_SCENE)


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


class Scene:
    """The seven arrays of RenderFrame's bind order plus the config."""

    def __init__(self, objects, tlas, lights, vertices, indices, blas, instances, config, name):
        self.objects, self.tlas, self.lights = objects, tlas, lights
        self.vertices, self.indices, self.blas, self.instances = vertices, indices, blas, instances
        self.config, self.name = config, name
        self.textures = None

    @property
    def triangles(self):
        return len(self.indices) // 3


def make_config(width, height, source, target, fov, depth, sky):
    """Config for a pinhole camera: Renderer::Initialize's defaults with the
    camera, sky and depth of the workload (renderer/renderer.cpp:104-120)."""
    c = np.zeros(1, L.CONFIG)[0]
    c["source_x"], c["source_y"], c["source_z"] = source
    c["target_x"], c["target_y"], c["target_z"] = target
    c["up_x"], c["up_y"], c["up_z"] = 0.0, 1.0, 0.0
    c["fov"], c["focus_dist"] = fov, 1.0
    c["width"], c["height"] = width, height
    c["samples"], c["batches"], c["depth"] = 1, 1, depth
    c["sky_r"], c["sky_g"], c["sky_b"] = sky
    c["exposure"] = 1.0
    c["traceScale"] = 1.0
    c["historyCap"] = 32.0
    c["zNear"], c["zFar"] = 0.1, 10000.0
    return c


def build_instanced(spec):
    """The packed scene of synth.instanced_meshes_spec(...) built by the
    reference's code.  Every instance is a Lambertian mesh."""
    lib = ctypes.CDLL(REF_SCENE)
    u32 = ctypes.c_uint32
    vertices, indices, blas, ranges = [], [], [], []
    nv = ni = nb = 0
    for rows, idx in spec["geometry"]:
        v = np.ascontiguousarray(rows, np.float32).view(L.VERTEX).reshape(-1)
        i = np.ascontiguousarray(idx, np.uint32)
        nodes = np.zeros(max(2 * (len(i) // 3), 1), L.NODE)
        out_idx = np.zeros(max(len(i), 1), np.uint32)
        local = np.zeros(6, np.float32)
        cnt = u32()
        lib.aeref_mesh_add_u32(_ptr(v), u32(len(v)), _ptr(i), u32(len(i)), _ptr(nodes), ctypes.byref(cnt),
                               _ptr(out_idx), _ptr(local))
        ranges.append(dict(vertexBase=nv, indexBase=ni, triangleCount=len(i) // 3, blasBase=nb, local=local))
        vertices.append(v)
        indices.append(out_idx[:len(i)])
        blas.append(nodes[:cnt.value])
        nv, ni, nb = nv + len(v), ni + len(i), nb + cnt.value

    ents = spec["instances"]
    n = len(ents)
    bounds = np.zeros((n, 6), np.float32)
    for k, e in enumerate(ents):
        local = ranges[e["mesh"]]["local"]
        s = np.float32(e["scale"])
        if s != 0 and s != 1:
            local = (local * s).astype(np.float32)
        pos = np.asarray(e["position"], np.float32)
        rot = np.asarray(e["rotation"], np.float32)
        lib.aeref_mesh_bounds(_ptr(pos), _ptr(rot), _ptr(np.ascontiguousarray(local)), _ptr(bounds[k]))
    tlas = np.zeros(max(2 * n, 1), L.NODE)
    order = np.zeros(max(n, 1), np.uint32)
    cnt = u32()
    lib.aeref_build_bvh(_ptr(bounds), u32(n), _ptr(tlas), ctypes.byref(cnt), _ptr(order))
    tlas = tlas[:cnt.value].copy()

    objects = np.zeros(n, L.OBJECT)
    instances = np.zeros(n, L.INSTANCE)
    lights = []
    for slot in range(n):
        e = ents[order[slot]]
        r = ranges[e["mesh"]]
        pos = np.asarray(e["position"], np.float32)
        rot = np.asarray(e["rotation"], np.float32)
        alb = np.asarray(e["albedo"], np.float32)
        kind = int(e.get("material", L.MAT_LAMBERTIAN))
        lib.aeref_mesh_object(_ptr(pos), _ptr(rot), _ptr(alb), u32(kind), ctypes.c_float(e.get("fuzz", 0.0)),
                              ctypes.c_float(e.get("ior", 1.0)), ctypes.c_float(e.get("emission", 0.0)),
                              ctypes.c_float(e.get("density", 0.0)), u32(slot), _ptr(objects[slot:slot + 1]))
        if kind == L.MAT_DIFFUSE_LIGHT:
            lights.append(slot)
        inst = instances[slot]
        inst["px"], inst["py"], inst["pz"] = pos
        inst["qx"], inst["qy"], inst["qz"], inst["qw"] = rot
        s = np.float32(e["scale"])
        inst["scale"] = s if (s != 0 and s != 1) else 0.0
        for f in ("vertexBase", "indexBase", "triangleCount", "blasBase"):
            inst[f] = r[f]
    cam = spec["camera"]
    cfg = make_config(cam["width"], cam["height"], cam["source"], cam["target"], cam["fov"], cam["depth"], cam["sky"])
    cfg["num_lights"] = len(lights)
    cfg["num_spheres"] = n
    return Scene(objects, tlas, np.array(lights, np.uint32), np.concatenate(vertices), np.concatenate(indices),
                 np.concatenate(blas), instances, cfg, "instanced_meshes")


def scene_digest(scene):
    """SHA-256 over the seven device arrays and the config, in bind order."""
    h = hashlib.sha256()
    for a in (scene.objects, scene.tlas, scene.lights, scene.vertices, scene.indices, scene.blas, scene.instances):
        h.update(np.ascontiguousarray(a).view(np.uint8).tobytes())
    h.update(np.ascontiguousarray(np.array(scene.config).reshape(1)).view(np.uint8).tobytes())
    return h.hexdigest()[:16]


def rays_digest(rays):
    return hashlib.sha256(np.ascontiguousarray(rays).view(np.uint8).tobytes()).hexdigest()[:16]
