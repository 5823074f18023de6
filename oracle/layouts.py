"""TEST INFRASTRUCTURE ONLY.  numpy dtypes of the reference's byte layouts, as
the oracle and the reference's own CPU code read them.

They restate the reference's structs so that nothing on the oracle side
imports the library under test:
  Vertex_GPU        scene/mesh_library.h:39-46       (32 B)
  BVHNode_GPU       scene/bvh.h:31-43                (48 B)
  Object_GPU        scene/gpu_types.h:26-81          (128 B)
  MeshInstance_GPU  scene/gpu_types.h:84-96          (48 B; pad0 carries the
                    workload's uniform instance scale, 0 = rigid)
  Config            renderer/renderer.h:76-159       (240 B)
  Ray / Hit         the closest-hit query records of the C ABI (32 B / 20 B)
tests/test_layouts.py checks them against the library's dtypes field by field.
"""
import numpy as np

VERTEX = np.dtype([("px", "<f4"), ("py", "<f4"), ("pz", "<f4"), ("nx", "<f4"), ("ny", "<f4"), ("nz", "<f4"),
                   ("u", "<f4"), ("v", "<f4")])
NODE = np.dtype([("min_x", "<f4"), ("min_y", "<f4"), ("min_z", "<f4"), ("pad0", "<f4"), ("max_x", "<f4"),
                 ("max_y", "<f4"), ("max_z", "<f4"), ("left", "<i4"), ("right", "<i4"), ("count", "<i4"),
                 ("padding", "<i4"), ("pad_trailing", "<i4")])
OBJECT = np.dtype([("x", "<f4"), ("y", "<f4"), ("z", "<f4"), ("prevRotX", "<f4"), ("x2", "<f4"), ("y2", "<f4"),
                   ("z2", "<f4"), ("radius", "<f4"), ("u_x", "<f4"), ("u_y", "<f4"), ("u_z", "<f4"),
                   ("prevRotY", "<f4"), ("v_x", "<f4"), ("v_y", "<f4"), ("v_z", "<f4"), ("prevRotZ", "<f4"),
                   ("half_x", "<f4"), ("half_y", "<f4"), ("half_z", "<f4"), ("rotation", "<f4"),
                   ("density", "<f4"), ("emission", "<f4"), ("instanceIndex", "<u4"), ("textureTint", "<f4"),
                   ("r", "<f4"), ("g", "<f4"), ("b", "<f4"), ("fuzz", "<f4"), ("refraction", "<f4"),
                   ("shapeType", "<u4"), ("colorType", "<u4"), ("textureID", "<u4")])
INSTANCE = np.dtype([("px", "<f4"), ("py", "<f4"), ("pz", "<f4"), ("scale", "<f4"), ("qx", "<f4"), ("qy", "<f4"),
                     ("qz", "<f4"), ("qw", "<f4"), ("vertexBase", "<u4"), ("indexBase", "<u4"),
                     ("triangleCount", "<u4"), ("blasBase", "<u4")])
RAY = np.dtype([("ox", "<f4"), ("oy", "<f4"), ("oz", "<f4"), ("tnear", "<f4"), ("dx", "<f4"), ("dy", "<f4"),
                ("dz", "<f4"), ("time", "<f4")])
HIT = np.dtype([("t", "<f4"), ("alpha", "<f4"), ("beta", "<f4"), ("object", "<u4"), ("prim", "<u4")])
CONFIG = np.dtype([("source_x", "<f4"), ("source_y", "<f4"), ("source_z", "<f4"), ("fov", "<f4"),
                   ("target_x", "<f4"), ("target_y", "<f4"), ("target_z", "<f4"), ("focus_dist", "<f4"),
                   ("defocus_angle", "<f4"), ("padding", "<f4", 3), ("up_x", "<f4"), ("up_y", "<f4"),
                   ("up_z", "<f4"), ("oof", "<f4"), ("sky_r", "<f4"), ("sky_g", "<f4"), ("sky_b", "<f4"),
                   ("width", "<u4"), ("horizon_r", "<f4"), ("horizon_g", "<f4"), ("horizon_b", "<f4"),
                   ("height", "<u4"), ("samples", "<u4"), ("batches", "<u4"), ("batch", "<u4"), ("depth", "<u4"),
                   ("num_spheres", "<u4"), ("renderType", "<u4"), ("num_lights", "<u4"), ("exposure", "<f4"),
                   ("debugView", "<u4"), ("zNear", "<f4"), ("zFar", "<f4"), ("jitter_x", "<f4"),
                   ("jitter_y", "<f4"), ("displayOnly", "<u4"), ("traceScale", "<f4"), ("frameIndex", "<u4"),
                   ("historyReset", "<u4"), ("cameraMoved", "<u4"), ("historyCap", "<f4"), ("padding3", "<f4"),
                   ("prevViewProj", "<f4", 16)])

# Shape and material enumerations (scene/gpu_types.h, scene/material.h:9-16).
SHAPE_MESH = 4
MAT_LAMBERTIAN, MAT_METAL, MAT_DIELECTRIC, MAT_DIFFUSE_LIGHT, MAT_ISOTROPIC = range(5)
MAT_GGX_METAL = 5  # the library's extension (rough metal, GGX microfacets); not a reference material
NO_TEXTURE = 0xFFFFFFFF  # kNoTexture, scene/texture.h
MISS = 0xFFFFFFFF

for _dt, _size in ((VERTEX, 32), (NODE, 48), (OBJECT, 128), (INSTANCE, 48), (RAY, 32), (HIT, 20), (CONFIG, 240)):
    assert _dt.itemsize == _size, (_dt, _size)
