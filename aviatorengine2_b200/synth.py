"""Seeded synthetic geometry of the measured workloads, in plain numpy.

This module imports nothing from the package and loads no native code: it is
the workload definition both sides of a comparison share (the library's scene
packing in scenes.py, and a CPU implementation that builds the same scene with
its own code).  Vertices come back as (n, 8) float32 rows p.xyz, n.xyz, uv -
the byte layout of Vertex_GPU (scene/mesh_library.h:39-46) - and indices as a
flat uint32 triangle list.
"""
import numpy as np


def vertex_rows(p, n, uv):
    """(n, 8) float32 rows of positions, normals and UVs."""
    out = np.zeros((len(p), 8), np.float32)
    out[:, 0:3] = p
    out[:, 3:6] = n
    out[:, 6:8] = uv
    return out


def icosphere(level, radius=1.0):
    """Icosahedron subdivided `level` times, projected to a sphere:
    20 * 4^level triangles."""
    t = (1.0 + 5 ** 0.5) / 2.0
    p = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], np.float64)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                  [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5], [2, 4, 11],
                  [6, 2, 10], [8, 6, 7], [9, 8, 1]], np.int64)
    p /= np.linalg.norm(p, axis=1, keepdims=True)
    for _ in range(level):
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        e.sort(axis=1)
        key = e[:, 0] * (len(p) + 1) + e[:, 1]
        uniq, inv = np.unique(key, return_inverse=True)
        a, b = uniq // (len(p) + 1), uniq % (len(p) + 1)
        mid = p[a] + p[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        m = (inv + len(p)).reshape(3, -1).T  # mids of edges 01, 12, 20
        p = np.concatenate([p, mid])
        f = np.concatenate([np.stack([f[:, 0], m[:, 0], m[:, 2]], 1), np.stack([f[:, 1], m[:, 1], m[:, 0]], 1),
                            np.stack([f[:, 2], m[:, 2], m[:, 1]], 1), m])
    n = p.astype(np.float32)
    pos = (p * radius).astype(np.float32)
    uv = np.stack([0.5 + np.arctan2(p[:, 2], p[:, 0]) / (2 * np.pi), 0.5 - np.arcsin(p[:, 1]) / np.pi], 1)
    return vertex_rows(pos, n, uv.astype(np.float32)), f.astype(np.uint32).ravel()


def value_noise(n, cells, rng):
    """Smooth value noise on an n x n grid: random lattice values on a
    (cells+1)^2 lattice, bicubic-smoothstep interpolated."""
    lat = rng.uniform(-1.0, 1.0, size=(cells + 1, cells + 1))
    x = np.linspace(0, cells, n, endpoint=False)
    i = np.floor(x).astype(int)
    fr = x - i
    s = fr * fr * (3 - 2 * fr)
    a = lat[np.ix_(i, i)]
    b = lat[np.ix_(i + 1, i)]
    c = lat[np.ix_(i, i + 1)]
    d = lat[np.ix_(i + 1, i + 1)]
    sy, sx = s[:, None], s[None, :]
    return (a * (1 - sy) + b * sy) * (1 - sx) + (c * (1 - sy) + d * sy) * sx


def heightfield(n, size, amplitude, rng):
    """n x n vertex grid over [-size/2, size/2]^2 in x/z with value-noise height
    (three octaves); 2 (n-1)^2 triangles."""
    h = (value_noise(n, 8, rng) + 0.5 * value_noise(n, 16, rng) + 0.25 * value_noise(n, 32, rng)) * amplitude
    g = np.linspace(-size / 2, size / 2, n)
    X, Z = np.meshgrid(g, g, indexing="xy")
    pos = np.stack([X, h, Z], -1).reshape(-1, 3)
    dx = np.gradient(h, g, axis=1)
    dz = np.gradient(h, g, axis=0)
    nrm = np.stack([-dx, np.ones_like(h), -dz], -1).reshape(-1, 3)
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    uu, vv = np.meshgrid(np.linspace(0, 1, n), np.linspace(0, 1, n), indexing="xy")
    uv = np.stack([uu, vv], -1).reshape(-1, 2)
    r = np.arange(n - 1)
    i00 = (r[:, None] * n + r[None, :]).ravel()
    i10, i01, i11 = i00 + 1, i00 + n, i00 + n + 1
    tris = np.stack([np.stack([i00, i01, i10], 1), np.stack([i10, i01, i11], 1)], 1).reshape(-1, 3)
    return vertex_rows(pos.astype(np.float32), nrm.astype(np.float32), uv.astype(np.float32)), \
        tris.astype(np.uint32).ravel()


def random_quat(rng):
    """Uniform random rotation (Shoemake's method), x,y,z,w."""
    u1, u2, u3 = rng.random(3)
    a, b = np.sqrt(1 - u1), np.sqrt(u1)
    return (a * np.sin(2 * np.pi * u2), a * np.cos(2 * np.pi * u2), b * np.sin(2 * np.pi * u3),
            b * np.cos(2 * np.pi * u3))


def instanced_meshes_spec(seed=2, width=1920, height=1080, levels=(7, 6, 6, 5, 5), grid=512, n_instances=64,
                          n_heightfields=3):
    """The closest-hit workload before any acceleration structure exists:
    8 unique meshes (3 value-noise heightfields of grid^2 vertices, icospheres
    at `levels`), 64 Lambertian instances with random rotation, scale uniform
    in [0.5, 2] and translation uniform in a 100^3 box, and the pinhole camera.
    Returns a dict: geometry [(vertex rows, indices)], instances [dict(position,
    rotation, scale, albedo, mesh)], camera dict(width, height, source, target,
    fov, depth, sky)."""
    rng = np.random.default_rng(seed)
    geometry = [heightfield(grid, 20.0, 2.5, rng) for _ in range(n_heightfields)]
    geometry += [icosphere(lv, 5.0) for lv in levels]
    instances = []
    for k in range(n_instances):
        pos = tuple(float(x) for x in rng.uniform(0.0, 100.0, 3))
        rot = random_quat(rng)
        scale = float(rng.uniform(0.5, 2.0))
        albedo = tuple(float(x) for x in rng.uniform(0.2, 0.8, 3))
        instances.append(dict(position=pos, rotation=rot, scale=scale, albedo=albedo, mesh=k % len(geometry)))
    camera = dict(width=width, height=height, source=(50.0, 55.0, 175.0), target=(50.0, 50.0, 50.0), fov=40.0,
                  depth=2, sky=(0.5, 0.6, 0.8))
    return dict(geometry=geometry, instances=instances, camera=camera)
