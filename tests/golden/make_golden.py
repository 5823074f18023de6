"""Generates the golden fixtures of tests/golden/ from the REFERENCE's own code
run on the CPU: its scene headers (BuildBVH, MeshLibrary::Add) and its
compute-only shader, both compiled by oracle/Makefile into oracle/_ref/ from a
reference checkout (located by oracle/Makefile, AE_REFERENCE_DIR).  Run in a tree where
oracle/_ref/ is built:

    make -C oracle ref && python tests/golden/make_golden.py

The fixtures are small subsamples; the full-size comparisons run live in the
tests wherever oracle/_ref/ exists.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import _oracle as O  # noqa: E402
from aviatorengine2_b200 import scenes  # noqa: E402


def main():
    rng = np.random.default_rng(1234)
    out = {}

    # BuildBVH on random boxes, including flat and coincident ones.
    for k, n in enumerate((1, 5, 37, 1000)):
        c = rng.uniform(-10, 10, (n, 3)).astype(np.float32)
        e = rng.uniform(0, 2, (n, 3)).astype(np.float32)
        e[rng.random((n, 3)) < 0.2] = 0.0
        if n > 10:
            c[: n // 5] = c[0]
        boxes = np.concatenate([c - e, c + e], 1).astype(np.float32)
        nodes, order = O.ref_build_bvh(boxes)
        out[f"bvh{k}_boxes"], out[f"bvh{k}_nodes"], out[f"bvh{k}_order"] = boxes, nodes.view(np.uint8), order
    np.savez_compressed(os.path.join(HERE, "bvh_build.npz"), **out)

    # The Cornell box: 4096 camera rays and their closest hits; 1024 pixels
    # over 4 accumulated frames.
    s = scenes.cornell_box()
    cfg = s.config.copy()
    rays = O.camera_rays(cfg)
    pick = np.sort(rng.choice(len(rays), 4096, replace=False))
    hits = O.ref_closest_hit(s, rays[pick])
    px = np.stack([pick % cfg["width"], pick // cfg["width"]], 1)[:1024].astype(np.uint32)
    acc = None
    frames = []
    for b in range(4):
        cfg["batch"] = b
        acc, _ = O.ref_render(s, cfg, acc, pixels=px)
        frames.append(acc[px[:, 1], px[:, 0]].copy())
    np.savez_compressed(os.path.join(HERE, "cornell_box.npz"), rays=rays[pick].view(np.uint8),
                        hits=hits.view(np.uint8), pixels=px, accum=np.stack(frames))

    # Instanced meshes at 240x135, rigid instances (the reference has no scale).
    s = scenes.instanced_meshes(width=240, height=135, levels=(4, 3, 3, 2, 2), grid=64)
    s.instances["scale"] = 0.0
    rays = O.camera_rays(s.config)
    pick = np.sort(rng.choice(len(rays), 4096, replace=False))
    hits = O.ref_closest_hit(s, rays[pick])
    np.savez_compressed(os.path.join(HERE, "instanced_small.npz"), rays=rays[pick].view(np.uint8),
                        hits=hits.view(np.uint8))
    print("golden fixtures written")


if __name__ == "__main__":
    main()
