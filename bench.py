"""Closest-hit throughput of the ray-tracing hot path on one B200 (or N
independent replicas), with the reference's CPU implementation timed beside it.

Workload (`instanced_meshes`, seeded): 64 instances of 8 procedural meshes,
2,099,206 unique triangles (3 value-noise heightfields of 512x512 vertices,
icospheres at levels 7, 6, 6, 5, 5), random rotation, uniform scale in
[0.5, 2], translation in a 100^3 box.  One step traces the 1920x1080 camera
rays of frame 0 (2,073,600) and then one diffuse bounce ray per primary hit,
closest hit each, ray set already resident in HBM.  L2 is flushed (a 512 MB
write) before every timed step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--variant plain|fast|quant]

Prints one JSON line (rank 0).  Under torchrun each rank is an independent
replica on its own GPU (the path does not shard across GPUs); value is the
sum over ranks, timed as the max over ranks.
"""
import argparse
import ctypes
import hashlib
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "closest-hit Mrays/s (1080p primary + diffuse bounce rays, 2.1M-triangle instanced scene)"
UNIT = "Mrays/s"
VARIANTS = {"plain": 0, "fast": 1, "quant": 2, "walk": 3}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
             "clocks_event_reasons.sw_power_cap"

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[4 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def max_over_ranks(x, pg, device=None):
    """The largest of x over all ranks (x itself with no process group): the
    step time every replica's throughput is divided by."""
    if pg is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def replica_value(units_per_rank, world, seconds):
    """Whole-job throughput of `world` independent replicas that each process
    `units_per_rank` in `seconds` (the max over ranks), in millions per second."""
    return units_per_rank * world / seconds / 1e6


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic():
    """DRAM bytes per ray of the closest-hit kernel from a committed ncu
    summary (profiles/k_closest_fast_instanced_meshes_traffic.json), or None."""
    p = os.path.join(ROOT, "profiles", "k_closest_fast_instanced_meshes_traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return None


def make_workload(ctx, scene):
    """Primary rays of frame 0 and one diffuse bounce per primary hit."""
    from aviatorengine2_b200 import _lib
    prim = ctx.camera_rays()
    hits = ctx.closest_hit(prim, _lib.VARIANT_PLAIN)
    bounce, valid = ctx.bounce_rays(prim, hits)
    return prim, bounce[valid].copy()


def _oracle_modules():
    """The oracle bindings (tests/_oracle.py) and the reference-scene packer
    (oracle/ref_scene.py).  Neither imports the library under test."""
    for d in (os.path.join(ROOT, "tests"), os.path.join(ROOT, "oracle")):
        if d not in sys.path:
            sys.path.insert(0, d)
    import _oracle as O
    import ref_scene as R
    return O, R


def digest(*arrays):
    """First 16 hex digits of SHA-256 over the arrays' bytes, in order."""
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).view(np.uint8).tobytes())
    return h.hexdigest()[:16]


def scene_digest(scene):
    """Digest of the seven device arrays (RenderFrame's bind order) and the config."""
    return digest(scene.objects, scene.tlas, scene.lights, scene.vertices, scene.indices, scene.blas,
                  scene.instances, np.array(scene.config).reshape(1))


def workload_config(W, H, n_prim, n_bounce, triangles, instances, scene_dig, rays_dig, world):
    """The `config` object both arms print: the workload and nothing about
    the implementation, so equal dicts mean equal work."""
    return {"workload": f"instanced_meshes {W}x{H} primary+bounce closest hit",
            "rays_per_step": int(n_prim + n_bounce), "primary_rays": int(n_prim), "bounce_rays": int(n_bounce),
            "triangles": int(triangles), "instances": int(instances), "instance_scale": "uniform in [0.5, 2]",
            "scene_sha256_16": scene_dig, "rays_sha256_16": rays_dig,
            "l2": "GPU arm: flushed before every step (512 MB write)", "parallelism": f"replicas x{world}"}


def cpu_reference(scene, rays, budget_s=12.0, impl="port"):
    """The reference's closest hit on the CPU over a bounded sample of the ray
    set, all host cores: a random subset when the whole set would take longer
    than the budget, otherwise the whole set traced repeatedly until about
    `budget_s`.  impl "port": the oracle's restatement of the reference's
    traversal (TraverseBVH/HitMesh, hybrid:600-917) with the instance-scale
    extension, which traces this workload's scaled instances; impl
    "reference": the reference's own shader compiled for the CPU
    (oracle/_ref), which has rigid instances only."""
    O, _ = _oracle_modules()
    cores = os.cpu_count() or 1
    if impl == "reference" and not O.ref_available():
        raise RuntimeError("oracle/_ref is not built")
    fn = O.ref_closest_hit if impl == "reference" else O.closest_hit
    rng = np.random.default_rng(0)
    n = min(len(rays), 65536)
    probe = rays[np.sort(rng.choice(len(rays), n, replace=False))]
    t0 = time.perf_counter()
    fn(scene, probe, threads=cores)
    rate = n / max(time.perf_counter() - t0, 1e-6)
    want = int(rate * budget_s)
    if want < len(rays):
        sample = rays[np.sort(rng.choice(len(rays), max(want, n), replace=False))]
        passes = 1
    else:
        sample = rays
        passes = max(1, int(round(want / len(rays))))
    t0 = time.perf_counter()
    for _ in range(passes):
        fn(scene, sample, threads=cores)
    dt = time.perf_counter() - t0
    total = len(sample) * passes
    what = (f"{len(sample)} rays drawn uniformly from the step's {len(rays)}" if passes == 1 else
            f"the step's {len(rays)} rays (primary + bounce) traced {passes} times")
    return {"value": total / dt / 1e6, "unit": UNIT, "cores": cores, "kind": impl,
            "sample": f"{what}, {dt:.2f} s"}


EDGE_EPS = 1e-2   # minimum barycentric of a hit counted as lying at a triangle edge
TIE_REL = 1e-6    # relative depth difference of two hits counted as a tie
MRE_EPS = 1e-3


def classify_ids(ref, wt):
    """Primary-ray ID disagreements between the reference's triangle test
    (hybrid:564-598) and the watertight one, by cause:
      crack     - the watertight hit is nearer (or the reference missed) and
                  lies within EDGE_EPS (barycentric) of an edge: the
                  reference's test let the ray through between triangles;
      leak      - the reference's hit is nearer (or the watertight test
                  missed) and lies within EDGE_EPS of an edge: the
                  reference's test took a ray just outside its triangle;
      depth tie - two different surfaces within TIE_REL of the same depth,
                  ranked by each test's own rounding of t;
    and the rest, unexplained (must be none)."""
    from aviatorengine2_b200 import _lib

    def min_bary(h):
        a, b = h["alpha"].astype(np.float64), h["beta"].astype(np.float64)
        return np.where(h["prim"] != _lib.MISS, np.minimum(np.minimum(a, b), 1.0 - a - b), np.inf)

    dis = (ref["object"] != wt["object"]) | (ref["prim"] != wt["prim"])
    rh, wh = ref["object"] != _lib.MISS, wt["object"] != _lib.MISS
    tr, tw = ref["t"].astype(np.float64), wt["t"].astype(np.float64)
    crack = dis & wh & (~rh | (tw < tr)) & (min_bary(wt) < EDGE_EPS)
    leak = dis & rh & (~wh | (tr < tw)) & (min_bary(ref) < EDGE_EPS)
    tie = dis & rh & wh & (np.abs(tr - tw) <= TIE_REL * np.maximum(tr, tw))
    explained = crack | leak | tie
    rest = np.flatnonzero(dis & ~explained)
    examples = [{"ray": int(i), "ref": [int(ref["object"][i]), int(ref["prim"][i]), float(ref["t"][i]),
                                        float(min_bary(ref[i:i + 1])[0])],
                 "wt": [int(wt["object"][i]), int(wt["prim"][i]), float(wt["t"][i]), float(min_bary(wt[i:i + 1])[0])]}
                for i in rest[:8]]
    n_expl = int((dis & explained).sum())
    return {"rays": int(len(ref)), "agreement": float(1.0 - dis.mean()), "disagree": int(dis.sum()),
            "crack": int(crack.sum()), "leak": int((leak & ~crack).sum()), "depth_tie": int((tie & ~crack & ~leak).sum()),
            "within_1e-3_of_an_edge": int((dis & ((min_bary(wt) < 1e-3) | (min_bary(ref) < 1e-3))).sum()),
            "unexplained": int(len(rest)),
            "agreement_excluding_explained": float(1.0 - len(rest) / max(1, len(ref) - n_expl)),
            "edge_eps": EDGE_EPS, "tie_rel": TIE_REL, "unexplained_examples": examples}


def precision_ids(ctx, rays):
    """The precision closest hit's primary-ray IDs: against the FP32-node form
    with the same watertight test (must be identical: 8-bit outward-rounded
    bounds lose no hit) and against the reference's triangle test
    (classified)."""
    from aviatorengine2_b200 import _lib
    plain = ctx.closest_hit(rays, _lib.VARIANT_PLAIN)
    fp32 = ctx.closest_hit(rays, _lib.VARIANT_PLAIN_WT)
    quant = ctx.closest_hit(rays, _lib.VARIANT_QUANT)
    ids = (quant["object"] == fp32["object"]) & (quant["prim"] == fp32["prim"])
    return {"vs_fp32_nodes_same_test": {"agreement": float(ids.mean()),
                                        "bit_exact_hits": bool(np.array_equal(quant.view(np.uint8),
                                                                              fp32.view(np.uint8)))},
            "vs_reference_triangle_test": classify_ids(plain, quant)}


def fp64_reference(scene, config, frames, pixels):
    """The FP64 oracle's accumulation after `frames` frames at `pixels` only
    (the checker of the MRE figures; host cores).  The buffers are reused
    across frames: only the listed pixels are written."""
    O, _ = _oracle_modules()
    s = O.oscene(scene)
    c = np.ascontiguousarray(np.array(config, dtype=O._lib.CONFIG).reshape(1))
    w, h = int(c["width"][0]), int(c["height"][0])
    acc = np.zeros((h, w, 4), np.float64)
    disp = np.zeros((h, w, 4), np.float64)
    frame = np.zeros((h, w, 4), np.float64)
    xy = np.ascontiguousarray(pixels, dtype=np.uint32).reshape(-1, 2)
    fn = O.oracle().oracle_render_frame_f64
    for b in range(frames):
        c["batch"][0] = b
        fn(ctypes.byref(s), O.ptr(c), O.ptr(acc), O.ptr(disp), O.ptr(frame), O.ptr(xy), ctypes.c_uint32(len(xy)),
           ctypes.c_int(os.cpu_count() or 1))
    return acc[xy[:, 1], xy[:, 0]].copy()


def seeded_pixels(width, height, n, seed):
    rng = np.random.default_rng(seed)
    pick = np.sort(rng.choice(width * height, min(n, width * height), replace=False))
    return np.stack([pick % width, pick // width], 1).astype(np.uint32)


def measure_paths(local, width, height, frames=2, mre_pixels=1024, mre_frames=16, target_tris=10_000_000,
                  n_instances=1024):
    """Mpaths/s of compute-only frames (1 spp) on the wavefront workload:
    the plain megakernel against the wavefront form (4-wide 8-bit quantised
    BVH, persistent stages, CUDA graph) and its precision form (watertight
    test, FP16 shading normals, compensated accumulation).  Frames are timed
    on the device around the whole frame; the plain and wavefront images are
    compared, and primary-ray IDs of both optimised closest hits against the
    plain kernel's.  The images are scored against the FP64 oracle after
    `mre_frames` frames (the frames past the timed ones continue the same
    accumulation)."""
    from aviatorengine2_b200 import Context, _lib, scenes
    scene = scenes.wavefront_scene(width=width, height=height, gpu_build=True, ggx=True, target_tris=target_tris,
                                   n_instances=n_instances)
    _lib.lib().ae_bvh_builder_release()  # the device builder's scratch is not needed past the build
    out = {"workload": f"wavefront_scene {width}x{height}, 1 spp, depth {int(scene.config['depth'])}, "
                       f"{len(scene.lights)} lights, materials 60% Lambertian / 25% GGX metal / 15% dielectric",
           "triangles": int(scene.triangles),
           "instances": int(len(scene.instances)), "paths_per_frame": width * height}
    imgs = {}
    px = seeded_pixels(width, height, mre_pixels, 17) if mre_pixels > 0 else None
    n_frames = max(frames + 1, mre_frames if px is not None else 0)
    ref64 = fp64_reference(scene, scene.config, n_frames, px) if px is not None else None
    mre = {}
    with Context(width, height, device=local) as ctx:
        ctx.upload(scene)
        # Primary-ray instance and triangle IDs of the optimised closest hits
        # against the reference-order kernel, on this frame's camera rays.
        rays = ctx.camera_rays()
        ref = ctx.closest_hit(rays, _lib.VARIANT_PLAIN)
        h = ctx.closest_hit(rays, _lib.VARIANT_FAST)
        out["primary_id_agreement_fast"] = float(((h["object"] == ref["object"]) & (h["prim"] == ref["prim"])).mean())
        out["primary_ids_precision"] = precision_ids(ctx, rays)
        out["primary_id_agreement_precision"] = \
            out["primary_ids_precision"]["vs_reference_triangle_test"]["agreement"]
        # Algorithmic bytes of one frame of paths (the reference megakernel's
        # traversals, counted on the device): the Mpaths/s roofline.
        ctx.set_config(scene.config)
        pc = np.zeros(7, np.uint64)
        _lib.check(_lib.lib().ae_path_counters(ctx.handle, _lib.ptr(pc)), ctx.handle)
        per = np.array([48, 128, 48, 48, 48, 60], np.float64)
        bytes_per_path = float((pc[:6].astype(np.float64) * per).sum()) / (width * height)
        for name, mode in (("plain", _lib.MODE_COMPUTE_ONLY), ("wavefront", _lib.MODE_WAVEFRONT),
                           ("precision", _lib.MODE_WAVEFRONT_PRECISION)):
            c = scene.config.copy()
            ms = []
            for b in range(n_frames):  # frame 0 warms up (and autotunes the wavefront)
                c["batch"] = b
                ctx.set_config(c)
                ctx.render_frame(mode)
                ctx.synchronize()
                if 1 <= b <= frames:
                    ms.append(ctx.last_kernel_ms())
                if b == frames:
                    imgs[name] = ctx.read_image(_lib.IMAGE_FRAME)
            out[f"{name}_ms"] = float(np.mean(ms))
            out[f"{name}_mpaths"] = width * height / (float(np.mean(ms)) / 1e3) / 1e6
            if ref64 is not None:
                mre[name] = ctx.image_error_pixels(px, ref64, eps=MRE_EPS)["mre"]
        info = ctx.wavefront_info()
        out["wavefront_extend"] = {"threads": info["threads"], "stack": info["stack"]}
        out["walker_runs"] = {"wavefront": ctx.wavefront_walk_info(False), "precision": ctx.wavefront_walk_info(True)}
    out["speedup"] = out["wavefront_mpaths"] / out["plain_mpaths"]
    out["precision_speedup"] = out["precision_mpaths"] / out["plain_mpaths"]
    peak, peak_kind = load_peaks()
    roof = peak * 1e9 / bytes_per_path / 1e6
    out["roofline"] = {"bound": "hbm", "algorithmic_bytes_per_path": bytes_per_path,
                       "traversals_per_path": float(pc[6]) / (width * height), "peak_gbs": peak,
                       "peak_source": peak_kind, "roofline_mpaths": roof,
                       "frac": {k: out[f"{k}_mpaths"] / roof for k in ("plain", "wavefront", "precision")}}
    if mre:
        out["mre"] = {"reference": f"FP64 oracle (same estimator and RNG stream in double) after {n_frames} "
                                   f"frames at {len(px)} seeded pixels; reduced on the GPU in FP64; eps {MRE_EPS}",
                      **mre, "precision_over_plain": mre["precision"] / max(mre["plain"], 1e-300),
                      "wavefront_over_plain": mre["wavefront"] / max(mre["plain"], 1e-300)}
    a, b = imgs["plain"], imgs["wavefront"]
    out["frames_bit_exact"] = bool(np.array_equal(a.view(np.uint32), b.view(np.uint32)))
    out["pixels_differing"] = int(np.any(a.view(np.uint32) != b.view(np.uint32), axis=-1).sum())
    return out


def measure_config1(local, frames=16, budget_s=8.0, check_pixels=1024):
    """The plain method's small case: the Cornell box (8 objects, 36
    triangles) at 320x240, `frames` frames of 1 spp (16 spp accumulated),
    depth 8.  GPU: the plain megakernel and the wavefront form, each frame
    timed on the device.  CPU: the reference's own compute shader compiled
    for the CPU (oracle/_ref), all host cores, whole frames until about
    `budget_s`; its accumulation after all frames at `check_pixels` seeded
    pixels is compared with the GPU's bit for bit."""
    from aviatorengine2_b200 import Context, _lib, scenes
    O, _ = _oracle_modules()
    scene = scenes.cornell_box()
    W, H = int(scene.config["width"]), int(scene.config["height"])
    out = {"workload": f"cornell_box {W}x{H}, {frames} frames of 1 spp, depth {int(scene.config['depth'])}",
           "triangles": int(scene.triangles), "objects": int(len(scene.objects))}
    accs = {}
    with Context(W, H, device=local) as ctx:
        ctx.upload(scene)
        for name, mode in (("plain", _lib.MODE_COMPUTE_ONLY), ("wavefront", _lib.MODE_WAVEFRONT)):
            c = scene.config.copy()
            ms = []
            for rep in range(2):  # the first pass warms up (and tunes the wavefront)
                for b in range(frames):
                    c["batch"] = b
                    ctx.set_config(c)
                    ctx.render_frame(mode)
                    ctx.synchronize()
                    if rep:
                        ms.append(ctx.last_kernel_ms())
            accs[name] = ctx.read_image(_lib.IMAGE_ACCUM)
            out[name] = {"ms_per_frame": float(np.mean(ms)), "ms_16spp": float(np.sum(ms)),
                         "mpaths": W * H / (float(np.mean(ms)) / 1e3) / 1e6}
    out["wavefront_equals_plain"] = bool(np.array_equal(accs["plain"].view(np.uint32),
                                                        accs["wavefront"].view(np.uint32)))
    if O.ref_available():
        cores = os.cpu_count() or 1
        px = seeded_pixels(W, H, check_pixels, 31)
        c = scene.config.copy()
        acc = None
        for b in range(frames):
            c["batch"] = b
            acc, _ = O.ref_render(scene, c, acc, threads=cores, pixels=px)
        out["bit_exact_vs_reference_sample"] = bool(np.array_equal(
            acc[px[:, 1], px[:, 0]].view(np.uint32), accs["plain"][px[:, 1], px[:, 0]].view(np.uint32)))
        acc = None
        t0 = time.perf_counter()
        done = 0
        while done < frames and (done == 0 or time.perf_counter() - t0 < budget_s):
            c["batch"] = done
            acc, _ = O.ref_render(scene, c, acc, threads=cores)
            done += 1
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": W * H * done / dt / 1e6, "unit": "Mpaths/s", "cores": cores,
                               "kind": "reference", "ms_per_frame": dt / done * 1e3,
                               "sample": f"{done} whole frames of the reference's compute shader on the CPU"}
        out["speedup_plain_vs_cpu"] = out["plain"]["mpaths"] / out["cpu_baseline"]["value"]
    return out


def timed_closest_hit(ctx, d_rays, n, d_hits, variant, flush, reps=5):
    """Mean CUDA-event time (ms) of one closest-hit launch over device rays,
    L2 flushed before each, on the context's stream."""
    import torch
    ext = torch.cuda.ExternalStream(ctx.stream)
    ctx.closest_hit_device(d_rays, n, d_hits, variant)  # warm-up (and prepare)
    ms = []
    for _ in range(reps):
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(ext):
            e0.record()
            ctx.closest_hit_device(d_rays, n, d_hits, variant)
            e1.record()
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    return float(np.mean(ms))


def measure_config4(local, frames=4096, mre_pixels=2048, width=960, height=540):
    """The precision variant of the closest-hit workload (the 2.1M-triangle
    instanced scene at 960x540):
      * primary-ray IDs of the precision closest hit (4-wide BVH, 8-bit child
        bounds rounded outward, watertight test) against the FP32-node form
        with the same test (identical when no hit is lost) and against the
        reference's triangle test (disagreements classified);
      * node bytes per ray, counted on the device over camera + bounce rays:
        the reference walk's 48-byte binary nodes against the precision
        walk's 48-byte TLAS nodes and 64-byte quantised BLAS nodes;
      * closest-hit Mrays/s (CUDA events, L2 flushed) of the FP32-node forms
        and the precision form;
      * `frames` frames of 1 spp each, the plain FP32 megakernel against the
        precision wavefront form (Kahan-compensated accumulation): ms/frame,
        Mpaths/s and MRE of the accumulation against the FP64 oracle at
        `mre_pixels` seeded pixels."""
    import torch
    from aviatorengine2_b200 import Context, _lib, scenes
    scene = scenes.instanced_meshes(width=width, height=height, gpu_build=True)
    _lib.lib().ae_bvh_builder_release()
    out = {"workload": f"instanced_meshes {width}x{height}, {frames} frames of 1 spp, depth "
                       f"{int(scene.config['depth'])}", "triangles": int(scene.triangles)}
    dev = torch.device("cuda", local)
    with Context(width, height, device=local) as ctx:
        ctx.upload(scene)
        ctx.prepare_fast()
        prim = ctx.camera_rays()
        out["primary_ids"] = precision_ids(ctx, prim)
        hits = ctx.closest_hit(prim, _lib.VARIANT_PLAIN)
        bounce, valid = ctx.bounce_rays(prim, hits)
        rays = np.concatenate([prim, bounce[valid]])
        d_rays = torch.from_numpy(rays.view(np.uint8)).to(dev)
        d_hits = torch.empty(len(rays) * 20, dtype=torch.uint8, device=dev)
        flush = torch.empty(512 * 1024 * 1024, dtype=torch.uint8, device=dev)
        torch.cuda.synchronize()
        L = _lib.lib()
        cnt = {}
        for name, var in (("plain", _lib.VARIANT_PLAIN), ("precision", _lib.VARIANT_QUANT)):
            c6 = np.zeros(6, np.uint64)
            _lib.check(L.ae_trace_counters_variant(ctx.handle, d_rays.data_ptr(), len(rays), var, _lib.ptr(c6)),
                       ctx.handle)
            cnt[name] = c6.astype(np.float64) / len(rays)
        out["node_bytes_per_ray"] = {
            "plain_fp32_binary": 48.0 * (cnt["plain"][0] + cnt["plain"][3]),
            "precision_quantised": 48.0 * cnt["precision"][0] + 64.0 * cnt["precision"][3],
            "plain_nodes_per_ray": float(cnt["plain"][0] + cnt["plain"][3]),
            "precision_nodes_per_ray": float(cnt["precision"][0] + cnt["precision"][3]),
            "plain_triangle_bytes_per_ray": 48.0 * cnt["plain"][4],
            "precision_triangle_bytes_per_ray": 48.0 * cnt["precision"][4],
            "rays": int(len(rays)), "note": "camera rays + one diffuse bounce per primary hit"}
        chit = {}
        for name, var in (("plain_fp32_nodes", _lib.VARIANT_PLAIN),
                          ("plain_fp32_nodes_watertight", _lib.VARIANT_PLAIN_WT), ("precision", _lib.VARIANT_QUANT)):
            ms = timed_closest_hit(ctx, d_rays.data_ptr(), len(rays), d_hits.data_ptr(), var, flush)
            chit[name] = {"ms": ms, "mrays": len(rays) / (ms / 1e3) / 1e6}
        out["closest_hit"] = chit
        del flush
        px = seeded_pixels(width, height, mre_pixels, 23) if mre_pixels > 0 else None
        ref64 = fp64_reference(scene, scene.config, frames, px) if px is not None else None
        for name, mode in (("plain", _lib.MODE_COMPUTE_ONLY), ("precision", _lib.MODE_WAVEFRONT_PRECISION)):
            c = scene.config.copy()
            ms = []
            for b in range(frames):
                c["batch"] = b
                ctx.set_config(c)
                ctx.render_frame(mode)
                ms.append(ctx.last_kernel_ms())
            ctx.synchronize()
            r = {"ms_per_frame": float(np.mean(ms[1:])) if frames > 1 else float(ms[0])}
            r["mpaths"] = width * height / (r["ms_per_frame"] / 1e3) / 1e6
            if ref64 is not None:
                r["mre"] = ctx.image_error_pixels(px, ref64, eps=MRE_EPS)["mre"]
            out[name] = r
    out["speedup"] = out["precision"]["mpaths"] / out["plain"]["mpaths"]
    if ref64 is not None:
        out["mre_reference"] = (f"FP64 oracle (same estimator and RNG stream in double) after {frames} frames at "
                                f"{len(px)} seeded pixels; reduced on the GPU in FP64; eps {MRE_EPS}")
        out["mre_precision_over_plain"] = out["precision"]["mre"] / max(out["plain"]["mre"], 1e-300)
    return out


def measure_build(local, reps=3):
    """BLAS builds of the wavefront workload's 32 meshes (10,067,490
    triangles): MeshLibrary::Add's triangle boxes, binned-SAH build and
    leaf-order index rewrite, on the GPU from device-resident vertex and index
    arrays (ae_mesh_blas_device_many: the 32 trees in one forest build; also
    ae_mesh_blas_device once per mesh; timed with CUDA events around all 32;
    the builder synchronises the stream between tree levels, and that host
    time is inside the events) against the host builder (ae_mesh_library_add,
    one thread, wall clock).  The device output is compared with the host's
    byte for byte."""
    import ctypes
    import torch
    from aviatorengine2_b200 import _lib, scenes
    from aviatorengine2_b200._lib import lib
    geometry, _ = scenes.wavefront_meshes(np.random.default_rng(4))
    tris = sum(len(i) // 3 for _, i in geometry)
    dev = torch.device("cuda", local)
    d_v = [torch.from_numpy(np.ascontiguousarray(v, _lib.VERTEX).view(np.uint8)).to(dev) for v, _ in geometry]
    d_i = [torch.from_numpy(np.ascontiguousarray(i, np.uint32).view(np.int32)).to(dev) for _, i in geometry]
    d_n = [torch.empty(2 * (len(i) // 3) * 48, dtype=torch.uint8, device=dev) for _, i in geometry]
    d_o = [torch.empty(len(i), dtype=torch.int32, device=dev) for _, i in geometry]
    counts = [ctypes.c_uint32() for _ in geometry]
    stream = torch.cuda.current_stream(dev)
    L = lib()

    k = len(geometry)
    P = ctypes.c_void_p
    arr_v = (P * k)(*[t.data_ptr() for t in d_v])
    arr_i = (P * k)(*[t.data_ptr() for t in d_i])
    arr_n = (P * k)(*[t.data_ptr() for t in d_n])
    arr_o = (P * k)(*[t.data_ptr() for t in d_o])
    nv = np.array([len(v) for v, _ in geometry], np.uint32)
    ni = np.array([len(i) for _, i in geometry], np.uint32)
    many_counts = np.zeros(k, np.uint32)

    def build_per_mesh():
        for m, (v, i) in enumerate(geometry):
            rc = L.ae_mesh_blas_device(d_v[m].data_ptr(), len(v), d_i[m].data_ptr(), len(i), d_n[m].data_ptr(),
                                       ctypes.byref(counts[m]), d_o[m].data_ptr(), P(stream.cuda_stream))
            if rc:
                raise _lib.AeError(rc, "ae_mesh_blas_device")

    def build_forest():
        rc = L.ae_mesh_blas_device_many(k, arr_v, _lib.ptr(nv), arr_i, _lib.ptr(ni), arr_n, _lib.ptr(many_counts),
                                        arr_o, P(stream.cuda_stream))
        if rc:
            raise _lib.AeError(rc, "ae_mesh_blas_device_many")

    def timed(fn):
        ms = []
        for r in range(reps + 1):  # the first pass grows the builder's scratch
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize(dev)
            if r:
                ms.append(e0.elapsed_time(e1))
        return float(np.mean(ms))

    per_mesh_ms = timed(build_per_mesh)
    ms = [timed(build_forest)]  # leaves the forest build's output in d_n / d_o
    host = scenes.MeshLibrary()
    t0 = time.perf_counter()
    for v, i in geometry:
        host.add(v, i)
    host_s = time.perf_counter() - t0
    _, h_idx, h_blas = host.arrays()
    g_blas = np.concatenate([d_n[m][: int(many_counts[m]) * 48].cpu().numpy() for m in range(k)])
    g_idx = np.concatenate([d_o[m].cpu().numpy().view(np.uint32) for m in range(k)])
    # The library's BLAS links are mesh-relative: the concatenation is the same bytes.
    exact = bool(np.array_equal(g_blas, h_blas.view(np.uint8).ravel()) and np.array_equal(g_idx, h_idx))
    gpu_ms = float(np.mean(ms))
    return {"workload": f"BLAS of wavefront_scene's {len(geometry)} meshes, {tris} triangles",
            "triangles": int(tris), "gpu_ms": gpu_ms, "gpu_mtris_per_s": tris / (gpu_ms / 1e3) / 1e6,
            "host_s": host_s, "host_mtris_per_s": tris / host_s / 1e6, "host_threads": 1,
            "speedup": host_s * 1e3 / gpu_ms, "bit_exact": exact, "reps": reps,
            "gpu_call": "ae_mesh_blas_device_many (the 32 trees built together)",
            "gpu_ms_per_mesh_calls": per_mesh_ms}


def measure_serving(local, n_requests=48, rate=0.5, seed=7, claim_policy=1, frame_hz=30.0, queue_run=0, slots=0):
    """The serving loop under a Poisson stream of requests over the 8 resident
    serving scenes: resolution uniform over {256^2, 640x480, 960x540,
    1920x1080}, spp from {1, 4, 16, 64} (as that many progressive frames).
    While the requests run, the world moves every frame: at `frame_hz` all
    4096 instances (512 per scene) take a random-walk step, submitted to the
    server as one move per scene (a GPU TLAS refit when applied; moves that
    no request renders are coalesced).  Latency = submit to images in host
    memory; frame latency = a request's latency over its progressive frames."""
    from aviatorengine2_b200 import Context, Server, scenes
    rng = np.random.default_rng(seed)
    t0 = time.perf_counter()
    S = scenes.serving_scenes(gpu_build=True)
    from aviatorengine2_b200 import _lib
    _lib.lib().ae_bvh_builder_release()
    ctxs = []
    for sc in S:
        c = Context(256, 256, device=local)
        c.upload(sc)
        ctxs.append(c)
    build_s = time.perf_counter() - t0
    res_choices = [(256, 256), (640, 480), (960, 540), (1920, 1080)]
    spp_choices = [1, 4, 16, 64]
    plan = [(int(rng.integers(0, len(S))), res_choices[int(rng.integers(0, 4))], spp_choices[int(rng.integers(0, 4))])
            for _ in range(n_requests)]
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n_requests))
    inst = [sc.instances.copy() for sc in S]
    with Server(device=local, arena_bytes=4 << 30, max_requests=64, claim_policy=claim_policy,
                queue_run=queue_run, slots=slots) as srv:
        ids = [srv.add_scene(c) for c in ctxs]
        # warm-up: one small request per scene
        for k in range(len(S)):
            c = S[k].config.copy()
            c["samples"], c["batches"] = 1, 1
            srv.wait(srv.submit(ids[k], 64, 64, 1, c, accum=False, display=False), 600000)
        srv.reset_stats()
        stop = threading.Event()
        moved = {"frames": 0, "moves": 0}
        mover_rng = np.random.default_rng(seed + 1000)

        def mover():
            period = 1.0 / frame_hz
            nxt = time.perf_counter()
            while not stop.is_set():
                for k in range(len(S)):
                    inst[k] = scenes.random_walk(inst[k], mover_rng)
                    srv.move_instances(ids[k], inst[k])
                    moved["moves"] += 1
                moved["frames"] += 1
                nxt += period
                stop.wait(max(0.0, nxt - time.perf_counter()))

        th = threading.Thread(target=mover, daemon=True) if frame_hz > 0 else None
        start = time.perf_counter()
        if th:
            th.start()
        rids = []
        for i, (sc, (w, h), spp) in enumerate(plan):
            while time.perf_counter() - start < arrivals[i]:
                time.sleep(0.0005)
            c = S[sc].config.copy()
            c["samples"], c["batches"] = 1, 1
            rids.append(srv.submit(ids[sc], w, h, spp, c))
        lat, per_frame = [], []
        for r, (_, _, spp) in zip(rids, plan):
            res, _, _ = srv.wait(r, 1800000)
            lat.append(res["done_ms"] - res["submit_ms"])
            per_frame.append(lat[-1] / spp)
        stop.set()
        if th:
            th.join()
        mover_s = time.perf_counter() - start
        srv.drain(600000)
        st = srv.stats()
    for c in ctxs:
        c.close()
    wall = (st["last_done_ms"] - st["first_submit_ms"]) / 1e3
    return {"workload": "8 resident scenes " + "/".join(f"{sc.triangles // 1000}k" for sc in S) +
                        " tris, 512 instances each (4096 in all) moving every frame; Poisson arrivals",
            "requests": n_requests, "rate_per_s": rate, "claim_policy": "shared" if claim_policy else "oldest_first",
            "queue_run": queue_run or "default (32)", "slots": slots or 1 << 20,
            "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "mean_ms": st["mean_ms"], "max_ms": st["max_ms"],
            # per progressive frame: a request's latency over its frame count
            "frame_p50_ms": float(np.percentile(per_frame, 50)), "frame_p99_ms": float(np.percentile(per_frame, 99)),
            "mpaths": st["paths"] / wall / 1e6, "mrays": st["rays"] / wall / 1e6, "paths": int(st["paths"]),
            "wall_s": wall, "frame_hz": frame_hz, "world_frames": int(moved["frames"]),
            "moves_submitted": int(moved["moves"]), "moves_applied": int(st["moves_applied"]),
            "moves_coalesced": int(st["moves_coalesced"]),
            "refits_per_s": st["moves_applied"] / mover_s, "instances_moved_per_frame": int(sum(len(i) for i in inst)),
            "peak_resident": int(st["peak_resident"]), "peak_arena_bytes": int(st["peak_arena_bytes"]),
            "errors": int(st["errors"]), "scene_build_s": build_s}


def run_reference_arm(args):
    """The reference's CPU implementation of the path on this box's host
    cores, over the same scene bytes and the same rays as our arm, with none
    of the library's code: the scene is packed by the reference's own scene
    code (oracle/ref_scene.py over oracle/_ref), the rays are made by the
    oracle, and the timed closest hit is the oracle's restatement of the
    reference traversal (kind "port"), because the reference's own traversal
    has rigid instances and this workload scales them.  The reference's own
    compiled traversal is timed beside it on the rigid twin of the scene
    (the same rays, every instance at scale 1): that figure and the port's on
    the same rigid scene show the port runs at the reference's speed."""
    rank, world, local = dist_env()
    if rank != 0:
        return 0
    O, R = _oracle_modules()
    import importlib.util
    spec_mod = importlib.util.spec_from_file_location("ae_synth", os.path.join(ROOT, "aviatorengine2_b200", "synth.py"))
    synth = importlib.util.module_from_spec(spec_mod)
    spec_mod.loader.exec_module(synth)
    if not R.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (the reference's scene code compiled "
                                                              "for the CPU) is not built"}), flush=True)
        return 0
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    scene = R.build_instanced(synth.instanced_meshes_spec(width=args.width, height=args.height))
    build_s = time.perf_counter() - t0
    prim = O.camera_rays(scene.config)
    hits = O.closest_hit(scene, prim, threads=cores)
    bounce, valid = O.bounce_rays(scene, scene.config, prim, hits)
    bounce = bounce[valid]
    rays = np.concatenate([prim, bounce])
    W, H = int(scene.config["width"]), int(scene.config["height"])
    config = workload_config(W, H, len(prim), len(bounce), scene.triangles, len(scene.instances),
                             scene_digest(scene), digest(prim, bounce), world)
    for _ in range(args.warmup):
        cpu_reference(scene, rays[:20000], budget_s=0.0)
    steps = []
    base = None
    for _ in range(args.steps):
        # about 60 s of CPU work over all steps
        base = cpu_reference(scene, rays, budget_s=max(1.0, min(6.0, 60.0 / max(args.steps, 1))))
        steps.append(base["value"])
    v = float(np.median(steps))
    base["value"] = v
    base["sample"] += f"; median of {args.steps} steps"
    rigid = None
    if O.ref_available():
        twin = R.Scene(scene.objects, scene.tlas, scene.lights, scene.vertices, scene.indices, scene.blas,
                       scene.instances.copy(), scene.config, "instanced_meshes (rigid twin)")
        twin.instances["scale"] = 0.0
        own = cpu_reference(twin, rays, budget_s=8.0, impl="reference")
        port = cpu_reference(twin, rays, budget_s=8.0, impl="port")
        rigid = {"workload": "the same rays against the rigid twin of the scene (every instance at scale 1)",
                 "reference_own_traversal": own, "port": port, "port_over_reference": port["value"] / own["value"]}
    native = sorted({ln.split()[-1] for ln in open("/proc/self/maps") if ln.rstrip().endswith(".so")
                     and ROOT in ln})
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": len(rays) / (v * 1e6) * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene and camera)",
            "config": config, "cpu_baseline": base,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "scene_build": {"by": "the reference's MeshLibrary::Add steps, MeshBounds, BuildBVH and MeshToGPU "
                                  "(oracle/_ref/libaeref_scene.so)", "seconds": build_s},
            "reference_rigid_twin": rigid, "repo_native_libraries_loaded": native}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--variant", default=os.environ.get("AE_BENCH_VARIANT", "best"))
    ap.add_argument("--bounce-variant", default="walk",
                    help="kernel family for the bounce rays ('same' = --variant's, or plain/fast/quant/walk); "
                         "walk: FAST's walk one step at a time per thread, the same hits, for incoherent rays")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer leg (profiling runs)")
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--no-paths", action="store_true", help="skip the Mpaths/s leg (plain vs wavefront frames)")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving leg")
    ap.add_argument("--no-build", action="store_true", help="skip the BVH build leg")
    ap.add_argument("--no-config4", action="store_true", help="skip the precision-variant leg (960x540)")
    ap.add_argument("--no-config1", action="store_true", help="skip the small plain-method leg (Cornell box)")
    ap.add_argument("--c4-frames", type=int, default=4096, help="frames (1 spp each) of the precision-variant leg")
    ap.add_argument("--mre-pixels", type=int, default=2048, help="seeded pixels scored against the FP64 oracle")
    ap.add_argument("--paths-tris", type=int, default=10_000_000, help="unique triangles of the wavefront scene")
    ap.add_argument("--paths-instances", type=int, default=1024, help="instances of the wavefront scene")
    ap.add_argument("--paths-mre-frames", type=int, default=16, help="frames accumulated before the MRE of the "
                    "wavefront-scene images")
    ap.add_argument("--serve-requests", type=int, default=48)
    ap.add_argument("--serve-frame-hz", type=float, default=30.0, help="world frames per second (every frame moves "
                    "all 4096 instances of the serving scenes)")
    ap.add_argument("--serve-rate", type=float, default=0.5, help="Poisson arrivals per second")
    ap.add_argument("--serve-sweep", default="", help="comma-separated arrival rates: also run the serving "
                    "leg at each (reported as serving_sweep)")
    ap.add_argument("--serve-claim", choices=["shared", "oldest"], default="shared",
                    help="how free slots pick the next pixel: spread over the admitted requests, or the oldest first")
    ap.add_argument("--serve-slots", type=int, default=0, help="server path slots (0: the library default, 2^20)")
    ap.add_argument("--serve-run", type=int, default=0,
                    help="walker stages' queue entries per warp claim in the server (0: default, 1: static)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    args.warmup = max(args.warmup, 3)

    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist

    from aviatorengine2_b200 import Context, _lib, scenes
    # BLAS built on the GPU: the same bytes as the host build (tests), and
    # seconds less of set-up per run.
    scene = scenes.instanced_meshes(width=args.width, height=args.height, gpu_build=True)
    _lib.lib().ae_bvh_builder_release()
    W, H = int(scene.config["width"]), int(scene.config["height"])
    ctx = Context(W, H, device=local)
    ctx.upload(scene)
    prim, bounce = make_workload(ctx, scene)
    n1, n2 = len(prim), len(bounce)
    variant = args.variant
    if variant == "best":
        try:
            ctx.prepare_fast()
            variant = "fast"
        except Exception:
            variant = "plain"
    vid = VARIANTS[variant]
    bounce_variant = variant if args.bounce_variant == "same" or variant != "fast" else args.bounce_variant
    vid2 = VARIANTS[bounce_variant]

    dev = torch.device("cuda", local)
    d_prim = torch.from_numpy(prim.view(np.uint8)).to(dev)
    d_bounce = torch.from_numpy(bounce.view(np.uint8)).to(dev)
    d_hits1 = torch.empty(n1 * 20, dtype=torch.uint8, device=dev)
    d_hits2 = torch.empty(n2 * 20, dtype=torch.uint8, device=dev)
    flush = torch.empty(512 * 1024 * 1024, dtype=torch.uint8, device=dev)
    torch.cuda.synchronize()
    ext = torch.cuda.ExternalStream(ctx.stream)

    def step(mid=None):
        ctx.closest_hit_device(d_prim.data_ptr(), n1, d_hits1.data_ptr(), vid)
        if mid is not None:
            mid.record()
        ctx.closest_hit_device(d_bounce.data_ptr(), n2, d_hits2.data_ptr(), vid2)

    for _ in range(args.warmup):
        step()
    ctx.synchronize()

    # Algorithmic bytes of the reference traversal over this ray set.
    cnt = np.zeros(6, np.uint64)
    _lib.check(_lib.lib().ae_trace_counters(ctx.handle, d_prim.data_ptr(), n1, _lib.ptr(cnt)), ctx.handle)
    cnt2 = np.zeros(6, np.uint64)
    _lib.check(_lib.lib().ae_trace_counters(ctx.handle, d_bounce.data_ptr(), n2, _lib.ptr(cnt2)), ctx.handle)
    per = np.array([48, 128, 48, 48, 48, 60], np.float64)
    alg_bytes_prim = float((cnt.astype(np.float64) * per).sum())
    alg_bytes_bounce = float((cnt2.astype(np.float64) * per).sum())
    alg_bytes_step = alg_bytes_prim + alg_bytes_bounce

    launches0 = ctx.launch_count
    times, t_prim, t_bounce = [], [], []
    with ClockSampler(local) as clk:
        if pg:
            pg.barrier()
        torch.cuda.synchronize()
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            e0, em, e1 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            with torch.cuda.stream(ext):
                e0.record()
                step(em)
                e1.record()
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
            t_prim.append(e0.elapsed_time(em))
            t_bounce.append(em.elapsed_time(e1))
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
    launches = ctx.launch_count - launches0
    ms = max_over_ranks(float(np.sum(times)) / args.steps, pg, dev)
    rays_step = n1 + n2
    value = replica_value(rays_step, world, ms / 1e3)

    e2e = None
    if not args.no_e2e:
        # End to end through the public call with host buffers: pinned host rays
        # in, hits out, per step.
        h_prim = torch.from_numpy(prim.view(np.uint8)).pin_memory()
        h_bounce = torch.from_numpy(bounce.view(np.uint8)).pin_memory()
        h_h1 = torch.empty(n1 * 20, dtype=torch.uint8).pin_memory()
        h_h2 = torch.empty(n2 * 20, dtype=torch.uint8).pin_memory()
        L = _lib.lib()

        def e2e_step():
            _lib.check(L.ae_closest_hit(ctx.handle, h_prim.data_ptr(), n1, h_h1.data_ptr(), vid), ctx.handle)
            _lib.check(L.ae_closest_hit(ctx.handle, h_bounce.data_ptr(), n2, h_h2.data_ptr(), vid2), ctx.handle)

        for _ in range(2):
            e2e_step()
        et = []
        for _ in range(max(3, args.steps // 2)):
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            e2e_step()
            et.append(time.perf_counter() - t0)
        e2e_s = max_over_ranks(float(np.mean(et)), pg, dev)
        e2e = {"value": replica_value(rays_step, world, e2e_s), "unit": UNIT, "h2d_bytes_per_step": int((n1 + n2) * 32),
               "d2h_bytes_per_step": int((n1 + n2) * 20),
               "note": "pinned host buffers, wall clock per step; the camera-ray call's kernel reads the rays and "
                       "writes the hits in host memory over the bus, the bounce-ray call copies chunks in and out "
                       "(cudaMemcpyAsync) around its launches"}

    peak, peak_kind = load_peaks()
    traffic = load_traffic()
    same_kernels = bool(traffic and traffic.get("variant") == variant
                        and traffic.get("bounce_variant", variant) == bounce_variant)
    ms_prim, ms_bounce = float(np.mean(t_prim)), float(np.mean(t_bounce))
    # Per launch: algorithmic bytes of that launch's ray set / its CUDA-event
    # duration inside the timed steps; traffic per launch from the committed
    # full-size ncu capture of the same kernels.
    kernels = {
        "camera_rays": {"kernel": f"closest hit, variant {variant}", "rays": n1, "ms": ms_prim,
                        "achieved": alg_bytes_prim / (ms_prim / 1e3) / 1e9,
                        "traffic": float(traffic["primary_launch_bytes"]) if same_kernels else None},
        "bounce_rays": {"kernel": f"closest hit, variant {bounce_variant}", "rays": n2, "ms": ms_bounce,
                        "achieved": alg_bytes_bounce / (ms_bounce / 1e3) / 1e9,
                        "traffic": float(traffic["bounce_launch_bytes"]) if same_kernels else None},
    }
    for k in kernels.values():
        k["frac"] = k["achieved"] / peak
    dominant = max(kernels, key=lambda k: kernels[k]["ms"])
    D = kernels[dominant]
    roofline = {"bound": "hbm", "kernel": f"{D['kernel']} ({dominant.replace('_', ' ')})", "achieved": D["achieved"],
                "peak": peak, "unit": "GB/s", "frac": D["frac"], "traffic": D["traffic"], "peak_source": peak_kind,
                "algorithmic_bytes_per_ray": (alg_bytes_bounce / n2) if dominant == "bounce_rays" else alg_bytes_prim / n1,
                "per_launch": kernels,
                "step": {"achieved": alg_bytes_step / (ms / 1e3) / 1e9, "frac": alg_bytes_step / (ms / 1e3) / 1e9 / peak},
                "l2_throughput_pct_of_peak": traffic.get("l2_throughput_pct_of_peak") if same_kernels else None,
                "note": "algorithmic bytes = reference-walk touches (48 B node, 128 B object, 48 B instance, "
                        "48 B triangle, 60 B winner) counted on the device over each launch's ray set; achieved = "
                        "those bytes / that launch's CUDA-event time; the working set is mostly L2-resident, so "
                        "DRAM traffic is far below the algorithmic bytes (l2_throughput_pct_of_peak: the committed ncu summary, its case named)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_reference(scene, np.concatenate([prim, bounce]))
        cpu["note"] = ("the oracle's restatement of the reference traversal, which traces the scaled instances; "
                       "--impl reference prints the reference's own compiled traversal on the rigid twin beside it")

    # Frame-level legs: single-GPU workloads, measured in the one-GPU run
    # (with N replicas they would repeat the same numbers on rank 0 while the
    # other GPUs wait).  A leg that fails reports its error in its own block;
    # the closest-hit line above stands.
    def leg(enabled, fn, *a, **kw):
        if not enabled or rank != 0 or world > 1:
            return None
        try:
            return fn(*a, **kw)
        except Exception as e:  # noqa: BLE001 - reported in the JSON line
            import traceback
            traceback.print_exc()
            return {"error": f"{type(e).__name__}: {e}"}

    paths = leg(not args.no_paths, measure_paths, local, args.width, args.height, mre_pixels=args.mre_pixels,
                mre_frames=args.paths_mre_frames, target_tris=args.paths_tris, n_instances=args.paths_instances)
    build = leg(not args.no_build, measure_build, local)
    config1 = leg(not args.no_config1, measure_config1, local)
    config4 = leg(not args.no_config4, measure_config4, local, args.c4_frames, args.mre_pixels)
    claim = 0 if args.serve_claim == "oldest" else 1
    serving = leg(not args.no_serve, measure_serving, local, args.serve_requests, args.serve_rate,
                  claim_policy=claim, frame_hz=args.serve_frame_hz, queue_run=args.serve_run, slots=args.serve_slots)
    sweep = None
    if args.serve_sweep:
        sweep = [leg(True, measure_serving, local, args.serve_requests, float(r), claim_policy=claim,
                     frame_hz=args.serve_frame_hz, queue_run=args.serve_run, slots=args.serve_slots)
                 for r in args.serve_sweep.split(",")]

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene and camera)",
            "config": workload_config(W, H, n1, n2, scene.triangles, len(scene.instances), scene_digest(scene),
                                      digest(prim, bounce), world),
            "kernels": {"camera_rays": variant, "bounce_rays": bounce_variant},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
            "clocks": clk.summary(),
            "per_step_ms": [round(t, 4) for t in times],
            "paths": paths, "config1": config1, "config4": config4, "serving": serving, "bvh_build": build}
    if sweep is not None:
        line["serving_sweep"] = sweep
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if pg:
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
