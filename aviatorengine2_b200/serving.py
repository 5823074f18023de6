"""Python handle on the render server (ae_serve_* in include/ae_b200.h).

The server keeps scenes resident on one GPU and renders frame requests with
continuous batching; see the header for the guarantees.  Typical use:

    with Context(w, h) as scene_ctx:
        scene_ctx.upload(packed)
        with Server() as srv:
            sid = srv.add_scene(scene_ctx)
            rid = srv.submit(sid, 640, 480, frames=4, config=packed.config)
            result, accum, display = srv.wait(rid)
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import lib, ptr


class Server:
    def __init__(self, slots=0, max_lights=0, max_requests=0, arena_bytes=0, ticks_per_launch=0, extend_threads=0,
                 max_scenes=0, claim_policy=_lib.CLAIM_OLDEST_FIRST, device=0, queue_run=0):
        s = np.zeros(1, _lib.SERVE_SETTINGS)
        s["device"], s["slots"], s["max_lights"], s["max_requests"] = device, slots, max_lights, max_requests
        s["arena_bytes"], s["ticks_per_launch"] = arena_bytes, ticks_per_launch
        s["extend_threads"], s["max_scenes"], s["claim_policy"] = extend_threads, max_scenes, claim_policy
        s["queue_run"] = queue_run
        self._h = lib().ae_serve_create(ptr(s))
        if not self._h:
            raise _lib.AeError(lib().ae_create_status(), "ae_serve_create failed (see stderr)")
        self._scenes = []    # contexts stay alive while the server holds them
        self._outputs = {}   # request id -> (accum, display) host buffers

    def close(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            lib().ae_serve_destroy(h)
        self._outputs = {}

    def __del__(self):
        # At interpreter exit the ctypes module state may already be gone;
        # the process is ending and the driver releases the device anyway.
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _chk(self, code):
        if code != 0:
            raise _lib.AeError(code, lib().ae_serve_last_error(self._h).decode())
        return code

    def add_scene(self, ctx):
        """Makes an uploaded Context resident; returns the scene id."""
        sid = ctypes.c_uint32(0)
        self._chk(lib().ae_serve_add_scene(self._h, ctx.handle, ctypes.byref(sid)))
        self._scenes.append(ctx)
        return sid.value

    def submit(self, scene, width, height, frames, config, accum=True, display=True, user=0):
        """Queues a request; returns its id.  The images land in host arrays
        that wait() returns."""
        r = np.zeros(1, _lib.SERVE_REQUEST)
        r["scene"], r["width"], r["height"], r["frames"] = scene, width, height, frames
        r["config"] = config
        acc = np.zeros((height, width, 4), np.float32) if accum else None
        dsp = np.zeros((height, width, 4), np.uint8) if display else None
        r["accum"] = acc.ctypes.data if acc is not None else 0
        r["display"] = dsp.ctypes.data if dsp is not None else 0
        r["user"] = user
        rid = ctypes.c_uint64(0)
        self._chk(lib().ae_serve_submit(self._h, ptr(r), ctypes.byref(rid)))
        self._outputs[rid.value] = (acc, dsp)
        return rid.value

    def move_instances(self, scene, instances):
        ins = np.ascontiguousarray(instances, _lib.INSTANCE)
        self._chk(lib().ae_serve_move_instances(self._h, scene, ptr(ins), len(ins)))

    def cancel(self, rid):
        """Withdraws a request (ae_serve_cancel); wait() then raises AeError
        with code -9 (AE_ERR_CANCELLED) for it."""
        self._chk(lib().ae_serve_cancel(self._h, rid))

    def debug_inject(self, fault, on=True):
        """Test hook (ae_serve_debug_inject)."""
        self._chk(lib().ae_serve_debug_inject(self._h, fault, 1 if on else 0))

    def wait(self, rid, timeout_ms=-1):
        """(result record, accum image, display image) of a finished request."""
        out = np.zeros(1, _lib.SERVE_RESULT)
        code = lib().ae_serve_wait(self._h, rid, timeout_ms, ptr(out))
        # AE_ERR_TIMEOUT is either the wait running out (the record is left
        # untouched) or the request's own status (a device wait gave up).
        if code == -6 and timeout_ms >= 0 and int(out[0]["id"]) != rid:
            raise TimeoutError(f"request {rid} not finished after {timeout_ms} ms")
        acc, dsp = self._outputs.pop(rid, (None, None))
        self._chk(code)
        return out[0], acc, dsp

    def drain(self, timeout_ms=-1):
        self._chk(lib().ae_serve_drain(self._h, timeout_ms))

    def stats(self):
        out = np.zeros(1, _lib.SERVE_STATS)
        self._chk(lib().ae_serve_get_stats(self._h, ptr(out)))
        return {k: out[0][k].item() for k in _lib.SERVE_STATS.names if k != "pad"}

    def reset_stats(self):
        self._chk(lib().ae_serve_reset_stats(self._h))


def simulate_policy(events, arena_bytes, max_resident, n_scenes, frame_sets=2, max_ticks=100000):
    """Runs the server's admission policy on a list of event dicts on the host
    (no GPU).  Returns (status, outcomes array)."""
    ev = np.zeros(len(events), _lib.POLICY_EVENT)
    for i, e in enumerate(events):
        ev[i]["kind"] = e.get("kind", _lib.POLICY_REQUEST)
        ev[i]["scene"] = e.get("scene", 0)
        ev[i]["tick"] = e["tick"]
        ev[i]["service_ticks"] = e.get("service_ticks", 1)
        ev[i]["footprint"] = e.get("footprint", 0)
    out = np.zeros(len(events), _lib.POLICY_OUTCOME)
    code = lib().ae_serve_policy_simulate(ptr(ev), len(ev), arena_bytes, max_resident, n_scenes, frame_sets, max_ticks,
                                          ptr(out))
    return code, out
