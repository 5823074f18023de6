// serve.cu - the render-serving loop: continuous batching of frame requests
// over scenes kept resident on one GPU.
//
// Device side.  A fixed pool of path slots is shared by every admitted
// request.  A slot owns one pixel of one request and renders all of that
// pixel's samples in order (frame by frame, sample by sample), so the
// pixel's arithmetic - seeds, RNG draws, sample sums, the running
// accumulation - is exactly that of `frames` compute-only frames of the plain
// megakernel, whatever else is in flight.  Work moves through one merged ray
// queue per tick:
//
//   begin    resets the next queues; adds the tick's ray counts to the stats
//   extend   closest hit of every queued ray, each against its own scene's
//            4-wide BVH (the scene is looked up per ray), on the step-wise
//            walker (or, with extend_threads set, CTAs that stage queue
//            tiles in shared memory with a bulk asynchronous copy)
//   shade    ColorRay's vertex work; surviving paths go to the next queue,
//            light samples to the shadow queue (warp-aggregated appends)
//   shadow   the reference's occlusion loop per light sample (walker)
//   connect  NEE sums in light order onto the path radiance
//   advance  finished paths close their sample; finished frames fold into the
//            pixel's running accumulation; a finished pixel is written to its
//            request's images, and the slot claims the next unclaimed pixel
//            of the oldest admitted request (warp-cooperative claim) and
//            queues that pixel's first camera ray; idle slots claim too
//
// A replay of one CUDA graph runs an even number of ticks; every parameter it
// reads lives in device memory (scene table, request table, admission order),
// so the graph is captured once.
//
// Host side.  A scheduler thread admits queued requests (serve_policy.h:
// arrival order, by image footprint inside an arena allocated once, and by
// resident request slots), applies instance moves with the GPU refit into a
// copy of the scene's per-frame arrays that no outstanding request renders
// (coalescing moves no request needs, serve_policy.h), replays the graph
// while any request is on the GPU (two replays in flight), and watches the
// per-request pixel counters.  A completion thread copies finished images to
// the caller's memory and releases their arena blocks.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "context.h"
#include "fast.h"
#include "fast_trace.cuh"
#include "fast_walk.cuh"
#include "kernels.h"
#include "serve_policy.h"
#include "shade.cuh"
#include "trace_common.cuh"
#include "wf_common.cuh"

namespace ae {
namespace {

constexpr uint32_t kServeMaxLights = 64;
constexpr uint32_t kServeMaxRequests = 1024;
constexpr int kServeStack = 24;  // shared-memory traversal entries per thread

struct SceneRec {
    DevScene S;
    FastView V;
};

struct ReqDev {
    FrameParams F;  // the request's camera at its own resolution; batch is the frame
    float4 *accum;
    uchar4 *display;
    uint32_t scene, n_pixels, frames, spp;
};

// SV_FAULT: the injected tile-wait failure of ae_serve_debug_inject (0 = none).
enum { SV_Q0 = 0, SV_Q1 = 1, SV_SH = 2, SV_ERR = 3, SV_TILE = 4, SV_IDLE0 = 5, SV_IDLE1 = 6, SV_NORDER = 7,
       SV_FAULT = 8, SV_RUN_EXT = 9, SV_RUN_SH = 10, SV_COUNT = 11 };
enum { ST_RAYS = 0, ST_SHADOW = 1, ST_COUNT = 2 };
// Default run of queue entries a warp of the walker stages takes at a time
// (ae_serve_settings.queue_run 0).
constexpr uint32_t kServeQueueRun = 32;

struct SvView {
    const SceneRec *scenes;
    const ReqDev *reqs;
    uint32_t *next, *done;  // per request-table entry: pixels claimed, pixels written
    const uint32_t *order;  // request-table entries in admission order, cnt[SV_NORDER] of them
    uint32_t *cnt;
    unsigned long long *stats;
    // per slot
    uint32_t *s_req, *s_pix, *s_frame, *s_sample, *s_bounce, *s_seed, *s_scene;
    float4 *s_thr, *s_acc, *s_col, *s_accp, *s_pend;
    uint8_t *s_nee, *s_end;
    // queues
    ae_ray *qray[2];
    uint32_t *qslot[2];
    ae_hit *qhit;
    uint32_t *idle[2];
    ShadowStore sh;  // entry = slot * max_lights + light
    uint32_t *sq;
    uint32_t max_lights;
    uint32_t claim_shared;  // 1: each warp starts its claim at a different request
};

__global__ void k_sv_init(SvView W, uint32_t slots) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < slots; i += gridDim.x * blockDim.x) {
        W.idle[0][i] = i;
        W.s_end[i] = 0;
        W.s_nee[i] = 0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        for (int k = 0; k < SV_COUNT; k++) W.cnt[k] = 0;
        W.cnt[SV_IDLE0] = slots;
        W.stats[ST_RAYS] = 0;
        W.stats[ST_SHADOW] = 0;
    }
}

__global__ void k_sv_begin(SvView W, int q) {
    W.stats[ST_RAYS] += W.cnt[q];
    W.stats[ST_SHADOW] += W.cnt[SV_SH];
    W.cnt[q ^ 1] = 0;
    W.cnt[SV_SH] = 0;
    W.cnt[SV_TILE] = 0;
    W.cnt[SV_RUN_EXT] = 0;
    W.cnt[SV_RUN_SH] = 0;
    W.cnt[SV_IDLE0 + (q ^ 1)] = 0;
}

// Withdraws request-table entry t from pixel claims: its claim counter is
// set to its pixel count (claim_pixel then passes it over), and the pixels
// claimed before - the ones still to finish - are reported.  Runs on the
// serving stream between replays, so no claim races with it.
__global__ void k_sv_cancel(SvView W, uint32_t t, uint32_t *claimed) {
    const uint32_t n = W.reqs[t].n_pixels;
    const uint32_t old = atomicExch(W.next + t, n);
    *claimed = old < n ? old : n;
}

template <int THREADS>
__global__ void __launch_bounds__(THREADS) k_sv_extend(SvView W, int q) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ae_ray *tile = reinterpret_cast<ae_ray *>(smem_raw);
    uint2 *stk = reinterpret_cast<uint2 *>(smem_raw + THREADS * sizeof(ae_ray));
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tile_index;
    const uint32_t count = W.cnt[q];
    // An injected failure issues no copy: the wait runs out with nothing in flight.
    const bool inject = W.cnt[SV_FAULT] != 0;
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    __syncthreads();
    uint32_t phase = 0;
    for (;;) {
        if (threadIdx.x == 0) tile_index = atomicAdd(&W.cnt[SV_TILE], 1u);
        __syncthreads();
        const uint32_t start = tile_index * THREADS;
        if (start >= count) break;
        const uint32_t m = min(uint32_t(THREADS), count - start);
        if (threadIdx.x == 0 && !inject) {
            mbar_expect_tx(&bar, m * uint32_t(sizeof(ae_ray)));
            bulk_g2s(tile, W.qray[q] + start, m * uint32_t(sizeof(ae_ray)), &bar);
        }
        const bool ok = __syncthreads_and(mbar_wait(&bar, phase, inject ? 64u : (1u << 24)) ? 1 : 0) != 0;
        if (!ok) {
            // As in the wavefront extend: a second bounded wait for a copy in
            // flight, then the block exits and reports the timeout.
            if (!inject) mbar_wait(&bar, phase, 1u << 24);
            if (threadIdx.x == 0) atomicOr(&W.cnt[SV_ERR], 1u);
            break;
        }
        phase ^= 1u;
        if (threadIdx.x < m) {
            const ae_ray r = tile[threadIdx.x];
            const uint32_t slot = W.qslot[q][start + threadIdx.x];
            const SceneRec &R = W.scenes[W.s_scene[slot]];
            const DevScene S = R.S;
            const FastView V = R.V;
            const Best b = closest_fast<false, kServeStack>(S, V, mk(r.ox, r.oy, r.oz), mk(r.dx, r.dy, r.dz), r.tnear,
                                                            r.time, stk, threadIdx.x, THREADS);
            const bool any = b.object != AE_MISS;
            ae_hit h;
            h.t = any ? b.t : 0.0f;
            h.alpha = any ? b.alpha : 0.0f;
            h.beta = any ? b.beta : 0.0f;
            h.object = b.object;
            h.prim = b.prim;
            W.qhit[start + threadIdx.x] = h;
        }
        __syncthreads();
    }
}

// Extend on the step-wise Walker: each thread steps its own queued ray (its
// own scene's) and takes the next one as soon as one finishes - k + grid size
// (DYN false) or from its warp's run of `run` consecutive queue entries (DYN
// true; ae_serve_settings.queue_run).
template <bool DYN>
__global__ void __launch_bounds__(128, kWalkBlocksPerSm) k_sv_extend_walk(SvView W, int q, uint32_t run) {
    extern __shared__ uint2 stk[];
    const uint32_t count = W.cnt[q];
    const uint32_t stride = gridDim.x * blockDim.x;
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    Walker<false> w;
    WalkStacks<> K;
    const SceneRec *R = nullptr;
    bool active = !DYN && k < count;
    bool need = DYN, exhausted = false;
    uint32_t cbase = 0, cend = 0;
    auto begin = [&]() {
        const ae_ray r = W.qray[q][k];
        R = W.scenes + W.s_scene[W.qslot[q][k]];
        w.start(R->V, mk(r.ox, r.oy, r.oz), mk(r.dx, r.dy, r.dz), r.tnear, r.time);
    };
    if (active) begin();
    uint32_t iter = 0;
    for (;;) {
        if (DYN && run_take(&W.cnt[SV_RUN_EXT], count, run, need, k, cbase, cend, exhausted)) {
            active = true;
            begin();
        }
        const uint32_t am = __ballot_sync(0xffffffffu, active);
        if (!am) break;
        // Only the warp's largest phase group steps (warp_pick_group).
        const uint32_t pick = warp_pick_group(active ? w.group() : 0u, active, am, iter);
        if (!active || w.group() != pick || !w.step(R->S, R->V, K, stk, threadIdx.x, blockDim.x)) continue;
        const Best &b = w.best;
        const bool any = b.object != AE_MISS;
        ae_hit h;
        h.t = any ? b.t : 0.0f;
        h.alpha = any ? b.alpha : 0.0f;
        h.beta = any ? b.beta : 0.0f;
        h.object = b.object;
        h.prim = b.prim;
        W.qhit[k] = h;
        if (DYN) {
            active = false;
            need = true;
            continue;
        }
        k += stride;
        active = k < count;
        if (active) begin();
    }
}

__global__ void __launch_bounds__(256) k_sv_shade(SvView W, int q) {
    // After an extend that gave up, hit records past its last tile were never
    // written: nothing of this queue is shaded (the host fails the requests).
    if (W.cnt[SV_ERR]) return;
    const uint32_t count = W.cnt[q];
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
        const uint32_t slot = W.qslot[q][k];
        const ae_ray r = W.qray[q][k];
        const ae_hit hr = W.qhit[k];
        const SceneRec &SR = W.scenes[W.s_scene[slot]];
        const DevScene S = SR.S;
        const ReqDev &R = W.reqs[W.s_req[slot]];
        const int bounce = int(W.s_bounce[slot]);
        const float4 t4 = W.s_thr[slot], a4 = W.s_acc[slot];
        f3 thr = mk(t4.x, t4.y, t4.z), acc = mk(a4.x, a4.y, a4.z);
        uint32_t seed = W.s_seed[slot];
        ae_ray nr;
        uint32_t n_shadow;
        const uint32_t e0 = slot * W.max_lights;
        const bool next = shade_vertex<false>(S, SR.V, PrecView{nullptr}, R.F.sky, R.F.depth, S.n_lights, bounce, r, hr,
                                              thr, acc, seed, W.sh, e0, W.s_nee + slot, W.s_pend + slot, n_shadow, nr);
        W.s_thr[slot] = make_float4(thr.x, thr.y, thr.z, 0.0f);
        W.s_acc[slot] = make_float4(acc.x, acc.y, acc.z, 0.0f);
        W.s_seed[slot] = seed;
        if (next) W.s_bounce[slot] = uint32_t(bounce + 1);
        else W.s_end[slot] = 1;
        const uint32_t qi = warp_append(&W.cnt[q ^ 1], next ? 1u : 0u);
        if (next) {
            W.qray[q ^ 1][qi] = nr;
            W.qslot[q ^ 1][qi] = slot;
        }
        const uint32_t sbase = warp_append(&W.cnt[SV_SH], n_shadow);
        if (n_shadow) push_shadow_entries(W.sh, e0, S.n_lights, W.sq, sbase);
    }
}

template <int THREADS, bool DYN>
__global__ void __launch_bounds__(THREADS, kWalkBlocksPerSm * 128 / THREADS) k_sv_shadow(SvView W, uint32_t run) {
    // The reference's shadow loop per light sample on the step-wise Walker:
    // a lane that finishes a sample starts its next one at once (k + grid
    // size, or from its warp's run of `run` queue entries when DYN).  The
    // sample's scene (its slot's) is read through the scene table.
    extern __shared__ uint2 stk[];
    const uint32_t count = W.cnt[SV_SH];
    const uint32_t stride = gridDim.x * THREADS;
    uint32_t k = blockIdx.x * THREADS + threadIdx.x;
    Walker<false> w;
    WalkStacks<> K;
    const SceneRec *R = nullptr;
    uint32_t e = 0;
    f3 so, sd, lp;
    int step = 0;
    bool active = !DYN && k < count;
    bool need = DYN, exhausted = false;
    uint32_t cbase = 0, cend = 0;
    auto begin = [&]() {
        e = W.sq[k];
        R = W.scenes + W.s_scene[e / W.max_lights];
        const float4 o4 = W.sh.o[e], d4 = W.sh.d[e], l4 = W.sh.lp[e];
        so = mk(o4.x, o4.y, o4.z); sd = mk(d4.x, d4.y, d4.z); lp = mk(l4.x, l4.y, l4.z);
        step = 0;
        w.start(R->V, so, sd, 0.001f, d4.w, AE_SUB(distance(lp, so), 0.001f));
    };
    if (active) begin();
    uint32_t iter = 0;
    for (;;) {
        if (DYN && run_take(&W.cnt[SV_RUN_SH], count, run, need, k, cbase, cend, exhausted)) {
            active = true;
            begin();
        }
        const uint32_t am = __ballot_sync(0xffffffffu, active);
        if (!am) break;
        // Only the warp's largest phase group steps (warp_pick_group).
        const uint32_t pick = warp_pick_group(active ? w.group() : 0u, active, am, iter);
        if (!active || w.group() != pick || !w.step(R->S, R->V, K, stk, threadIdx.x, THREADS)) continue;
        const Best &b = w.best;
        int verdict = 0;  // 0 unoccluded, 1 occluded, 2 through glass
        if (b.object != AE_MISS && b.t < AE_SUB(distance(lp, so), 0.001f)) {
            const uint32_t mt = load_head(R->S.objects + b.object).material;
            verdict = mt == AE_MAT_DIFFUSE_LIGHT ? 0 : (mt != AE_MAT_DIELECTRIC ? 1 : 2);
        }
        if (verdict == 2) {
            so = (so + sd * b.t) + sd * 0.001f;
            if (++step < 4) {
                w.start(R->V, so, sd, 0.001f, w.time, AE_SUB(distance(lp, so), 0.001f));
                continue;
            }
            verdict = 0;
        }
        W.sh.occ[e] = uint8_t(verdict);
        if (DYN) {
            active = false;
            need = true;
            continue;
        }
        k += stride;
        active = k < count;
        if (active) begin();
    }
}

__global__ void __launch_bounds__(256) k_sv_connect(SvView W, int q) {
    const uint32_t count = W.cnt[q];
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
        const uint32_t slot = W.qslot[q][k];
        if (!W.s_nee[slot]) continue;
        W.s_nee[slot] = 0;
        const uint32_t n_lights = W.scenes[W.s_scene[slot]].S.n_lights;
        const f3 dl = nee_total(W.sh, size_t(slot) * W.max_lights, n_lights);
        const float4 t4 = W.s_pend[slot], a4 = W.s_acc[slot];
        const f3 acc = mk(a4.x, a4.y, a4.z) + mk(t4.x, t4.y, t4.z) * dl;
        W.s_acc[slot] = make_float4(acc.x, acc.y, acc.z, 0.0f);
    }
}

// Warp-cooperative claim: the lanes with `need` take consecutive pixels of
// the oldest request that still has unclaimed ones (with the shared policy:
// of the first such request from a per-warp starting point in the admission
// order), moving to the next request when it runs out.  A request's counter is only advanced while it
// has pixels left, so it never runs far past its pixel count.  Every lane of
// the calling warp that is in the loop must call this.
AE_DEV bool claim_pixel(const SvView &W, bool need, uint32_t &req, uint32_t &pix) {
    const unsigned mask = __activemask();
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t n_order = W.cnt[SV_NORDER];
    bool got = false;
    const uint32_t start =
        W.claim_shared && n_order ? ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) % n_order : 0u;
    for (uint32_t i = 0; i < n_order; i++) {
        const unsigned want = __ballot_sync(mask, need && !got);
        if (!want) break;
        const uint32_t r = W.order[start + i < n_order ? start + i : start + i - n_order];
        const uint32_t n = W.reqs[r].n_pixels;
        const int leader = __ffs(want) - 1;
        uint32_t base = n;
        if (int(lane) == leader) {
            const uint32_t seen = *reinterpret_cast<volatile const uint32_t *>(W.next + r);
            if (seen < n) base = atomicAdd(W.next + r, uint32_t(__popc(want)));
        }
        base = __shfl_sync(mask, base, leader);
        if (need && !got) {
            const uint32_t p = base + uint32_t(__popc(want & ((1u << lane) - 1u)));
            if (p < n) {
                req = r;
                pix = p;
                got = true;
            }
        }
    }
    return got;
}

__global__ void __launch_bounds__(256) k_sv_advance(SvView W, int q) {
    const uint32_t cq = W.cnt[q], ci = W.cnt[SV_IDLE0 + q];
    const uint32_t total = cq + ci;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x) {
        uint32_t slot;
        bool ended = false;
        const bool idle = k >= cq;
        if (!idle) {
            slot = W.qslot[q][k];
            ended = W.s_end[slot] != 0;
        } else {
            slot = W.idle[q][k - cq];
        }
        bool need = idle, finished_pixel = false;
        uint32_t req = 0, pix = 0, frame = 0, sample = 0, seed = 0;
        if (ended) {
            W.s_end[slot] = 0;
            req = W.s_req[slot];
            pix = W.s_pix[slot];
            const ReqDev &R = W.reqs[req];
            frame = W.s_frame[slot];
            sample = W.s_sample[slot] + 1;
            seed = W.s_seed[slot];
            const float4 a4 = W.s_acc[slot], c4 = W.s_col[slot];
            f3 col = mk(c4.x, c4.y, c4.z) + mk(a4.x, a4.y, a4.z);
            if (sample == R.spp) {
                // End of a frame: hybrid:1383-1403 for this pixel.
                const f3 color = col / AE_U2F(R.spp);
                f3 accp;
                if (frame == 0) {
                    accp = color;
                } else {
                    const float4 p4 = W.s_accp[slot];
                    accp = lerp(mk(p4.x, p4.y, p4.z), color, AE_DIV(1.0f, AE_U2F(frame + 1)));
                }
                frame++;
                sample = 0;
                col = splat(0.0f);
                if (frame == R.frames) {
                    R.accum[pix] = make_float4(accp.x, accp.y, accp.z, 1.0f);
                    R.display[pix] = display_texel(accp, R.F.exposure);
                    finished_pixel = true;
                    need = true;
                } else {
                    W.s_accp[slot] = make_float4(accp.x, accp.y, accp.z, 1.0f);
                }
            }
            W.s_col[slot] = make_float4(col.x, col.y, col.z, 0.0f);
        }
        // One atomic per request per warp for the finished pixels.
        {
            const unsigned amask = __activemask();
            const unsigned same = __match_any_sync(amask, finished_pixel ? req : 0xffffffffu);
            if (finished_pixel && int(threadIdx.x & 31) == __ffs(same) - 1) atomicAdd(W.done + req, uint32_t(__popc(same)));
        }
        uint32_t creq = 0, cpix = 0;
        const bool got = claim_pixel(W, need, creq, cpix);
        if (need && got) {
            req = creq;
            pix = cpix;
            frame = 0;
            sample = 0;
            W.s_req[slot] = req;
            W.s_pix[slot] = pix;
            W.s_scene[slot] = W.reqs[req].scene;
            W.s_col[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
        const bool start = (ended && !need) || (need && got);
        ae_ray r;
        if (start) {
            const ReqDev &R = W.reqs[req];
            FrameParams F = R.F;
            F.batch = frame;
            const uint32_t x = pix % F.width, y = pix / F.width;
            f3 o, d;
            float time;
            if (sample == 0) camera_ray(F, x, y, o, d, time, seed);
            else camera_sample(F, x, y, o, d, time, seed);
            W.s_frame[slot] = frame;
            W.s_sample[slot] = sample;
            W.s_seed[slot] = seed;
            W.s_bounce[slot] = 0;
            W.s_thr[slot] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
            W.s_acc[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            r.ox = o.x; r.oy = o.y; r.oz = o.z; r.tnear = 0.001f;
            r.dx = d.x; r.dy = d.y; r.dz = d.z; r.time = time;
        }
        const uint32_t qi = warp_append(&W.cnt[q ^ 1], start ? 1u : 0u);
        if (start) {
            W.qray[q ^ 1][qi] = r;
            W.qslot[q ^ 1][qi] = slot;
        }
        const bool still_idle = need && !got;
        const uint32_t ii = warp_append(&W.cnt[SV_IDLE0 + (q ^ 1)], still_idle ? 1u : 0u);
        if (still_idle) W.idle[q ^ 1][ii] = slot;
    }
}

// ---------------------------------------------------------------------------
// Host
// ---------------------------------------------------------------------------
double now_ms(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

struct HostReq {
    uint64_t id = 0, user = 0;
    uint32_t scene = 0, width = 0, height = 0, frames = 0, spp = 0;
    ae_config config{};
    float *dst_accum = nullptr;
    uint8_t *dst_display = nullptr;
    uint64_t footprint = 0, offset = 0, accum_bytes = 0, display_bytes = 0;
    uint32_t version = 0;
    int table = -1;
    uint64_t admit_launch = 0;
    double t_submit = 0, t_admit = -1, t_done = -1;
    int status = 1;  // 1 = not finished
    int stage = 0;   // 0 queued, 1 on the GPU, 2 result being copied
    uint32_t target = 0;  // finished pixels that complete it (lowered to the claimed ones on cancel)
    uint32_t copy = 0;    // the copy of its scene's per-frame arrays it renders from
    bool cancel = false;  // withdrawn by ae_serve_cancel while on the GPU
};

struct MoveOp {
    uint32_t scene;
    uint32_t version = 0;  // the scene version this move creates
    uint32_t copy = 0;     // the copy of the per-frame arrays it is written into
    std::vector<ae_instance> inst;
};

// One copy of a scene's per-frame arrays.  Version v of a scene is rendered
// from copy v % 2, so a move is prepared in the other copy while requests of
// the current version keep running.
struct FrameSet {
    DevBuf<ae_object> objects;
    DevBuf<ae_bvh_node> tlas;
    DevBuf<ae_instance> instances;
    DevBuf<FastInst> inst;
    DevBuf<QNode> tnodes;  // the optimised walks' instance-level tree
};
constexpr uint32_t kFrameSets = AE_SERVE_FRAME_SETS;

typedef void (*SvExtendFn)(SvView, int);

}  // namespace

struct Server {
    ae_serve_settings st{};
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    cudaStream_t stream = nullptr, copy_stream = nullptr, stats_stream = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    bool ev_live[2] = {false, false};
    cudaGraphExec_t graph = nullptr;
    int sms = 148;

    // slot pool and queues
    DevBuf<uint32_t> s_u32;  // 7 arrays of slots
    DevBuf<float4> s_f4;     // 5 arrays of slots
    DevBuf<uint8_t> s_u8;    // 2 arrays of slots
    DevBuf<ae_ray> qray;     // 2 x slots
    DevBuf<uint32_t> qslot, idle;
    DevBuf<ae_hit> qhit;
    DevBuf<float4> sh4;      // 4 x slots x max_lights
    DevBuf<uint8_t> sh8;     // 2 x slots x max_lights
    DevBuf<uint32_t> sq;
    DevBuf<uint32_t> cnt, next, done, order;
    DevBuf<unsigned long long> stats;
    DevBuf<SceneRec> scenes_d;
    DevBuf<ReqDev> reqs_d;
    unsigned char *arena = nullptr;
    SvView view{};

    // pinned staging
    ReqDev *h_req = nullptr;      // 2 x max_requests
    uint32_t *h_order = nullptr;  // 2 x (max_requests + 1)
    uint32_t *h_done = nullptr;   // 2 x (max_requests + 1): done counters, then the error word

    // state shared with the API threads
    std::mutex mu;
    std::condition_variable cv_sched, cv_done, cv_copy;
    std::string err;
    Policy policy;
    std::vector<Ctx *> scene_ctx;
    std::vector<std::unique_ptr<FrameSet[]>> frame_sets;  // kFrameSets per scene
    std::map<uint64_t, std::unique_ptr<HostReq>> reqs;
    std::vector<std::deque<MoveOp>> moves;
    std::deque<HostReq *> copy_queue;
    std::vector<HostReq *> cancels;  // admitted requests withdrawn, for the scheduler
    DevBuf<uint32_t> cancel_claimed;
    std::vector<HostReq *> table;
    std::vector<int> table_free;
    std::vector<int> order_host;  // table entries in admission order
    bool order_dirty = true;
    uint64_t next_id = 1;
    uint64_t outstanding = 0;  // requests + moves not finished
    bool stop = false, stop_copy = false, failed = false;
    std::thread sched, completer;

    // statistics
    std::vector<double> latencies;
    uint64_t submitted = 0, completed = 0, rejected = 0, n_failed = 0, paths = 0, launches = 0;
    double first_submit = -1, last_done = -1;
    uint64_t peak_arena = 0;
    uint32_t peak_resident = 0, moves_applied = 0, moves_coalesced = 0, dev_errors = 0, n_cancelled = 0;
    unsigned long long rays_base = 0;

    int fail_locked(int code, const char *fmt, ...) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        std::vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        err = buf;
        return code;
    }
    int init();
    int build_graph();
    void run();
    void run_completer();
    void fail_all(int code, const std::string &why);
    int apply_move(MoveOp &m);
    int fill_frame_set(uint32_t scene, uint32_t copy);
    ~Server();
};

namespace {

const SvExtendFn kSvExtend[3] = {k_sv_extend<64>, k_sv_extend<128>, k_sv_extend<256>};

int extend_index(uint32_t threads) { return threads == 256 ? 2 : threads == 128 ? 1 : 0; }

size_t sv_extend_smem(int threads) { return size_t(threads) * sizeof(ae_ray) + size_t(threads) * kServeStack * sizeof(uint2); }

}  // namespace

int Server::init() {
    const uint32_t S = st.slots, L = st.max_lights, R = st.max_requests;
    if (cudaSetDevice(st.device) != cudaSuccess) { cudaGetLastError(); err = "cudaSetDevice failed"; return AE_ERR_CUDA; }
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, st.device);
    if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&stats_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        err = "stream or event creation failed";
        return AE_ERR_CUDA;
    }
    const size_t SL = size_t(S) * L;
    if (s_u32.reserve(size_t(S) * 7) || s_f4.reserve(size_t(S) * 5) || s_u8.reserve(size_t(S) * 2) ||
        qray.reserve(size_t(S) * 2) || qslot.reserve(size_t(S) * 2) || idle.reserve(size_t(S) * 2) ||
        qhit.reserve(S) || sh4.reserve(SL * 4) || sh8.reserve(SL * 2) || sq.reserve(SL) || cnt.reserve(SV_COUNT) ||
        next.reserve(R) || done.reserve(R) || order.reserve(R) || stats.reserve(ST_COUNT) ||
        scenes_d.reserve(size_t(st.max_scenes) * kFrameSets) || reqs_d.reserve(R) || cancel_claimed.reserve(1)) {
        err = "slot pool allocation failed";
        return AE_ERR_OOM;
    }
    if (dev_alloc(reinterpret_cast<void **>(&arena), st.arena_bytes) != cudaSuccess) {
        cudaGetLastError();
        arena = nullptr;
        err = "image arena allocation failed";
        return AE_ERR_OOM;
    }
    if (cudaMallocHost(&h_req, sizeof(ReqDev) * 2 * R) != cudaSuccess ||
        cudaMallocHost(&h_order, sizeof(uint32_t) * 2 * (R + 1)) != cudaSuccess ||
        cudaMallocHost(&h_done, sizeof(uint32_t) * 2 * (R + 1)) != cudaSuccess) {
        cudaGetLastError();
        err = "pinned staging allocation failed";
        return AE_ERR_OOM;
    }
    SvView &W = view;
    W.scenes = scenes_d.ptr;
    W.reqs = reqs_d.ptr;
    W.next = next.ptr;
    W.done = done.ptr;
    W.order = order.ptr;
    W.cnt = cnt.ptr;
    W.stats = stats.ptr;
    uint32_t *u = s_u32.ptr;
    W.s_req = u; W.s_pix = u + S; W.s_frame = u + 2 * size_t(S); W.s_sample = u + 3 * size_t(S);
    W.s_bounce = u + 4 * size_t(S); W.s_seed = u + 5 * size_t(S); W.s_scene = u + 6 * size_t(S);
    float4 *f = s_f4.ptr;
    W.s_thr = f; W.s_acc = f + S; W.s_col = f + 2 * size_t(S); W.s_accp = f + 3 * size_t(S); W.s_pend = f + 4 * size_t(S);
    W.s_nee = s_u8.ptr; W.s_end = s_u8.ptr + S;
    W.qray[0] = qray.ptr; W.qray[1] = qray.ptr + S;
    W.qslot[0] = qslot.ptr; W.qslot[1] = qslot.ptr + S;
    W.qhit = qhit.ptr;
    W.idle[0] = idle.ptr; W.idle[1] = idle.ptr + S;
    W.sh = ShadowStore{sh4.ptr, sh4.ptr + SL, sh4.ptr + 2 * SL, sh4.ptr + 3 * SL, sh8.ptr, sh8.ptr + SL};
    W.sq = sq.ptr;
    W.max_lights = L;
    W.claim_shared = st.claim_policy == AE_CLAIM_SHARED ? 1u : 0u;
    cudaMemsetAsync(next.ptr, 0, sizeof(uint32_t) * R, stream);
    cudaMemsetAsync(done.ptr, 0, sizeof(uint32_t) * R, stream);
    k_sv_init<<<sms * 4, 256, 0, stream>>>(W, S);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(stream) != cudaSuccess) {
        cudaGetLastError();
        err = "slot pool initialisation failed";
        return AE_ERR_CUDA;
    }
    policy.configure(st.arena_bytes, st.max_requests, kFrameSets);
    scene_ctx.reserve(st.max_scenes);
    frame_sets.reserve(st.max_scenes);
    moves.reserve(st.max_scenes);
    table.assign(R, nullptr);
    for (int i = int(R) - 1; i >= 0; i--) table_free.push_back(i);
    int rc = build_graph();
    if (rc) return rc;
    sched = std::thread([this] { run(); });
    completer = std::thread([this] { run_completer(); });
    return AE_OK;
}

// One replay = ticks_per_launch ticks of six stages; launch shapes fixed here.
// The extend stage runs on the step-wise walker (the merged queue mixes
// requests, scenes and bounces; measured on the B200 serving mix: p50/p99
// 1.35/5.52 s with the tile-staged extend, 0.97/4.34 s with the walker), or
// tile-staged with an explicit extend_threads.
int Server::build_graph() {
    const bool walk = st.extend_threads == 0;
    const int ei = extend_index(st.extend_threads);
    const int et = walk ? 128 : (ei == 2 ? 256 : ei == 1 ? 128 : 64);
    // Walker stages: runs of queue_run entries per warp, or (queue_run 1)
    // the static assignment.
    const bool dyn = st.queue_run > 1;
    const uint32_t run = st.queue_run;
    const void *wfn = dyn ? reinterpret_cast<const void *>(k_sv_extend_walk<true>)
                          : reinterpret_cast<const void *>(k_sv_extend_walk<false>);
    const void *efn = walk ? wfn : reinterpret_cast<const void *>(kSvExtend[ei]);
    const void *shfn = dyn ? reinterpret_cast<const void *>(k_sv_shadow<128, true>)
                           : reinterpret_cast<const void *>(k_sv_shadow<128, false>);
    const size_t shsmem = size_t(kSharedStack) * 128 * sizeof(uint2);
    const size_t esmem = walk ? shsmem : sv_extend_smem(et);
    cudaFuncSetAttribute(efn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(esmem));
    cudaFuncSetAttribute(shfn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(shsmem));
    int e_per_sm = 0, sh_per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&e_per_sm, efn, et, esmem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&sh_per_sm, shfn, 128, shsmem);
    const int egrid = std::max(1, e_per_sm) * sms, shgrid = std::max(1, sh_per_sm) * sms, g256 = sms * 8;
    if (cudaGetLastError() != cudaSuccess) { err = "launch shape query failed"; return AE_ERR_CUDA; }
    cudaGraph_t g;
    if (cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        err = "graph capture failed";
        return AE_ERR_CUDA;
    }
    const SvView W = view;
    for (uint32_t t = 0; t < st.ticks_per_launch; t++) {
        const int q = int(t & 1);
        k_sv_begin<<<1, 1, 0, stream>>>(W, q);
        if (!walk) kSvExtend[ei]<<<egrid, et, esmem, stream>>>(W, q);
        else if (dyn) k_sv_extend_walk<true><<<egrid, et, esmem, stream>>>(W, q, run);
        else k_sv_extend_walk<false><<<egrid, et, esmem, stream>>>(W, q, 0u);
        k_sv_shade<<<g256, 256, 0, stream>>>(W, q);
        if (dyn) k_sv_shadow<128, true><<<shgrid, 128, shsmem, stream>>>(W, run);
        else k_sv_shadow<128, false><<<shgrid, 128, shsmem, stream>>>(W, 0u);
        k_sv_connect<<<g256, 256, 0, stream>>>(W, q);
        k_sv_advance<<<g256, 256, 0, stream>>>(W, q);
    }
    const cudaError_t le = cudaGetLastError();
    cudaError_t ce = cudaStreamEndCapture(stream, &g);
    if (le != cudaSuccess || ce != cudaSuccess) { cudaGetLastError(); err = "graph capture failed"; return AE_ERR_CUDA; }
    ce = cudaGraphInstantiate(&graph, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) { cudaGetLastError(); err = "graph instantiate failed"; return AE_ERR_CUDA; }
    return AE_OK;
}

// Copies the scene context's current per-frame arrays into one of the
// scene's frame sets and points that set's row of the device scene table at
// it (geometry and the optimised BLAS stay shared).
int Server::fill_frame_set(uint32_t scene, uint32_t copy) {
    Ctx *c = scene_ctx[scene];
    FrameSet &fs = frame_sets[scene][copy];
    FastScene &F = *c->fast;
    const size_t no = std::max<size_t>(c->n_objects, 1), nn = std::max<size_t>(c->n_nodes, 1),
                 ni = std::max<size_t>(c->n_instances, 1);
    const size_t nt = std::max<size_t>(F.n_tnodes, 1);
    if (fs.objects.reserve(no) || fs.tlas.reserve(nn) || fs.instances.reserve(ni) || fs.inst.reserve(ni) ||
        fs.tnodes.reserve(nt))
        return AE_ERR_OOM;
    cudaStream_t cs = c->stream;
    cudaError_t e = cudaSuccess;
    if (c->n_objects)
        e = cudaMemcpyAsync(fs.objects.ptr, c->objects.ptr, c->n_objects * sizeof(ae_object), cudaMemcpyDeviceToDevice, cs);
    if (e == cudaSuccess && c->n_nodes)
        e = cudaMemcpyAsync(fs.tlas.ptr, c->tlas.ptr, c->n_nodes * sizeof(ae_bvh_node), cudaMemcpyDeviceToDevice, cs);
    if (e == cudaSuccess && c->n_instances)
        e = cudaMemcpyAsync(fs.instances.ptr, c->instances.ptr, c->n_instances * sizeof(ae_instance),
                            cudaMemcpyDeviceToDevice, cs);
    if (e == cudaSuccess && c->n_instances)
        e = cudaMemcpyAsync(fs.inst.ptr, F.inst.ptr, c->n_instances * sizeof(FastInst), cudaMemcpyDeviceToDevice, cs);
    if (e == cudaSuccess && F.n_tnodes)
        e = cudaMemcpyAsync(fs.tnodes.ptr, F.tnodes.ptr, F.n_tnodes * sizeof(QNode), cudaMemcpyDeviceToDevice, cs);
    if (e == cudaSuccess) e = cudaStreamSynchronize(cs);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return AE_ERR_CUDA;
    }
    DevScene S = c->scene();
    S.objects = fs.objects.ptr;
    S.tlas = fs.tlas.ptr;
    S.instances = fs.instances.ptr;
    const SceneRec rec{S, fast_view(F, fs.inst.ptr, fs.tnodes.ptr)};
    // Stream order puts the row before any replay that reads it.
    if (cudaMemcpyAsync(scenes_d.ptr + size_t(scene) * kFrameSets + copy, &rec, sizeof(rec), cudaMemcpyHostToDevice,
                        stream) != cudaSuccess) {
        cudaGetLastError();
        return AE_ERR_CUDA;
    }
    return AE_OK;
}

// Applies one queued move: refit on the scene's context (which always holds
// the newest version), its optimised instance records, then a copy into the
// frame set of the new version.
int Server::apply_move(MoveOp &m) {
    Ctx *c = scene_ctx[m.scene];
    int rc = ae_refit_instances(reinterpret_cast<ae_ctx *>(c), m.inst.data(), uint32_t(m.inst.size()));
    if (rc == AE_OK) rc = prepare_fast(c);
    if (rc == AE_OK) rc = c->cuda(cudaStreamSynchronize(c->stream), "refit");
    if (rc == AE_OK) rc = fill_frame_set(m.scene, m.copy);
    if (rc != AE_OK) {
        std::lock_guard<std::mutex> lk(mu);
        err = "instance move: " + (c->err.empty() ? std::string("frame set copy failed") : c->err);
    }
    return rc;
}

void Server::fail_all(int code, const std::string &why) {
    // called with mu held
    failed = true;
    if (err.empty()) err = why;
    for (auto &kv : reqs) {
        HostReq *r = kv.second.get();
        if (r->status == 1 && r->stage < 2) {  // results already being copied still complete
            r->status = code;
            r->t_done = now_ms(t0);
            n_failed++;
        }
    }
    outstanding = copy_queue.size();
    cv_done.notify_all();
}

void Server::run() {
    cudaSetDevice(st.device);
    uint64_t issued = 0, observed = 0;
    for (;;) {
        std::vector<MoveOp> todo_moves;
        std::vector<HostReq *> admitted, todo_cancels;
        bool active;
        {
            std::unique_lock<std::mutex> lk(mu);
            if (stop || failed) break;
            todo_cancels.swap(cancels);
            uint32_t s, v, cp;
            bool coalesced = false;
            while (policy.next_move(s, v, cp)) {
                // Moves below version v are superseded by it (absolute transforms).
                while (!moves[s].empty() && moves[s].front().version < v) {
                    moves[s].pop_front();
                    moves_coalesced++;
                    coalesced = true;
                    if (outstanding) outstanding--;
                }
                if (moves[s].empty() || moves[s].front().version != v) break;  // not reached: v was submitted
                todo_moves.push_back(std::move(moves[s].front()));
                moves[s].pop_front();
                todo_moves.back().copy = cp;
                policy.move_applied(s, v, cp);  // requests of version v wait for this iteration's upload
            }
            if (coalesced) cv_done.notify_all();
            PolicyRequest pr;
            uint64_t off;
            while (!table_free.empty() && policy.next_admission(pr, off)) {
                HostReq *r = reqs[pr.id].get();
                r->offset = off;
                r->table = table_free.back();
                table_free.pop_back();
                table[r->table] = r;
                r->t_admit = now_ms(t0);
                r->stage = 1;
                r->copy = pr.copy;
                r->target = r->width * r->height;
                r->admit_launch = issued;
                order_host.push_back(r->table);
                order_dirty = true;
                admitted.push_back(r);
            }
            peak_resident = std::max(peak_resident, policy.resident());
            peak_arena = std::max(peak_arena, policy.arena().used());
            active = !order_host.empty();
            if (!active && todo_moves.empty() && issued == observed) {
                cv_sched.wait_for(lk, std::chrono::milliseconds(20));
                continue;
            }
        }
        for (MoveOp &m : todo_moves) {
            if (apply_move(m) != AE_OK) {
                std::lock_guard<std::mutex> lk(mu);
                fail_all(AE_ERR_CUDA, err);
                break;
            }
            std::lock_guard<std::mutex> lk(mu);
            moves_applied++;
            if (outstanding) outstanding--;
            cv_done.notify_all();
        }
        // Descriptors of the admitted requests and the admission order go
        // through pinned staging half h = parity of the next replay; the
        // replay two before it (the last reader of half h) has always been
        // observed by now, and copies not followed by a replay are waited for.
        const int h = int(issued & 1);
        bool staged = false;
        if (!admitted.empty() || order_dirty) {
            if (ev_live[h]) cudaEventSynchronize(ev[h]);
            staged = true;
            ReqDev *hr = h_req + size_t(h) * st.max_requests;
            for (size_t i = 0; i < admitted.size(); i++) {
                HostReq *r = admitted[i];
                ae_config cfg = r->config;
                cfg.width = r->width;
                cfg.height = r->height;
                cfg.batch = 0;
                ReqDev &d = hr[i];
                d.F = make_frame_params(cfg);
                d.accum = reinterpret_cast<float4 *>(arena + r->offset);
                d.display = reinterpret_cast<uchar4 *>(arena + r->offset + r->accum_bytes);
                d.scene = r->scene * kFrameSets + r->copy;
                d.n_pixels = r->width * r->height;
                d.frames = r->frames;
                d.spp = d.F.spp;
                cudaMemcpyAsync(reqs_d.ptr + r->table, &d, sizeof(ReqDev), cudaMemcpyHostToDevice, stream);
                cudaMemsetAsync(next.ptr + r->table, 0, sizeof(uint32_t), stream);
                cudaMemsetAsync(done.ptr + r->table, 0, sizeof(uint32_t), stream);
            }
            uint32_t *ho = h_order + size_t(h) * (st.max_requests + 1);
            {
                std::lock_guard<std::mutex> lk(mu);
                for (size_t i = 0; i < order_host.size(); i++) ho[i] = uint32_t(order_host[i]);
                ho[st.max_requests] = uint32_t(order_host.size());
                order_dirty = false;
            }
            if (ho[st.max_requests]) cudaMemcpyAsync(order.ptr, ho, sizeof(uint32_t) * ho[st.max_requests],
                                                     cudaMemcpyHostToDevice, stream);
            cudaMemcpyAsync(cnt.ptr + SV_NORDER, ho + st.max_requests, sizeof(uint32_t), cudaMemcpyHostToDevice, stream);
        }
        // Withdrawn requests stop claiming pixels before the next replay; the
        // pixels already claimed finish and complete them.
        for (HostReq *r : todo_cancels) {
            if (r->stage != 1 || r->table < 0) continue;
            uint32_t claimed = 0;
            k_sv_cancel<<<1, 1, 0, stream>>>(view, uint32_t(r->table), cancel_claimed.ptr);
            cudaError_t ce = cudaMemcpyAsync(&claimed, cancel_claimed.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                             stream);
            if (ce == cudaSuccess) ce = cudaStreamSynchronize(stream);
            std::lock_guard<std::mutex> lk(mu);
            if (ce != cudaSuccess) {
                fail_all(AE_ERR_CUDA, std::string("cancel: ") + cudaGetErrorString(ce));
                break;
            }
            r->target = claimed;
        }
        if (active) {
            cudaGraphLaunch(graph, stream);
            uint32_t *hd = h_done + size_t(h) * (st.max_requests + 1);
            cudaMemcpyAsync(hd, done.ptr, sizeof(uint32_t) * st.max_requests, cudaMemcpyDeviceToHost, stream);
            cudaMemcpyAsync(hd + st.max_requests, cnt.ptr + SV_ERR, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream);
            cudaEventRecord(ev[h], stream);
            ev_live[h] = true;
            issued++;
            launches++;
            const cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) {
                std::lock_guard<std::mutex> lk(mu);
                fail_all(AE_ERR_CUDA, std::string("graph replay: ") + cudaGetErrorString(e));
                break;
            }
        }
        else if (staged) {
            cudaStreamSynchronize(stream);
        }
        // Observe finished replays: wait while two are in flight (or nothing
        // new was queued), otherwise only poll.
        bool broke = false;
        while (observed < issued) {
            const int k = int(observed & 1);
            const bool must = (issued - observed) >= 2 || !active;
            cudaError_t e = must ? cudaEventSynchronize(ev[k]) : cudaEventQuery(ev[k]);
            if (e == cudaErrorNotReady) break;
            if (e != cudaSuccess) {
                std::lock_guard<std::mutex> lk(mu);
                fail_all(AE_ERR_CUDA, std::string("serving replay: ") + cudaGetErrorString(e));
                broke = true;
                break;
            }
            ev_live[k] = false;
            const uint32_t *hd = h_done + size_t(k) * (st.max_requests + 1);
            std::lock_guard<std::mutex> lk(mu);
            if (hd[st.max_requests]) {
                dev_errors = hd[st.max_requests];
                fail_all(AE_ERR_TIMEOUT, "a bounded queue-tile wait gave up on the device");
                broke = true;
                break;
            }
            for (size_t i = 0; i < order_host.size();) {
                const int t = order_host[i];
                HostReq *r = table[t];
                if (r && r->admit_launch <= observed && hd[t] >= r->target) {
                    table[t] = nullptr;
                    table_free.push_back(t);
                    order_host.erase(order_host.begin() + long(i));
                    order_dirty = true;
                    r->stage = 2;
                    copy_queue.push_back(r);
                    cv_copy.notify_one();
                } else {
                    i++;
                }
            }
            observed++;
        }
        if (broke) break;
    }
    cudaStreamSynchronize(stream);
}

void Server::run_completer() {
    cudaSetDevice(st.device);
    for (;;) {
        HostReq *r;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_copy.wait(lk, [this] { return stop_copy || !copy_queue.empty(); });
            if (copy_queue.empty()) return;
            r = copy_queue.front();
            copy_queue.pop_front();
        }
        cudaError_t e = cudaSuccess;
        if (r->cancel) {
            // Withdrawn: its pixels in flight have finished; nothing is copied.
            std::lock_guard<std::mutex> lk(mu);
            policy.completed(r->id);
            if (r->status == 1) {
                r->status = AE_ERR_CANCELLED;
                r->t_done = now_ms(t0);
                n_cancelled++;
                if (outstanding) outstanding--;
            }
            cv_done.notify_all();
            cv_sched.notify_one();
            continue;
        }
        if (r->dst_accum)
            e = cudaMemcpyAsync(r->dst_accum, arena + r->offset, r->accum_bytes, cudaMemcpyDeviceToHost, copy_stream);
        if (e == cudaSuccess && r->dst_display)
            e = cudaMemcpyAsync(r->dst_display, arena + r->offset + r->accum_bytes, r->display_bytes,
                                cudaMemcpyDeviceToHost, copy_stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(copy_stream);
        std::lock_guard<std::mutex> lk(mu);
        policy.completed(r->id);
        if (r->status == 1) {
            r->t_done = now_ms(t0);
            if (e == cudaSuccess) {
                r->status = AE_OK;
                completed++;
                paths += uint64_t(r->width) * r->height * r->frames * r->spp;
                latencies.push_back(r->t_done - r->t_submit);
                last_done = std::max(last_done, r->t_done);
            } else {
                cudaGetLastError();
                r->status = AE_ERR_CUDA;
                n_failed++;
                err = std::string("result copy: ") + cudaGetErrorString(e);
            }
            if (outstanding) outstanding--;
        }
        cv_done.notify_all();
        cv_sched.notify_one();
    }
}

Server::~Server() {
    {
        std::lock_guard<std::mutex> lk(mu);
        stop = true;
    }
    cv_sched.notify_all();
    cv_copy.notify_all();
    if (sched.joinable()) sched.join();
    // Copies already queued still complete; the completer exits after them.
    {
        std::lock_guard<std::mutex> lk(mu);
        stop_copy = true;
    }
    cv_copy.notify_all();
    if (completer.joinable()) completer.join();
    if (graph) cudaGraphExecDestroy(graph);
    if (stream) cudaStreamSynchronize(stream);
    if (arena) dev_free(arena);
    if (h_req) cudaFreeHost(h_req);
    if (h_order) cudaFreeHost(h_order);
    if (h_done) cudaFreeHost(h_done);
    for (cudaEvent_t e : ev)
        if (e) cudaEventDestroy(e);
    if (stream) cudaStreamDestroy(stream);
    if (copy_stream) cudaStreamDestroy(copy_stream);
    if (stats_stream) cudaStreamDestroy(stats_stream);
}

}  // namespace ae

using namespace ae;

struct ae_server : Server {};

extern "C" ae_server *ae_serve_create(const ae_serve_settings *settings) {
    set_create_status(AE_ERR_INVALID);
    ae_serve_settings s{};
    if (settings) s = *settings;
    if (!s.slots) s.slots = 1u << 20;
    if (!s.max_lights) s.max_lights = 16;
    if (!s.max_requests) s.max_requests = 64;
    if (!s.arena_bytes) s.arena_bytes = 1ull << 30;
    if (!s.ticks_per_launch) s.ticks_per_launch = 4;
    if (s.extend_threads != 0 && s.extend_threads != 64 && s.extend_threads != 128 && s.extend_threads != 256)
        return nullptr;
    if (!s.max_scenes) s.max_scenes = 16;
    if (!s.queue_run) s.queue_run = kServeQueueRun;
    if (s.max_lights > kServeMaxLights || s.max_requests > kServeMaxRequests || (s.ticks_per_launch & 1) ||
        s.claim_policy > AE_CLAIM_SHARED || s.queue_run > 1024 ||
        s.slots > (1u << 26) || uint64_t(s.slots) * s.max_lights > 0xffffffffull)
        return nullptr;
    ae_server *srv = new (std::nothrow) ae_server();
    if (!srv) {
        set_create_status(AE_ERR_OOM);
        return nullptr;
    }
    srv->st = s;
    const int rc = srv->init();
    if (rc != AE_OK) {
        std::fprintf(stderr, "ae_serve_create: %s\n", srv->err.c_str());
        delete srv;
        set_create_status(rc);
        return nullptr;
    }
    set_create_status(AE_OK);
    return srv;
}

extern "C" void ae_serve_destroy(ae_server *srv) {
    if (!srv) return;
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        for (uint64_t id : srv->policy.cancel_pending()) {
            auto it = srv->reqs.find(id);
            if (it != srv->reqs.end() && it->second->status == 1) it->second->status = AE_ERR_STATE;
        }
        srv->cv_done.notify_all();
    }
    delete srv;
}

extern "C" const char *ae_serve_last_error(ae_server *srv) {
    if (!srv) return "null server";
    std::lock_guard<std::mutex> lk(srv->mu);
    return srv->err.c_str();
}

extern "C" int ae_serve_add_scene(ae_server *srv, ae_ctx *scene, uint32_t *scene_id) {
    if (!srv || !scene) return AE_ERR_INVALID;
    Ctx *c = reinterpret_cast<Ctx *>(scene);
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        if (srv->scene_ctx.size() >= srv->st.max_scenes)
            return srv->fail_locked(AE_ERR_OVERSIZE, "at most %u resident scenes", srv->st.max_scenes);
        if (c->settings.device != srv->st.device)
            return srv->fail_locked(AE_ERR_INVALID, "scene context is on device %d, server on %d", c->settings.device,
                                    srv->st.device);
        if (c->n_lights > srv->st.max_lights)
            return srv->fail_locked(AE_ERR_OVERSIZE, "scene has %u lights; server takes %u", c->n_lights,
                                    srv->st.max_lights);
        for (Ctx *o : srv->scene_ctx)
            if (o == c) return srv->fail_locked(AE_ERR_INVALID, "scene context already resident");
    }
    // The optimised BVH build can take seconds; it runs without the lock.
    int rc = prepare_fast(c);
    if (rc == AE_OK) rc = c->cuda(cudaStreamSynchronize(c->stream), "prepare scene");
    std::lock_guard<std::mutex> lk(srv->mu);
    if (rc != AE_OK) return srv->fail_locked(rc, "scene: %s", c->err.c_str());
    if (srv->scene_ctx.size() >= srv->st.max_scenes)
        return srv->fail_locked(AE_ERR_OVERSIZE, "at most %u resident scenes", srv->st.max_scenes);
    const uint32_t id = uint32_t(srv->scene_ctx.size());
    std::unique_ptr<FrameSet[]> sets(new (std::nothrow) FrameSet[kFrameSets]);
    if (!sets) return srv->fail_locked(AE_ERR_OOM, "frame sets");
    srv->scene_ctx.push_back(c);  // capacity reserved at creation: the scheduler reads it unlocked
    srv->frame_sets.push_back(std::move(sets));
    for (uint32_t k = 0; k < kFrameSets; k++) {
        if ((rc = srv->fill_frame_set(id, k)) != AE_OK) {
            srv->scene_ctx.pop_back();
            srv->frame_sets.pop_back();
            return srv->fail_locked(rc, "scene %u: frame set copy failed", id);
        }
    }
    if (cudaStreamSynchronize(srv->stream) != cudaSuccess) {
        cudaGetLastError();
        return srv->fail_locked(AE_ERR_CUDA, "scene table upload failed");
    }
    srv->moves.emplace_back();
    srv->policy.add_scene();
    if (scene_id) *scene_id = id;
    return AE_OK;
}

extern "C" int ae_serve_submit(ae_server *srv, const ae_serve_request *req, uint64_t *id) {
    if (!srv || !req) return AE_ERR_INVALID;
    std::unique_ptr<HostReq> r(new (std::nothrow) HostReq());
    if (!r) return AE_ERR_OOM;
    std::lock_guard<std::mutex> lk(srv->mu);
    if (srv->failed) return AE_ERR_STATE;
    if (req->scene >= srv->scene_ctx.size()) return srv->fail_locked(AE_ERR_INVALID, "unknown scene %u", req->scene);
    if (!req->width || !req->height || !req->frames || uint64_t(req->width) * req->height > (1ull << 30))
        return srv->fail_locked(AE_ERR_INVALID, "bad request size %ux%u x %u frames", req->width, req->height, req->frames);
    if (req->config.depth == 0 || req->config.depth > 64) return srv->fail_locked(AE_ERR_INVALID, "depth %u outside 1..64", req->config.depth);
    r->id = srv->next_id++;
    r->user = req->user;
    r->scene = req->scene;
    r->width = req->width;
    r->height = req->height;
    r->frames = req->frames;
    r->config = req->config;
    const uint32_t per = req->config.batches ? req->config.samples / req->config.batches : req->config.samples;
    r->spp = per > 1u ? per : 1u;
    r->dst_accum = req->accum;
    r->dst_display = req->display;
    const uint64_t px = uint64_t(req->width) * req->height;
    r->accum_bytes = align_up(px * 16, Arena::kAlign);
    r->display_bytes = px * 4;
    r->footprint = r->accum_bytes + align_up(px * 4, Arena::kAlign);
    r->t_submit = now_ms(srv->t0);
    PolicyRequest pr;
    pr.id = r->id;
    pr.scene = r->scene;
    pr.footprint = r->footprint;
    srv->submitted++;
    if (srv->first_submit < 0) srv->first_submit = r->t_submit;
    if (!srv->policy.submit(pr)) {
        srv->rejected++;
        return srv->fail_locked(AE_ERR_REJECTED, "request of %llu image bytes exceeds the %llu-byte arena",
                                (unsigned long long)r->footprint, (unsigned long long)srv->st.arena_bytes);
    }
    r->version = pr.version;
    if (id) *id = r->id;
    srv->reqs[r->id] = std::move(r);
    srv->outstanding++;
    srv->cv_sched.notify_one();
    return AE_OK;
}

extern "C" int ae_serve_move_instances(ae_server *srv, uint32_t scene, const ae_instance *instances, uint32_t n) {
    if (!srv || (n && !instances)) return AE_ERR_INVALID;
    std::lock_guard<std::mutex> lk(srv->mu);
    if (srv->failed) return AE_ERR_STATE;
    if (scene >= srv->scene_ctx.size()) return srv->fail_locked(AE_ERR_INVALID, "unknown scene %u", scene);
    Ctx *c = srv->scene_ctx[scene];
    if (n != c->n_instances) return srv->fail_locked(AE_ERR_INVALID, "scene %u has %u instances, got %u", scene, c->n_instances, n);
    MoveOp m;
    m.scene = scene;
    m.inst.assign(instances, instances + n);
    m.version = srv->policy.move(scene);
    srv->moves[scene].push_back(std::move(m));
    srv->outstanding++;
    srv->cv_sched.notify_one();
    return AE_OK;
}

extern "C" int ae_serve_cancel(ae_server *srv, uint64_t id) {
    if (!srv) return AE_ERR_INVALID;
    std::lock_guard<std::mutex> lk(srv->mu);
    auto it = srv->reqs.find(id);
    if (it == srv->reqs.end()) return srv->fail_locked(AE_ERR_INVALID, "unknown request %llu", (unsigned long long)id);
    HostReq *r = it->second.get();
    if (r->status != 1 || r->stage == 2 || r->cancel)
        return srv->fail_locked(AE_ERR_STATE, "request %llu has finished or is being cancelled", (unsigned long long)id);
    if (r->stage == 0) {
        if (!srv->policy.withdraw(id)) return srv->fail_locked(AE_ERR_STATE, "request %llu is not queued", (unsigned long long)id);
        r->status = AE_ERR_CANCELLED;
        r->t_done = now_ms(srv->t0);
        srv->n_cancelled++;
        if (srv->outstanding) srv->outstanding--;
        srv->cv_done.notify_all();
        srv->cv_sched.notify_one();
        return AE_OK;
    }
    r->cancel = true;
    srv->cancels.push_back(r);
    srv->cv_sched.notify_one();
    return AE_OK;
}

// Test hook: the tile-staged extend of every later replay issues no copy and
// lets its bounded wait run out (AE_FAULT_TILE_WAIT), so the timeout path runs
// with nothing in flight.
extern "C" int ae_serve_debug_inject(ae_server *srv, int fault, uint32_t on) {
    if (!srv) return AE_ERR_INVALID;
    if (fault != AE_FAULT_TILE_WAIT) return AE_ERR_INVALID;
    const uint32_t v = on ? 1u : 0u;
    std::lock_guard<std::mutex> lk(srv->mu);
    if (cudaMemcpy(srv->cnt.ptr + SV_FAULT, &v, sizeof(v), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaGetLastError();
        return AE_ERR_CUDA;
    }
    return AE_OK;
}

extern "C" int ae_serve_wait(ae_server *srv, uint64_t id, int32_t timeout_ms, ae_serve_result *out) {
    if (!srv) return AE_ERR_INVALID;
    std::unique_lock<std::mutex> lk(srv->mu);
    auto it = srv->reqs.find(id);
    if (it == srv->reqs.end()) return srv->fail_locked(AE_ERR_INVALID, "unknown request %llu", (unsigned long long)id);
    HostReq *r = it->second.get();
    auto ready = [r] { return r->status != 1; };
    if (timeout_ms < 0) srv->cv_done.wait(lk, ready);
    else if (!srv->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) return AE_ERR_TIMEOUT;
    if (out) {
        out->id = r->id;
        out->user = r->user;
        out->status = r->status;
        out->scene_version = r->version;
        out->submit_ms = r->t_submit;
        out->admit_ms = r->t_admit;
        out->done_ms = r->t_done;
        out->paths = uint64_t(r->width) * r->height * r->frames * r->spp;
        out->footprint = r->footprint;
    }
    const int status = r->status;
    srv->reqs.erase(it);
    return status;
}

extern "C" int ae_serve_drain(ae_server *srv, int32_t timeout_ms) {
    if (!srv) return AE_ERR_INVALID;
    std::unique_lock<std::mutex> lk(srv->mu);
    auto ready = [srv] { return srv->outstanding == 0 || srv->failed; };
    if (timeout_ms < 0) srv->cv_done.wait(lk, ready);
    else if (!srv->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) return AE_ERR_TIMEOUT;
    return srv->failed ? AE_ERR_STATE : AE_OK;
}

extern "C" int ae_serve_get_stats(ae_server *srv, ae_serve_stats *out) {
    if (!srv || !out) return AE_ERR_INVALID;
    unsigned long long dev[ST_COUNT] = {0, 0};
    if (cudaMemcpyAsync(dev, srv->stats.ptr, sizeof(dev), cudaMemcpyDeviceToHost, srv->stats_stream) != cudaSuccess ||
        cudaStreamSynchronize(srv->stats_stream) != cudaSuccess) {
        cudaGetLastError();
        return AE_ERR_CUDA;
    }
    std::lock_guard<std::mutex> lk(srv->mu);
    std::memset(out, 0, sizeof(*out));
    out->submitted = srv->submitted;
    out->completed = srv->completed;
    out->rejected = srv->rejected;
    out->failed = srv->n_failed;
    out->paths = srv->paths;
    out->rays = dev[ST_RAYS] + dev[ST_SHADOW] - srv->rays_base;
    out->first_submit_ms = srv->first_submit;
    out->last_done_ms = srv->last_done;
    std::vector<double> l = srv->latencies;
    if (!l.empty()) {
        std::sort(l.begin(), l.end());
        auto pct = [&l](double p) {
            const double pos = p * double(l.size() - 1);
            const size_t lo = size_t(pos);
            const size_t hi = std::min(lo + 1, l.size() - 1);
            return l[lo] + (l[hi] - l[lo]) * (pos - double(lo));
        };
        out->p50_ms = pct(0.50);
        out->p99_ms = pct(0.99);
        double s = 0;
        for (double v : l) s += v;
        out->mean_ms = s / double(l.size());
        out->max_ms = l.back();
    }
    out->launches = srv->launches;
    out->peak_arena_bytes = srv->peak_arena;
    out->peak_resident = srv->peak_resident;
    out->moves_applied = srv->moves_applied;
    out->moves_coalesced = srv->moves_coalesced;
    out->errors = srv->dev_errors;
    out->cancelled = srv->n_cancelled;
    return AE_OK;
}

extern "C" int ae_serve_reset_stats(ae_server *srv) {
    if (!srv) return AE_ERR_INVALID;
    unsigned long long dev[ST_COUNT] = {0, 0};
    if (cudaMemcpyAsync(dev, srv->stats.ptr, sizeof(dev), cudaMemcpyDeviceToHost, srv->stats_stream) != cudaSuccess ||
        cudaStreamSynchronize(srv->stats_stream) != cudaSuccess) {
        cudaGetLastError();
        return AE_ERR_CUDA;
    }
    std::lock_guard<std::mutex> lk(srv->mu);
    srv->latencies.clear();
    srv->submitted = srv->completed = srv->rejected = srv->n_failed = srv->paths = srv->launches = 0;
    srv->n_cancelled = 0;
    srv->first_submit = srv->last_done = -1;
    srv->peak_arena = srv->policy.arena().used();
    srv->peak_resident = srv->policy.resident();
    srv->moves_applied = 0;
    srv->moves_coalesced = 0;
    srv->rays_base = dev[ST_RAYS] + dev[ST_SHADOW];
    return AE_OK;
}
