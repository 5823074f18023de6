// wavefront.cu - the compute-only path tracer (ColorRay, hybrid:1230-1325)
// restructured into persistent stages over compacted queues, so every stage
// runs coherent work at full occupancy instead of one divergent megakernel:
//
//   generate  camera rays (main, hybrid:1346-1373) into the ray queue
//   extend    closest hit of every queued ray (the optimised 4-wide walk);
//             for the camera rays each CTA stages a tile of the ray queue in
//             shared memory with a bulk asynchronous copy (cp.async.bulk,
//             completion on an mbarrier with a bounded wait); the incoherent
//             bounce queues run on the step-wise walker (fast_walk.cuh)
//   shade     miss / emission / NEE light sampling / bounce / Russian
//             roulette; surviving paths are appended to the next ray queue
//             and shadow rays to the shadow queue with warp-aggregated
//             atomics (ballot + prefix over the warp)
//   shadow    the reference's shadow test: up to four closest hits stepping
//             through glass (hybrid:1167-1191), on the step-wise walker
//   connect   NEE sums in light order, the luma clamp of 8, added to the path
//   finish    samples into the frame, the running accumulation and display
//
// RNG draws happen in shade in the reference's order (two per quad light,
// then the bounce, then roulette), and every arithmetic step is the plain
// megakernel's, so a wavefront frame equals the plain frame bit for bit.
//
// One frame is captured into a CUDA graph (all stage launches for Depth
// bounces, queue counts read on the device), replayed per frame with only the
// frame parameters copied in.  The extend stage's block size, queue tile and
// shared-memory stack depth come from an autotuner that times the candidates
// on the scene's own first-bounce queue.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "context.h"
#include "fast.h"
#include "fast_trace.cuh"
#include "kernels.h"
#include "shade.cuh"
#include "trace_common.cuh"
#include "fast_walk.cuh"
#include "wf_common.cuh"

namespace ae {

constexpr int kMaxLights = 64;  // NEE entries per path vertex

struct WfParams {
    FrameParams F;
    uint32_t n_paths, sample, spp, n_lights;
    uint32_t kahan;  // precision form: compensated accumulation
};

// Device counters: [0],[1] ray queue sizes (ping-pong), [2] shadow queue,
// [3] error flags, [4..4+kMaxBounce) extend tile counters, then shadow tiles.
constexpr int kMaxBounce = 64;
// C_FAULT: the injected tile-wait failure of ae_debug_inject (0 = none).
enum { C_Q0 = 0, C_Q1 = 1, C_SH = 2, C_ERR = 3, C_TILE = 4, C_SHTILE = 4 + kMaxBounce, C_FAULT = 4 + 2 * kMaxBounce,
       C_COUNT = 5 + 2 * kMaxBounce };

struct WfView {
    ae_ray *qray[2];
    uint32_t *qpid[2];
    ae_hit *qhit;
    float4 *thr, *acc, *col, *pend;
    uint32_t *seed;
    uint8_t *nee;
    ShadowStore sh;  // light-sample entries, index = path * n_lights + light
    uint32_t *sq;
    uint32_t *cnt;
    const WfParams *P;
    float4 *accum, *frame;
    uchar4 *display;
    float4 *ksum, *kcomp;  // precision form: compensated sum of frame colours
    PrecView prec;
};

struct Wavefront {
    uint32_t cap = 0, n_lights = 0;
    DevBuf<ae_ray> qray[2];
    DevBuf<uint32_t> qpid[2];
    DevBuf<ae_hit> qhit;
    DevBuf<float4> thr, acc, col, pend;
    DevBuf<uint32_t> seed;
    DevBuf<uint8_t> nee;
    DevBuf<float4> sh_o, sh_d, sh_lp, sh_c;
    DevBuf<uint8_t> sh_valid, sh_occ;
    DevBuf<uint32_t> sq;
    DevBuf<uint32_t> cnt;
    DevBuf<WfParams> params;
    DevBuf<float4> ksum, kcomp;
    WfParams *host_params = nullptr;  // pinned
    cudaGraphExec_t graph = nullptr;
    uint64_t graph_key = ~0ull;
    int sms = 148;
    // autotuned extend configuration
    int ext_threads = 128, ext_stack = 24;
    bool tuned = false;
    float tune_ms[9] = {0};
    // autotuned queue assignment of the walker stages, per form (index:
    // precision form), as a run length (0: static assignment)
    uint32_t walk_run[2] = {0, 0}, shadow_run[2] = {0, 0};
    // and register bound, as an index into kWalkMinBlocks (6 or 7 blocks per SM)
    int walk_mb[2] = {1, 1}, shadow_mb[2] = {1, 1};
    bool walk_tuned[2] = {false, false};
    // per stage (shadow, then the bounce extend): kRunCfgs x {6, 7} blocks per SM
    float walk_tune_ms[2][16] = {};
    ~Wavefront() {
        if (graph) cudaGraphExecDestroy(graph);
        if (host_params) cudaFreeHost(host_params);
    }
};

void destroy_wavefront(Ctx *c) {
    delete c->wave;
    c->wave = nullptr;
}

// ---------------------------------------------------------------------------
// Stages
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_wf_generate(WfView W) {
    const WfParams &P = *W.P;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        W.cnt[C_Q0] = P.n_paths;
        W.cnt[C_Q1] = 0;
        W.cnt[C_SH] = 0;
        for (int k = 0; k < 2 * kMaxBounce; k++) W.cnt[C_TILE + k] = 0;
    }
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < P.n_paths; p += gridDim.x * blockDim.x) {
        const uint32_t x = p % P.F.width, y = p / P.F.width;
        uint32_t seed;
        f3 o, d;
        float time;
        if (P.sample == 0) {
            camera_ray(P.F, x, y, o, d, time, seed);
        } else {
            // Later samples of the frame continue the pixel's stream (the
            // samples loop of main, hybrid:1366-1381).
            seed = W.seed[p];
            camera_sample(P.F, x, y, o, d, time, seed);
        }
        W.seed[p] = seed;
        ae_ray r;
        r.ox = o.x; r.oy = o.y; r.oz = o.z; r.tnear = 0.001f;
        r.dx = d.x; r.dy = d.y; r.dz = d.z; r.time = time;
        W.qray[0][p] = r;
        W.qpid[0][p] = p;
        W.thr[p] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
        W.acc[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (P.sample == 0) W.col[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        W.nee[p] = 0;
    }
}

// Extend: persistent CTAs take tiles of the ray queue; one elected thread
// bulk-copies the tile into shared memory and every thread traces one ray.
template <int THREADS, int SS, bool WT>
__global__ void __launch_bounds__(THREADS) k_wf_extend(DevScene S, FastView V, WfView W, int bounce) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ae_ray *tile = reinterpret_cast<ae_ray *>(smem_raw);
    uint2 *stk = reinterpret_cast<uint2 *>(smem_raw + THREADS * sizeof(ae_ray));
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tile_index;
    const int q = bounce & 1;
    const uint32_t count = W.cnt[q];
    // An injected failure (ae_debug_inject) issues no copy and waits on the
    // unarmed phase for a few polls: the timeout path runs with nothing in
    // flight.
    const bool inject = W.cnt[C_FAULT] != 0;
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    __syncthreads();
    uint32_t phase = 0;
    for (;;) {
        if (threadIdx.x == 0) tile_index = atomicAdd(&W.cnt[C_TILE + bounce], 1u);
        __syncthreads();
        const uint32_t start = tile_index * THREADS;
        if (start >= count) break;
        const uint32_t m = min(uint32_t(THREADS), count - start);
        if (threadIdx.x == 0 && !inject) {
            mbar_expect_tx(&bar, m * uint32_t(sizeof(ae_ray)));
            bulk_g2s(tile, W.qray[q] + start, m * uint32_t(sizeof(ae_ray)), &bar);
        }
        // Every thread polls the barrier (bounded); the block then agrees on
        // the outcome so no thread leaves while others wait at a barrier.
        const bool ok = __syncthreads_and(mbar_wait(&bar, phase, inject ? 64u : (1u << 24)) ? 1 : 0) != 0;
        if (!ok) {
            // A copy that has not landed after 2^24 polls gets a second
            // bounded wait before the block exits and reports the timeout.
            // Should it still be outstanding then, the block exits with a
            // bulk copy into its shared memory in flight, which PTX leaves
            // undefined; the bound keeps a kernel from hanging the GPU
            // instead.  A global-to-shared copy of at most 8 KB has never
            // come near it.
            if (!inject) mbar_wait(&bar, phase, 1u << 24);
            if (threadIdx.x == 0) atomicOr(&W.cnt[C_ERR], 1u);
            break;
        }
        phase ^= 1u;
        if (threadIdx.x < m) {
            const ae_ray r = tile[threadIdx.x];
            const Best b = closest_fast<WT, SS>(S, V, mk(r.ox, r.oy, r.oz), mk(r.dx, r.dy, r.dz), r.tnear, r.time,
                                                stk, threadIdx.x, THREADS);
            const bool any = b.object != AE_MISS;
            ae_hit h;
            h.t = any ? b.t : 0.0f;
            h.alpha = any ? b.alpha : 0.0f;
            h.beta = any ? b.beta : 0.0f;
            h.object = b.object;
            h.prim = b.prim;
            W.qhit[start + threadIdx.x] = h;
        }
        __syncthreads();  // the tile buffer is reused by the next copy
    }
}

// Extend on the step-wise Walker: a persistent grid, each thread stepping
// its own queued ray and taking the next one when one finishes - static
// assignment (DYN false: k + grid size) or runs of `run` consecutive queue
// entries per warp claimed from the bounce's counter (DYN true), compiled
// for MINB resident blocks per SM; the autotuner picks per scene.  For
// incoherent queues (bounces past the camera rays).
template <bool WT, bool DYN, int MINB>
__global__ void __launch_bounds__(128, MINB) k_wf_extend_walk(DevScene S, FastView V, WfView W, int bounce,
                                                                          uint32_t run) {
    extern __shared__ uint2 stk[];
    const int q = bounce & 1;
    const uint32_t count = W.cnt[q];
    const uint32_t stride = gridDim.x * blockDim.x;
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    Walker<WT> w;
    WalkStacks<> K;
    bool active = !DYN && k < count;
    bool need = DYN, exhausted = false;
    uint32_t cbase = 0, cend = 0;
    if (active) {
        const ae_ray r = W.qray[q][k];
        w.start(V, mk(r.ox, r.oy, r.oz), mk(r.dx, r.dy, r.dz), r.tnear, r.time);
    }
    uint32_t iter = 0;
    for (;;) {
        if (DYN && run_take(&W.cnt[C_TILE + bounce], count, run, need, k, cbase, cend, exhausted)) {
            active = true;
            const ae_ray r = W.qray[q][k];
            w.start(V, mk(r.ox, r.oy, r.oz), mk(r.dx, r.dy, r.dz), r.tnear, r.time);
        }
        const uint32_t am = __ballot_sync(0xffffffffu, active);
        if (!am) break;
        // Only the warp's largest phase group steps (warp_pick_group).
        const uint32_t pick = warp_pick_group(active ? w.group() : 0u, active, am, iter);
        if (!active || w.group() != pick || !w.step(S, V, K, stk, threadIdx.x, blockDim.x)) continue;
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
        if (active) {
            const ae_ray r = W.qray[q][k];
            w.start(V, mk(r.ox, r.oy, r.oz), mk(r.dx, r.dy, r.dz), r.tnear, r.time);
        }
    }
}

// Shade: one queued path per thread (ColorRay's body after the traversal).
template <bool PREC>
__global__ void __launch_bounds__(256) k_wf_shade(DevScene S, FastView V, WfView W, int bounce) {
    // After an extend that gave up, hit records past its last tile were never
    // written: nothing is shaded, the frame ends and reports the timeout.
    if (W.cnt[C_ERR]) return;
    const WfParams &P = *W.P;
    const int q = bounce & 1;
    const uint32_t count = W.cnt[q];
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
        const uint32_t pid = W.qpid[q][k];
        const ae_ray r = W.qray[q][k];
        const ae_hit hr = W.qhit[k];
        float4 t4 = W.thr[pid], a4 = W.acc[pid];
        f3 thr = mk(t4.x, t4.y, t4.z), acc = mk(a4.x, a4.y, a4.z);
        uint32_t seed = W.seed[pid];
        ae_ray nr;
        uint32_t n_shadow;
        const size_t e0 = size_t(pid) * P.n_lights;
        const bool next = shade_vertex<PREC>(S, V, W.prec, P.F.sky, P.F.depth, P.n_lights, bounce, r, hr, thr, acc,
                                             seed, W.sh, e0, W.nee + pid, W.pend + pid, n_shadow, nr);
        W.thr[pid] = make_float4(thr.x, thr.y, thr.z, 0.0f);
        W.acc[pid] = make_float4(acc.x, acc.y, acc.z, 0.0f);
        W.seed[pid] = seed;
        // Compaction into the next ray queue and the shadow queue.
        const uint32_t slot = warp_append(&W.cnt[q ^ 1], next ? 1u : 0u);
        if (next) {
            W.qray[q ^ 1][slot] = nr;
            W.qpid[q ^ 1][slot] = pid;
        }
        const uint32_t sbase = warp_append(&W.cnt[C_SH], n_shadow);
        if (n_shadow) push_shadow_entries(W.sh, pid * P.n_lights, P.n_lights, W.sq, sbase);
    }
}

// Shadow: the reference's occlusion loop per entry (hybrid:1167-1191: up to
// four closest hits, stepping through glass), run on a step-wise Walker so a
// lane that finishes an entry starts its next one at once instead of waiting
// for the warp's longest traversal.  The loop only asks whether the closest
// hit lies before |lp - so| - 0.001 (a hit at or beyond it, or none, leaves
// the sample unoccluded), so each walk starts with that distance as its
// bound: the verdict and the glass step are those of the unbounded walk.
// Entries are taken statically (k + grid size) or, DYN, in runs of `run`
// consecutive queue entries per warp; MINB is the resident blocks per SM the
// kernel is compiled for (its register bound).  The autotuner picks both.
template <int THREADS, bool WT, bool DYN, int MINB>
__global__ void __launch_bounds__(THREADS, MINB * 128 / THREADS)
    k_wf_shadow(DevScene S, FastView V, WfView W, int bounce, uint32_t run) {
    extern __shared__ uint2 stk[];
    const uint32_t count = W.cnt[C_SH];
    const uint32_t stride = gridDim.x * THREADS;
    uint32_t k = blockIdx.x * THREADS + threadIdx.x;
    Walker<WT> w;
    WalkStacks<> K;
    uint32_t e = 0;
    float lim = 0.0f;  // the sample's cut-off |lp - so| - 0.001; the ray itself lives in the walker (w.o, w.d)
    int step = 0;
    bool active = !DYN && k < count;
    bool need = DYN, exhausted = false;
    uint32_t cbase = 0, cend = 0;
    // Starts sample k of the queue.
    auto begin = [&]() {
        e = W.sq[k];
        const float4 o4 = W.sh.o[e], d4 = W.sh.d[e], l4 = W.sh.lp[e];
        const f3 so = mk(o4.x, o4.y, o4.z);
        step = 0;
        lim = AE_SUB(distance(mk(l4.x, l4.y, l4.z), so), 0.001f);
        w.start(V, so, mk(d4.x, d4.y, d4.z), 0.001f, d4.w, lim);
    };
    if (active) begin();
    uint32_t iter = 0;
    for (;;) {
        if (DYN && run_take(&W.cnt[C_SHTILE + bounce], count, run, need, k, cbase, cend, exhausted)) {
            active = true;
            begin();
        }
        const uint32_t am = __ballot_sync(0xffffffffu, active);
        if (!am) break;
        // Only the warp's largest phase group steps (warp_pick_group).
        const uint32_t pick = warp_pick_group(active ? w.group() : 0u, active, am, iter);
        if (!active || w.group() != pick || !w.step(S, V, K, stk, threadIdx.x, THREADS)) continue;
        const Best &b = w.best;
        int verdict = 0;  // 0 unoccluded, 1 occluded, 2 through glass
        if (b.object != AE_MISS && b.t < lim) {
            const uint32_t mt = load_head(S.objects + b.object).material;
            verdict = mt == AE_MAT_DIFFUSE_LIGHT ? 0 : (mt != AE_MAT_DIELECTRIC ? 1 : 2);
        }
        if (verdict == 2) {
            // Through the glass: the reference's re-origin, from the walker's
            // copy of the ray; the light point is read again.
            const f3 so = (w.o + w.d * b.t) + w.d * 0.001f;
            if (++step < 4) {
                const float4 l4 = W.sh.lp[e];
                lim = AE_SUB(distance(mk(l4.x, l4.y, l4.z), so), 0.001f);
                w.start(V, so, w.d, 0.001f, w.time, lim);
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

// Connect: NEE in light order, clamped, onto the path radiance.
__global__ void __launch_bounds__(256) k_wf_connect(WfView W, int bounce) {
    const WfParams &P = *W.P;
    const int q = bounce & 1;
    const uint32_t count = W.cnt[q];
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
        const uint32_t pid = W.qpid[q][k];
        if (!W.nee[pid]) continue;
        W.nee[pid] = 0;
        const f3 dl = nee_total(W.sh, size_t(pid) * P.n_lights, P.n_lights);
        const float4 t4 = W.pend[pid], a4 = W.acc[pid];
        const f3 acc = mk(a4.x, a4.y, a4.z) + mk(t4.x, t4.y, t4.z) * dl;
        W.acc[pid] = make_float4(acc.x, acc.y, acc.z, 0.0f);
    }
}

// The shadow queue of a bounce starts empty; the next ray queue too.
__global__ void k_wf_reset(WfView W, int bounce) {
    W.cnt[(bounce & 1) ^ 1] = 0;
    W.cnt[C_SH] = 0;
}

// Finish: this sample's path radiance into the pixel's sum; at the last
// sample, the frame colour, the running accumulation and the display
// (hybrid:1383-1403).
__global__ void __launch_bounds__(256) k_wf_finish(WfView W) {
    const WfParams &P = *W.P;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < P.n_paths; p += gridDim.x * blockDim.x) {
        const float4 a = W.acc[p], c0 = W.col[p];
        const f3 col = mk(c0.x, c0.y, c0.z) + mk(a.x, a.y, a.z);
        W.col[p] = make_float4(col.x, col.y, col.z, 0.0f);
        if (P.sample + 1 < P.spp) continue;
        const f3 color = col / AE_U2F(P.spp);
        if (W.frame) W.frame[p] = make_float4(color.x, color.y, color.z, 1.0f);
        f3 accum;
        if (P.kahan) {
            // Compensated (Kahan) sum of the frame colours, divided by the
            // frame count: the precision form's accumulation.
            f3 sum, comp;
            if (P.F.batch == 0) {
                sum = color;
                comp = splat(0.0f);
            } else {
                const float4 s4 = W.ksum[p], c4 = W.kcomp[p];
                const f3 y = color - mk(c4.x, c4.y, c4.z);
                const f3 prev = mk(s4.x, s4.y, s4.z);
                sum = prev + y;
                comp = (sum - prev) - y;
            }
            W.ksum[p] = make_float4(sum.x, sum.y, sum.z, 0.0f);
            W.kcomp[p] = make_float4(comp.x, comp.y, comp.z, 0.0f);
            accum = sum / AE_U2F(P.F.batch + 1);
        } else if (P.F.batch == 0) {
            accum = color;
        } else {
            const float4 prev = W.accum[p];
            accum = lerp(mk(prev.x, prev.y, prev.z), color, AE_DIV(1.0f, AE_U2F(P.F.batch + 1)));
        }
        W.accum[p] = make_float4(accum.x, accum.y, accum.z, 1.0f);
        W.display[p] = display_texel(accum, P.F.exposure);
    }
}

// ---------------------------------------------------------------------------
// Host
// ---------------------------------------------------------------------------
typedef void (*ExtendFn)(DevScene, FastView, WfView, int);
struct ExtendCfg {
    int threads, stack;
    ExtendFn fn;
};
// [0]: the reference triangle test; [1]: the watertight test (precision form).
static const ExtendCfg kExtendCfgs[2][9] = {
    {{64, 16, k_wf_extend<64, 16, false>}, {64, 24, k_wf_extend<64, 24, false>}, {64, 32, k_wf_extend<64, 32, false>},
     {128, 16, k_wf_extend<128, 16, false>}, {128, 24, k_wf_extend<128, 24, false>},
     {128, 32, k_wf_extend<128, 32, false>}, {256, 16, k_wf_extend<256, 16, false>},
     {256, 24, k_wf_extend<256, 24, false>}, {256, 32, k_wf_extend<256, 32, false>}},
    {{64, 16, k_wf_extend<64, 16, true>}, {64, 24, k_wf_extend<64, 24, true>}, {64, 32, k_wf_extend<64, 32, true>},
     {128, 16, k_wf_extend<128, 16, true>}, {128, 24, k_wf_extend<128, 24, true>},
     {128, 32, k_wf_extend<128, 32, true>}, {256, 16, k_wf_extend<256, 16, true>},
     {256, 24, k_wf_extend<256, 24, true>}, {256, 32, k_wf_extend<256, 32, true>}},
};

static size_t extend_smem(int threads, int stack) {
    return size_t(threads) * sizeof(ae_ray) + size_t(threads) * stack * sizeof(uint2);
}

static int extend_grid(Ctx *c, const ExtendCfg &e) {
    int per_sm = 0;
    cudaFuncSetAttribute(reinterpret_cast<const void *>(e.fn), cudaFuncAttributeMaxDynamicSharedMemorySize,
                         int(extend_smem(e.threads, e.stack)));
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, reinterpret_cast<const void *>(e.fn), e.threads,
                                                  extend_smem(e.threads, e.stack));
    return std::max(1, per_sm) * c->wave->sms;
}

static WfView view_of(Ctx *c) {
    Wavefront &Wf = *c->wave;
    WfView W;
    for (int k = 0; k < 2; k++) { W.qray[k] = Wf.qray[k].ptr; W.qpid[k] = Wf.qpid[k].ptr; }
    W.qhit = Wf.qhit.ptr;
    W.thr = Wf.thr.ptr; W.acc = Wf.acc.ptr; W.col = Wf.col.ptr; W.pend = Wf.pend.ptr;
    W.seed = Wf.seed.ptr;
    W.nee = Wf.nee.ptr;
    W.sh = ShadowStore{Wf.sh_o.ptr, Wf.sh_d.ptr, Wf.sh_lp.ptr, Wf.sh_c.ptr, Wf.sh_valid.ptr, Wf.sh_occ.ptr};
    W.sq = Wf.sq.ptr;
    W.cnt = Wf.cnt.ptr;
    W.P = Wf.params.ptr;
    W.accum = c->accum.ptr;
    W.frame = c->frame.ptr;
    W.display = c->display.ptr;
    W.ksum = Wf.ksum.ptr;
    W.kcomp = Wf.kcomp.ptr;
    W.prec = PrecView{c->fast->shade16.ptr};
    return W;
}

static int ensure_wavefront(Ctx *c) {
    int rc = prepare_fast(c);
    if (rc) return rc;
    if (!c->wave) c->wave = new (std::nothrow) Wavefront();
    if (!c->wave) return c->fail(AE_ERR_OOM, "wavefront state");
    Wavefront &Wf = *c->wave;
    const uint32_t n = c->settings.width * c->settings.height;
    const uint32_t nl = c->n_lights;
    if (nl > uint32_t(kMaxLights)) return c->fail(AE_ERR_LAYOUT, "wavefront NEE supports at most %d lights", kMaxLights);
    if (c->config.depth > uint32_t(kMaxBounce)) return c->fail(AE_ERR_INVALID, "depth above %d", kMaxBounce);
    if (Wf.cap < n || Wf.n_lights < std::max(nl, 1u)) {
        const size_t ne = size_t(n) * std::max(nl, 1u);
        if (Wf.qray[0].reserve(n) || Wf.qray[1].reserve(n) || Wf.qpid[0].reserve(n) || Wf.qpid[1].reserve(n) ||
            Wf.qhit.reserve(n) || Wf.thr.reserve(n) || Wf.acc.reserve(n) || Wf.col.reserve(n) || Wf.pend.reserve(n) ||
            Wf.seed.reserve(n) || Wf.nee.reserve(n) || Wf.sh_o.reserve(ne) || Wf.sh_d.reserve(ne) ||
            Wf.sh_lp.reserve(ne) || Wf.sh_c.reserve(ne) || Wf.sh_valid.reserve(ne) || Wf.sh_occ.reserve(ne) ||
            Wf.sq.reserve(ne) || Wf.cnt.reserve(C_COUNT) || Wf.params.reserve(1))
            return c->fail(AE_ERR_OOM, "wavefront queues (%u paths x %u lights)", n, nl);
        Wf.cap = n;
        Wf.n_lights = std::max(nl, 1u);
        if (Wf.graph) { cudaGraphExecDestroy(Wf.graph); Wf.graph = nullptr; }
        cudaMemsetAsync(Wf.cnt.ptr, 0, C_COUNT * sizeof(uint32_t), c->stream);
    }
    if (!Wf.host_params) {
        if (cudaMallocHost(&Wf.host_params, sizeof(WfParams)) != cudaSuccess)
            return c->fail(AE_ERR_OOM, "pinned frame parameters");
    }
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&Wf.sms, cudaDevAttrMultiProcessorCount, dev);
    return AE_OK;
}

// Records one sample's stages onto `st` (graph capture or direct).
struct Grids {
    int grid256, egrid, shgrid, wgrid;
    size_t esmem, shsmem;
};

// The walker stages' kernels by [precision form][runs][register bound]:
// compiled for 6 or 7 resident 128-thread blocks per SM (kWalkMinBlocks).
using ShadowFn = void (*)(DevScene, FastView, WfView, int, uint32_t);
using ExtendWalkFn = void (*)(DevScene, FastView, WfView, int, uint32_t);
constexpr int kWalkMinBlocks[2] = {6, 7};
static const ShadowFn kShadowFns[2][2][2] = {
    {{k_wf_shadow<128, false, false, 6>, k_wf_shadow<128, false, false, 7>},
     {k_wf_shadow<128, false, true, 6>, k_wf_shadow<128, false, true, 7>}},
    {{k_wf_shadow<128, true, false, 6>, k_wf_shadow<128, true, false, 7>},
     {k_wf_shadow<128, true, true, 6>, k_wf_shadow<128, true, true, 7>}}};
static const ExtendWalkFn kExtendWalkFns[2][2][2] = {
    {{k_wf_extend_walk<false, false, 6>, k_wf_extend_walk<false, false, 7>},
     {k_wf_extend_walk<false, true, 6>, k_wf_extend_walk<false, true, 7>}},
    {{k_wf_extend_walk<true, false, 6>, k_wf_extend_walk<true, false, 7>},
     {k_wf_extend_walk<true, true, 6>, k_wf_extend_walk<true, true, 7>}}};
static const void *shadow_fn(bool prec, bool dyn, int mb) {
    return reinterpret_cast<const void *>(kShadowFns[prec][dyn][mb]);
}
static const void *extend_walk_fn(bool prec, bool dyn, int mb) {
    return reinterpret_cast<const void *>(kExtendWalkFns[prec][dyn][mb]);
}
// Persistent grid of a walker kernel: its resident blocks per SM x the SMs
// (an occupancy query: never while a stream is being captured).
static int walk_grid(Ctx *c, const void *fn) {
    const size_t smem = size_t(kSharedStack) * 128 * sizeof(uint2);
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 128, smem);
    return std::max(1, per_sm) * c->wave->sms;
}

// Launch shapes, fixed before capture (no attribute or occupancy query runs
// while a stream is being captured).
static Grids grids_for(Ctx *c, int cfg_index, bool prec) {
    Wavefront &Wf = *c->wave;
    Grids g;
    g.grid256 = Wf.sms * 8;
    const ExtendCfg &e = kExtendCfgs[prec][cfg_index];
    g.egrid = extend_grid(c, e);
    g.esmem = extend_smem(e.threads, e.stack);
    g.shsmem = size_t(kSharedStack) * 128 * sizeof(uint2);
    g.shgrid = walk_grid(c, shadow_fn(prec, Wf.shadow_run[prec] != 0, Wf.shadow_mb[prec]));
    g.wgrid = walk_grid(c, extend_walk_fn(prec, Wf.walk_run[prec] != 0, Wf.walk_mb[prec]));
    return g;
}

// The walker stages with a queue assignment (run 0: static, else runs of
// `run` entries per warp) and a register bound (kWalkMinBlocks[mb] resident
// blocks per SM), launched on `grid` blocks.
static void launch_extend_walk(bool prec, uint32_t run, int mb, int grid, const Grids &G, cudaStream_t st,
                               const DevScene &S, const FastView &V, const WfView &W, int b) {
    const ExtendWalkFn fn = kExtendWalkFns[prec][run != 0][mb];
    fn<<<grid, 128, G.shsmem, st>>>(S, V, W, b, run);
}

static void launch_shadow(bool prec, uint32_t run, int mb, int grid, const Grids &G, cudaStream_t st,
                          const DevScene &S, const FastView &V, const WfView &W, int b) {
    const ShadowFn fn = kShadowFns[prec][run != 0][mb];
    fn<<<grid, 128, G.shsmem, st>>>(S, V, W, b, run);
}

static int record_sample(Ctx *c, cudaStream_t st, int cfg_index, const Grids &G, bool prec) {
    const WfView W = view_of(c);
    const DevScene S = c->scene();
    FastScene &F = *c->fast;
    const FastView V = fast_view(F);
    const Wavefront &Wf = *c->wave;
    const ExtendCfg &e = kExtendCfgs[prec][cfg_index];
    const int grid256 = G.grid256, egrid = G.egrid;
    const size_t esmem = G.esmem;
    k_wf_generate<<<grid256, 256, 0, st>>>(W);
    for (uint32_t b = 0; b < c->config.depth; b++) {
        k_wf_reset<<<1, 1, 0, st>>>(W, int(b));
        // Camera rays are coherent: the autotuned tile-staged extend.  Bounce
        // queues are not: the step-wise walk keeps warps full (measured 6 %
        // more paths/s on the 10M-triangle scene).
        if (b == 0) e.fn<<<egrid, e.threads, esmem, st>>>(S, V, W, int(b));
        else launch_extend_walk(prec, Wf.walk_run[prec], Wf.walk_mb[prec], G.wgrid, G, st, S, V, W, int(b));
        if (prec) k_wf_shade<true><<<grid256, 256, 0, st>>>(S, V, W, int(b));
        else k_wf_shade<false><<<grid256, 256, 0, st>>>(S, V, W, int(b));
        launch_shadow(prec, Wf.shadow_run[prec], Wf.shadow_mb[prec], G.shgrid, G, st, S, V, W, int(b));
        k_wf_connect<<<grid256, 256, 0, st>>>(W, int(b));
    }
    k_wf_finish<<<grid256, 256, 0, st>>>(W);
    return c->cuda(cudaGetLastError(), "wavefront launch");
}

static uint64_t launches_per_sample(const Ctx *c) { return 2 + 5ull * c->config.depth; }

// Times every extend configuration on this scene's first bounce and keeps
// the fastest.
static int autotune(Ctx *c) {
    Wavefront &Wf = *c->wave;
    const WfView W = view_of(c);
    const DevScene S = c->scene();
    FastScene &F = *c->fast;
    const FastView V = fast_view(F);
    int best = 4;
    float best_ms = 1e30f;
    for (int k = 0; k < 9; k++) {
        const ExtendCfg &e = kExtendCfgs[0][k];
        const int egrid = extend_grid(c, e);
        float total = 0.0f;
        for (int rep = 0; rep < 2; rep++) {
            k_wf_generate<<<Wf.sms * 8, 256, 0, c->stream>>>(W);
            k_wf_reset<<<1, 1, 0, c->stream>>>(W, 0);
            cudaEventRecord(c->ev0, c->stream);
            e.fn<<<egrid, e.threads, extend_smem(e.threads, e.stack), c->stream>>>(S, V, W, 0);
            cudaEventRecord(c->ev1, c->stream);
            int rc = c->cuda(cudaEventSynchronize(c->ev1), "autotune");
            if (rc) return rc;
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, c->ev0, c->ev1);
            if (rep == 1) total = ms;
            c->launches += 3;
        }
        Wf.tune_ms[k] = total;
        if (total < best_ms) { best_ms = total; best = k; }
    }
    Wf.ext_threads = kExtendCfgs[0][best].threads;
    Wf.ext_stack = kExtendCfgs[0][best].stack;
    Wf.tuned = true;
    return c->cuda(cudaGetLastError(), "autotune");
}

static int best_cfg_index(const Wavefront &Wf) {
    for (int k = 0; k < 9; k++)
        if (kExtendCfgs[0][k].threads == Wf.ext_threads && kExtendCfgs[0][k].stack == Wf.ext_stack) return k;
    return 4;
}

// Queue assignments the walker stages are timed with: static, then runs of
// 32, 64 and 256 queue entries per warp.
static const uint32_t kRunCfgs[4] = {0, 32, 64, 256};

// Times the shadow stage on sample 0's first shadow queue and the step-wise
// extend on its second ray queue under every assignment of kRunCfgs, each
// compiled for 6 and for 7 resident blocks per SM, and keeps the fastest of
// each for this form.  Runs before the first frame of
// the form; the frame's generate stage then starts every path afresh.
static int autotune_walkers(Ctx *c, bool prec) {
    Wavefront &Wf = *c->wave;
    const WfView W = view_of(c);
    const DevScene S = c->scene();
    const FastView V = fast_view(*c->fast);
    const int ci = best_cfg_index(Wf);
    const Grids G = grids_for(c, ci, prec);
    const ExtendCfg &e = kExtendCfgs[prec][ci];
    cudaStream_t st = c->stream;
    k_wf_generate<<<G.grid256, 256, 0, st>>>(W);
    k_wf_reset<<<1, 1, 0, st>>>(W, 0);
    e.fn<<<G.egrid, e.threads, G.esmem, st>>>(S, V, W, 0);
    if (prec) k_wf_shade<true><<<G.grid256, 256, 0, st>>>(S, V, W, 0);
    else k_wf_shade<false><<<G.grid256, 256, 0, st>>>(S, V, W, 0);
    c->launches += 4;
    int rc = c->cuda(cudaGetLastError(), "autotune");
    if (rc) return rc;
    for (int stage = 0; stage < 2; stage++) {
        uint32_t *counter = Wf.cnt.ptr + (stage == 0 ? C_SHTILE + 0 : C_TILE + 1);
        int best = 0;
        for (int k = 0; k < 8; k++) {
            const uint32_t run = kRunCfgs[k & 3];
            const int mb = k >> 2;
            const int grid = walk_grid(c, stage == 0 ? shadow_fn(prec, run != 0, mb) : extend_walk_fn(prec, run != 0, mb));
            float ms = 0.0f;
            for (int rep = 0; rep < 2; rep++) {
                if ((rc = c->cuda(cudaMemsetAsync(counter, 0, sizeof(uint32_t), st), "autotune"))) return rc;
                cudaEventRecord(c->ev0, st);
                if (stage == 0) launch_shadow(prec, run, mb, grid, G, st, S, V, W, 0);
                else launch_extend_walk(prec, run, mb, grid, G, st, S, V, W, 1);
                cudaEventRecord(c->ev1, st);
                if ((rc = c->cuda(cudaEventSynchronize(c->ev1), "autotune"))) return rc;
                if (rep == 1) cudaEventElapsedTime(&ms, c->ev0, c->ev1);
                c->launches++;
            }
            Wf.walk_tune_ms[prec][stage * 8 + k] = ms;
            if (ms < Wf.walk_tune_ms[prec][stage * 8 + best]) best = k;
        }
        (stage == 0 ? Wf.shadow_run : Wf.walk_run)[prec] = kRunCfgs[best & 3];
        (stage == 0 ? Wf.shadow_mb : Wf.walk_mb)[prec] = best >> 2;
    }
    Wf.walk_tuned[prec] = true;
    return c->cuda(cudaGetLastError(), "autotune");
}

int render_wavefront(Ctx *c, bool prec) {
    int rc = ensure_wavefront(c);
    if (rc) return rc;
    Wavefront &Wf = *c->wave;
    const uint32_t n_px = c->settings.width * c->settings.height;
    if (prec) {
        if ((rc = prepare_precision(c))) return rc;
        if (Wf.ksum.reserve(n_px) || Wf.kcomp.reserve(n_px))
            return c->fail(AE_ERR_OOM, "compensated accumulation (%u pixels)", n_px);
    }
    WfParams hp;
    std::memset(&hp, 0, sizeof(hp));
    hp.F = make_frame_params(c->config);
    hp.n_paths = n_px;
    hp.spp = hp.F.spp;
    hp.n_lights = c->n_lights;
    hp.kahan = prec ? 1u : 0u;
    if (hp.F.display_only) {
        // Re-grade only: the compute-only kernel's display-only branch.
        if ((rc = c->timed_begin())) return rc;
        if ((rc = c->cuda(launch_render_plain(c->scene(), hp.F, c->accum.ptr, c->display.ptr, c->frame.ptr, c->stream),
                          "display only")))
            return rc;
        return c->timed_end();
    }
    if (!Wf.tuned || !Wf.walk_tuned[prec]) {
        if ((rc = c->cuda(cudaStreamSynchronize(c->stream), "params"))) return rc;
        *Wf.host_params = hp;
        if ((rc = c->cuda(cudaMemcpyAsync(Wf.params.ptr, Wf.host_params, sizeof(WfParams), cudaMemcpyHostToDevice,
                                          c->stream), "params")))
            return rc;
        if (!Wf.tuned && (rc = autotune(c))) return rc;
        if (!Wf.walk_tuned[prec] && (rc = autotune_walkers(c, prec))) return rc;
    }
    // One graph per (scene upload, frame shape); frame parameters travel
    // through device memory so the graph is replayed unchanged.
    const uint64_t key = (c->scene_version << 21) ^ (uint64_t(prec) << 20) ^ (uint64_t(c->config.depth) << 8) ^
                         hp.n_lights;
    if (!Wf.graph || Wf.graph_key != key) {
        if (Wf.graph) { cudaGraphExecDestroy(Wf.graph); Wf.graph = nullptr; }
        cudaGraph_t g;
        const int ci = best_cfg_index(Wf);
        const Grids G = grids_for(c, ci, prec);
        if ((rc = c->cuda(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal), "capture"))) return rc;
        rc = record_sample(c, c->stream, ci, G, prec);
        cudaError_t ce = cudaStreamEndCapture(c->stream, &g);
        if (rc) return rc;
        if ((rc = c->cuda(ce, "end capture"))) return rc;
        ce = cudaGraphInstantiate(&Wf.graph, g, 0);
        cudaGraphDestroy(g);
        if ((rc = c->cuda(ce, "graph instantiate"))) return rc;
        Wf.graph_key = key;
    }
    // The error word counts this frame only; the fault word carries an
    // injected failure (ae_debug_inject) into the extend kernels.
    if ((rc = c->cuda(cudaMemsetAsync(Wf.cnt.ptr + C_ERR, 0, sizeof(uint32_t), c->stream), "reset error word")) ||
        (rc = c->cuda(cudaMemsetAsync(Wf.cnt.ptr + C_FAULT, c->fault_tile_wait ? 0xff : 0, sizeof(uint32_t),
                                      c->stream), "fault word")))
        return rc;
    if ((rc = c->timed_begin())) return rc;
    for (uint32_t s = 0; s < hp.spp; s++) {
        hp.sample = s;
        // The pinned block is rewritten only after the previous copy finished.
        if ((rc = c->cuda(cudaStreamSynchronize(c->stream), "params"))) return rc;
        *Wf.host_params = hp;
        if ((rc = c->cuda(cudaMemcpyAsync(Wf.params.ptr, Wf.host_params, sizeof(WfParams), cudaMemcpyHostToDevice,
                                          c->stream), "params")))
            return rc;
        if ((rc = c->cuda(cudaGraphLaunch(Wf.graph, c->stream), "graph launch"))) return rc;
        c->launches += launches_per_sample(c);
    }
    c->launches--;  // timed_end counts one
    if ((rc = c->timed_end())) return rc;
    // A bounded device-side wait that gave up makes the frame incomplete.
    uint32_t e = 0;
    if ((rc = c->cuda(cudaMemcpyAsync(&e, Wf.cnt.ptr + C_ERR, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream),
                      "read error word")) ||
        (rc = c->cuda(cudaStreamSynchronize(c->stream), "frame")))
        return rc;
    if (e) return c->fail(AE_ERR_TIMEOUT, "a bounded queue-tile wait gave up on the device; the frame is incomplete");
    return AE_OK;
}

}  // namespace ae

using namespace ae;

extern "C" int ae_wavefront_walk_info(ae_ctx *ctx, int precision, uint32_t *shadow_run, uint32_t *extend_run,
                                      uint32_t *shadow_blocks, uint32_t *extend_blocks, float *tune_ms16) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return AE_ERR_INVALID;
    const int f = precision ? 1 : 0;
    if (!c->wave || !c->wave->walk_tuned[f]) return c->fail(AE_ERR_STATE, "no wavefront frame of this form yet");
    const Wavefront &Wf = *c->wave;
    if (shadow_run) *shadow_run = Wf.shadow_run[f];
    if (extend_run) *extend_run = Wf.walk_run[f];
    if (shadow_blocks) *shadow_blocks = uint32_t(kWalkMinBlocks[Wf.shadow_mb[f]]);
    if (extend_blocks) *extend_blocks = uint32_t(kWalkMinBlocks[Wf.walk_mb[f]]);
    if (tune_ms16) std::memcpy(tune_ms16, Wf.walk_tune_ms[f], sizeof(Wf.walk_tune_ms[f]));
    return AE_OK;
}

extern "C" int ae_wavefront_set_walk_runs(ae_ctx *ctx, int precision, uint32_t shadow_run, uint32_t extend_run,
                                          uint32_t shadow_blocks, uint32_t extend_blocks) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return AE_ERR_INVALID;
    if (shadow_run > (1u << 20) || extend_run > (1u << 20))
        return c->fail(AE_ERR_INVALID, "run lengths above 2^20 (got %u, %u)", shadow_run, extend_run);
    auto mb_of = [](uint32_t blocks) { return blocks == 0 || blocks == 7 ? 1 : blocks == 6 ? 0 : -1; };
    const int smb = mb_of(shadow_blocks), emb = mb_of(extend_blocks);
    if (smb < 0 || emb < 0)
        return c->fail(AE_ERR_INVALID, "resident blocks per SM must be 6 or 7 (got %u, %u)", shadow_blocks,
                       extend_blocks);
    if (!c->wave) c->wave = new (std::nothrow) Wavefront();
    if (!c->wave) return c->fail(AE_ERR_OOM, "wavefront state");
    Wavefront &Wf = *c->wave;
    const int f = precision ? 1 : 0;
    Wf.shadow_run[f] = shadow_run;
    Wf.walk_run[f] = extend_run;
    Wf.shadow_mb[f] = smb;
    Wf.walk_mb[f] = emb;
    Wf.walk_tuned[f] = true;
    if (Wf.graph) {
        cudaGraphExecDestroy(Wf.graph);
        Wf.graph = nullptr;
    }
    return AE_OK;
}

// Wavefront statistics: the autotuned extend configuration and the error flag.
extern "C" int ae_wavefront_info(ae_ctx *ctx, int32_t *threads, int32_t *stack, float *tune_ms9, uint32_t *errors) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return AE_ERR_INVALID;
    if (!c->wave) return c->fail(AE_ERR_STATE, "no wavefront frame yet");
    if (threads) *threads = c->wave->ext_threads;
    if (stack) *stack = c->wave->ext_stack;
    if (tune_ms9) std::memcpy(tune_ms9, c->wave->tune_ms, sizeof(c->wave->tune_ms));
    if (errors) {
        uint32_t e = 0;
        int rc = c->cuda(cudaMemcpyAsync(&e, c->wave->cnt.ptr + C_ERR, 4, cudaMemcpyDeviceToHost, c->stream), "copy");
        if (!rc) rc = c->cuda(cudaStreamSynchronize(c->stream), "sync");
        if (rc) return rc;
        *errors = e;
    }
    return AE_OK;
}
