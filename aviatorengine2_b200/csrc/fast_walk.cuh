// fast_walk.cuh - the optimised closest hit (closest_fast, fast_trace.cuh)
// re-expressed as a state machine that advances one step per call: one node
// of the instance-level tree, one object entry, or one BLAS node (a leaf's
// triangles included).
//
// Why: the nested form runs an instance-tree loop and a BLAS loop inside one
// another, and the lanes of a warp wait at the end of each inner loop for the
// slowest lane.  On incoherent rays (bounces, shadow samples)
// only a few lanes were active per instruction.  A kernel built on Walker
// keeps every lane stepping its own ray and lets a lane that finishes start
// its next ray at once, so warps stay full.
//
// Each ray takes exactly the steps of closest_fast in the same order with the
// same arithmetic (same ToLocal, child order, stack discipline, ranking of
// equal distances), so the Best it returns is bit-identical.
#pragma once
#include "fast_trace.cuh"

namespace ae {

enum : uint32_t { kWalkTlas = 0, kWalkObject = 1, kWalkBlas = 2, kWalkDone = 3 };

// Minimum resident 128-thread blocks per SM asked of the compiler for every
// kernel built on Walker (extend and shadow, wavefront and serving): caps them
// at 72 registers.  Measured at 1920x1080 on the 10M-triangle wavefront scene:
// 7 blocks (28-108 bytes of spills) beat both the unbounded build (79-87
// registers, 6 blocks) and 8 blocks (64 registers, 110-280 bytes of spills) -
// wavefront frame 177 ms against 192 ms and 179 ms.
constexpr int kWalkBlocksPerSm = 7;

// The walk's per-thread local stacks: the instance-tree stack and the BLAS
// entries beyond the shared-memory part.  Kept out of Walker so its scalar
// state can live in registers.
template <int SS = kSharedStack>
struct WalkStacks {
    uint32_t tstack[kTlas4Stack];
    float tdist[kTlas4Stack];
    uint2 spill[kFastStack - SS];
};

template <bool WT, int SS = kSharedStack>
struct Walker {
    // ray
    f3 o, d, tinv;
    float tn, time;
    Best best;
    uint32_t phase;
    // instance tree: the current node, or the leaf (object) being entered
    uint32_t tcur;
    int tsp;
    // current mesh instance
    f3 lo, ld, linv;
    WtRay W;
    uint32_t tri_base, cur, slot;
    uint64_t orank;
    int bsp;

    // tmax below kFarStart starts the walk as if a hit at tmax were already
    // found: every hit nearer than tmax is still found, with the same tie
    // ranking, and nothing at or beyond it is reported as nearer.
    AE_DEV void start(const FastView &V, f3 o_, f3 d_, float tn_, float time_, float tmax = kFarStart) {
        o = o_;
        d = d_;
        tn = tn_;
        time = time_;
        best.t = tmax; best.alpha = 0.0f; best.beta = 0.0f;
        best.object = AE_MISS; best.prim = AE_MISS; best.orank = 0; best.lrank = 0;
        tsp = 0;
        tinv = mk(slab_inv(d.x), slab_inv(d.y), slab_inv(d.z));
        tcur = V.troot;
        phase = (tcur & kLeafBit) ? (leaf_count(tcur) ? kWalkObject : kWalkDone) : kWalkTlas;
    }

    // Next instance-tree stack entry no farther than the best hit, or done.
    AE_DEV void tlas_pop(const WalkStacks<SS> &K) {
        while (tsp > 0) {
            tsp--;
            if (K.tdist[tsp] <= best.t) {
                tcur = K.tstack[tsp];
                phase = (tcur & kLeafBit) ? kWalkObject : kWalkTlas;
                return;
            }
        }
        phase = kWalkDone;
    }

    // Next BLAS stack entry no farther than the best hit, or back to the
    // instance tree.
    AE_DEV void blas_pop(const WalkStacks<SS> &K, const uint2 *stk, int tid, int nt) {
        while (bsp > 0) {
            bsp--;
            const uint2 e = bsp < SS ? stk[bsp * nt + tid] : K.spill[bsp - SS];
            if (__uint_as_float(e.y) <= best.t) {
                cur = e.x;
                return;
            }
        }
        tlas_pop(K);
    }

    // The walk's phase group for warp-level step scheduling: 0 interior node
    // of either tree (the instance-level tree and the BLAS share the 4-wide
    // node format and its child test), 1 object entry, 2 BLAS leaf.
    AE_DEV uint32_t group() const {
        return phase == kWalkObject ? 1u : ((phase == kWalkBlas && (cur & kLeafBit)) ? 2u : 0u);
    }

    // One step; returns true once the ray is finished (best is final).
    AE_DEV bool step(const DevScene &S, const FastView &V, WalkStacks<SS> &K, uint2 *stk, int tid, int nt) {
        if (phase == kWalkBlas && (cur & kLeafBit)) {
            const uint32_t first = leaf_first(cur), cnt = leaf_count(cur);
            const float4 *tris = V.tris + size_t(tri_base) * 3;
            for (uint32_t k = 0; k < cnt; k++) {
                const uint32_t s = first + k;
                const float4 *r = tris + size_t(s) * 3;
                const float4 r0 = __ldg(r), r1 = __ldg(r + 1), r2 = __ldg(r + 2);
                float t, a, b;
                const bool h = WT ? tri_test_wt(lo, W, tn, best.t, r0, r1, r2, t, a, b)
                                  : tri_test_ref(lo, ld, tn, best.t, r0, r1, r2, t, a, b);
                if (h && takes(best, t, orank, ~first, s)) {
                    best.t = t; best.alpha = a; best.beta = b;
                    best.object = slot; best.prim = s;
                    best.orank = orank; best.lrank = ~first;
                }
            }
            blas_pop(K, stk, tid, nt);
            return phase == kWalkDone;
        }
        if (phase == kWalkObject) {
            slot = leaf_first(tcur);
            const uint4 m = __ldg(V.meta + slot);
            orank = object_rank(m, slot);
            const uint32_t shape = m.x & 0xff;
            if (shape == AE_SHAPE_MESH) {
                // ToLocal (hybrid:534-543), as trace_mesh.
                const float4 *ip = reinterpret_cast<const float4 *>(V.inst + m.y);
                const float4 a = __ldg(ip), b = __ldg(ip + 1), c = __ldg(ip + 2);
                lo = quat_rotate(-b.x, -b.y, -b.z, b.w, o - mk(a.x, a.y, a.z));
                ld = quat_rotate(-b.x, -b.y, -b.z, b.w, d);
                if (a.w != 0.0f && a.w != 1.0f) {
                    const float inv = AE_DIV(1.0f, a.w);
                    lo = lo * inv;
                    ld = ld * inv;
                }
                linv = mk(slab_inv(ld.x), slab_inv(ld.y), slab_inv(ld.z));
                if (WT) W = wt_setup(ld);
                tri_base = __float_as_uint(c.y);
                cur = __float_as_uint(c.x);
                bsp = 0;
                phase = kWalkBlas;
                return false;
            }
            DHit h;
            const ae_object *obj = S.objects + slot;
            bool hit;
            if (shape == AE_SHAPE_SPHERE) hit = hit_sphere_ref(obj, o, d, time, tn, best.t, h);
            else if (shape == AE_SHAPE_QUAD) hit = hit_planar_ref(obj, false, o, d, tn, best.t, h);
            else if (shape == AE_SHAPE_TRIANGLE) hit = hit_planar_ref(obj, true, o, d, tn, best.t, h);
            else hit = hit_box_ref(obj, o, d, tn, best.t, h);
            if (hit && takes(best, h.t, orank, 0u, 0u)) {
                best.t = h.t; best.alpha = h.alpha; best.beta = h.beta;
                best.object = slot; best.prim = AE_MISS; best.orank = orank; best.lrank = 0;
            }
            tlas_pop(K);
            return phase == kWalkDone;
        }
        if (phase == kWalkDone) return true;
        // An interior node of the instance-level tree (world ray) or of the
        // current mesh's BLAS (local ray): one code path for both, so the
        // lanes of a warp at either level step together.
        const bool top = phase == kWalkTlas;
        float tm[4];
        uint32_t ch[4];
        child_hits(top ? V.tnodes + tcur : V.nodes + cur, top ? o : lo, top ? tinv : linv, tn, best.t, tm, ch);
        const int nh = sort_hits(tm, ch);
        if (nh > 0) {
            if (top) {
                for (int k = nh - 1; k >= 1; k--) {
                    if (tsp < kTlas4Stack) {
                        K.tstack[tsp] = ch[k];
                        K.tdist[tsp] = tm[k];
                        tsp++;
                    }
                }
                tcur = ch[0];
                phase = (tcur & kLeafBit) ? kWalkObject : kWalkTlas;
            } else {
                for (int k = nh - 1; k >= 1; k--) {
                    if (bsp < SS) stk[bsp * nt + tid] = make_uint2(ch[k], __float_as_uint(tm[k]));
                    else if (bsp < kFastStack) K.spill[bsp - SS] = make_uint2(ch[k], __float_as_uint(tm[k]));
                    bsp = bsp < kFastStack ? bsp + 1 : bsp;
                }
                cur = ch[0];
            }
            return false;
        }
        if (top) tlas_pop(K);
        else blas_pop(K, stk, tid, nt);
        return phase == kWalkDone;
    }
};

// Run assignment for a persistent walker grid: the lanes of a warp that need
// work (need) take the next indices of the warp's current run of `run`
// consecutive queue entries, in lane order, and the warp claims a new run from
// `counter` when its run is used up, so the entries a warp has in flight stay
// neighbours in the queue.  cbase, cend and exhausted are the same in every
// lane.  Returns true in the lanes that got an index (k).  All 32 lanes must
// call this together.
AE_DEV bool run_take(uint32_t *counter, uint32_t n, uint32_t run, bool &need, uint32_t &k, uint32_t &cbase,
                     uint32_t &cend, bool &exhausted) {
    const uint32_t lane = threadIdx.x & 31u, below = (1u << lane) - 1u;
    bool got = false;
    uint32_t m = __ballot_sync(0xffffffffu, need);
    while (m && !exhausted) {
        if (cbase >= cend) {
            uint32_t b = 0;
            if (lane == 0) b = atomicAdd(counter, run);
            b = __shfl_sync(0xffffffffu, b, 0);
            if (b >= n) {
                exhausted = true;
                break;
            }
            cbase = b;
            cend = min(b + run, n);
        }
        const uint32_t take = min(cend - cbase, uint32_t(__popc(m)));
        if (need && uint32_t(__popc(m & below)) < take) {
            k = cbase + uint32_t(__popc(m & below));
            need = false;
            got = true;
        }
        cbase += take;
        m = __ballot_sync(0xffffffffu, need);
    }
    return got;
}

// Which phase group a warp steps this iteration: the largest group among its
// active lanes, so the lanes that step run the same code; every fourth
// iteration the group of the next active lane at or after a rotating
// position, so every lane steps at least once every 128 iterations.  `am` is
// the warp's ballot of `active`; `group` of an inactive lane is ignored.  All
// 32 lanes must call this together.  Scheduling only: each lane's own
// sequence of steps, and so its result, is unchanged.
AE_DEV uint32_t warp_pick_group(uint32_t group, bool active, uint32_t am, uint32_t &iter) {
    uint32_t pick;
    if ((iter & 3u) == 3u) {
        const uint32_t r = (iter >> 2) & 31u;
        const uint32_t rot = (am >> r) | (r ? (am << (32u - r)) : 0u);
        const uint32_t src = (r + uint32_t(__ffs(rot)) - 1u) & 31u;
        pick = __shfl_sync(0xffffffffu, group, int(src));
    } else {
        // Lane counts of groups 0 and 1 by ballot, group 2 by difference;
        // ties go to the lower group.
        const uint32_t c0 = uint32_t(__popc(__ballot_sync(0xffffffffu, active && group == 0u)));
        const uint32_t c1 = uint32_t(__popc(__ballot_sync(0xffffffffu, active && group == 1u)));
        const uint32_t c2 = uint32_t(__popc(am)) - c0 - c1;
        pick = c1 > c0 ? 1u : 0u;
        if (c2 > max(c0, c1)) pick = 2u;
    }
    iter++;
    return pick;
}

}  // namespace ae
