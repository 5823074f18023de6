// bvh_build.cu - the binned-SAH BVH build (BuildBVH, scene/bvh.h:120-295) on
// the GPU.  It produces the host builder's tree node for node and slot for
// slot (host_scene.cpp SahBuilder, itself pinned to the reference).
//
// The reference recursion is sequential, but what it does at a node depends
// only on that node's primitive range as the ancestors' partitions left it.
// The device builds the same tree in two phases:
//
//   * nodes of more than kWarpTask primitives, one tree level per round:
//     blocks of kChunk positions reduce the node box and centroid bounds,
//     bin the 3 x 12 SAH buckets in shared memory and partition;
//   * every node of at most kWarpTask primitives: one warp builds its whole
//     subtree with the reference's pre-order work list, each per-node loop
//     spread over the 32 lanes.
//
// Node indices are the recursion's pre-order; they are assigned at the end
// from the subtree sizes.  Leaf slots are positions in the permuted index
// array, which is the reference's outOrder.
//
// Exactness:
//   * Every float operation is the reference's, with _rn intrinsics (no
//     contraction): the centroid (min + max) * 0.5, the bucket
//     (c - cmin) * (12 / extent) truncated, HalfArea, the costs.
//   * The node box folds with std::min / std::max, which keep the FIRST of
//     equal values.  Equal floats differ in bits only as +0 / -0, so the box
//     reductions carry (value, position) keys and the smallest position among
//     equal values wins.  Centroid bounds and bucket boxes only reach
//     differences, products and comparisons, where +0 and -0 act alike, and
//     reduce by value.
//   * std::partition (libstdc++, the bidirectional form random-access
//     iterators use) scans from the left for an element failing the predicate
//     and from the right for one passing it, swaps them and repeats until the
//     scans meet.  The result: with T passing elements in the range, the k-th
//     failing element of [start, start + T) counted from the left trades
//     places with the k-th passing element of [start + T, end) counted from
//     the right, and every other element stays.  The device finds those ranks
//     with scans and moves the pairs through a stash.
#include <cuda_runtime.h>

#include <cfloat>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/ae_b200.h"
#include "ae_math.h"
#include "devmem.h"

namespace ae {
namespace {

// scene/bvh.h:13, 93, 101 and scene/aabb.h:12
constexpr int kLeafSize = 4;
constexpr int kBins = 12;
constexpr int kMaxDepth = 20;
constexpr float kBoundsMinimum = 0.0001f;
constexpr float kHalfMinimum = kBoundsMinimum * 0.5f;

// Subtrees of at most this many primitives are built by one warp (the
// default; any threshold gives the same tree).  Measured over the BLAS builds
// of a 10M-triangle, 32-mesh scene: 32 -> 86 ms, 64 -> 71 ms, 128 -> 64 ms,
// 256 -> 61 ms, 512 -> 65 ms, 1024 -> 87 ms.  Smaller subtrees give more
// warps to run at once but more tree levels to run as rounds.
constexpr uint32_t kWarpTask = 256;
constexpr int kWarpsPerBlock = 8;
// Positions per block in the level-by-level phase: 256 threads x 8.
constexpr int kThreads = 256;
constexpr int kPer = 8;
constexpr uint32_t kChunk = kThreads * kPer;
// Bucket record: ordered min x,y,z, ordered max x,y,z, count.
constexpr int kBinWords = 7;
constexpr int kBinTable = 3 * kBins * kBinWords;
// Pre-order work list of one warp: at most one pending right child per depth
// plus the current left child.
constexpr int kWarpStack = kMaxDepth + 4;

struct Chunk { uint32_t task, begin, end; };
struct BigTask { uint32_t start, end, depth; };
// A subtree for one warp.  root: the first position of its tree's range
// (leaf slots are relative to it); out: where its tree's nodes start in the
// output array.
struct SmallTask { uint32_t start, end, depth, root, out; };

// Per large task, reset every round.
struct TaskAcc {
    unsigned long long bmin[3], bmax[3];  // (ordered value, position) keys
    uint32_t cmin[3], cmax[3];            // ordered centroid bounds
    uint32_t bins[kBinTable];
};

struct Decision {
    ae_aabb box;       // union of the node's primitive boxes (not yet widened)
    int32_t leaf;      // 1: the node is a leaf
    int32_t axis;      // winning axis, -1 = no plane separates (median split)
    int32_t split;     // first bucket on the right
    float cmin, scale; // bucket mapping on the winning axis
};

// Order-preserving map of floats onto unsigned integers (-0 below +0).
__device__ __forceinline__ uint32_t ord(float f) {
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float unord(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// Keys for the first-occurrence box fold.  Position 0 stands for the fold's
// starting value (AABB::Empty), which comes before every primitive.
__device__ __forceinline__ unsigned long long min_key(float v, uint32_t pos) {
    const float z = v == 0.0f ? 0.0f : v;
    return (static_cast<unsigned long long>(ord(z)) << 32) | (pos + 1u);
}
__device__ __forceinline__ unsigned long long max_key(float v, uint32_t pos) {
    const float z = v == 0.0f ? 0.0f : v;
    return (static_cast<unsigned long long>(ord(z)) << 32) | (0xffffffffu - (pos + 1u));
}
__device__ __forceinline__ unsigned long long min_key_empty() {
    return static_cast<unsigned long long>(ord(FLT_MAX)) << 32;
}
__device__ __forceinline__ unsigned long long max_key_empty() {
    return (static_cast<unsigned long long>(ord(-FLT_MAX)) << 32) | 0xffffffffu;
}
__device__ __forceinline__ float min_from_key(unsigned long long k, const ae_aabb *pb, int axis) {
    const uint32_t lo = static_cast<uint32_t>(k);
    return lo == 0u ? FLT_MAX : (&pb[lo - 1u].min_x)[axis];
}
__device__ __forceinline__ float max_from_key(unsigned long long k, const ae_aabb *pb, int axis) {
    const uint32_t lo = 0xffffffffu - static_cast<uint32_t>(k);
    return lo == 0u ? -FLT_MAX : (&pb[lo - 1u].min_x)[axis + 3];
}

__device__ __forceinline__ float centre(const ae_aabb &b, int axis) {
    const float *f = &b.min_x;
    return AE_MUL(AE_ADD(f[axis], f[axis + 3]), 0.5f);
}
__device__ __forceinline__ int bucket(float c, float cmin, float scale) {
    // c >= cmin, so the product is >= 0 (or NaN -> 0); max() only keeps an
    // overflowing extent inside the table.
    return max(0, min(kBins - 1, __float2int_rz(AE_MUL(AE_SUB(c, cmin), scale))));
}
__device__ __forceinline__ float half_area(const float lo[3], const float hi[3]) {
    const float dx = AE_SUB(hi[0], lo[0]), dy = AE_SUB(hi[1], lo[1]), dz = AE_SUB(hi[2], lo[2]);
    return AE_ADD(AE_ADD(AE_MUL(dx, dy), AE_MUL(dy, dz)), AE_MUL(dz, dx));
}

// MakeNode, scene/bvh.h:58-89.
__device__ __forceinline__ ae_bvh_node make_node(const ae_aabb &b, int left, int right, int count) {
    ae_bvh_node n;
    n.min_x = b.min_x; n.min_y = b.min_y; n.min_z = b.min_z; n.pad0 = 0.0f;
    n.max_x = b.max_x; n.max_y = b.max_y; n.max_z = b.max_z;
    if (AE_SUB(n.max_x, n.min_x) < kBoundsMinimum) { n.min_x = AE_SUB(n.min_x, kHalfMinimum); n.max_x = AE_ADD(n.max_x, kHalfMinimum); }
    if (AE_SUB(n.max_y, n.min_y) < kBoundsMinimum) { n.min_y = AE_SUB(n.min_y, kHalfMinimum); n.max_y = AE_ADD(n.max_y, kHalfMinimum); }
    if (AE_SUB(n.max_z, n.min_z) < kBoundsMinimum) { n.min_z = AE_SUB(n.min_z, kHalfMinimum); n.max_z = AE_ADD(n.max_z, kHalfMinimum); }
    n.left = left; n.right = right; n.count = count; n.padding = 0; n.pad_trailing = 0;
    return n;
}

// The bucket sweep of one axis (scene/bvh.h:203-236) over a bucket table of
// ordered bounds and counts.  Returns the axis's cheapest plane in the
// reference's visiting order (right to left, strict <), cost FLT_MAX if none.
__device__ void sweep_axis(const uint32_t *bins, float &best_cost, int &best_split) {
    float left_cost[kBins - 1];
    int left_count[kBins - 1];
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    int acc = 0;
    for (int s = 0; s < kBins - 1; s++) {
        const uint32_t *b = bins + s * kBinWords;
        for (int a = 0; a < 3; a++) {
            lo[a] = fminf(lo[a], unord(b[a]));
            hi[a] = fmaxf(hi[a], unord(b[3 + a]));
        }
        acc += int(b[6]);
        left_count[s] = acc;
        left_cost[s] = acc > 0 ? AE_MUL(half_area(lo, hi), float(acc)) : 0.0f;
    }
    for (int a = 0; a < 3; a++) { lo[a] = FLT_MAX; hi[a] = -FLT_MAX; }
    acc = 0;
    best_cost = FLT_MAX;
    best_split = 0;
    for (int s = kBins - 1; s > 0; s--) {
        const uint32_t *b = bins + s * kBinWords;
        for (int a = 0; a < 3; a++) {
            lo[a] = fminf(lo[a], unord(b[a]));
            hi[a] = fmaxf(hi[a], unord(b[3 + a]));
        }
        acc += int(b[6]);
        if (left_count[s - 1] == 0 || acc == 0) continue;
        const float cost = AE_ADD(left_cost[s - 1], AE_MUL(half_area(lo, hi), float(acc)));
        if (cost < best_cost) { best_cost = cost; best_split = s; }
    }
}

__device__ __forceinline__ void bins_reset(uint32_t *bins, int i) {
    const int w = i % kBinWords;
    bins[i] = w < 3 ? ord(FLT_MAX) : (w < 6 ? ord(-FLT_MAX) : 0u);
}

// Centroid extent of one axis -> bucket mapping; false when the reference
// skips the axis (extent <= 0).
__device__ __forceinline__ bool axis_mapping(uint32_t ocmin, uint32_t ocmax, float &cmin, float &scale) {
    cmin = unord(ocmin);
    const float extent = AE_SUB(unord(ocmax), cmin);
    if (extent <= 0.0f) return false;
    scale = AE_DIV(float(kBins), extent);
    return true;
}

// ---------------------------------------------------------------------------
// Setup: copy the boxes into the permuted array, identity order, and flag a
// coordinate that is not finite.
// ---------------------------------------------------------------------------
__global__ void k_setup(const ae_aabb *bounds, uint32_t n, uint32_t *idx, ae_aabb *pb, int *bad) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const ae_aabb b = bounds[i];
    const float *f = &b.min_x;
    bool finite = true;
    for (int a = 0; a < 6; a++) finite &= isfinite(f[a]);
    if (!finite) atomicExch(bad, 1);
    idx[i] = i;
    pb[i] = b;
}

// ---------------------------------------------------------------------------
// Level-by-level phase (nodes larger than kWarpTask).
// ---------------------------------------------------------------------------
__global__ void k_acc_reset(TaskAcc *acc, uint32_t ntasks) {
    const uint32_t t = blockIdx.x;
    if (t >= ntasks) return;
    TaskAcc &A = acc[t];
    if (threadIdx.x < 3) {
        A.bmin[threadIdx.x] = min_key_empty();
        A.bmax[threadIdx.x] = max_key_empty();
        A.cmin[threadIdx.x] = ord(FLT_MAX);
        A.cmax[threadIdx.x] = ord(-FLT_MAX);
    }
    for (int i = threadIdx.x; i < kBinTable; i += blockDim.x) bins_reset(A.bins, i);
}

template <class T, class Op>
__device__ __forceinline__ T warp_all(T v, Op op) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = op(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
struct MinOp { template <class T> __device__ T operator()(T a, T b) const { return b < a ? b : a; } };
struct MaxOp { template <class T> __device__ T operator()(T a, T b) const { return a < b ? b : a; } };

// Box keys and centroid bounds of one chunk, folded into its task.
__global__ void __launch_bounds__(kThreads) k_big_reduce(const Chunk *chunks, const ae_aabb *pb, TaskAcc *acc) {
    const Chunk C = chunks[blockIdx.x];
    unsigned long long kmin[3], kmax[3];
    uint32_t cmin[3], cmax[3];
    for (int a = 0; a < 3; a++) {
        kmin[a] = min_key_empty(); kmax[a] = max_key_empty();
        cmin[a] = ord(FLT_MAX); cmax[a] = ord(-FLT_MAX);
    }
    for (uint32_t p = C.begin + threadIdx.x; p < C.end; p += kThreads) {
        const ae_aabb b = pb[p];
        const float *f = &b.min_x;
        for (int a = 0; a < 3; a++) {
            kmin[a] = MinOp()(kmin[a], min_key(f[a], p));
            kmax[a] = MaxOp()(kmax[a], max_key(f[a + 3], p));
            const uint32_t c = ord(centre(b, a));
            cmin[a] = min(cmin[a], c);
            cmax[a] = max(cmax[a], c);
        }
    }
    __shared__ unsigned long long skmin[kThreads / 32][3], skmax[kThreads / 32][3];
    __shared__ uint32_t scmin[kThreads / 32][3], scmax[kThreads / 32][3];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int a = 0; a < 3; a++) {
        kmin[a] = warp_all(kmin[a], MinOp());
        kmax[a] = warp_all(kmax[a], MaxOp());
        cmin[a] = __reduce_min_sync(0xffffffffu, cmin[a]);
        cmax[a] = __reduce_max_sync(0xffffffffu, cmax[a]);
        if (lane == 0) { skmin[w][a] = kmin[a]; skmax[w][a] = kmax[a]; scmin[w][a] = cmin[a]; scmax[w][a] = cmax[a]; }
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        const int a = threadIdx.x;
        unsigned long long m0 = skmin[0][a], m1 = skmax[0][a];
        uint32_t c0 = scmin[0][a], c1 = scmax[0][a];
        for (int i = 1; i < kThreads / 32; i++) {
            m0 = MinOp()(m0, skmin[i][a]); m1 = MaxOp()(m1, skmax[i][a]);
            c0 = min(c0, scmin[i][a]); c1 = max(c1, scmax[i][a]);
        }
        TaskAcc &A = acc[C.task];
        atomicMin(&A.bmin[a], m0);
        atomicMax(&A.bmax[a], m1);
        atomicMin(&A.cmin[a], c0);
        atomicMax(&A.cmax[a], c1);
    }
}

// The 3 x 12 buckets of one chunk, in shared memory, folded into its task.
__global__ void __launch_bounds__(kThreads) k_big_bin(const Chunk *chunks, const BigTask *tasks, const ae_aabb *pb,
                                                      TaskAcc *acc) {
    const Chunk C = chunks[blockIdx.x];
    const BigTask T = tasks[C.task];
    if (T.depth >= uint32_t(kMaxDepth)) return;  // a leaf: no buckets
    TaskAcc &A = acc[C.task];
    __shared__ uint32_t sb[kBinTable];
    for (int i = threadIdx.x; i < kBinTable; i += kThreads) bins_reset(sb, i);
    float cmin[3], scale[3];
    bool ok[3];
    for (int a = 0; a < 3; a++) ok[a] = axis_mapping(A.cmin[a], A.cmax[a], cmin[a], scale[a]);
    __syncthreads();
    for (uint32_t p = C.begin + threadIdx.x; p < C.end; p += kThreads) {
        const ae_aabb b = pb[p];
        const float *f = &b.min_x;
        for (int a = 0; a < 3; a++) {
            if (!ok[a]) continue;
            uint32_t *r = sb + (a * kBins + bucket(centre(b, a), cmin[a], scale[a])) * kBinWords;
            for (int k = 0; k < 3; k++) {
                atomicMin(r + k, ord(f[k]));
                atomicMax(r + 3 + k, ord(f[k + 3]));
            }
            atomicAdd(r + 6, 1u);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kBinTable; i += kThreads) {
        const int rec = i / kBinWords, wd = i % kBinWords;
        if (sb[rec * kBinWords + 6] == 0u) continue;
        if (wd < 3) atomicMin(&A.bins[i], sb[i]);
        else if (wd < 6) atomicMax(&A.bins[i], sb[i]);
        else atomicAdd(&A.bins[i], sb[i]);
    }
}

// The node box, leaf or not, the SAH plane (scene/bvh.h:148-247), from the
// task's accumulated keys and buckets.
__device__ Decision decide(const BigTask &T, const TaskAcc &A, const ae_aabb *pb) {
    Decision D;
    float *bx = &D.box.min_x;
    for (int a = 0; a < 3; a++) {
        bx[a] = min_from_key(A.bmin[a], pb, a);
        bx[a + 3] = max_from_key(A.bmax[a], pb, a);
    }
    const uint32_t count = T.end - T.start;
    D.leaf = (count <= uint32_t(kLeafSize) || T.depth >= uint32_t(kMaxDepth)) ? 1 : 0;
    D.axis = -1; D.split = 0; D.cmin = 0.0f; D.scale = 0.0f;
    if (!D.leaf) {
        float best = FLT_MAX;
        for (int a = 0; a < 3; a++) {
            float cm, sc;
            if (!axis_mapping(A.cmin[a], A.cmax[a], cm, sc)) continue;
            float c; int s;
            sweep_axis(A.bins + a * kBins * kBinWords, c, s);
            if (c < best) { best = c; D.axis = a; D.split = s; D.cmin = cm; D.scale = sc; }
        }
    }
    return D;
}

__device__ __forceinline__ bool goes_left(const ae_aabb &b, const Decision &D) {
    return bucket(centre(b, D.axis), D.cmin, D.scale) < D.split;
}

// Each block decides its task (the task's first chunk publishes the
// decision) and counts the chunk's elements that go left.
__global__ void __launch_bounds__(kThreads) k_big_count(const Chunk *chunks, const BigTask *tasks, const TaskAcc *acc,
                                                        const ae_aabb *pb, Decision *dec, uint32_t *chunk_true) {
    const Chunk C = chunks[blockIdx.x];
    __shared__ Decision sD;
    __shared__ uint32_t s[kThreads / 32];
    if (threadIdx.x == 0) {
        const BigTask T = tasks[C.task];
        sD = decide(T, acc[C.task], pb);
        if (C.begin == T.start) dec[C.task] = sD;
    }
    __syncthreads();
    const Decision D = sD;
    if (D.leaf || D.axis < 0) {
        if (threadIdx.x == 0) chunk_true[blockIdx.x] = 0;
        return;
    }
    uint32_t n = 0;
    for (uint32_t p = C.begin + threadIdx.x; p < C.end; p += kThreads) n += goes_left(pb[p], D) ? 1u : 0u;
    n = __reduce_add_sync(0xffffffffu, n);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = n;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int i = 0; i < kThreads / 32; i++) t += s[i];
        chunk_true[blockIdx.x] = t;
    }
}

// Misplaced elements of a splitting task go to the stash: the k-th failing
// element left of the boundary to start + k, the k-th passing element right
// of it (counted from the right) to end - 1 - k.  kinfo[p] = k + 1, bit 31
// set for the passing kind, 0 for an element that stays.
__global__ void __launch_bounds__(kThreads) k_big_stash(const Chunk *chunks, const BigTask *tasks, const Decision *dec,
                                                        const uint32_t *task_true, const uint32_t *chunk_base,
                                                        const uint32_t *idx, const ae_aabb *pb, uint32_t *stash_idx,
                                                        ae_aabb *stash_pb, uint32_t *kinfo) {
    const Chunk C = chunks[blockIdx.x];
    const Decision D = dec[C.task];
    if (D.leaf || D.axis < 0) return;
    const BigTask T = tasks[C.task];
    const uint32_t ntrue = task_true[C.task];
    const uint32_t boundary = T.start + ntrue;
    // Each thread takes kPer consecutive positions.
    const uint32_t p0 = C.begin + threadIdx.x * kPer;
    bool pass[kPer];
    uint32_t mine = 0;
    for (int j = 0; j < kPer; j++) {
        const uint32_t p = p0 + j;
        pass[j] = p < C.end && goes_left(pb[p], D);
        mine += pass[j] ? 1u : 0u;
    }
    // Block exclusive scan of the per-thread counts.
    __shared__ uint32_t s[kThreads / 32];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t incl = mine;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) s[w] = incl;
    __syncthreads();
    uint32_t before = chunk_base[blockIdx.x] + incl - mine;
    for (int i = 0; i < w; i++) before += s[i];
    for (int j = 0; j < kPer; j++) {
        const uint32_t p = p0 + j;
        if (p >= C.end) break;
        uint32_t info = 0;
        if (p < boundary && !pass[j]) {
            const uint32_t k = (p - T.start) - before;
            stash_idx[T.start + k] = idx[p];
            stash_pb[T.start + k] = pb[p];
            info = k + 1u;
        } else if (p >= boundary && pass[j]) {
            const uint32_t k = ntrue - before - 1u;
            stash_idx[T.end - 1u - k] = idx[p];
            stash_pb[T.end - 1u - k] = pb[p];
            info = (k + 1u) | 0x80000000u;
        }
        kinfo[p] = info;
        before += pass[j] ? 1u : 0u;
    }
}

// Each misplaced element takes its partner's record from the stash.
__global__ void __launch_bounds__(kThreads) k_big_unstash(const Chunk *chunks, const BigTask *tasks, const Decision *dec,
                                                          const uint32_t *kinfo, const uint32_t *stash_idx,
                                                          const ae_aabb *stash_pb, uint32_t *idx, ae_aabb *pb) {
    const Chunk C = chunks[blockIdx.x];
    const Decision D = dec[C.task];
    if (D.leaf || D.axis < 0) return;
    const BigTask T = tasks[C.task];
    for (uint32_t p = C.begin + threadIdx.x; p < C.end; p += kThreads) {
        const uint32_t info = kinfo[p];
        if (info == 0u) continue;
        const uint32_t k = (info & 0x7fffffffu) - 1u;
        const uint32_t from = (info & 0x80000000u) ? T.start + k : T.end - 1u - k;
        idx[p] = stash_idx[from];
        pb[p] = stash_pb[from];
    }
}

// ---------------------------------------------------------------------------
// One warp per subtree of at most kWarpTask primitives.
// ---------------------------------------------------------------------------
struct WarpWork { uint32_t start, end, depth; int32_t parent, right; };

__global__ void __launch_bounds__(kWarpsPerBlock * 32) k_warp_build(const SmallTask *tasks, uint32_t ntasks,
                                                                   uint32_t *idx, ae_aabb *pb, uint32_t *stash_idx,
                                                                   ae_aabb *stash_pb, uint32_t *kinfo,
                                                                   ae_bvh_node *tmp, uint32_t *sub_count) {
    __shared__ uint32_t sbins[kWarpsPerBlock][kBinTable];
    __shared__ WarpWork sstack[kWarpsPerBlock][kWarpStack];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t t = blockIdx.x * kWarpsPerBlock + w;
    if (t >= ntasks) return;
    uint32_t *bins = sbins[w];
    WarpWork *stack = sstack[w];
    const SmallTask task = tasks[t];
    ae_bvh_node *out = tmp + 2ull * task.start;
    if (lane == 0) stack[0] = WarpWork{task.start, task.end, task.depth, -1, 0};
    int sp = 1;
    int li = 0;
    __syncwarp();
    while (sp > 0) {
        const WarpWork wk = stack[--sp];
        __syncwarp();
        const int self = li++;
        if (lane == 0 && wk.parent >= 0) {
            if (wk.right) out[wk.parent].right = self;
            else out[wk.parent].left = self;
        }
        // Box and centroid bounds.  Each lane folds its positions (ascending,
        // strict comparisons: the first of equal values stays); across lanes
        // the extreme value wins, then the smallest position holding it.
        // Position 0 is the fold's starting value (AABB::Empty).
        uint32_t vmin[3], pmin[3], vmax[3], pmax[3], cmn[3], cmx[3];
        for (int a = 0; a < 3; a++) {
            vmin[a] = ord(FLT_MAX); pmin[a] = 0u;
            vmax[a] = ord(-FLT_MAX); pmax[a] = 0u;
            cmn[a] = ord(FLT_MAX); cmx[a] = ord(-FLT_MAX);
        }
        for (uint32_t p = wk.start + lane; p < wk.end; p += 32) {
            const ae_aabb b = pb[p];
            const float *f = &b.min_x;
            for (int a = 0; a < 3; a++) {
                const uint32_t lo = ord(f[a] == 0.0f ? 0.0f : f[a]);
                const uint32_t hi = ord(f[a + 3] == 0.0f ? 0.0f : f[a + 3]);
                if (lo < vmin[a]) { vmin[a] = lo; pmin[a] = p + 1u; }
                if (hi > vmax[a]) { vmax[a] = hi; pmax[a] = p + 1u; }
                const uint32_t c = ord(centre(b, a));
                cmn[a] = min(cmn[a], c);
                cmx[a] = max(cmx[a], c);
            }
        }
        ae_aabb box;
        float *bx = &box.min_x;
        for (int a = 0; a < 3; a++) {
            const uint32_t wmin = __reduce_min_sync(0xffffffffu, vmin[a]);
            const uint32_t wmax = __reduce_max_sync(0xffffffffu, vmax[a]);
            const uint32_t fmin = __reduce_min_sync(0xffffffffu, vmin[a] == wmin ? pmin[a] : 0xffffffffu);
            const uint32_t fmax = __reduce_min_sync(0xffffffffu, vmax[a] == wmax ? pmax[a] : 0xffffffffu);
            bx[a] = fmin == 0u ? FLT_MAX : (&pb[fmin - 1u].min_x)[a];
            bx[a + 3] = fmax == 0u ? -FLT_MAX : (&pb[fmax - 1u].min_x)[a + 3];
            cmn[a] = __reduce_min_sync(0xffffffffu, cmn[a]);
            cmx[a] = __reduce_max_sync(0xffffffffu, cmx[a]);
        }
        const uint32_t count = wk.end - wk.start;
        if (count <= uint32_t(kLeafSize) || wk.depth >= uint32_t(kMaxDepth)) {
            if (lane == 0) out[self] = make_node(box, int(wk.start - task.root), -1, int(count));
            __syncwarp();
            continue;
        }
        // Buckets.
        float cmin[3], scale[3];
        bool ok[3];
        for (int a = 0; a < 3; a++) ok[a] = axis_mapping(cmn[a], cmx[a], cmin[a], scale[a]);
        for (int i = lane; i < kBinTable; i += 32) bins_reset(bins, i);
        __syncwarp();
        if (ok[0] || ok[1] || ok[2]) {
            for (uint32_t p = wk.start + lane; p < wk.end; p += 32) {
                const ae_aabb b = pb[p];
                const float *f = &b.min_x;
                for (int a = 0; a < 3; a++) {
                    if (!ok[a]) continue;
                    uint32_t *r = bins + (a * kBins + bucket(centre(b, a), cmin[a], scale[a])) * kBinWords;
                    for (int k = 0; k < 3; k++) {
                        atomicMin(r + k, ord(f[k]));
                        atomicMax(r + 3 + k, ord(f[k + 3]));
                    }
                    atomicAdd(r + 6, 1u);
                }
            }
        }
        __syncwarp();
        // Lanes 0-2 sweep one axis each; axes are then taken in order with
        // strict <, as the reference's single loop over axes does.
        float c = FLT_MAX;
        int s = 0;
        if (lane < 3 && ok[lane]) sweep_axis(bins + lane * kBins * kBinWords, c, s);
        const float c0 = __shfl_sync(0xffffffffu, c, 0), c1 = __shfl_sync(0xffffffffu, c, 1),
                    c2 = __shfl_sync(0xffffffffu, c, 2);
        const int s0 = __shfl_sync(0xffffffffu, s, 0), s1 = __shfl_sync(0xffffffffu, s, 1),
                  s2 = __shfl_sync(0xffffffffu, s, 2);
        float best = FLT_MAX;
        int axis = -1, split = 0;
        if (c0 < best) { best = c0; axis = 0; split = s0; }
        if (c1 < best) { best = c1; axis = 1; split = s1; }
        if (c2 < best) { best = c2; axis = 2; split = s2; }
        uint32_t mid = wk.start + count / 2;
        if (axis >= 0) {
            Decision D;
            D.axis = axis; D.split = split; D.cmin = cmin[axis]; D.scale = scale[axis];
            uint32_t ntrue = 0;
            for (uint32_t base = wk.start; base < wk.end; base += 32) {
                const uint32_t p = base + lane;
                ntrue += __popc(__ballot_sync(0xffffffffu, p < wk.end && goes_left(pb[p], D)));
            }
            const uint32_t boundary = wk.start + ntrue;
            uint32_t before = 0;
            for (uint32_t base = wk.start; base < wk.end; base += 32) {
                const uint32_t p = base + lane;
                const bool pass = p < wk.end && goes_left(pb[p], D);
                const uint32_t m = __ballot_sync(0xffffffffu, pass);
                const uint32_t b = before + __popc(m & ((1u << lane) - 1u));
                if (p < wk.end) {
                    uint32_t info = 0;
                    if (p < boundary && !pass) {
                        const uint32_t k = (p - wk.start) - b;
                        stash_idx[wk.start + k] = idx[p];
                        stash_pb[wk.start + k] = pb[p];
                        info = k + 1u;
                    } else if (p >= boundary && pass) {
                        const uint32_t k = ntrue - b - 1u;
                        stash_idx[wk.end - 1u - k] = idx[p];
                        stash_pb[wk.end - 1u - k] = pb[p];
                        info = (k + 1u) | 0x80000000u;
                    }
                    kinfo[p] = info;
                }
                before += __popc(m);
            }
            __syncwarp();
            for (uint32_t p = wk.start + lane; p < wk.end; p += 32) {
                const uint32_t info = kinfo[p];
                if (info == 0u) continue;
                const uint32_t k = (info & 0x7fffffffu) - 1u;
                const uint32_t from = (info & 0x80000000u) ? wk.start + k : wk.end - 1u - k;
                idx[p] = stash_idx[from];
                pb[p] = stash_pb[from];
            }
            __syncwarp();
            mid = boundary;
        }
        if (mid <= wk.start || mid >= wk.end) mid = wk.start + count / 2;
        if (lane == 0) {
            out[self] = make_node(box, -1, -1, 0);
            stack[sp] = WarpWork{mid, wk.end, wk.depth + 1, self, 1};
            stack[sp + 1] = WarpWork{wk.start, mid, wk.depth + 1, self, 0};
        }
        sp += 2;
        __syncwarp();
    }
    if (lane == 0) sub_count[t] = uint32_t(li);
}

// ---------------------------------------------------------------------------
// Final numbering.
// ---------------------------------------------------------------------------
// One block per warp-built subtree: local node indices -> global.
// sub_base: the subtree's first node index within its tree (links are
// relative to the tree); the nodes land at the tree's offset in `out`.
__global__ void k_place_subtrees(const SmallTask *tasks, const uint32_t *sub_count, const uint32_t *sub_base,
                                 const ae_bvh_node *tmp, ae_bvh_node *out) {
    const uint32_t t = blockIdx.x;
    const ae_bvh_node *src = tmp + 2ull * tasks[t].start;
    const uint32_t base = sub_base[t], n = sub_count[t];
    ae_bvh_node *dst = out + tasks[t].out;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        ae_bvh_node nd = src[i];
        if (nd.count == 0) {
            nd.left += int(base);
            nd.right += int(base);
        }
        dst[base + i] = nd;
    }
}

struct TopPlace { uint32_t at; int32_t left, right; uint32_t start, count; int32_t leaf; };

__global__ void k_place_top(const TopPlace *place, const Decision *dec_all, uint32_t ntop, ae_bvh_node *out) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntop) return;
    const TopPlace P = place[t];
    const ae_aabb box = dec_all[t].box;
    out[P.at] = P.leaf ? make_node(box, int(P.start), -1, int(P.count)) : make_node(box, P.left, P.right, 0);
}

// Triangle boxes: Surround2Points(a, b) then SurroundPoint(c),
// scene/aabb.h:96-103, with std::min / std::max (first of equal values).
__device__ __forceinline__ float smin(float a, float b) { return b < a ? b : a; }
__device__ __forceinline__ float smax(float a, float b) { return a < b ? b : a; }

__global__ void k_triangle_boxes(const ae_vertex *v, uint32_t nv, const uint32_t *idx, uint32_t tris, ae_aabb *out,
                                 int *bad) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= tris) return;
    const uint32_t i0 = idx[3 * t], i1 = idx[3 * t + 1], i2 = idx[3 * t + 2];
    if (i0 >= nv || i1 >= nv || i2 >= nv) {
        atomicExch(bad, 1);
        return;
    }
    const ae_vertex a = v[i0], b = v[i1], c = v[i2];
    ae_aabb e;
    e.min_x = smin(smin(a.px, b.px), c.px);
    e.min_y = smin(smin(a.py, b.py), c.py);
    e.min_z = smin(smin(a.pz, b.pz), c.pz);
    e.max_x = smax(smax(a.px, b.px), c.px);
    e.max_y = smax(smax(a.py, b.py), c.py);
    e.max_z = smax(smax(a.pz, b.pz), c.pz);
    out[t] = e;
}

// Indices in leaf-slot order (scene/mesh_library.h:147-153); `order` holds
// triangle numbers offset by `first` (a mesh's range in a forest build).
__global__ void k_reorder_indices(const uint32_t *idx, const uint32_t *order, uint32_t first, uint32_t tris,
                                  uint32_t *out) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= tris) return;
    const uint32_t t = order[s] - first;
    out[3 * s] = idx[3 * t];
    out[3 * s + 1] = idx[3 * t + 1];
    out[3 * s + 2] = idx[3 * t + 2];
}

// RebuildAcceleration's packing after the build (renderer/renderer.cpp:
// 1096-1121): objects in slot order, each mesh numbered by its rank among the
// meshes in slot order (PackObjects), lights as the slots of emissive objects
// in slot order (LightIndices).  One block walks the slots in order with
// block-wide scans.  flags: bit 0 mesh, bit 1 light.
__global__ void __launch_bounds__(1024) k_assemble(uint32_t n, const uint32_t *order, const uint32_t *flags,
                                                   const ae_object *obj_t, const ae_instance *inst_t,
                                                   ae_object *objects, ae_instance *instances, uint32_t *lights,
                                                   uint32_t *counts) {
    __shared__ uint32_t wm[32], wl[32];
    __shared__ uint32_t base_m, base_l;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (threadIdx.x == 0) { base_m = 0; base_l = 0; }
    __syncthreads();
    for (uint32_t b = 0; b < n; b += blockDim.x) {
        const uint32_t slot = b + threadIdx.x;
        const uint32_t e = slot < n ? order[slot] : 0u;
        const uint32_t f = slot < n ? flags[e] : 0u;
        const uint32_t mesh = f & 1u, light = (f >> 1) & 1u;
        const uint32_t mm = __ballot_sync(0xffffffffu, mesh), ml = __ballot_sync(0xffffffffu, light);
        const uint32_t below = (1u << lane) - 1u;
        if (lane == 0) { wm[w] = __popc(mm); wl[w] = __popc(ml); }
        __syncthreads();
        uint32_t rm = base_m + __popc(mm & below), rl = base_l + __popc(ml & below);
        for (int i = 0; i < w; i++) { rm += wm[i]; rl += wl[i]; }
        if (slot < n) {
            ae_object o = obj_t[e];
            if (mesh) {
                o.instanceIndex = rm;
                instances[rm] = inst_t[e];
            }
            objects[slot] = o;
            if (light) lights[rl] = slot;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t tm = 0, tl = 0;
            for (int i = 0; i < int(blockDim.x >> 5); i++) { tm += wm[i]; tl += wl[i]; }
            base_m += tm;
            base_l += tl;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) { counts[0] = base_m; counts[1] = base_l; }
}

// ---------------------------------------------------------------------------
// Host driver.
// ---------------------------------------------------------------------------
// Device scratch that only grows, kept between builds (cudaMalloc and
// cudaFree synchronise the device and cost more than a small build).
template <class T> struct Grow {
    T *p = nullptr;
    size_t cap = 0;
    cudaError_t need(size_t n) {
        if (n <= cap && p) return cudaSuccess;
        if (p) dev_free(p);
        p = nullptr;
        cap = 0;
        const size_t want = n + n / 4 + 16;
        void *q = nullptr;
        const cudaError_t e = dev_alloc(&q, want * sizeof(T));
        p = static_cast<T *>(q);
        if (e == cudaSuccess) cap = want;
        return e;
    }
    void release() {
        if (p) dev_free(p);
        p = nullptr;
        cap = 0;
    }
};

#define AE_CK(x)                                  \
    do {                                          \
        if ((x) != cudaSuccess) {                 \
            cudaGetLastError();                   \
            return AE_ERR_CUDA;                   \
        }                                         \
    } while (0)

struct Scratch {
    Grow<ae_aabb> pb, stash_pb;
    Grow<uint32_t> stash_idx, kinfo;
    Grow<ae_bvh_node> tmp;
    Grow<int> bad;
    Grow<TaskAcc> acc;
    Grow<BigTask> tasks;
    Grow<Chunk> chunks;
    Grow<Decision> dec, top_dec;
    Grow<uint32_t> chunk_true, chunk_base, task_true, sub_count, sub_base;
    Grow<SmallTask> small;
    Grow<TopPlace> place;
    // mesh builds
    Grow<ae_vertex> v;
    Grow<uint32_t> idx, order, out_idx;
    Grow<ae_aabb> box;
    Grow<ae_bvh_node> nodes, mesh_nodes;
    // scene packing
    Grow<ae_object> obj_t, objects;
    Grow<ae_instance> inst_t, instances;
    Grow<uint32_t> flags, lights, counts;
    void release() {
        obj_t.release(); objects.release(); inst_t.release(); instances.release(); flags.release();
        lights.release(); counts.release();
        pb.release(); stash_pb.release(); stash_idx.release(); kinfo.release(); tmp.release(); bad.release();
        acc.release(); tasks.release(); chunks.release(); dec.release(); top_dec.release(); chunk_true.release();
        chunk_base.release(); task_true.release(); sub_count.release(); sub_base.release(); small.release();
        place.release(); v.release(); idx.release(); order.release(); out_idx.release(); box.release();
        nodes.release(); mesh_nodes.release();
    }
};
Scratch g_scratch;
std::mutex g_mutex;  // one build at a time per process: they share g_scratch

struct TopNode {
    BigTask task;
    uint32_t tree = 0;            // index of the tree (root range) it belongs to
    int32_t left = 0, right = 0;  // >= 0: top node; < 0: warp subtree -1 - id
    bool leaf = false;
};

}  // namespace

// Builds the tree over `d_bounds` (device, n boxes) on `st`.  On success
// d_nodes (2n capacity) holds the nodes, d_order the leaf-slot permutation,
// *node_count their number.
// A forest: one tree per range [first[r], first[r + 1]) of the n boxes
// (first[0] = 0, first[n_trees] = n), all built in the same level rounds and
// warp launch.  Tree r's nodes go to d_nodes + 2 * first[r] (room for its
// 2 * count - 1), with links and leaf slots relative to its own range, so
// each tree is exactly the one built over its range alone;
// node_counts[r] = its node count.  d_order: per position, the index of the
// box there (positions of a range hold that range's boxes).
int gpu_build_forest(const ae_aabb *d_bounds, const uint32_t *first, uint32_t n_trees, ae_bvh_node *d_nodes,
                     uint32_t *d_order, uint32_t *node_counts, cudaStream_t st, uint32_t warp_subtree) {
    for (uint32_t r = 0; r < n_trees; r++) node_counts[r] = 0;
    const uint32_t n = first[n_trees];
    if (n == 0) return AE_OK;
    Scratch &S = g_scratch;
    auto &pb = S.pb, &stash_pb = S.stash_pb;
    auto &stash_idx = S.stash_idx, &kinfo = S.kinfo;
    auto &tmp = S.tmp;
    auto &bad = S.bad;
    AE_CK(pb.need(n));
    AE_CK(stash_pb.need(n));
    AE_CK(stash_idx.need(n));
    AE_CK(kinfo.need(n));
    AE_CK(tmp.need(2ull * n));
    AE_CK(bad.need(1));
    AE_CK(cudaMemsetAsync(bad.p, 0, sizeof(int), st));
    uint32_t *idx = d_order;
    k_setup<<<(n + 255) / 256, 256, 0, st>>>(d_bounds, n, idx, pb.p, bad.p);
    int h_bad = 0;
    AE_CK(cudaMemcpyAsync(&h_bad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    AE_CK(cudaStreamSynchronize(st));
    if (h_bad) return AE_ERR_INVALID;

    std::vector<TopNode> top;
    std::vector<SmallTask> small;
    std::vector<Decision> top_dec;
    std::vector<BigTask> level;
    std::vector<uint32_t> level_top;  // top node of each task of the level
    std::vector<int32_t> tree_root(n_trees, 0);  // ref of each tree's root (see TopNode::left)
    std::vector<char> tree_empty(n_trees, 0);
    for (uint32_t r = 0; r < n_trees; r++) {
        const uint32_t a = first[r], b = first[r + 1];
        if (b <= a) {
            tree_empty[r] = 1;
            continue;
        }
        if (b - a > warp_subtree) {
            tree_root[r] = int32_t(top.size());
            level.push_back(BigTask{a, b, 0});
            level_top.push_back(uint32_t(top.size()));
            top.push_back(TopNode{});
            top.back().task = level.back();
            top.back().tree = r;
        } else {
            tree_root[r] = -1 - int32_t(small.size());
            small.push_back(SmallTask{a, b, 0, a, 2 * a});
        }
    }
    auto &acc = S.acc;
    auto &d_tasks = S.tasks;
    auto &d_chunks = S.chunks;
    auto &d_dec = S.dec;
    auto &d_chunk_true = S.chunk_true, &d_chunk_base = S.chunk_base, &d_task_true = S.task_true;
    std::vector<Chunk> chunks;
    std::vector<Decision> dec;
    std::vector<uint32_t> chunk_true, chunk_base, task_true;
    while (!level.empty()) {
        const uint32_t nt = uint32_t(level.size());
        chunks.clear();
        for (uint32_t t = 0; t < nt; t++)
            for (uint32_t b = level[t].start; b < level[t].end; b += kChunk)
                chunks.push_back(Chunk{t, b, b + kChunk < level[t].end ? b + kChunk : level[t].end});
        const uint32_t nc = uint32_t(chunks.size());
        AE_CK(acc.need(nt));
        AE_CK(d_tasks.need(nt));
        AE_CK(d_dec.need(nt));
        AE_CK(d_task_true.need(nt));
        AE_CK(d_chunks.need(nc));
        AE_CK(d_chunk_true.need(nc));
        AE_CK(d_chunk_base.need(nc));
        AE_CK(cudaMemcpyAsync(d_tasks.p, level.data(), nt * sizeof(BigTask), cudaMemcpyHostToDevice, st));
        AE_CK(cudaMemcpyAsync(d_chunks.p, chunks.data(), nc * sizeof(Chunk), cudaMemcpyHostToDevice, st));
        k_acc_reset<<<nt, 128, 0, st>>>(acc.p, nt);
        k_big_reduce<<<nc, kThreads, 0, st>>>(d_chunks.p, pb.p, acc.p);
        k_big_bin<<<nc, kThreads, 0, st>>>(d_chunks.p, d_tasks.p, pb.p, acc.p);
        k_big_count<<<nc, kThreads, 0, st>>>(d_chunks.p, d_tasks.p, acc.p, pb.p, d_dec.p, d_chunk_true.p);
        dec.resize(nt);
        chunk_true.resize(nc);
        AE_CK(cudaMemcpyAsync(dec.data(), d_dec.p, nt * sizeof(Decision), cudaMemcpyDeviceToHost, st));
        AE_CK(cudaMemcpyAsync(chunk_true.data(), d_chunk_true.p, nc * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        AE_CK(cudaStreamSynchronize(st));
        task_true.assign(nt, 0);
        chunk_base.resize(nc);
        for (uint32_t c = 0; c < nc; c++) {
            chunk_base[c] = task_true[chunks[c].task];
            task_true[chunks[c].task] += chunk_true[c];
        }
        AE_CK(cudaMemcpyAsync(d_chunk_base.p, chunk_base.data(), nc * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
        AE_CK(cudaMemcpyAsync(d_task_true.p, task_true.data(), nt * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
        k_big_stash<<<nc, kThreads, 0, st>>>(d_chunks.p, d_tasks.p, d_dec.p, d_task_true.p, d_chunk_base.p, idx, pb.p,
                                             stash_idx.p, stash_pb.p, kinfo.p);
        k_big_unstash<<<nc, kThreads, 0, st>>>(d_chunks.p, d_tasks.p, d_dec.p, kinfo.p, stash_idx.p, stash_pb.p, idx,
                                               pb.p);
        AE_CK(cudaGetLastError());
        // Children of this level.  The copies above were staged from pageable
        // memory, so the host arrays may be reused at once.
        std::vector<BigTask> next;
        std::vector<uint32_t> next_top;
        if (top_dec.size() < top.size()) top_dec.resize(top.size());
        for (uint32_t t = 0; t < nt; t++) {
            const BigTask T = level[t];
            const uint32_t id = level_top[t];
            top_dec[id] = dec[t];
            if (dec[t].leaf) {
                top[id].leaf = true;
                continue;
            }
            const uint32_t count = T.end - T.start;
            uint32_t mid = dec[t].axis >= 0 ? T.start + task_true[t] : T.start + count / 2;
            if (mid <= T.start || mid >= T.end) mid = T.start + count / 2;
            const BigTask kids[2] = {BigTask{T.start, mid, T.depth + 1}, BigTask{mid, T.end, T.depth + 1}};
            for (int side = 0; side < 2; side++) {
                const BigTask &K = kids[side];
                int32_t ref;
                const uint32_t tree = top[id].tree;
                if (K.end - K.start > warp_subtree) {
                    ref = int32_t(top.size());
                    top.push_back(TopNode{});
                    top.back().task = K;
                    top.back().tree = tree;
                    next.push_back(K);
                    next_top.push_back(uint32_t(ref));
                } else {
                    ref = -1 - int32_t(small.size());
                    small.push_back(SmallTask{K.start, K.end, K.depth, first[tree], 2 * first[tree]});
                }
                if (side == 0) top[id].left = ref;
                else top[id].right = ref;
            }
        }
        level.swap(next);
        level_top.swap(next_top);
    }

    // Warp-built subtrees.
    const uint32_t ns = uint32_t(small.size());
    auto &d_small = S.small;
    auto &d_sub_count = S.sub_count, &d_sub_base = S.sub_base;
    AE_CK(d_small.need(ns));
    AE_CK(d_sub_count.need(ns));
    AE_CK(d_sub_base.need(ns));
    std::vector<uint32_t> sub_count(ns), sub_base(ns);
    if (ns) {
        AE_CK(cudaMemcpyAsync(d_small.p, small.data(), ns * sizeof(SmallTask), cudaMemcpyHostToDevice, st));
        k_warp_build<<<(ns + kWarpsPerBlock - 1) / kWarpsPerBlock, kWarpsPerBlock * 32, 0, st>>>(
            d_small.p, ns, idx, pb.p, stash_idx.p, stash_pb.p, kinfo.p, tmp.p, d_sub_count.p);
        AE_CK(cudaGetLastError());
        AE_CK(cudaMemcpyAsync(sub_count.data(), d_sub_count.p, ns * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        AE_CK(cudaStreamSynchronize(st));
    }
    // Pre-order numbering per tree: a node, then its left subtree, then its
    // right.
    std::vector<TopPlace> place(top.size());
    std::vector<int32_t> work;
    std::vector<uint32_t> root_of_top(top.size());
    for (uint32_t r = 0; r < n_trees; r++) {
        if (tree_empty[r]) continue;
        uint32_t next_index = 0;
        work.push_back(tree_root[r]);
        while (!work.empty()) {
            const int32_t ref = work.back();
            work.pop_back();
            if (ref >= 0) {
                root_of_top[ref] = next_index++;
                if (!top[ref].leaf) {
                    work.push_back(top[ref].right);
                    work.push_back(top[ref].left);
                }
            } else {
                const uint32_t s = uint32_t(-1 - ref);
                sub_base[s] = next_index;
                next_index += sub_count[s];
            }
        }
        node_counts[r] = next_index;
    }
    for (size_t i = 0; i < top.size(); i++) {
        TopPlace &P = place[i];
        const uint32_t tree_first = first[top[i].tree];
        P.at = 2 * tree_first + root_of_top[i];
        P.leaf = top[i].leaf ? 1 : 0;
        P.start = top[i].task.start - tree_first;
        P.count = top[i].task.end - top[i].task.start;
        auto root = [&](int32_t r) { return r >= 0 ? int32_t(root_of_top[r]) : int32_t(sub_base[-1 - r]); };
        P.left = P.leaf ? 0 : root(top[i].left);
        P.right = P.leaf ? 0 : root(top[i].right);
    }
    if (ns) {
        AE_CK(cudaMemcpyAsync(d_sub_base.p, sub_base.data(), ns * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
        k_place_subtrees<<<ns, 256, 0, st>>>(d_small.p, d_sub_count.p, d_sub_base.p, tmp.p, d_nodes);
    }
    if (!top.empty()) {
        auto &d_place = S.place;
        auto &d_top_dec = S.top_dec;
        AE_CK(d_place.need(top.size()));
        AE_CK(d_top_dec.need(top.size()));
        AE_CK(cudaMemcpyAsync(d_place.p, place.data(), top.size() * sizeof(TopPlace), cudaMemcpyHostToDevice, st));
        AE_CK(cudaMemcpyAsync(d_top_dec.p, top_dec.data(), top.size() * sizeof(Decision), cudaMemcpyHostToDevice, st));
        k_place_top<<<uint32_t((top.size() + 127) / 128), 128, 0, st>>>(d_place.p, d_top_dec.p, uint32_t(top.size()),
                                                                         d_nodes);
        AE_CK(cudaGetLastError());
        AE_CK(cudaStreamSynchronize(st));
    }
    AE_CK(cudaGetLastError());
    AE_CK(cudaStreamSynchronize(st));
    return AE_OK;
}

// One tree over all n boxes.
int gpu_build_bvh(const ae_aabb *d_bounds, uint32_t n, ae_bvh_node *d_nodes, uint32_t *d_order,
                  uint32_t *node_count, cudaStream_t st, uint32_t warp_subtree = kWarpTask) {
    const uint32_t first[2] = {0, n};
    return gpu_build_forest(d_bounds, first, 1, d_nodes, d_order, node_count, st, warp_subtree);
}

// MeshLibrary::Add's device part on device arrays: the triangle boxes, the
// BLAS and the indices in leaf-slot order.
int gpu_mesh_blas_device(const ae_vertex *d_v, uint32_t nv, const uint32_t *d_idx, uint32_t ni, ae_bvh_node *d_nodes,
                         uint32_t *out_count, uint32_t *d_out_idx, cudaStream_t st) {
    *out_count = 0;
    const uint32_t tris = ni / 3;
    if (tris == 0) return AE_OK;
    Scratch &S = g_scratch;
    AE_CK(S.box.need(tris));
    AE_CK(S.order.need(tris));
    AE_CK(S.bad.need(1));
    AE_CK(cudaMemsetAsync(S.bad.p, 0, sizeof(int), st));
    k_triangle_boxes<<<(tris + 255) / 256, 256, 0, st>>>(d_v, nv, d_idx, tris, S.box.p, S.bad.p);
    int h_bad = 0;
    AE_CK(cudaMemcpyAsync(&h_bad, S.bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    AE_CK(cudaStreamSynchronize(st));
    if (h_bad) return AE_ERR_LAYOUT;
    const int rc = gpu_build_bvh(S.box.p, tris, d_nodes, S.order.p, out_count, st);
    if (rc != AE_OK) return rc;
    k_reorder_indices<<<(tris + 255) / 256, 256, 0, st>>>(d_idx, S.order.p, 0u, tris, d_out_idx);
    AE_CK(cudaGetLastError());
    AE_CK(cudaStreamSynchronize(st));
    return AE_OK;
}

// The BLAS of k meshes at once: one forest build over all their triangles,
// so the meshes share the level rounds and the warp launch.  Arrays of device
// pointers, one entry per mesh; each mesh's output equals
// gpu_mesh_blas_device's.
int gpu_mesh_blas_many(uint32_t k, const ae_vertex *const *d_v, const uint32_t *nv, const uint32_t *const *d_idx,
                       const uint32_t *ni, ae_bvh_node *const *d_nodes, uint32_t *out_counts,
                       uint32_t *const *d_out_idx, cudaStream_t st) {
    std::vector<uint32_t> first(size_t(k) + 1, 0);
    for (uint32_t m = 0; m < k; m++) {
        out_counts[m] = 0;
        if (ni[m] % 3 != 0) return AE_ERR_INVALID;
        if (ni[m] && (!d_v[m] || !d_idx[m] || !d_nodes[m] || !d_out_idx[m])) return AE_ERR_INVALID;
        first[m + 1] = first[m] + ni[m] / 3;
    }
    const uint32_t total = first[k];
    if (total == 0) return AE_OK;
    Scratch &S = g_scratch;
    AE_CK(S.box.need(total));
    AE_CK(S.order.need(total));
    AE_CK(S.nodes.need(2ull * total));
    AE_CK(S.bad.need(1));
    AE_CK(cudaMemsetAsync(S.bad.p, 0, sizeof(int), st));
    for (uint32_t m = 0; m < k; m++) {
        const uint32_t tris = first[m + 1] - first[m];
        if (tris)
            k_triangle_boxes<<<(tris + 255) / 256, 256, 0, st>>>(d_v[m], nv[m], d_idx[m], tris, S.box.p + first[m],
                                                                  S.bad.p);
    }
    int h_bad = 0;
    AE_CK(cudaMemcpyAsync(&h_bad, S.bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    AE_CK(cudaStreamSynchronize(st));
    if (h_bad) return AE_ERR_LAYOUT;
    const int rc = gpu_build_forest(S.box.p, first.data(), k, S.nodes.p, S.order.p, out_counts, st, kWarpTask);
    if (rc != AE_OK) return rc;
    for (uint32_t m = 0; m < k; m++) {
        const uint32_t tris = first[m + 1] - first[m];
        if (!tris) continue;
        k_reorder_indices<<<(tris + 255) / 256, 256, 0, st>>>(d_idx[m], S.order.p + first[m], first[m], tris,
                                                               d_out_idx[m]);
        AE_CK(cudaMemcpyAsync(d_nodes[m], S.nodes.p + 2ull * first[m], size_t(out_counts[m]) * sizeof(ae_bvh_node),
                              cudaMemcpyDeviceToDevice, st));
    }
    AE_CK(cudaGetLastError());
    AE_CK(cudaStreamSynchronize(st));
    return AE_OK;
}

namespace {
struct OwnStream {
    cudaStream_t s = nullptr;
    cudaError_t make() { return cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking); }
    ~OwnStream() { if (s) cudaStreamDestroy(s); }
};
}  // namespace

// k meshes with host arrays (indices already checked against nv): staged
// into device buffers, built as one forest, copied back.  out_nodes[m] holds
// 2 * ni[m] / 3 nodes, out_indices[m] ni[m] indices.
int gpu_mesh_blas_many_host(uint32_t k, const ae_vertex *const *v, const uint32_t *nv, const uint32_t *const *idx,
                            const uint32_t *ni, ae_bvh_node *const *out_nodes, uint32_t *out_counts,
                            uint32_t *const *out_indices) {
    std::lock_guard<std::mutex> lock(g_mutex);
    OwnStream st;
    AE_CK(st.make());
    Scratch &S = g_scratch;
    std::vector<size_t> vo(size_t(k) + 1, 0), io(size_t(k) + 1, 0);
    for (uint32_t m = 0; m < k; m++) {
        vo[m + 1] = vo[m] + nv[m];
        io[m + 1] = io[m] + ni[m];
        if (ni[m] % 3 != 0) return AE_ERR_INVALID;
    }
    AE_CK(S.v.need(vo[k]));
    AE_CK(S.idx.need(io[k]));
    AE_CK(S.out_idx.need(io[k]));
    // Node room per mesh: 2 * tris, laid out like the forest's own array.
    Grow<ae_bvh_node> &staged = S.mesh_nodes;
    AE_CK(staged.need(2 * (io[k] / 3) + 1));
    std::vector<const ae_vertex *> dv(k);
    std::vector<const uint32_t *> di(k);
    std::vector<ae_bvh_node *> dn(k);
    std::vector<uint32_t *> dout(k);
    for (uint32_t m = 0; m < k; m++) {
        if (nv[m]) AE_CK(cudaMemcpyAsync(S.v.p + vo[m], v[m], size_t(nv[m]) * sizeof(ae_vertex), cudaMemcpyHostToDevice, st.s));
        if (ni[m]) AE_CK(cudaMemcpyAsync(S.idx.p + io[m], idx[m], size_t(ni[m]) * sizeof(uint32_t), cudaMemcpyHostToDevice, st.s));
        dv[m] = S.v.p + vo[m];
        di[m] = S.idx.p + io[m];
        dn[m] = staged.p + 2 * (io[m] / 3);
        dout[m] = S.out_idx.p + io[m];
    }
    const int rc = gpu_mesh_blas_many(k, dv.data(), nv, di.data(), ni, dn.data(), out_counts, dout.data(), st.s);
    if (rc != AE_OK) return rc;
    for (uint32_t m = 0; m < k; m++) {
        if (!ni[m]) continue;
        AE_CK(cudaMemcpyAsync(out_nodes[m], dn[m], size_t(out_counts[m]) * sizeof(ae_bvh_node), cudaMemcpyDeviceToHost, st.s));
        AE_CK(cudaMemcpyAsync(out_indices[m], dout[m], size_t(ni[m]) * sizeof(uint32_t), cudaMemcpyDeviceToHost, st.s));
    }
    AE_CK(cudaStreamSynchronize(st.s));
    return AE_OK;
}

// The same with host arrays (indices already checked against nv).
int gpu_mesh_blas(const ae_vertex *v, uint32_t nv, const uint32_t *idx, uint32_t ni, ae_bvh_node *out_nodes,
                  uint32_t *out_count, uint32_t *out_indices) {
    *out_count = 0;
    const uint32_t tris = ni / 3;
    if (tris == 0) return AE_OK;
    std::lock_guard<std::mutex> lock(g_mutex);
    OwnStream st;
    AE_CK(st.make());
    Scratch &S = g_scratch;
    AE_CK(S.v.need(nv));
    AE_CK(S.idx.need(ni));
    AE_CK(S.out_idx.need(ni));
    AE_CK(S.nodes.need(2ull * tris));
    AE_CK(cudaMemcpyAsync(S.v.p, v, size_t(nv) * sizeof(ae_vertex), cudaMemcpyHostToDevice, st.s));
    AE_CK(cudaMemcpyAsync(S.idx.p, idx, size_t(ni) * sizeof(uint32_t), cudaMemcpyHostToDevice, st.s));
    uint32_t count = 0;
    const int rc = gpu_mesh_blas_device(S.v.p, nv, S.idx.p, ni, S.nodes.p, &count, S.out_idx.p, st.s);
    if (rc != AE_OK) return rc;
    AE_CK(cudaMemcpyAsync(out_nodes, S.nodes.p, size_t(count) * sizeof(ae_bvh_node), cudaMemcpyDeviceToHost, st.s));
    AE_CK(cudaMemcpyAsync(out_indices, S.out_idx.p, size_t(ni) * sizeof(uint32_t), cudaMemcpyDeviceToHost, st.s));
    AE_CK(cudaStreamSynchronize(st.s));
    *out_count = count;
    return AE_OK;
}

// ae_pack_scene's per-entity part (host_scene.cpp).
int pack_templates(const ae_entity *ents, uint32_t n, const ae_mesh_library *lib, ae_aabb *bounds,
                   ae_object *objects, ae_instance *instances, uint32_t *flags);

}  // namespace ae

extern "C" int ae_pack_scene_gpu(const ae_entity *ents, uint32_t n, const ae_mesh_library *lib,
                                 ae_object *out_objects, ae_bvh_node *out_nodes, uint32_t *out_node_count,
                                 uint32_t *out_lights, uint32_t *out_light_count, ae_instance *out_instances,
                                 uint32_t *out_instance_count, uint32_t *out_order) {
    if (!out_node_count || !out_light_count || !out_instance_count) return AE_ERR_INVALID;
    *out_node_count = *out_light_count = *out_instance_count = 0;
    if (n == 0) return AE_OK;
    if (!ents || !out_objects || !out_nodes || !out_lights || !out_instances || !out_order) return AE_ERR_INVALID;
    std::vector<ae_aabb> bounds(n);
    std::vector<ae_object> obj_t(n);
    std::vector<ae_instance> inst_t(n);
    std::vector<uint32_t> flags(n);
    int rc = ae::pack_templates(ents, n, lib, bounds.data(), obj_t.data(), inst_t.data(), flags.data());
    if (rc != AE_OK) return rc;
    std::lock_guard<std::mutex> lock(ae::g_mutex);
    ae::OwnStream st;
    AE_CK(st.make());
    ae::Scratch &S = ae::g_scratch;
    if (S.box.need(n) != cudaSuccess || S.order.need(n) != cudaSuccess || S.nodes.need(2ull * n) != cudaSuccess ||
        S.obj_t.need(n) != cudaSuccess || S.objects.need(n) != cudaSuccess || S.inst_t.need(n) != cudaSuccess ||
        S.instances.need(n) != cudaSuccess || S.flags.need(n) != cudaSuccess || S.lights.need(n) != cudaSuccess ||
        S.counts.need(2) != cudaSuccess) {
        cudaGetLastError();
        return AE_ERR_OOM;
    }
    AE_CK(cudaMemcpyAsync(S.box.p, bounds.data(), size_t(n) * sizeof(ae_aabb), cudaMemcpyHostToDevice, st.s));
    AE_CK(cudaMemcpyAsync(S.obj_t.p, obj_t.data(), size_t(n) * sizeof(ae_object), cudaMemcpyHostToDevice, st.s));
    AE_CK(cudaMemcpyAsync(S.inst_t.p, inst_t.data(), size_t(n) * sizeof(ae_instance), cudaMemcpyHostToDevice, st.s));
    AE_CK(cudaMemcpyAsync(S.flags.p, flags.data(), size_t(n) * sizeof(uint32_t), cudaMemcpyHostToDevice, st.s));
    uint32_t nodes = 0;
    rc = ae::gpu_build_bvh(S.box.p, n, S.nodes.p, S.order.p, &nodes, st.s);
    if (rc != AE_OK) return rc;
    ae::k_assemble<<<1, 1024, 0, st.s>>>(n, S.order.p, S.flags.p, S.obj_t.p, S.inst_t.p, S.objects.p, S.instances.p,
                                         S.lights.p, S.counts.p);
    AE_CK(cudaGetLastError());
    uint32_t counts[2] = {0, 0};
    AE_CK(cudaMemcpyAsync(counts, S.counts.p, sizeof(counts), cudaMemcpyDeviceToHost, st.s));
    AE_CK(cudaStreamSynchronize(st.s));
    AE_CK(cudaMemcpyAsync(out_objects, S.objects.p, size_t(n) * sizeof(ae_object), cudaMemcpyDeviceToHost, st.s));
    AE_CK(cudaMemcpyAsync(out_nodes, S.nodes.p, size_t(nodes) * sizeof(ae_bvh_node), cudaMemcpyDeviceToHost, st.s));
    AE_CK(cudaMemcpyAsync(out_order, S.order.p, size_t(n) * sizeof(uint32_t), cudaMemcpyDeviceToHost, st.s));
    if (counts[0])
        AE_CK(cudaMemcpyAsync(out_instances, S.instances.p, size_t(counts[0]) * sizeof(ae_instance),
                              cudaMemcpyDeviceToHost, st.s));
    if (counts[1])
        AE_CK(cudaMemcpyAsync(out_lights, S.lights.p, size_t(counts[1]) * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                              st.s));
    AE_CK(cudaStreamSynchronize(st.s));
    *out_node_count = nodes;
    *out_instance_count = counts[0];
    *out_light_count = counts[1];
    return AE_OK;
}

extern "C" int ae_build_bvh_gpu_ex(const ae_aabb *bounds, uint32_t n, uint32_t warp_subtree, ae_bvh_node *out_nodes,
                                   uint32_t *out_node_count, uint32_t *out_order) {
    if (!out_node_count) return AE_ERR_INVALID;
    *out_node_count = 0;
    if (n == 0) return AE_OK;
    if (!bounds || !out_nodes || !out_order) return AE_ERR_INVALID;
    std::lock_guard<std::mutex> lock(ae::g_mutex);
    ae::OwnStream st;
    AE_CK(st.make());
    ae::Scratch &S = ae::g_scratch;
    if (S.box.need(n) != cudaSuccess || S.order.need(n) != cudaSuccess || S.nodes.need(2ull * n) != cudaSuccess) {
        cudaGetLastError();
        return AE_ERR_OOM;
    }
    AE_CK(cudaMemcpyAsync(S.box.p, bounds, size_t(n) * sizeof(ae_aabb), cudaMemcpyHostToDevice, st.s));
    uint32_t count = 0;
    const int rc = ae::gpu_build_bvh(S.box.p, n, S.nodes.p, S.order.p, &count, st.s, warp_subtree);
    if (rc != AE_OK) return rc;
    AE_CK(cudaMemcpyAsync(out_nodes, S.nodes.p, size_t(count) * sizeof(ae_bvh_node), cudaMemcpyDeviceToHost, st.s));
    AE_CK(cudaMemcpyAsync(out_order, S.order.p, size_t(n) * sizeof(uint32_t), cudaMemcpyDeviceToHost, st.s));
    AE_CK(cudaStreamSynchronize(st.s));
    *out_node_count = count;
    return AE_OK;
}

extern "C" int ae_build_bvh_gpu(const ae_aabb *bounds, uint32_t n, ae_bvh_node *out_nodes, uint32_t *out_node_count,
                                uint32_t *out_order) {
    return ae_build_bvh_gpu_ex(bounds, n, ae::kWarpTask, out_nodes, out_node_count, out_order);
}

extern "C" int ae_build_bvh_device(const ae_aabb *d_bounds, uint32_t n, uint32_t warp_subtree, ae_bvh_node *d_nodes,
                                   uint32_t *out_node_count, uint32_t *d_order, void *stream) {
    if (!out_node_count) return AE_ERR_INVALID;
    *out_node_count = 0;
    if (n == 0) return AE_OK;
    if (!d_bounds || !d_nodes || !d_order) return AE_ERR_INVALID;
    std::lock_guard<std::mutex> lock(ae::g_mutex);
    return ae::gpu_build_bvh(d_bounds, n, d_nodes, d_order, out_node_count, static_cast<cudaStream_t>(stream),
                             warp_subtree);
}

extern "C" int ae_mesh_blas_device(const ae_vertex *d_vertices, uint32_t nv, const uint32_t *d_indices, uint32_t ni,
                                   ae_bvh_node *d_nodes, uint32_t *out_node_count, uint32_t *d_out_indices,
                                   void *stream) {
    if (!out_node_count) return AE_ERR_INVALID;
    *out_node_count = 0;
    if (ni % 3 != 0) return AE_ERR_INVALID;
    if (ni == 0) return AE_OK;
    if (!d_vertices || !d_indices || !d_nodes || !d_out_indices) return AE_ERR_INVALID;
    std::lock_guard<std::mutex> lock(ae::g_mutex);
    return ae::gpu_mesh_blas_device(d_vertices, nv, d_indices, ni, d_nodes, out_node_count, d_out_indices,
                                    static_cast<cudaStream_t>(stream));
}

extern "C" int ae_mesh_blas_device_many(uint32_t k, const ae_vertex *const *d_vertices, const uint32_t *nv,
                                        const uint32_t *const *d_indices, const uint32_t *ni,
                                        ae_bvh_node *const *d_nodes, uint32_t *out_node_counts,
                                        uint32_t *const *d_out_indices, void *stream) {
    if (k && (!d_vertices || !nv || !d_indices || !ni || !d_nodes || !out_node_counts || !d_out_indices))
        return AE_ERR_INVALID;
    std::lock_guard<std::mutex> lock(ae::g_mutex);
    return ae::gpu_mesh_blas_many(k, d_vertices, nv, d_indices, ni, d_nodes, out_node_counts, d_out_indices,
                                  static_cast<cudaStream_t>(stream));
}

extern "C" void ae_bvh_builder_release(void) {
    std::lock_guard<std::mutex> lock(ae::g_mutex);
    ae::g_scratch.release();
}
