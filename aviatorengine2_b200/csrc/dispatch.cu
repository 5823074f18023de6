// dispatch.cu - kernel-family selection for closest hit, and the context's
// destructor (it owns the optimised structures).
#include "context.h"
#include "kernels.h"
#include "fast.h"

namespace ae {

Ctx::~Ctx() {
    destroy_fast(this);
    destroy_wavefront(this);
    destroy_deferred(this);
    destroy_refit(this);
    if (side_stream) cudaStreamDestroy(side_stream);
    if (side_stream2) cudaStreamDestroy(side_stream2);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (stream) cudaStreamDestroy(stream);
}

int prepare_variant(Ctx *c, int variant) {
    switch (variant) {
    case AE_VARIANT_PLAIN:
    case AE_VARIANT_PLAIN_WT: return AE_OK;
    case AE_VARIANT_PLAIN_CHECKED:
        if (!c->check_word.ptr) {
            if (c->check_word.reserve(1)) return c->fail(AE_ERR_OOM, "check word");
            return c->cuda(cudaMemset(c->check_word.ptr, 0, sizeof(uint32_t)), "check word");
        }
        return AE_OK;
    case AE_VARIANT_FAST:
    case AE_VARIANT_QUANT:
    case AE_VARIANT_FAST_WALK: return prepare_fast(c);
    default: return c->fail(AE_ERR_INVALID, "unknown kernel variant %d", variant);
    }
}

// The debug walk's limits: the uploaded arrays' true lengths and the walk's
// stack capacities, or (AE_FAULT_CHECK_LIMITS) stacks of 2 and half of every
// length, so the checks fire while every access made stays in bounds.
static Checks checks_of(const Ctx *c) {
    Checks C;
    C.flags = c->check_word.ptr;
    const bool lim = c->fault_check_limits != 0;
    C.n_nodes = lim ? c->n_nodes / 2 : c->n_nodes;
    C.n_objects = lim ? c->n_objects / 2 : c->n_objects;
    C.n_instances = lim ? c->n_instances / 2 : c->n_instances;
    C.n_blas = uint32_t(lim ? c->n_blas / 2 : c->n_blas);
    C.n_indices = uint32_t(lim ? c->n_indices / 2 : c->n_indices);
    C.n_vertices = uint32_t(lim ? c->n_vertices / 2 : c->n_vertices);
    C.tlas_stack = lim ? 2 : kTlasStack;
    C.blas_stack = lim ? 2 : kBlasStack;
    return C;
}

int closest_hit_dispatch(Ctx *c, const ae_ray *rays, uint32_t n, ae_hit *hits, int variant, cudaStream_t st,
                         bool timed) {
    int rc = prepare_variant(c, variant);
    if (rc) return rc;
    if (n == 0) return AE_OK;
    // The kernels read a ray as two 16-byte loads.
    if (reinterpret_cast<uintptr_t>(rays) & 15u)
        return c->fail(AE_ERR_INVALID, "device rays must start on a 16-byte boundary");
    if (timed && (rc = c->cuda(cudaEventRecord(c->ev0, st), "event"))) return rc;
    cudaError_t e;
    if (variant == AE_VARIANT_PLAIN || variant == AE_VARIANT_PLAIN_WT)
        e = launch_closest_plain(c->scene(), rays, n, hits, st, variant == AE_VARIANT_PLAIN_WT);
    else if (variant == AE_VARIANT_PLAIN_CHECKED) e = launch_closest_checked(c->scene(), checks_of(c), rays, n, hits, st);
    else if (variant == AE_VARIANT_FAST_WALK) e = launch_closest_walk(c, rays, n, hits, st);
    else e = launch_closest_fast(c, rays, n, hits, variant == AE_VARIANT_QUANT, st);
    if ((rc = c->cuda(e, "closest hit launch"))) return rc;
    c->launches++;
    if (timed) {
        c->timed = true;
        if ((rc = c->cuda(cudaEventRecord(c->ev1, st), "event"))) return rc;
    }
    return AE_OK;
}

}  // namespace ae

static int trace_counters(ae::Ctx *c, const ae_ray *d_rays, uint32_t n, int variant, uint64_t *counters) {
    if (!c->scene_uploaded) return c->fail(AE_ERR_STATE, "counters before ae_upload_scene");
    if (reinterpret_cast<uintptr_t>(d_rays) & 15u)
        return c->fail(AE_ERR_INVALID, "device rays must start on a 16-byte boundary");
    if (variant != AE_VARIANT_PLAIN && variant != AE_VARIANT_FAST && variant != AE_VARIANT_QUANT)
        return c->fail(AE_ERR_INVALID, "touch counters exist for PLAIN, FAST and QUANT (got variant %d)", variant);
    int rc = ae::prepare_variant(c, variant);
    if (rc) return rc;
    ae::DevBuf<unsigned long long> tot;
    if (tot.reserve(6)) return c->fail(AE_ERR_OOM, "counter buffer");
    rc = c->cuda(cudaMemsetAsync(tot.ptr, 0, 6 * sizeof(unsigned long long), c->stream), "memset");
    if (!rc)
        rc = c->cuda(variant == AE_VARIANT_PLAIN
                         ? ae::launch_count_plain(c->scene(), d_rays, n, tot.ptr, c->stream)
                         : ae::launch_count_fast(c, d_rays, n, variant == AE_VARIANT_QUANT, tot.ptr, c->stream),
                     "count launch");
    c->launches++;
    if (!rc) rc = c->cuda(cudaMemcpyAsync(counters, tot.ptr, 6 * sizeof(uint64_t), cudaMemcpyDeviceToHost, c->stream), "copy");
    if (!rc) rc = c->cuda(cudaStreamSynchronize(c->stream), "counters");
    return rc;
}

extern "C" int ae_trace_counters(ae_ctx *ctx, const ae_ray *d_rays, uint32_t n, uint64_t *counters) {
    ae::Ctx *c = reinterpret_cast<ae::Ctx *>(ctx);
    if (!c || !counters || (n && !d_rays)) return AE_ERR_INVALID;
    return trace_counters(c, d_rays, n, AE_VARIANT_PLAIN, counters);
}

extern "C" int ae_trace_counters_variant(ae_ctx *ctx, const ae_ray *d_rays, uint32_t n, int variant,
                                         uint64_t *counters) {
    ae::Ctx *c = reinterpret_cast<ae::Ctx *>(ctx);
    if (!c || !counters || (n && !d_rays)) return AE_ERR_INVALID;
    return trace_counters(c, d_rays, n, variant, counters);
}

extern "C" int ae_path_counters(ae_ctx *ctx, uint64_t *counters) {
    ae::Ctx *c = reinterpret_cast<ae::Ctx *>(ctx);
    if (!c || !counters) return AE_ERR_INVALID;
    if (!c->scene_uploaded || !c->geometry_uploaded) return c->fail(AE_ERR_STATE, "path counters before the uploads");
    const ae::FrameParams F = ae::make_frame_params(c->config);
    ae::DevBuf<unsigned long long> tot;
    if (tot.reserve(7)) return c->fail(AE_ERR_OOM, "counter buffer");
    int rc = c->cuda(cudaMemsetAsync(tot.ptr, 0, 7 * sizeof(unsigned long long), c->stream), "memset");
    if (!rc) rc = c->cuda(ae::launch_count_paths(c->scene(), F, tot.ptr, c->stream), "count launch");
    c->launches++;
    if (!rc) rc = c->cuda(cudaMemcpyAsync(counters, tot.ptr, 7 * sizeof(uint64_t), cudaMemcpyDeviceToHost, c->stream), "copy");
    if (!rc) rc = c->cuda(cudaStreamSynchronize(c->stream), "path counters");
    return rc;
}

extern "C" int ae_prepare_fast(ae_ctx *ctx) {
    ae::Ctx *c = reinterpret_cast<ae::Ctx *>(ctx);
    if (!c) return AE_ERR_INVALID;
    return ae::prepare_fast(c);
}
