// fast.h - entry points of the optimised closest-hit path and the other
// kernel families that own per-context state.
#pragma once
#include "context.h"

namespace ae {
int prepare_fast(Ctx *c);
int prepare_precision(Ctx *c);
void destroy_fast(Ctx *c);
cudaError_t launch_closest_fast(Ctx *c, const ae_ray *rays, uint32_t n, ae_hit *hits, bool quant, cudaStream_t st);
cudaError_t launch_closest_walk(Ctx *c, const ae_ray *rays, uint32_t n, ae_hit *hits, cudaStream_t st);
cudaError_t launch_count_fast(Ctx *c, const ae_ray *rays, uint32_t n, bool quant, unsigned long long *totals,
                              cudaStream_t st);
void destroy_wavefront(Ctx *c);
void destroy_deferred(Ctx *c);
void destroy_refit(Ctx *c);
// World box of an analytic (non-mesh) object record, as the scene packer
// computes it (refit.cu).
ae_aabb analytic_box(const ae_object &o);
}  // namespace ae
