// TEST INFRASTRUCTURE ONLY (oracle).  Runs the reference's hybrid compute
// passes - shaders/deferred.comp.hlsl and shaders/upsample.comp.hlsl,
// transpiled by hlsl2cpp.py into _ref/deferred.inc and _ref/upsample.inc - on
// the CPU, one invocation per cell or pixel, over caller-provided G-buffer and
// history planes (all float4 per texel; depth one float).  The library never
// uses this; tests compare the oracle restatement and the kernels with it.
#include <omp.h>

#include <cstring>

#include "../include/ae_b200.h"
#include "hlsl_shim.h"

namespace hlsl {
namespace d {
#include "_ref/deferred.inc"
}
namespace u {
#include "_ref/upsample.inc"
}
}  // namespace hlsl

namespace {

template <class NS_Config>
void dummy(NS_Config) {}

#define AE_SET_CONFIG(NS)                                                        \
    NS::Source = float3(c->source_x, c->source_y, c->source_z);                  \
    NS::Fov = c->fov;                                                            \
    NS::Target = float3(c->target_x, c->target_y, c->target_z);                  \
    NS::Focus = c->focus_dist;                                                   \
    NS::Defocus_angle = c->defocus_angle;                                        \
    NS::Up = float3(c->up_x, c->up_y, c->up_z);                                  \
    NS::Sky = float3(c->sky_r, c->sky_g, c->sky_b);                              \
    NS::Width = c->width;                                                        \
    NS::Horizon = float3(c->horizon_r, c->horizon_g, c->horizon_b);              \
    NS::Height = c->height;                                                      \
    NS::Samples = c->samples;                                                    \
    NS::Batches = c->batches;                                                    \
    NS::Batch = c->batch;                                                        \
    NS::Depth = c->depth;                                                        \
    NS::NumLights = c->num_lights;                                               \
    NS::Exposure = c->exposure;                                                  \
    NS::DebugView = c->debugView;                                                \
    NS::ZNear = c->zNear;                                                        \
    NS::ZFar = c->zFar;                                                          \
    NS::JitterX = c->jitter_x;                                                   \
    NS::JitterY = c->jitter_y;                                                   \
    NS::DisplayOnly = c->displayOnly;                                            \
    NS::TraceScale = c->traceScale;                                              \
    NS::FrameIndex = c->frameIndex;                                              \
    NS::HistoryReset = c->historyReset;                                          \
    NS::CameraMoved = c->cameraMoved;                                            \
    NS::HistoryCap = c->historyCap;                                              \
    for (int r = 0; r < 4; r++)                                                  \
        for (int k = 0; k < 4; k++) NS::PrevViewProj.m[r][k] = c->prevViewProj[4 * r + k];

template <class T> void bind_tex(hlsl::Texture2D<T> &t, const void *data, uint32_t w, uint32_t h) {
    t.data = static_cast<const T *>(data);
    t.width = w;
    t.height = h;
}
template <class T> void bind_rw(hlsl::RWTexture2D<T> &t, void *data, uint32_t w, uint32_t h) {
    t.data = static_cast<T *>(data);
    t.width = w;
    t.height = h;
}

}  // namespace

extern "C" {

void aeref_d_bind(const ae_object *objects, uint32_t n_objects, const ae_bvh_node *tlas, uint32_t n_nodes,
                  const uint32_t *lights, uint32_t n_lights, const ae_vertex *vertices, uint32_t nv,
                  const uint32_t *indices, uint32_t ni, const ae_bvh_node *blas, uint32_t nb,
                  const ae_instance *instances, uint32_t n_instances) {
    using namespace hlsl;
    d::objects.data = reinterpret_cast<const d::Object *>(objects);
    d::bvh.data = reinterpret_cast<const d::BVHNode *>(tlas);
    d::lightIDs.data = lights;
    d::vertices.data = reinterpret_cast<const d::Vertex *>(vertices);
    d::meshIndex.data = indices;
    d::blas.data = reinterpret_cast<const d::BVHNode *>(blas);
    d::instances.data = reinterpret_cast<const d::MeshInstance *>(instances);
    u::objects.data = reinterpret_cast<const u::Object *>(objects);
    u::instances.data = reinterpret_cast<const u::MeshInstance *>(instances);
    (void)n_objects; (void)n_nodes; (void)n_lights; (void)nv; (void)ni; (void)nb; (void)n_instances;
}

// The material texture array (GlobalTextureArray): RGBA8 sRGB words.
void aeref_d_bind_textures(const uint32_t *texels, uint32_t width, uint32_t height, uint32_t layers) {
    hlsl::d::GlobalTextureArray.texels = texels;
    hlsl::d::GlobalTextureArray.width = width;
    hlsl::d::GlobalTextureArray.height = height;
    hlsl::d::GlobalTextureArray.layers = layers;
}

void aeref_d_set_config(const ae_config *c) {
    using namespace hlsl;
    AE_SET_CONFIG(d)
    AE_SET_CONFIG(u)
}

// planes: gpos, gnrm, galb (float4 = byte/255), gdepth (float), prev_img,
// prev_geo (read); img, display, reduced, cur_geo (written).  reduced is
// red_w x red_h float4.
void aeref_deferred(const float *gpos, const float *gnrm, const float *galb, const float *gdepth,
                    const float *prev_img, const float *prev_geo, float *img, float *display, float *reduced,
                    uint32_t red_w, uint32_t red_h, float *cur_geo, int threads) {
    using namespace hlsl;
    if (threads > 0) omp_set_num_threads(threads);
    const uint32_t W = d::Width, H = d::Height;
    bind_tex(d::gPosition, gpos, W, H);
    bind_tex(d::gNormal, gnrm, W, H);
    bind_tex(d::gAlbedo, galb, W, H);
    bind_tex(d::gDepth, gdepth, W, H);
    bind_tex(d::previousImage, prev_img, W, H);
    bind_tex(d::previousGeometry, prev_geo, W, H);
    bind_rw(d::image, img, W, H);
    bind_rw(d::displayImage, display, W, H);
    bind_rw(d::lightingReduced, reduced, red_w, red_h);
    bind_rw(d::currentGeometry, cur_geo, W, H);
    const bool reduced_grid = d::TraceScale < 1.0f;
    const uint32_t ew = reduced_grid ? red_w : W, eh = reduced_grid ? red_h : H;
#pragma omp parallel for schedule(dynamic, 1)
    for (int y = 0; y < int(eh); y++)
        for (uint32_t x = 0; x < ew; x++) d::main(uint3(x, uint32_t(y), 0u));
}

void aeref_upsample(const float *gpos, const float *gnrm, const float *galb, const float *reduced, uint32_t red_w,
                    uint32_t red_h, const float *prev_img, const float *prev_geo, float *img, float *display,
                    float *cur_geo, int threads) {
    using namespace hlsl;
    if (threads > 0) omp_set_num_threads(threads);
    const uint32_t W = u::Width, H = u::Height;
    bind_tex(u::gPosition, gpos, W, H);
    bind_tex(u::gNormal, gnrm, W, H);
    bind_tex(u::gAlbedo, galb, W, H);
    bind_tex(u::lightingReduced, reduced, red_w, red_h);
    bind_tex(u::previousImage, prev_img, W, H);
    bind_tex(u::previousGeometry, prev_geo, W, H);
    bind_rw(u::image, img, W, H);
    bind_rw(u::displayImage, display, W, H);
    bind_rw(u::currentGeometry, cur_geo, W, H);
#pragma omp parallel for schedule(dynamic, 1)
    for (int y = 0; y < int(H); y++)
        for (uint32_t x = 0; x < W; x++) u::main(uint3(x, uint32_t(y), 0u));
}

}  // extern "C"
