// TEST INFRASTRUCTURE ONLY (oracle).  Runs the reference's compute-only
// shader (shaders/ray_trace.comp.hybrid.hlsl, transpiled by hlsl2cpp.py into
// _ref/hybrid.inc) on the CPU, one invocation per pixel or per ray, so the
// oracle restatement can be checked against the reference's own code on the
// same inputs.  Used by tests and by bench.py's CPU baseline, never by the
// library.
#include <omp.h>

#include <cstring>

#include "../include/ae_b200.h"
#include "hlsl_shim.h"

namespace hlsl {
#include "_ref/hybrid.inc"
}

static_assert(sizeof(hlsl::Object) == sizeof(ae_object), "Object stride");
static_assert(sizeof(hlsl::BVHNode) == sizeof(ae_bvh_node), "BVHNode stride");
static_assert(sizeof(hlsl::MeshInstance) == sizeof(ae_instance), "MeshInstance stride");
static_assert(sizeof(hlsl::Vertex) == sizeof(ae_vertex), "Vertex stride");

extern "C" {

void aeref_bind(const ae_object *objects, uint32_t n_objects, const ae_bvh_node *tlas, uint32_t n_nodes,
                const uint32_t *lights, uint32_t n_lights, const ae_vertex *vertices, uint32_t nv,
                const uint32_t *indices, uint32_t ni, const ae_bvh_node *blas, uint32_t nb,
                const ae_instance *instances, uint32_t n_instances) {
    hlsl::objects.data = reinterpret_cast<const hlsl::Object *>(objects);
    hlsl::objects.count = n_objects;
    hlsl::bvh.data = reinterpret_cast<const hlsl::BVHNode *>(tlas);
    hlsl::bvh.count = n_nodes;
    hlsl::lightIDs.data = lights;
    hlsl::lightIDs.count = n_lights;
    hlsl::vertices.data = reinterpret_cast<const hlsl::Vertex *>(vertices);
    hlsl::vertices.count = nv;
    hlsl::meshIndex.data = indices;
    hlsl::meshIndex.count = ni;
    hlsl::blas.data = reinterpret_cast<const hlsl::BVHNode *>(blas);
    hlsl::blas.count = nb;
    hlsl::instances.data = reinterpret_cast<const hlsl::MeshInstance *>(instances);
    hlsl::instances.count = n_instances;
}

// The material texture array (GlobalTextureArray): RGBA8 sRGB words.
void aeref_bind_textures(const uint32_t *texels, uint32_t width, uint32_t height, uint32_t layers) {
    hlsl::GlobalTextureArray.texels = texels;
    hlsl::GlobalTextureArray.width = width;
    hlsl::GlobalTextureArray.height = height;
    hlsl::GlobalTextureArray.layers = layers;
}

// One texture sample through the shader's own binding (test of the sampler).
void aeref_sample_texture(float u, float v, uint32_t layer, float *rgb) {
    const hlsl::float4 t = hlsl::GlobalTextureArray.SampleLevel(hlsl::GlobalSampler, hlsl::float3(u, v, float(layer)), 0.0f);
    rgb[0] = t.x; rgb[1] = t.y; rgb[2] = t.z;
}

void aeref_set_config(const ae_config *c) {
    using namespace hlsl;
    Source = float3(c->source_x, c->source_y, c->source_z);
    Fov = c->fov;
    Target = float3(c->target_x, c->target_y, c->target_z);
    Focus = c->focus_dist;
    Defocus_angle = c->defocus_angle;
    Up = float3(c->up_x, c->up_y, c->up_z);
    Oof = c->oof;
    Sky = float3(c->sky_r, c->sky_g, c->sky_b);
    Width = c->width;
    Horizon = float3(c->horizon_r, c->horizon_g, c->horizon_b);
    Height = c->height;
    Samples = c->samples;
    Batches = c->batches;
    Batch = c->batch;
    Depth = c->depth;
    NumSpheres = c->num_spheres;
    RenderType = c->renderType;
    NumLights = c->num_lights;
    Exposure = c->exposure;
    DisplayOnly = c->displayOnly;
}

// TraverseBVH(ray, ray.tnear) per ray (hybrid:862-917).
void aeref_closest_hit(const ae_ray *rays, uint32_t n, ae_hit *hits, int threads) {
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t i = 0; i < int64_t(n); i++) {
        const ae_ray &r = rays[i];
        hlsl::seed = 1u;
        hlsl::Ray ray;
        ray.Origin = hlsl::float3(r.ox, r.oy, r.oz);
        ray.Direction = hlsl::float3(r.dx, r.dy, r.dz);
        ray.time = r.time;
        hlsl::Hit h;
        ae_hit out{0.0f, 0.0f, 0.0f, AE_MISS, AE_MISS};
        if (hlsl::TraverseBVH(ray, r.tnear, h)) {
            out.t = h.Offset;
            out.object = h.aeObjSlot;
            if (h.aeTriBase != 0xFFFFFFFFu) {
                const hlsl::MeshInstance &inst = hlsl::instances[h.Object.InstanceIndex];
                out.prim = (h.aeTriBase - inst.indexBase) / 3u;
                out.alpha = h.aeAlpha;
                out.beta = h.aeBeta;
            } else {
                out.alpha = h.surface_uv.x;
                out.beta = h.surface_uv.y;
            }
        }
        hits[i] = out;
    }
}

// The shader's main for every pixel (hybrid:1328-1404).  image/display are
// width*height float4; image holds the running accumulation in and out.
void aeref_render(float *image, float *display, int threads) {
    if (threads > 0) omp_set_num_threads(threads);
    hlsl::image.data = reinterpret_cast<hlsl::float4 *>(image);
    hlsl::image.width = hlsl::Width;
    hlsl::image.height = hlsl::Height;
    hlsl::displayImage.data = reinterpret_cast<hlsl::float4 *>(display);
    hlsl::displayImage.width = hlsl::Width;
    hlsl::displayImage.height = hlsl::Height;
    const int w = int(hlsl::Width), h = int(hlsl::Height);
#pragma omp parallel for schedule(dynamic, 1)
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) hlsl::main(hlsl::uint3(uint32_t(x), uint32_t(y), 0u));
}

// The same invocation for an explicit list of pixels (a bounded sample).
void aeref_render_pixels(const uint32_t *xy, uint32_t n, float *image, float *display, int threads) {
    if (threads > 0) omp_set_num_threads(threads);
    hlsl::image.data = reinterpret_cast<hlsl::float4 *>(image);
    hlsl::image.width = hlsl::Width;
    hlsl::image.height = hlsl::Height;
    hlsl::displayImage.data = reinterpret_cast<hlsl::float4 *>(display);
    hlsl::displayImage.width = hlsl::Width;
    hlsl::displayImage.height = hlsl::Height;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < int64_t(n); i++) hlsl::main(hlsl::uint3(xy[2 * i], xy[2 * i + 1], 0u));
}

}  // extern "C"
