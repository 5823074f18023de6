// context.cu - the device context behind the C ABI: the Renderer of
// renderer/renderer.h:325-603 without a window.  It owns the scene's device
// buffers (sized once, like CreateSceneBuffers, renderer/renderer.cpp:553-628),
// the accumulation/display images, one CUDA stream, and the derived
// structures of the optimised kernels.
//
// Every upload is validated on the host before it reaches the device: a
// kernel must never be handed an index that leaves its buffers.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "context.h"
#include "kernels.h"
#include "trace_common.cuh"

using namespace ae;

namespace ae {

// Device allocations (devmem.h): live count and the failure injected by
// ae_debug_fail_alloc_after (the n-th call from now fails; -1 = none).
static std::atomic<long long> g_fail_after{-1};
static std::atomic<long long> g_live_allocations{0};

cudaError_t dev_alloc(void **p, size_t bytes) {
    long long n = g_fail_after.load();
    while (n >= 0 && !g_fail_after.compare_exchange_weak(n, n - 1)) {
    }
    if (n == 0) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    const cudaError_t e = cudaMalloc(p, bytes);
    if (e == cudaSuccess && *p) g_live_allocations++;
    return e;
}

void dev_free(void *p) {
    if (!p) return;
    cudaFree(p);
    g_live_allocations--;
}

static thread_local int g_create_status = AE_OK;
void set_create_status(int status) { g_create_status = status; }
int create_status() { return g_create_status; }

int Ctx::fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    err = buf;
    return code;
}

int Ctx::cuda(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return AE_OK;
    return fail(AE_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

DevScene Ctx::scene() const {
    DevScene S;
    S.objects = objects.ptr;
    S.tlas = tlas.ptr;
    S.lights = lights.ptr;
    S.vertices = vertices.ptr;
    S.indices = indices.ptr;
    S.blas = blas.ptr;
    S.instances = instances.ptr;
    S.n_objects = n_objects;
    S.n_nodes = n_nodes;
    S.n_lights = n_lights;
    S.n_instances = n_instances;
    S.tex = tex.ptr;
    S.srgb = srgb_lut.ptr;
    S.tex_w = tex_w;
    S.tex_h = tex_h;
    S.tex_layers = tex_layers;
    return S;
}

int Ctx::timed_begin() { return cuda(cudaEventRecord(ev0, stream), "cudaEventRecord"); }
int Ctx::timed_end() {
    launches++;
    timed = true;
    return cuda(cudaEventRecord(ev1, stream), "cudaEventRecord");
}

// Camera basis and per-frame constants of main, hybrid:1346-1373.
FrameParams make_frame_params(const ae_config &c) {
    FrameParams F;
    std::memset(&F, 0, sizeof(F));
    F.width = c.width;
    F.height = c.height;
    F.batch = c.batch;
    const uint32_t per = c.batches ? c.samples / c.batches : c.samples;
    F.spp = per > 1u ? per : 1u;
    F.depth = c.depth;
    F.display_only = c.displayOnly;
    F.frame_index = c.frameIndex;
    F.exposure = c.exposure;
    F.defocus_angle = c.defocus_angle;
    F.source = mk(c.source_x, c.source_y, c.source_z);
    const f3 target = mk(c.target_x, c.target_y, c.target_z), up = mk(c.up_x, c.up_y, c.up_z);
    const f3 w = normalize(F.source - target);
    const f3 u = normalize(cross(up, w));
    const f3 v = cross(w, u);
    const float vh = AE_MUL(AE_MUL(2.0f, tanf_(radians(AE_DIV(c.fov, 2.0f)))), c.focus_dist);
    const float vw = AE_DIV(AE_MUL(vh, AE_U2F(c.width)), AE_U2F(c.height));
    const f3 vu = vw * u, vv = vh * -v;
    F.pixel_u = vu / AE_U2F(c.width);
    F.pixel_v = vv / AE_U2F(c.height);
    F.pixel0 = F.source - c.focus_dist * w - vu / 2.0f - vv / 2.0f + F.pixel_u / 2.0f + F.pixel_v / 2.0f;
    const float dr = AE_MUL(c.focus_dist, tanf_(radians(AE_DIV(c.defocus_angle, 2.0f))));
    F.defocus_u = u * dr;
    F.defocus_v = v * dr;
    F.sky = mk(c.sky_r, c.sky_g, c.sky_b);
    F.cam_u = u;
    F.cam_v = v;
    F.cam_w = w;
    return F;
}

}  // namespace ae

namespace {

template <class T> int upload(Ctx *c, DevBuf<T> &buf, const T *src, size_t n, const char *what) {
    if (n == 0) return AE_OK;
    int rc = buf.reserve(n);
    if (rc != AE_OK) return c->fail(rc, "cudaMalloc(%s, %zu elements) failed", what, n);
    return c->cuda(cudaMemcpyAsync(buf.ptr, src, n * sizeof(T), cudaMemcpyHostToDevice, c->stream), what);
}

// Walks a tree exactly as the kernels' depth-first loop does (pop one, push
// left then right) and checks that every node it reaches lies in
// [base, base + limit_nodes), every leaf addresses primitives below
// leaf_limit, the stack never exceeds stack_cap and no node is reached twice
// (no cycles).  Returns an empty string when the tree is safe to traverse.
std::string check_tree(const ae_bvh_node *nodes, uint64_t base, uint64_t limit_nodes, uint64_t leaf_limit,
                       int stack_cap) {
    if (limit_nodes == 0) return "empty tree";
    std::vector<int64_t> stack;
    std::vector<uint8_t> seen(limit_nodes, 0);
    stack.push_back(0);
    size_t max_sp = 1;
    while (!stack.empty()) {
        const int64_t rel = stack.back();
        stack.pop_back();
        if (rel < 0 || uint64_t(rel) >= limit_nodes) return "node link outside its tree";
        if (seen[rel]++) return "node reached twice";
        const ae_bvh_node &n = nodes[base + rel];
        if (n.count > 0) {
            if (n.left < 0 || uint64_t(n.left) + uint64_t(n.count) > leaf_limit) return "leaf range outside its primitives";
        } else {
            stack.push_back(n.left);
            stack.push_back(n.right);
            max_sp = std::max(max_sp, stack.size());
        }
    }
    if (max_sp > size_t(stack_cap)) return "tree too deep for the traversal stack";
    return "";
}

int validate_scene(Ctx *c, const ae_object *objects, uint32_t n_objects, const ae_bvh_node *tlas, uint32_t n_nodes,
                   const uint32_t *lights, uint32_t n_lights, const ae_instance *inst, uint32_t n_inst) {
    if (n_nodes) {
        const std::string e = check_tree(tlas, 0, n_nodes, n_objects, ae::kTlasStack);
        if (!e.empty()) return c->fail(AE_ERR_LAYOUT, "TLAS: %s", e.c_str());
    }
    for (uint32_t i = 0; i < n_lights; i++)
        if (lights[i] >= n_objects) return c->fail(AE_ERR_LAYOUT, "light %u -> object %u of %u", i, lights[i], n_objects);
    for (uint32_t i = 0; i < n_objects; i++) {
        const ae_object &o = objects[i];
        if (o.shapeType > AE_SHAPE_MESH) return c->fail(AE_ERR_LAYOUT, "object %u has shape %u", i, o.shapeType);
        if (o.shapeType == AE_SHAPE_MESH && o.instanceIndex >= n_inst)
            return c->fail(AE_ERR_LAYOUT, "object %u -> instance %u of %u", i, o.instanceIndex, n_inst);
    }
    for (uint32_t i = 0; i < n_inst; i++) {
        const ae_instance &m = inst[i];
        const auto key = std::make_tuple(m.vertexBase, m.indexBase, m.triangleCount, m.blasBase);
        if (c->checked_meshes.count(key)) continue;
        if (uint64_t(m.indexBase) + 3ull * m.triangleCount > c->n_indices)
            return c->fail(AE_ERR_LAYOUT, "instance %u: triangles outside the index buffer", i);
        if (m.triangleCount == 0 || m.blasBase >= c->n_blas)
            return c->fail(AE_ERR_LAYOUT, "instance %u: BLAS root %u outside %llu nodes", i, m.blasBase,
                           (unsigned long long)c->n_blas);
        const std::string e = check_tree(c->host_blas.data(), m.blasBase, c->n_blas - m.blasBase, m.triangleCount,
                                         ae::kBlasStack);
        if (!e.empty()) return c->fail(AE_ERR_LAYOUT, "instance %u BLAS: %s", i, e.c_str());
        for (uint64_t k = m.indexBase; k < uint64_t(m.indexBase) + 3ull * m.triangleCount; k++)
            if (uint64_t(m.vertexBase) + c->host_indices[k] >= c->n_vertices)
                return c->fail(AE_ERR_LAYOUT, "instance %u: vertex index outside the vertex buffer", i);
        c->checked_meshes[key] = true;
    }
    return AE_OK;
}

}  // namespace

extern "C" {

ae_ctx *ae_create(const ae_settings *s) {
    ae::set_create_status(AE_OK);
    if (!s || s->width == 0 || s->height == 0) {
        fprintf(stderr, "ae_create: invalid settings\n");
        ae::set_create_status(AE_ERR_INVALID);
        return nullptr;
    }
    Ctx *c = new (std::nothrow) Ctx();
    if (!c) {
        ae::set_create_status(AE_ERR_OOM);
        return nullptr;
    }
    c->settings = *s;
    if (c->settings.trace_scale <= 0.0f) c->settings.trace_scale = 1.0f;
    if (c->settings.hybrid_max_depth == 0) c->settings.hybrid_max_depth = 3;
    if (c->settings.history_while_moving == 0) c->settings.history_while_moving = 32;
    cudaError_t e = cudaSetDevice(s->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&c->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&c->ev1);
    if (e != cudaSuccess) {
        fprintf(stderr, "ae_create: %s\n", cudaGetErrorString(e));
        cudaGetLastError();
        delete c;
        ae::set_create_status(AE_ERR_CUDA);
        return nullptr;
    }
    // Config defaults of Renderer::Initialize (renderer/renderer.cpp:104-120).
    std::memset(&c->config, 0, sizeof(c->config));
    c->config.width = s->width;
    c->config.height = s->height;
    c->config.samples = s->samples ? s->samples : 1;
    c->config.batches = 1;
    c->config.up_y = 1.0f;
    c->config.exposure = 0.1f;
    c->config.fov = 40.0f;
    c->config.focus_dist = 1.0f;
    c->config.depth = 8;
    c->config.traceScale = c->settings.trace_scale;
    c->config.historyCap = float(c->settings.history_while_moving);
    const size_t px = size_t(s->width) * s->height;
    if (c->accum.reserve(px) || c->frame.reserve(px) || c->display.reserve(px)) {
        fprintf(stderr, "ae_create: image allocation failed\n");
        delete c;
        ae::set_create_status(AE_ERR_OOM);
        return nullptr;
    }
    cudaMemsetAsync(c->accum.ptr, 0, px * sizeof(float4), c->stream);
    cudaMemsetAsync(c->frame.ptr, 0, px * sizeof(float4), c->stream);
    cudaMemsetAsync(c->display.ptr, 0, px * sizeof(uchar4), c->stream);
    return reinterpret_cast<ae_ctx *>(c);
}

void ae_destroy(ae_ctx *ctx) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return;
    cudaSetDevice(c->settings.device);
    cudaStreamSynchronize(c->stream);
    delete c;
}

const char *ae_last_error(const ae_ctx *ctx) {
    const Ctx *c = reinterpret_cast<const Ctx *>(ctx);
    return c ? c->err.c_str() : "null context";
}

int ae_upload_geometry(ae_ctx *ctx, const ae_vertex *v, uint32_t nv, const uint32_t *idx, uint32_t ni,
                       const ae_bvh_node *blas, uint32_t nb) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return AE_ERR_INVALID;
    if ((nv && !v) || (ni && !idx) || (nb && !blas) || ni % 3) return c->fail(AE_ERR_INVALID, "bad geometry arguments");
    // BLAS links are mesh-relative, so each tree is checked when an instance
    // first names it (validate_scene).
    c->checked_meshes.clear();
    c->n_vertices = nv;
    c->n_indices = ni;
    c->n_blas = nb;
    int rc;
    if ((rc = upload(c, c->vertices, v, nv, "vertices")) || (rc = upload(c, c->indices, idx, ni, "indices")) ||
        (rc = upload(c, c->blas, blas, nb, "blas")))
        return rc;
    c->host_indices.assign(idx, idx + ni);
    c->host_blas.assign(blas, blas + nb);
    c->host_vertices.assign(v, v + nv);
    c->fast_ready = false;
    // The optimised structures and any captured frame graph derive from the
    // old geometry: both are rebuilt on next use.
    c->geometry_version++;
    c->scene_version++;
    c->geometry_uploaded = true;
    return c->cuda(cudaStreamSynchronize(c->stream), "upload geometry");
}

// The material texture array: TextureLibrary::BuildGPUArray's result
// (scene/texture.h:110-230) as plain bytes, plus the 256-entry sRGB decode
// table every sample uses.
int ae_upload_textures(ae_ctx *ctx, const uint8_t *texels, uint32_t width, uint32_t height, uint32_t layers) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return AE_ERR_INVALID;
    if (layers && (!texels || !width || !height)) return c->fail(AE_ERR_INVALID, "bad texture array arguments");
    if (layers && (width > 2048u || height > 2048u))
        return c->fail(AE_ERR_OVERSIZE, "texture layers are at most 2048x2048 (kMaxTextureArrayDimension)");
    if (layers > 2048u) return c->fail(AE_ERR_OVERSIZE, "at most 2048 texture layers");
    cudaSetDevice(c->settings.device);
    if (!c->srgb_lut.ptr) {
        float lut[256];
        for (uint32_t b = 0; b < 256; b++) lut[b] = srgb_to_linear(b);
        int rc;
        if (c->srgb_lut.reserve(256)) return c->fail(AE_ERR_OOM, "sRGB table");
        if ((rc = c->cuda(cudaMemcpyAsync(c->srgb_lut.ptr, lut, sizeof(lut), cudaMemcpyHostToDevice, c->stream),
                          "upload sRGB table")))
            return rc;
        if ((rc = c->cuda(cudaStreamSynchronize(c->stream), "upload sRGB table"))) return rc;
    }
    const size_t words = size_t(width) * height * layers;
    int rc = upload(c, c->tex, reinterpret_cast<const uint32_t *>(texels), words, "textures");
    if (rc) return rc;
    c->tex_w = layers ? width : 0;
    c->tex_h = layers ? height : 0;
    c->tex_layers = layers;
    c->scene_version++;
    return c->cuda(cudaStreamSynchronize(c->stream), "upload textures");
}

int ae_reserve_scene(ae_ctx *ctx, uint32_t max_objects, uint32_t max_lights) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return AE_ERR_INVALID;
    max_objects = std::max(max_objects, 1u);
    max_lights = std::max(max_lights, 1u);
    if (c->objects.reserve(max_objects) || c->tlas.reserve(size_t(max_objects) * 2 + 1) || c->lights.reserve(max_lights) ||
        c->instances.reserve(max_objects))
        return c->fail(AE_ERR_OOM, "scene buffer allocation failed");
    c->max_objects = max_objects;
    c->max_lights = max_lights;
    return AE_OK;
}

int ae_upload_scene(ae_ctx *ctx, const ae_object *objects, uint32_t n_objects, const ae_bvh_node *tlas,
                    uint32_t n_nodes, const uint32_t *light_ids, uint32_t n_lights, const ae_instance *instances,
                    uint32_t n_instances) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return AE_ERR_INVALID;
    if ((n_objects && !objects) || (n_nodes && !tlas) || (n_lights && !light_ids) || (n_instances && !instances))
        return c->fail(AE_ERR_INVALID, "bad scene arguments");
    if (c->max_objects == 0) {
        int rc = ae_reserve_scene(ctx, n_objects, n_lights);
        if (rc) return rc;
    }
    // renderer/renderer.cpp:938-949: refuse anything beyond the sized buffers.
    if (n_objects > c->max_objects || n_nodes > c->max_objects * 2 + 1 || n_lights > c->max_lights ||
        n_instances > c->max_objects)
        return c->fail(AE_ERR_OVERSIZE, "scene too large for its buffers: %u/%u objects, %u/%u nodes, %u/%u lights",
                       n_objects, c->max_objects, n_nodes, c->max_objects * 2 + 1, n_lights, c->max_lights);
    int rc = validate_scene(c, objects, n_objects, tlas, n_nodes, light_ids, n_lights, instances, n_instances);
    if (rc) return rc;
    c->n_objects = n_objects;
    c->n_nodes = n_nodes;
    c->n_lights = n_lights;
    c->n_instances = n_instances;
    if ((rc = upload(c, c->objects, objects, n_objects, "objects")) || (rc = upload(c, c->tlas, tlas, n_nodes, "tlas")) ||
        (rc = upload(c, c->lights, light_ids, n_lights, "lights")) ||
        (rc = upload(c, c->instances, instances, n_instances, "instances")))
        return rc;
    c->host_objects.assign(objects, objects + n_objects);
    c->host_tlas.assign(tlas, tlas + n_nodes);
    c->host_instances.assign(instances, instances + n_instances);
    c->host_lights.assign(light_ids, light_ids + n_lights);
    c->scene_has_ggx = false;
    for (uint32_t i = 0; i < n_objects; i++)
        if (objects[i].colorType == AE_MAT_GGX_METAL) c->scene_has_ggx = true;
    c->scene_uploaded = true;
    c->scene_version++;
    c->scene_version_layout++;
    c->config.num_spheres = n_objects;
    c->config.num_lights = n_lights;
    return c->cuda(cudaStreamSynchronize(c->stream), "upload scene");
}

int ae_set_config(ae_ctx *ctx, const ae_config *cfg) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c || !cfg) return AE_ERR_INVALID;
    if (cfg->width != c->settings.width || cfg->height != c->settings.height)
        return c->fail(AE_ERR_INVALID, "config %ux%u does not match the context's %ux%u images", cfg->width,
                       cfg->height, c->settings.width, c->settings.height);
    c->config = *cfg;
    return AE_OK;
}

int ae_get_config(const ae_ctx *ctx, ae_config *cfg) {
    const Ctx *c = reinterpret_cast<const Ctx *>(ctx);
    if (!c || !cfg) return AE_ERR_INVALID;
    *cfg = c->config;
    return AE_OK;
}

int ae_reset_accumulation(ae_ctx *ctx) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return AE_ERR_INVALID;
    c->config.batch = 0;
    c->config.historyReset = 1;
    return AE_OK;
}

int ae_debug_fail_alloc_after(int64_t n) {
    ae::g_fail_after.store(n < 0 ? -1 : (long long)n);
    return AE_OK;
}

int64_t ae_debug_live_allocations(void) { return (int64_t)ae::g_live_allocations.load(); }

int ae_create_status(void) { return ae::create_status(); }

int ae_debug_inject(ae_ctx *ctx, int fault, uint32_t on) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return AE_ERR_INVALID;
    if (fault == AE_FAULT_TILE_WAIT) c->fault_tile_wait = on ? 1u : 0u;
    else if (fault == AE_FAULT_CHECK_LIMITS) c->fault_check_limits = on ? 1u : 0u;
    else return c->fail(AE_ERR_INVALID, "unknown fault %d", fault);
    return AE_OK;
}

int ae_debug_flags(ae_ctx *ctx, uint32_t *flags) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c || !flags) return AE_ERR_INVALID;
    *flags = 0;
    if (!c->check_word.ptr) return AE_OK;  // the debug walk has not run
    int rc = c->cuda(cudaMemcpyAsync(flags, c->check_word.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream),
                     "read check word");
    if (!rc) rc = c->cuda(cudaMemsetAsync(c->check_word.ptr, 0, sizeof(uint32_t), c->stream), "clear check word");
    if (!rc) rc = c->cuda(cudaStreamSynchronize(c->stream), "check word");
    return rc;
}

int ae_render_frame(ae_ctx *ctx, int mode, const ae_gbuffer *gb) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return AE_ERR_INVALID;
    if (!c->scene_uploaded) return c->fail(AE_ERR_STATE, "render before ae_upload_scene");
    cudaSetDevice(c->settings.device);
    const FrameParams F = make_frame_params(c->config);
    int rc;
    switch (mode) {
    case AE_MODE_COMPUTE_ONLY:
        if ((rc = c->timed_begin())) return rc;
        if ((rc = c->cuda(launch_render_plain(c->scene(), F, c->accum.ptr, c->display.ptr, c->frame.ptr, c->stream),
                          "render (compute-only)")))
            return rc;
        return c->timed_end();
    case AE_MODE_DEFERRED:
        if (c->scene_has_ggx)
            return c->fail(AE_ERR_STATE, "the hybrid passes have no GGX metal (an extension of the compute-only "
                                         "forms); render this scene compute-only, wavefront or served");
        return render_deferred(c, gb);
    case AE_MODE_WAVEFRONT:
        return render_wavefront(c, false);
    case AE_MODE_WAVEFRONT_PRECISION:
        return render_wavefront(c, true);
    default:
        return c->fail(AE_ERR_INVALID, "unknown render mode %d", mode);
    }
}

int ae_read_image(ae_ctx *ctx, int which, void *dst, size_t bytes) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c || !dst) return AE_ERR_INVALID;
    const size_t px = size_t(c->settings.width) * c->settings.height;
    const void *src = nullptr;
    size_t need = 0;
    switch (which) {
    case AE_IMAGE_ACCUM: src = c->accum.ptr; need = px * sizeof(float4); break;
    case AE_IMAGE_DISPLAY: src = c->display.ptr; need = px * sizeof(uchar4); break;
    case AE_IMAGE_FRAME: src = c->frame.ptr; need = px * sizeof(float4); break;
    default: return read_image_extra(c, which, dst, bytes);
    }
    if (bytes < need) return c->fail(AE_ERR_INVALID, "image needs %zu bytes, got %zu", need, bytes);
    int rc = c->cuda(cudaMemcpyAsync(dst, src, need, cudaMemcpyDeviceToHost, c->stream), "read image");
    if (rc) return rc;
    return c->cuda(cudaStreamSynchronize(c->stream), "read image");
}

int ae_closest_hit_device(ae_ctx *ctx, const ae_ray *rays, uint32_t n, ae_hit *hits, int variant) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return AE_ERR_INVALID;
    if (n && (!rays || !hits)) return c->fail(AE_ERR_INVALID, "null ray or hit buffer");
    if (!c->scene_uploaded) return c->fail(AE_ERR_STATE, "trace before ae_upload_scene");
    return closest_hit_dispatch(c, rays, n, hits, variant, c->stream, true);
}

int ae_closest_hit(ae_ctx *ctx, const ae_ray *rays, uint32_t n, ae_hit *hits, int variant) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return AE_ERR_INVALID;
    if (n && (!rays || !hits)) return c->fail(AE_ERR_INVALID, "null ray or hit buffer");
    if (!c->scene_uploaded) return c->fail(AE_ERR_STATE, "trace before ae_upload_scene");
    if (n == 0) return AE_OK;
    cudaSetDevice(c->settings.device);
    int rc = prepare_variant(c, variant);
    if (rc) return rc;
    // The one-ray-per-thread optimised kernels over page-locked host buffers
    // the device can address (cudaHostAlloc'd, or cudaHostRegister'd), rays
    // on a 16-byte boundary (anything else takes the staged pipeline): the
    // kernel reads the rays and writes the hits over the bus itself, one
    // launch and no staging copies.  Each thread reads its ray once when its
    // block starts, and the resident blocks hide the bus latency (1080p
    // camera rays: 2.38 -> 2.20 ms per call).  The walker variant keeps the
    // staged pipeline: its lanes take new rays all through the launch, and
    // each such read waiting on the bus cost more than the copies (1.3M
    // bounce rays: 2.25 -> 4.45 ms).
    if (variant == AE_VARIANT_FAST || variant == AE_VARIANT_QUANT) {
        cudaPointerAttributes ar{}, ah{};
        const bool mapped = cudaPointerGetAttributes(&ar, rays) == cudaSuccess &&
                            cudaPointerGetAttributes(&ah, hits) == cudaSuccess && ar.type == cudaMemoryTypeHost &&
                            ah.type == cudaMemoryTypeHost && ar.devicePointer && ah.devicePointer &&
                            (reinterpret_cast<uintptr_t>(ar.devicePointer) & 15u) == 0;
        cudaGetLastError();  // pageable memory is not an error here
        if (mapped) {
            if ((rc = closest_hit_dispatch(c, static_cast<const ae_ray *>(ar.devicePointer), n,
                                           static_cast<ae_hit *>(ah.devicePointer), variant, c->stream, false)))
                return rc;
            return c->cuda(cudaStreamSynchronize(c->stream), "closest hit");
        }
    }
    // Host -> device -> host in chunks over three streams, each with its own
    // staging slot, so the copies of one chunk overlap the tracing of the
    // others.  Chunks ramp 64K -> 512K rays at the start and back down at the
    // end, so the first kernel starts after a short copy and the last copy
    // back is short.
    constexpr uint32_t kBig = 1u << 19;
    static const uint32_t kRamp[3] = {1u << 16, 1u << 17, 1u << 18};
    std::vector<uint32_t> plan;
    const uint32_t ramp_total = 2 * (kRamp[0] + kRamp[1] + kRamp[2]);
    if (n <= ramp_total) {
        const uint32_t parts = std::max(1u, (n + kRamp[1] - 1) / kRamp[1]);
        for (uint32_t i = 0; i < parts; i++) plan.push_back(n / parts + (i < n % parts ? 1u : 0u));
    } else {
        for (uint32_t r : kRamp) plan.push_back(r);
        for (uint32_t mid = n - ramp_total; mid > 0;) {
            const uint32_t m = std::min(kBig, mid);
            plan.push_back(m);
            mid -= m;
        }
        for (int i = 2; i >= 0; i--) plan.push_back(kRamp[i]);
    }
    const uint32_t chunk = *std::max_element(plan.begin(), plan.end());
    if (!c->side_stream) {
        if ((rc = c->cuda(cudaStreamCreateWithFlags(&c->side_stream, cudaStreamNonBlocking), "stream"))) return rc;
    }
    if (!c->side_stream2) {
        if ((rc = c->cuda(cudaStreamCreateWithFlags(&c->side_stream2, cudaStreamNonBlocking), "stream"))) return rc;
    }
    for (int k = 0; k < Ctx::kIoSlots; k++)
        if (c->io_rays[k].reserve(chunk) || c->io_hits[k].reserve(chunk))
            return c->fail(AE_ERR_OOM, "staging allocation failed");
    cudaStream_t st[Ctx::kIoSlots] = {c->stream, c->side_stream, c->side_stream2};
    uint32_t off = 0;
    for (size_t i = 0; i < plan.size(); i++) {
        const int k = int(i % Ctx::kIoSlots);
        const uint32_t m = plan[i];
        if ((rc = c->cuda(cudaMemcpyAsync(c->io_rays[k].ptr, rays + off, size_t(m) * sizeof(ae_ray),
                                          cudaMemcpyHostToDevice, st[k]), "copy rays")))
            return rc;
        if ((rc = closest_hit_dispatch(c, c->io_rays[k].ptr, m, c->io_hits[k].ptr, variant, st[k], false))) return rc;
        if ((rc = c->cuda(cudaMemcpyAsync(hits + off, c->io_hits[k].ptr, size_t(m) * sizeof(ae_hit),
                                          cudaMemcpyDeviceToHost, st[k]), "copy hits")))
            return rc;
        off += m;
    }
    if ((rc = c->cuda(cudaStreamSynchronize(c->side_stream2), "closest hit"))) return rc;
    if ((rc = c->cuda(cudaStreamSynchronize(c->side_stream), "closest hit"))) return rc;
    return c->cuda(cudaStreamSynchronize(c->stream), "closest hit");
}

int ae_synchronize(ae_ctx *ctx) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return AE_ERR_INVALID;
    int rc = c->cuda(cudaStreamSynchronize(c->stream), "synchronize");
    if (rc) return rc;
    return c->cuda(cudaGetLastError(), "synchronize");
}

int ae_last_kernel_ms(ae_ctx *ctx, float *ms) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c || !ms) return AE_ERR_INVALID;
    if (!c->timed) return c->fail(AE_ERR_STATE, "no timed launch yet");
    int rc = c->cuda(cudaEventSynchronize(c->ev1), "event");
    if (rc) return rc;
    return c->cuda(cudaEventElapsedTime(ms, c->ev0, c->ev1), "event elapsed");
}

void *ae_stream(ae_ctx *ctx) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    return c ? reinterpret_cast<void *>(c->stream) : nullptr;
}

uint64_t ae_launch_count(const ae_ctx *ctx) {
    const Ctx *c = reinterpret_cast<const Ctx *>(ctx);
    return c ? c->launches : 0;
}

}  // extern "C"
