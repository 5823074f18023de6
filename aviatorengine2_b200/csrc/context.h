// context.h - the device context (ae_ctx) and its buffers.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/ae_b200.h"
#include "devmem.h"
#include "trace_common.cuh"

namespace ae {

// A device array that only grows.
template <class T> struct DevBuf {
    T *ptr = nullptr;
    size_t cap = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    int reserve(size_t n) {
        if (n <= cap) return AE_OK;
        release();
        void *p = nullptr;
        if (dev_alloc(&p, n * sizeof(T)) != cudaSuccess) {
            cudaGetLastError();
            return AE_ERR_OOM;
        }
        ptr = static_cast<T *>(p);
        cap = n;
        return AE_OK;
    }
    void release() {
        if (ptr) dev_free(ptr);
        ptr = nullptr;
        cap = 0;
    }
};

struct FastScene;   // derived structures of the optimised closest-hit kernels
struct Wavefront;   // queues of the wavefront path tracer
struct Deferred;    // G-buffer and history of the deferred resolve
struct Refit;       // bottom-up TLAS refit state

struct Ctx {
    ae_settings settings{};
    ae_config config{};
    cudaStream_t stream = nullptr;
    cudaStream_t side_stream = nullptr;
    cudaStream_t side_stream2 = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::string err;
    uint64_t launches = 0;
    bool timed = false;

    // Geometry, uploaded once (UploadMeshGeometry).
    DevBuf<ae_vertex> vertices;
    DevBuf<uint32_t> indices;
    DevBuf<ae_bvh_node> blas;
    uint64_t n_vertices = 0, n_indices = 0, n_blas = 0;
    std::vector<uint32_t> host_indices;
    std::vector<ae_bvh_node> host_blas;
    std::vector<ae_vertex> host_vertices;
    bool geometry_uploaded = false;
    // Meshes already checked: (vertexBase, indexBase, triangleCount, blasBase).
    std::map<std::tuple<uint32_t, uint32_t, uint32_t, uint32_t>, bool> checked_meshes;

    // Per-frame scene (UploadScene).
    DevBuf<ae_object> objects;
    DevBuf<ae_bvh_node> tlas;
    DevBuf<uint32_t> lights;
    DevBuf<ae_instance> instances;
    uint32_t n_objects = 0, n_nodes = 0, n_lights = 0, n_instances = 0;
    uint32_t max_objects = 0, max_lights = 0;
    std::vector<ae_object> host_objects;
    std::vector<ae_bvh_node> host_tlas;
    std::vector<ae_instance> host_instances;
    std::vector<uint32_t> host_lights;
    bool scene_uploaded = false;
    bool scene_has_ggx = false;  // an object uses AE_MAT_GGX_METAL (not shaded by the hybrid passes)
    uint32_t fault_tile_wait = 0;  // ae_debug_inject(AE_FAULT_TILE_WAIT)
    uint32_t fault_check_limits = 0;  // ae_debug_inject(AE_FAULT_CHECK_LIMITS)
    DevBuf<uint32_t> check_word;      // AE_CHECK_* bits of the debug walk (ae_debug_flags)
    uint64_t scene_version = 0;         // bumps on every change of scene content
    uint64_t geometry_version = 0;      // bumps on every ae_upload_geometry
    uint64_t scene_version_layout = 0;  // bumps when arrays are re-uploaded (topology may change)
    DevBuf<float> obj_box;              // world box per object (refit)

    // Material texture array (ae_upload_textures) and its sRGB decode table.
    DevBuf<uint32_t> tex;
    DevBuf<float> srgb_lut;
    uint32_t tex_w = 0, tex_h = 0, tex_layers = 0;

    // Images.
    DevBuf<float4> accum, frame;
    DevBuf<uchar4> display;

    // Host-buffer tracing staging.
    // Staging slots of the host-buffer closest hit (ae_closest_hit).
    static constexpr int kIoSlots = 3;
    DevBuf<ae_ray> io_rays[kIoSlots];
    DevBuf<ae_hit> io_hits[kIoSlots];

    // Optimised forms.
    FastScene *fast = nullptr;
    bool fast_ready = false;
    uint64_t fast_version = 0;
    Wavefront *wave = nullptr;
    Deferred *deferred = nullptr;
    Refit *refit = nullptr;

    ~Ctx();
    int fail(int code, const char *fmt, ...);
    int cuda(cudaError_t e, const char *what);
    DevScene scene() const;
    int timed_begin();
    int timed_end();
};

// Implemented by the optimised-kernel translation units.
int prepare_variant(Ctx *c, int variant);
int closest_hit_dispatch(Ctx *c, const ae_ray *rays, uint32_t n, ae_hit *hits, int variant, cudaStream_t st,
                         bool timed);
int render_deferred(Ctx *c, const ae_gbuffer *gb);
int render_wavefront(Ctx *c, bool precision);
int read_image_extra(Ctx *c, int which, void *dst, size_t bytes);

}  // namespace ae
