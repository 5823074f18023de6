/*
 * ae_b200.h - C ABI of the B200 ray/path-tracing library.
 *
 * This header is the drop-in boundary that replaces the SDL_gpu compute
 * dispatch of AviatorEngine2's renderer.  Everything crossing it is a plain C
 * type: byte layouts identical to the reference's shader contract, pointers
 * and sizes.  No CUDA or torch type appears in a signature.
 *
 * Byte contract (each struct re-declared here with its size pinned):
 *   ae_object      == Object_GPU        scene/gpu_types.h:26-81     (128 B)
 *   ae_instance    == MeshInstance_GPU  scene/gpu_types.h:84-96     (48 B)
 *   ae_bvh_node    == BVHNode_GPU       scene/bvh.h:31-43           (48 B)
 *   ae_vertex      == Vertex_GPU        scene/mesh_library.h:39-46  (32 B)
 *   ae_config      == Config            renderer/renderer.h:76-147  (240 B)
 *
 * Extension: ae_instance.scale occupies MeshInstance_GPU::pad0 (offset 12).
 * The reference transform is rigid (scene/gpu_types.h:83); a value of 0 or 1
 * means "no scale", so reference-packed instances (pad0 = 0) trace unchanged.
 *
 * Every entry point returns AE_OK (0) or a negative ae_status; the message of
 * the last failure on a context is available from ae_last_error().  The
 * reference returns bool + SDL_Log (renderer/renderer.cpp:938-949); the status
 * codes name the same failure classes.
 *
 * Threading: one host thread per context, as the reference drives its Renderer
 * from the main loop (main.cpp:157-369).  Calls on one context are not
 * re-entrant.  The serving API (ae_serve_*) is internally threaded and is the
 * one exception: it may be called from any thread.
 */
#ifndef AE_B200_H
#define AE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* Status codes                                                              */
/* ------------------------------------------------------------------------ */
typedef enum ae_status {
    AE_OK = 0,
    AE_ERR_INVALID = -1,     /* bad argument (null pointer, zero size, bad enum) */
    AE_ERR_OOM = -2,         /* device or host allocation failed                 */
    AE_ERR_OVERSIZE = -3,    /* upload larger than the buffers sized at creation  */
    AE_ERR_LAYOUT = -4,      /* scene arrays are inconsistent (index out of range) */
    AE_ERR_CUDA = -5,        /* a CUDA runtime call failed                        */
    AE_ERR_TIMEOUT = -6,     /* a bounded device-side wait gave up                */
    AE_ERR_STATE = -7,       /* call order violated (e.g. trace before upload)    */
    AE_ERR_REJECTED = -8,    /* serving: request refused at admission             */
    AE_ERR_CANCELLED = -9    /* serving: request withdrawn by ae_serve_cancel      */
} ae_status;

/* ------------------------------------------------------------------------ */
/* Byte contract                                                             */
/* ------------------------------------------------------------------------ */

/* BodyShape, scene/gpu_types.h:14-21 */
enum { AE_SHAPE_SPHERE = 0, AE_SHAPE_QUAD = 1, AE_SHAPE_BOX = 2, AE_SHAPE_TRIANGLE = 3, AE_SHAPE_MESH = 4 };
/* MaterialType, scene/material.h:11-18, plus one extension: GGX_METAL, a
 * rough metal with GGX microfacet reflection (Walter et al., EGSR 2007;
 * roughness alpha in Object_GPU::fuzz, F0 = albedo).  The compute-only,
 * wavefront, precision and serving forms shade it; the hybrid (deferred)
 * passes refuse scenes that use it. */
enum { AE_MAT_LAMBERTIAN = 0, AE_MAT_METAL = 1, AE_MAT_DIELECTRIC = 2, AE_MAT_DIFFUSE_LIGHT = 3, AE_MAT_ISOTROPIC = 4,
       AE_MAT_GGX_METAL = 5 };
/* kNoTexture, scene/texture.h:19 */
#define AE_NO_TEXTURE 0xFFFFFFFFu

/* Object_GPU, scene/gpu_types.h:26-81 (128 B). */
typedef struct ae_object {
    float x, y, z;          /*   0 position                        */
    float prevRotX;         /*  12                                  */
    float x2, y2, z2;       /*  16 previous position                */
    float radius;           /*  28                                  */
    float u_x, u_y, u_z;    /*  32 quad/triangle edge u             */
    float prevRotY;         /*  44                                  */
    float v_x, v_y, v_z;    /*  48 quad/triangle edge v             */
    float prevRotZ;         /*  60                                  */
    float half_x, half_y, half_z; /* 64 box half extents            */
    float rotation;         /*  76 yaw                              */
    float density;          /*  80                                  */
    float emission;         /*  84                                  */
    uint32_t instanceIndex; /*  88                                  */
    float textureTint;      /*  92                                  */
    float r, g, b;          /*  96 albedo                           */
    float fuzz;             /* 108                                  */
    float refraction;       /* 112                                  */
    uint32_t shapeType;     /* 116                                  */
    uint32_t colorType;     /* 120                                  */
    uint32_t textureID;     /* 124                                  */
} ae_object;

/* MeshInstance_GPU, scene/gpu_types.h:84-96 (48 B).  `scale` is pad0. */
typedef struct ae_instance {
    float px, py, pz;
    float scale;            /* 12: uniform scale, 0 or 1 = rigid (reference) */
    float qx, qy, qz, qw;   /* 16: rotation, x,y,z,w memory order            */
    uint32_t vertexBase;    /* 32 */
    uint32_t indexBase;     /* 36 */
    uint32_t triangleCount; /* 40 */
    uint32_t blasBase;      /* 44 */
} ae_instance;

/* BVHNode_GPU, scene/bvh.h:31-43 (48 B).  count > 0: leaf, left = first slot. */
typedef struct ae_bvh_node {
    float min_x, min_y, min_z;
    float pad0;
    float max_x, max_y, max_z;
    int32_t left;
    int32_t right;
    int32_t count;
    int32_t padding;
    int32_t pad_trailing;
} ae_bvh_node;

/* Vertex_GPU, scene/mesh_library.h:39-46 (32 B). */
typedef struct ae_vertex {
    float px, py, pz;
    float nx, ny, nz;
    float u, v;
} ae_vertex;

/* AABB, scene/aabb.h:14-22 (24 B). */
typedef struct ae_aabb {
    float min_x, min_y, min_z;
    float max_x, max_y, max_z;
} ae_aabb;

/* Config, renderer/renderer.h:76-147 (240 B). */
typedef struct ae_config {
    float source_x, source_y, source_z;
    float fov;
    float target_x, target_y, target_z;
    float focus_dist;
    float defocus_angle;
    float padding[3];
    float up_x, up_y, up_z;
    float oof;
    float sky_r, sky_g, sky_b;
    uint32_t width;
    float horizon_r, horizon_g, horizon_b;
    uint32_t height;
    uint32_t samples;
    uint32_t batches;
    uint32_t batch;
    uint32_t depth;
    uint32_t num_spheres;
    uint32_t renderType;
    uint32_t num_lights;
    float exposure;          /* 124 */
    uint32_t debugView;      /* 128 */
    float zNear, zFar;
    float jitter_x, jitter_y;
    uint32_t displayOnly;    /* 148 */
    float traceScale;        /* 152 */
    uint32_t frameIndex;     /* 156 */
    uint32_t historyReset;
    uint32_t cameraMoved;
    float historyCap;        /* 168 */
    float padding3;
    float prevViewProj[16];  /* 176, row-major Mat4 (math/mat4.h) */
} ae_config;

/* ------------------------------------------------------------------------ */
/* Ray and hit records of the closest-hit / any-hit entry points             */
/* ------------------------------------------------------------------------ */

/* A ray as the shaders build it (hybrid:32-41): origin, near bound, direction,
 * time.  The far bound starts at 1e6 as TraverseBVH does (hybrid:869). */
typedef struct ae_ray {
    float ox, oy, oz;
    float tnear;
    float dx, dy, dz;
    float time;
} ae_ray;

/* The closest hit.  object = slot in the object buffer (the TLAS leaf order),
 * AE_MISS on a miss.  prim = triangle slot inside the mesh (leaf order of its
 * BLAS, i.e. (bestBase - indexBase) / 3 in hybrid:600-707), AE_MISS for
 * analytic objects.  alpha/beta are HitMeshTriangle's weights of v1 and v2
 * (hybrid:564-598) or HitQuad's plane coordinates for quads. */
typedef struct ae_hit {
    float t;
    float alpha;
    float beta;
    uint32_t object;
    uint32_t prim;
} ae_hit;
#define AE_MISS 0xFFFFFFFFu

/* ------------------------------------------------------------------------ */
/* Host-side acceleration structure (the reference's CPU side)               */
/* ------------------------------------------------------------------------ */

/* Binned-SAH BVH over `n` boxes; BuildBVH, scene/bvh.h:275-295.
 * out_nodes must hold 2*n nodes (the builder never emits more than 2n-1);
 * out_order receives the n-entry leaf-slot permutation.  *out_node_count is
 * set to the number of nodes written.  n == 0 writes nothing. */
int ae_build_bvh(const ae_aabb *bounds, uint32_t n,
                 ae_bvh_node *out_nodes, uint32_t *out_node_count,
                 uint32_t *out_order);

/* ae_build_bvh on the GPU (the current device): the same nodes and the same
 * leaf-slot order, bit for bit.  Host arrays in and out with the capacities
 * of ae_build_bvh.  AE_ERR_INVALID for a NaN or infinite coordinate (the
 * reference's bucket index is undefined for those). */
int ae_build_bvh_gpu(const ae_aabb *bounds, uint32_t n,
                     ae_bvh_node *out_nodes, uint32_t *out_node_count,
                     uint32_t *out_order);
/* ae_build_bvh_gpu with the subtree size at or below which one warp builds a
 * whole subtree (ae_build_bvh_gpu uses 256).  Nodes above it are built one
 * tree level per round by blocks of 2048 boxes.  Every value gives the same
 * tree; it only moves work between the two phases. */
int ae_build_bvh_gpu_ex(const ae_aabb *bounds, uint32_t n, uint32_t warp_subtree,
                        ae_bvh_node *out_nodes, uint32_t *out_node_count,
                        uint32_t *out_order);

/* The device builder on device arrays (all pointers device memory except
 * out_node_count), enqueued on `stream` (a cudaStream_t; NULL = the legacy
 * default stream).  d_nodes holds 2n nodes, d_order n.  Returns once the
 * build has finished; it synchronises `stream` between tree levels. */
int ae_build_bvh_device(const ae_aabb *d_bounds, uint32_t n, uint32_t warp_subtree,
                        ae_bvh_node *d_nodes, uint32_t *out_node_count,
                        uint32_t *d_order, void *stream);

/* MeshLibrary::Add's device part on device arrays: triangle boxes (as
 * Surround2Points + SurroundPoint), the BLAS over them and the indices in
 * leaf-slot order (scene/mesh_library.h:130-153).  d_nodes holds 2*(ni/3)
 * nodes, d_out_indices ni.  AE_ERR_LAYOUT for an index >= nv. */
int ae_mesh_blas_device(const ae_vertex *d_vertices, uint32_t nv,
                        const uint32_t *d_indices, uint32_t ni,
                        ae_bvh_node *d_nodes, uint32_t *out_node_count,
                        uint32_t *d_out_indices, void *stream);

/* ae_mesh_blas_device for k meshes at once (arrays of k device pointers and
 * sizes, held in host memory): the k trees are built together - they share
 * the builder's level rounds and its warp launch - and each mesh's nodes,
 * count and indices equal its own ae_mesh_blas_device call's. */
int ae_mesh_blas_device_many(uint32_t k, const ae_vertex *const *d_vertices, const uint32_t *nv,
                             const uint32_t *const *d_indices, const uint32_t *ni,
                             ae_bvh_node *const *d_nodes, uint32_t *out_node_counts,
                             uint32_t *const *d_out_indices, void *stream);

/* The device builder keeps its scratch (about 150 bytes per box of the
 * largest build so far) between calls; this frees it. */
void ae_bvh_builder_release(void);

/* Mesh library: MeshLibrary, scene/mesh_library.h:64-159, with 32-bit input
 * indices (the reference's Mesh is uint16, scene/mesh.h:24, too small for a
 * 512x512 grid).  Add() appends local vertices, builds the BLAS over the
 * triangles' AABBs and appends the indices in BLAS leaf order. */
typedef struct ae_mesh_library ae_mesh_library;
typedef struct ae_mesh_range {
    uint32_t vertexBase, indexBase, triangleCount, blasBase;
    ae_aabb localBounds;
    uint32_t doubleSided;
} ae_mesh_range;

ae_mesh_library *ae_mesh_library_create(void);
void ae_mesh_library_destroy(ae_mesh_library *lib);
/* Returns the mesh handle (>= 0) or a negative ae_status. */
int ae_mesh_library_add(ae_mesh_library *lib, const ae_vertex *vertices, uint32_t nv,
                        const uint32_t *indices, uint32_t ni, int double_sided);
/* ae_mesh_library_add with the triangle boxes, the BLAS build and the
 * leaf-order index rewrite on the GPU; appends the same bytes. */
int ae_mesh_library_add_gpu(ae_mesh_library *lib, const ae_vertex *vertices, uint32_t nv,
                            const uint32_t *indices, uint32_t ni, int double_sided);
/* k calls of ae_mesh_library_add_gpu in one (host arrays of k pointers and
 * sizes; double_sided may be NULL): the k BLAS are built together on the GPU
 * and appended in order, each exactly as its own call would append it.
 * out_handles[m] receives mesh m's handle; nothing is appended on failure. */
int ae_mesh_library_add_many_gpu(ae_mesh_library *lib, uint32_t k, const ae_vertex *const *vertices,
                                 const uint32_t *nv, const uint32_t *const *indices, const uint32_t *ni,
                                 const int *double_sided, int *out_handles);
int ae_mesh_library_range(const ae_mesh_library *lib, uint32_t handle, ae_mesh_range *out);
/* Sizes of the flattened arrays (elements). */
void ae_mesh_library_sizes(const ae_mesh_library *lib, uint64_t *nv, uint64_t *ni, uint64_t *nb);
/* Borrowed pointers into the flattened arrays; valid until the next add. */
const ae_vertex *ae_mesh_library_vertices(const ae_mesh_library *lib);
const uint32_t *ae_mesh_library_indices(const ae_mesh_library *lib);
const ae_bvh_node *ae_mesh_library_blas(const ae_mesh_library *lib);

/* One renderable entity, the host-side union of TransformComponent,
 * MaterialComponent and the shape component (scene/components.h:31-148). */
typedef struct ae_entity {
    uint32_t shape;          /* AE_SHAPE_*                                   */
    uint32_t material;       /* AE_MAT_*                                     */
    float position[3];       /* TransformComponent::position                 */
    float rotation[4];       /* TransformComponent::rotation, x,y,z,w        */
    float scale;             /* mesh instances only: uniform scale (1 = rigid) */
    float albedo[3];
    float fuzz, ior, emission, density;
    float texture_tint;
    uint32_t texture_id;
    float radius;            /* sphere                                       */
    float u[3], v[3];        /* quad / triangle edges (local, unrotated)     */
    float half_extent[3];    /* box                                          */
    uint32_t mesh;           /* mesh handle for AE_SHAPE_MESH                */
    float prev_position[3];  /* last frame's transform (Object_GPU x2..)     */
    float prev_rotation[4];
} ae_entity;

/* TLAS assembly: GatherRenderables (scene/shapes.h:379-426) + BuildBVH +
 * entity reorder + LightIndices (renderer/renderer.cpp:803-813) + PackObjects
 * (renderer/renderer.cpp:815-929).  Entities are taken in the caller's order
 * (the reference's gather order is per shape type: spheres, quads, boxes,
 * triangles, meshes; callers that need its exact slot order pass them so).
 * Capacities: out_objects/out_instances n, out_nodes 2n+1, out_lights n,
 * out_order n.  Counts are written through the count pointers. */
int ae_pack_scene(const ae_entity *entities, uint32_t n, const ae_mesh_library *lib,
                  ae_object *out_objects, ae_bvh_node *out_nodes, uint32_t *out_node_count,
                  uint32_t *out_lights, uint32_t *out_light_count,
                  ae_instance *out_instances, uint32_t *out_instance_count,
                  uint32_t *out_order);

/* ae_pack_scene with the TLAS build and the slot-order packing (objects,
 * instance numbering, light list) on the GPU: the same arrays, bit for bit.
 * World boxes and per-entity records are made on the host as in
 * ae_pack_scene. */
int ae_pack_scene_gpu(const ae_entity *entities, uint32_t n, const ae_mesh_library *lib,
                      ae_object *out_objects, ae_bvh_node *out_nodes, uint32_t *out_node_count,
                      uint32_t *out_lights, uint32_t *out_light_count,
                      ae_instance *out_instances, uint32_t *out_instance_count,
                      uint32_t *out_order);

/* World bounds of one entity (SphereBounds/QuadBounds/BoxBounds/
 * TriangleBounds/MeshBounds, scene/shapes.h:70-145). */
int ae_entity_bounds(const ae_entity *e, const ae_mesh_library *lib, ae_aabb *out);

/* ------------------------------------------------------------------------ */
/* Device context: Renderer, renderer/renderer.h:325-411                     */
/* ------------------------------------------------------------------------ */

typedef struct ae_ctx ae_ctx;

/* RendererSettings, renderer/renderer.h:225-274 (window/shader-name fields
 * dropped: there is no window; the kernels are compiled in). */
typedef struct ae_settings {
    uint32_t width, height;
    uint32_t samples;          /* samples per pixel per frame                 */
    uint32_t max_samples;      /* 0 = accumulate forever                      */
    uint32_t hybrid;           /* 1 = deferred resolve, 0 = compute-only      */
    uint32_t hybrid_max_depth; /* path segments in hybrid mode (default 3)    */
    float trace_scale;         /* 1, 0.75, 0.5 (TraceResolution)              */
    uint32_t history_while_moving;
    int32_t device;            /* CUDA device ordinal                         */
    uint32_t reserved[7];
} ae_settings;

/* Kernel families.  PLAIN reproduces the reference order of operations;
 * FAST is the optimised closest-hit (ordered traversal, packed triangles);
 * QUANT adds 8-bit child bounds and the watertight triangle test; FAST_WALK
 * is FAST's walk run one step at a time per thread on a persistent grid (the
 * same hits; for incoherent sets such as bounce rays); PLAIN_WT is PLAIN's
 * walk over the FP32 binary BVH with QUANT's watertight triangle test - the
 * FP32-node form QUANT's 8-bit nodes are checked against (identical hits).
 * PLAIN_CHECKED is PLAIN's walk in a debug mode: every stack push checked
 * against the stack's capacity and every buffer index (TLAS node, object,
 * instance, BLAS node, index triple, vertex) against its array's length; a
 * violation skips that access and sets AE_CHECK_STACK or AE_CHECK_INDEX in
 * the context's check word (ae_debug_flags).  On a valid scene its hits are
 * PLAIN's. */
enum { AE_VARIANT_PLAIN = 0, AE_VARIANT_FAST = 1, AE_VARIANT_QUANT = 2, AE_VARIANT_FAST_WALK = 3, AE_VARIANT_PLAIN_WT = 4,
       AE_VARIANT_PLAIN_CHECKED = 5 };
enum { AE_CHECK_STACK = 1, AE_CHECK_INDEX = 2 };

/* Render modes for ae_render_frame.  AE_MODE_WAVEFRONT_PRECISION is the
 * wavefront tracer in the precision form: watertight triangle test, FP16
 * shading normals and UVs, and the accumulation image kept as a compensated
 * (Kahan) FP32 sum of the frame colours divided by the frame count. */
enum { AE_MODE_COMPUTE_ONLY = 0, AE_MODE_DEFERRED = 1, AE_MODE_WAVEFRONT = 2, AE_MODE_WAVEFRONT_PRECISION = 3 };

/* Image identifiers for ae_read_image. */
enum {
    AE_IMAGE_ACCUM = 0,    /* float4 linear accumulation (RGBA32F)           */
    AE_IMAGE_DISPLAY = 1,  /* uint8x4 sRGB display image                     */
    AE_IMAGE_FRAME = 2,    /* float4 this frame's radiance before blending   */
    AE_IMAGE_REDUCED = 3,  /* float4 lightingReduced (deferred, reduced grid) */
    AE_IMAGE_HISTORY_GEOMETRY = 4 /* float4 historyGeometry[write]           */
};

/* Renderer::Initialize.  Returns NULL on failure; the reason is printed to
 * stderr (there is no context to hold it yet). */
ae_ctx *ae_create(const ae_settings *settings);
/* Renderer::Shutdown. */
void ae_destroy(ae_ctx *ctx);
const char *ae_last_error(const ae_ctx *ctx);

/* Renderer::UploadMeshGeometry (renderer/renderer.cpp:706-785): vertices,
 * indices and BLAS nodes, once.  Sizes the geometry buffers. */
int ae_upload_geometry(ae_ctx *ctx, const ae_vertex *vertices, uint32_t nv,
                       const uint32_t *indices, uint32_t ni,
                       const ae_bvh_node *blas, uint32_t nb);

/* Renderer::CreateSceneBuffers (renderer/renderer.cpp:553-628): worst-case
 * capacities for the per-frame arrays.  Optional: ae_upload_scene sizes them
 * on first use. */
int ae_reserve_scene(ae_ctx *ctx, uint32_t max_objects, uint32_t max_lights);

/* The material texture array GlobalTextureArray (TextureLibrary::BuildGPUArray,
 * scene/texture.h:110-230): `layers` RGBA8 sRGB images of width x height
 * texels (at most 2048 x 2048), row-major, one after another.  Objects name a
 * layer with textureID; AE_NO_TEXTURE keeps the flat albedo.  Sampled as the
 * shaders' SampleLevel(uv, layer, 0) with the renderer's linear REPEAT sampler
 * (renderer/renderer.cpp:226-233).  With no array uploaded, textured
 * materials sample white, as BuildGPUArray's 1x1 fallback layer. */
int ae_upload_textures(ae_ctx *ctx, const uint8_t *texels, uint32_t width, uint32_t height, uint32_t layers);

/* Renderer::UploadScene (renderer/renderer.cpp:931-1027): objects, TLAS,
 * light IDs and instances, in the storage-buffer order of RenderFrame
 * (renderer/renderer.cpp:1456-1459).  Fails with AE_ERR_OVERSIZE beyond the
 * reserved capacity, like the reference. */
int ae_upload_scene(ae_ctx *ctx, const ae_object *objects, uint32_t n_objects,
                    const ae_bvh_node *tlas, uint32_t n_nodes,
                    const uint32_t *light_ids, uint32_t n_lights,
                    const ae_instance *instances, uint32_t n_instances);

/* SDL_PushGPUComputeUniformData(Config) (renderer/renderer.cpp:1426). */
int ae_set_config(ae_ctx *ctx, const ae_config *config);
int ae_get_config(const ae_ctx *ctx, ae_config *config);

/* Per-frame state of RenderFrame (renderer/renderer.cpp:1332-1588):
 * Renderer::ResetAccumulation / CameraMoved / MarkSceneDirty equivalents. */
int ae_reset_accumulation(ae_ctx *ctx);

/* G-buffer planes consumed by the deferred resolve, host or device pointers
 * per `on_device`.  Layout of renderer/renderer.cpp:370-421: position RGBA32F
 * (w = object slot as float), normal RGBA32F here (w = coverage; the
 * reference stores RGBA16F), albedo RGBA8 (a = 0 for view-dependent), depth
 * float. */
typedef struct ae_gbuffer {
    const float *position;
    const float *normal;
    const uint8_t *albedo;
    const float *depth;
    uint32_t on_device;
} ae_gbuffer;

/* One dispatch: the compute-only megakernel (hybrid:1328-1404), or the
 * deferred resolve (deferred:1879-2010) followed by the temporal upsample
 * (upsample:280-390) when config.traceScale < 1, or the wavefront path
 * tracer.  Uses the config set by ae_set_config (batch/frameIndex included). */
int ae_render_frame(ae_ctx *ctx, int mode, const ae_gbuffer *gbuffer);

/* Produce the G-buffer on the device by ray casting the primary hit with the
 * reference camera (the raster pass gbuffer.vert/frag writes the same planes).
 * The planes stay resident and feed the next deferred frame. */
int ae_build_gbuffer(ae_ctx *ctx);

/* Copy an image to host memory.  dst_bytes must be >= the image size. */
int ae_read_image(ae_ctx *ctx, int which, void *dst, size_t dst_bytes);

/* Error of an image against a reference image, reduced on the GPU in FP64
 * (no counterpart in the reference).  `reference` is host memory holding
 * width*height RGBA doubles (e.g. the FP64 CPU oracle's accumulation); the RGB
 * channels are compared.  out[0] = mean relative error
 * mean(|x - r| / (|r| + eps)), out[1] = mean absolute error, out[2] = largest
 * absolute error, out[3] = root mean square error.  The sums are reduced in a
 * fixed order, so the result is the same on every run. */
int ae_image_error(ae_ctx *ctx, int which, const double *reference, double eps, double *out4);
/* The same over a pixel subset: xy holds n_px (x, y) pairs, reference n_px
 * RGBA doubles in that order (e.g. the FP64 oracle rendered at those pixels
 * only).  Coordinates outside the image are refused with AE_ERR_INVALID. */
int ae_image_error_pixels(ae_ctx *ctx, int which, const uint32_t *xy, uint32_t n_px, const double *reference,
                          double eps, double *out4);

/* Closest hit for a batch of HOST rays: copies in, traces, copies out,
 * pipelined in chunks over streams.  variant = AE_VARIANT_*.  With FAST or
 * QUANT and page-locked buffers the device can address (cudaHostAlloc'd or
 * cudaHostRegister'd), the kernel reads the rays and writes the hits in host
 * memory directly, in one launch.  The hits are ae_closest_hit_device's
 * either way. */
int ae_closest_hit(ae_ctx *ctx, const ae_ray *rays, uint32_t n, ae_hit *hits, int variant);
/* Same with DEVICE pointers, on the context's stream, no synchronisation.
 * d_rays must start on a 16-byte boundary (AE_ERR_INVALID otherwise). */
int ae_closest_hit_device(ae_ctx *ctx, const ae_ray *d_rays, uint32_t n, ae_hit *d_hits, int variant);
/* Closest hit for HOST rays with no device allocation: the variant of
 * ae_closest_hit for callers that cannot let a library call cudaMalloc (a
 * frame loop that must not stall on the device synchronisation cudaMalloc and
 * cudaFree imply, or a process whose device memory another allocator already
 * holds).  It has no counterpart in the reference.  Rays and hits are staged
 * through one fixed array compiled into the library, AE_NOALLOC_MAX_RAYS rays
 * (3.25 MiB, held by every GPU that loads the library until exit); larger
 * batches are refused with AE_ERR_OVERSIZE.  The first call on a device looks
 * up the array's device address and should come before any stream capture;
 * that cached address is stale after cudaDeviceReset, so do not use this
 * entry point across a device reset.  All calls on a device share the array:
 * calls that overlap on the GPU race.  Variants: AE_VARIANT_PLAIN, and
 * AE_VARIANT_FAST / AE_VARIANT_QUANT once ae_prepare_fast (which allocates)
 * has accepted the current scene (AE_ERR_STATE otherwise, also for scenes
 * with participating media); AE_VARIANT_FAST_WALK is refused because its
 * launch reserves counters in memory the library allocates.  The calling
 * thread's current device is restored on return. */
#define AE_NOALLOC_MAX_RAYS 65536u
int ae_closest_hit_noalloc(ae_ctx *ctx, const ae_ray *rays, uint32_t n, ae_hit *hits, int variant);

/* Any hit in [tnear, tmax] with the deferred shader's rules (Occluded,
 * deferred:1115-1171: glass and lights do not block).  out[i] = 1 when
 * occluded.  Host pointers. */
int ae_any_hit(ae_ctx *ctx, const ae_ray *rays, const float *tmax, uint32_t n, uint8_t *out);

/* Ray sets of the closest-hit workload, host buffers.
 * ae_camera_rays: the width*height primary rays of the current config's
 * Batch in row-major pixel order, as main builds them (hybrid:1346-1373).
 * ae_bounce_rays: for ray i (pixel i) and its closest hit, one diffuse
 * bounce (n + RandomDirection(), hybrid:980-986) drawn from pixel i's RNG
 * stream after its camera ray, origin offset 0.001 along the facing normal
 * (hybrid:1294-1296).  valid[i] = 0 where the primary missed (out[i] is then
 * a copy of the primary ray). */
int ae_camera_rays(ae_ctx *ctx, ae_ray *out);
int ae_bounce_rays(ae_ctx *ctx, const ae_ray *primary, const ae_hit *hits, uint32_t n, ae_ray *out, uint8_t *valid);

/* Algorithmic traffic of the reference traversal over DEVICE rays: the
 * touches of TraverseBVH/HitMesh (hybrid:600-917) summed over the set, as
 * counters[6] = TLAS nodes, object records, instance records, BLAS nodes,
 * triangles tested, closest-hit winners.  The roofline's bytes per ray are
 * 48, 128, 48, 48, 48 and 60 bytes per touch respectively. */
int ae_trace_counters(ae_ctx *ctx, const ae_ray *d_rays, uint32_t n, uint64_t *counters);
/* The fetches of one kernel family's walk over DEVICE rays (no counterpart in
 * the reference).  PLAIN: as ae_trace_counters.  FAST / QUANT (after
 * ae_prepare_fast): counters[6] = TLAS nodes (48 B), object metadata records
 * (16 B), instance records (48 B), 4-wide quantised BLAS nodes (64 B),
 * triangle records (48 B), rays that hit. */
int ae_trace_counters_variant(ae_ctx *ctx, const ae_ray *d_rays, uint32_t n, int variant, uint64_t *counters);
/* Algorithmic traffic of one compute-only frame of the current config: every
 * traversal of main/ColorRay/CalculateDirectLight (hybrid:1122-1404) with its
 * touches counted as in ae_trace_counters, summed over all pixels.
 * counters[7] = the six touch counts, then the number of traversals. */
int ae_path_counters(ae_ctx *ctx, uint64_t *counters);

/* Wavefront path tracer state after an AE_MODE_WAVEFRONT frame: the extend
 * stage's autotuned block size and shared-memory stack depth, the nine
 * candidate timings in milliseconds (threads 64/128/256 x stack 16/24/32),
 * and the device error flags (non-zero: a bounded wait gave up). */
int ae_wavefront_info(ae_ctx *ctx, int32_t *threads, int32_t *stack, float *tune_ms9, uint32_t *errors);
/* The walker stages' autotuned launch for one form (precision 0:
 * AE_MODE_WAVEFRONT, 1: AE_MODE_WAVEFRONT_PRECISION), after that form's first
 * frame: for the shadow stage and the bounce extend, the run length of queue
 * entries a warp claims at a time (0: static assignment, entry k + grid
 * size) and the resident blocks per SM the kernel is compiled for (6 or 7:
 * its register bound), and the sixteen timings in milliseconds behind them
 * (shadow stage, then extend; each for static, 32, 64 and 256 at 6 blocks,
 * then the same at 7).  AE_ERR_STATE before that frame.  No counterpart in
 * the reference (its passes have no autotuner). */
int ae_wavefront_walk_info(ae_ctx *ctx, int precision, uint32_t *shadow_run, uint32_t *extend_run,
                           uint32_t *shadow_blocks, uint32_t *extend_blocks, float *tune_ms16);
/* Pins that launch for one form instead of autotuning it (runs: 0 static,
 * otherwise a run length, at most 2^20; blocks: 6 or 7, 0 = 7): every choice
 * gives the same hits and images, so this only fixes the launch shape
 * (comparisons, tests). */
int ae_wavefront_set_walk_runs(ae_ctx *ctx, int precision, uint32_t shadow_run, uint32_t extend_run,
                               uint32_t shadow_blocks, uint32_t extend_blocks);

/* Synchronise the context's stream.  Returns AE_ERR_CUDA on a sticky error. */
int ae_synchronize(ae_ctx *ctx);
/* Device time in milliseconds of the last kernel launch that the context
 * timed (events recorded on the launching stream). */
int ae_last_kernel_ms(ae_ctx *ctx, float *ms);
/* Raw CUDA stream of the context (cudaStream_t), for callers that order their
 * own work against it. */
void *ae_stream(ae_ctx *ctx);
/* Number of kernel launches issued by this context since creation. */
uint64_t ae_launch_count(const ae_ctx *ctx);

/* Rebuild the derived device structures (packed triangles, 4-wide quantised
 * BVH) after ae_upload_geometry.  Called implicitly on first use. */
int ae_prepare_fast(ae_ctx *ctx);

/* The 4-wide BVH of the optimised kernels, host side, for one mesh: binary
 * BLAS nodes (mesh-relative links, scene/bvh.h layout) collapsed to 64-byte
 * nodes holding four child boxes quantised to 8 bits and rounded outward.
 * Leaves are the binary tree's (same triangle slots).  Layout of a node:
 * float origin[3]; int8 exp[3]; uint8 nchild; uint8 lo[3][4]; uint8 hi[3][4];
 * uint32 child[4] (bit 31 = leaf: count in bits 24-30, first slot in 0-23);
 * uint32 pad[2].  Writes up to `capacity` nodes; *out_count, *out_root (node
 * index or leaf ref) and *out_stack (worst-case traversal stack) are always
 * set on AE_OK or AE_ERR_OVERSIZE. */
int ae_build_wide_bvh(const ae_bvh_node *blas, uint32_t n_nodes, uint32_t tri_count, void *out_nodes,
                      uint32_t capacity, uint32_t *out_count, uint32_t *out_root, int32_t *out_stack);

/* RebuildAcceleration + UploadScene (renderer/renderer.cpp:1087-1130):
 * ae_pack_scene_gpu of the entities, then ae_upload_scene.  The context's
 * scene is then exactly the reference's after a rebuild (SAH TLAS, objects
 * in slot order), unlike ae_refit_instances, which keeps the tree. */
int ae_rebuild_scene(ae_ctx *ctx, const ae_entity *entities, uint32_t n, const ae_mesh_library *lib);

/* GPU TLAS refit: new instance transforms on the device; recompute world
 * bounds of every mesh object bottom-up without rebuilding topology
 * (replaces the per-frame CPU rebuild of renderer/renderer.cpp:1087-1130
 * when only transforms changed). */
int ae_refit_instances(ae_ctx *ctx, const ae_instance *instances, uint32_t n);

/* Copies of the device's per-frame arrays as the kernels see them (after any
 * refit): objects, TLAS nodes, instances, each sized as last uploaded.  Null
 * pointers are skipped. */
int ae_download_scene(ae_ctx *ctx, ae_object *objects, ae_bvh_node *tlas, ae_instance *instances);
/* Element counts of the current scene arrays (null pointers skipped). */
int ae_scene_sizes(const ae_ctx *ctx, uint32_t *n_objects, uint32_t *n_nodes, uint32_t *n_lights,
                   uint32_t *n_instances);

/* ------------------------------------------------------------------------ */
/* Render serving (no counterpart in the reference, which renders one scene  */
/* for one window per process)                                               */
/* ------------------------------------------------------------------------ */

/* A server keeps several scenes resident on one GPU and renders frame
 * requests against them with continuous batching: a fixed pool of path slots
 * is shared by every admitted request, one merged ray queue carries rays of
 * all requests and scenes, and a request is admitted as soon as resident
 * slots and image memory free up, while others are still on the GPU.  Each
 * slot renders all samples of one pixel in order, so a request's image does
 * not depend on what else is being served: it equals `frames` compute-only
 * frames (Batch = 0 .. frames-1) of ae_render_frame on the same scene and
 * config, bit for bit.
 *
 * Threading: the server runs a scheduler thread and a completion thread;
 * every ae_serve_* call may be made from any thread.  A context handed to
 * ae_serve_add_scene belongs to the server until ae_serve_destroy (no other
 * call may use it meanwhile) and must outlive the server. */
typedef struct ae_server ae_server;

typedef struct ae_serve_settings {
    int32_t device;
    uint32_t slots;            /* paths in flight over all requests; 0 = 1,048,576 */
    uint32_t max_lights;       /* light samples per path vertex; 0 = 16, at most 64 */
    uint32_t max_requests;     /* requests resident at once; 0 = 64, at most 1024 */
    uint64_t arena_bytes;      /* device memory for request images; 0 = 1 GiB */
    uint32_t ticks_per_launch; /* queue ticks per graph replay (even); 0 = 4 */
    uint32_t extend_threads;   /* 0 = step-wise walker (default); 64, 128 or 256 = tile-staged extend */
    uint32_t max_scenes;       /* resident scenes; 0 = 16 */
    uint32_t claim_policy;     /* AE_CLAIM_OLDEST_FIRST (0) or AE_CLAIM_SHARED (1) */
    uint32_t queue_run;        /* walker extend and shadow stages: queue entries a warp takes at a time
                                  (runs of consecutive entries); 0 = default (32), 1 = static assignment
                                  (entry k + grid size); at most 1024 */
    uint32_t reserved[3];
} ae_serve_settings;

/* How free slots pick the next pixel: from the oldest admitted request that
 * still has unclaimed pixels, or spread over all admitted requests (each warp
 * starts its search at a different request), which lets short requests
 * finish while long ones run. */
enum { AE_CLAIM_OLDEST_FIRST = 0, AE_CLAIM_SHARED = 1 };

typedef struct ae_serve_request {
    uint32_t scene;            /* id from ae_serve_add_scene */
    uint32_t width, height;    /* image size (overrides config.width/height) */
    uint32_t frames;           /* progressive frames; spp = frames x samples */
    ae_config config;          /* camera, samples per frame, depth, sky, exposure; batch is ignored */
    float *accum;              /* host destination: width*height RGBA float32, or NULL */
    uint8_t *display;          /* host destination: width*height RGBA8, or NULL */
    uint64_t user;             /* opaque tag returned in the result */
} ae_serve_request;

typedef struct ae_serve_result {
    uint64_t id, user;
    int32_t status;            /* AE_OK, or why the request failed */
    uint32_t scene_version;    /* instance moves of the scene applied before it */
    double submit_ms, admit_ms, done_ms;  /* server clock: ms since ae_serve_create */
    uint64_t paths;            /* width * height * frames * samples per frame */
    uint64_t footprint;        /* bytes of image memory it held */
} ae_serve_result;

typedef struct ae_serve_stats {
    uint64_t submitted, completed, rejected, failed;
    uint64_t paths;            /* paths of completed requests */
    uint64_t rays;             /* closest-hit rays traced (extend + shadow tests) */
    double first_submit_ms, last_done_ms;
    double p50_ms, p99_ms, mean_ms, max_ms;  /* latency: submit -> result in host memory */
    uint64_t launches;         /* graph replays */
    uint64_t peak_arena_bytes;
    uint32_t peak_resident, moves_applied;
    uint32_t errors;           /* device error flags (bounded waits that gave up) */
    uint32_t cancelled;        /* requests ended by ae_serve_cancel */
    uint32_t moves_coalesced;  /* moves superseded by a later one before any request needed them */
    uint32_t pad;
} ae_serve_stats;

ae_server *ae_serve_create(const ae_serve_settings *settings);
/* Stops the threads; queued requests fail with AE_ERR_STATE. */
void ae_serve_destroy(ae_server *srv);
const char *ae_serve_last_error(ae_server *srv);
/* Makes an uploaded context's scene resident (prepares its optimised BVH). */
int ae_serve_add_scene(ae_server *srv, ae_ctx *scene, uint32_t *scene_id);
/* Queues a request; AE_ERR_REJECTED when its images exceed the whole arena. */
int ae_serve_submit(ae_server *srv, const ae_serve_request *req, uint64_t *id);
/* Queues new transforms for every instance of a scene (refit on the GPU);
 * requests submitted earlier render the old ones, later ones the new.  The
 * server keeps AE_SERVE_FRAME_SETS copies of each scene's per-frame arrays
 * (objects, TLAS, instances): a move is refit into a copy that no
 * outstanding request renders, while requests of older versions still run.
 * Moves that no request will render (several per frame interval, none
 * submitted between them) are coalesced into the next: a move carries
 * absolute transforms. */
#define AE_SERVE_FRAME_SETS 8u
int ae_serve_move_instances(ae_server *srv, uint32_t scene, const ae_instance *instances, uint32_t n);
/* Withdraws a request (no counterpart in the reference).  A queued request
 * ends at once; one on the GPU stops claiming pixels, its pixels in flight
 * finish, and then its slots and its image block in the arena go back to the
 * pool; requests beside it are unaffected.  Its result is not copied out;
 * ae_serve_wait returns AE_ERR_CANCELLED for it.  AE_ERR_STATE when the
 * request has already finished or is having its result copied. */
int ae_serve_cancel(ae_server *srv, uint64_t id);
/* Waits for a request (timeout_ms < 0: forever); returns its status, or
 * AE_ERR_TIMEOUT when the wait runs out.  A finished request fills `out`
 * (its status too, which is AE_ERR_TIMEOUT itself for a request ended by a
 * device wait that gave up); a wait that ran out leaves `out` untouched.  The
 * record is released once it has been returned. */
int ae_serve_wait(ae_server *srv, uint64_t id, int32_t timeout_ms, ae_serve_result *out);
/* Waits until every submitted request and move has finished. */
int ae_serve_drain(ae_server *srv, int32_t timeout_ms);
int ae_serve_get_stats(ae_server *srv, ae_serve_stats *out);
/* Clears latency samples and counters (not the resident scenes). */
int ae_serve_reset_stats(ae_server *srv);

/* The admission policy of the server run on a synthetic event list on the
 * host, with no GPU: requests (footprint, service ticks) and instance moves
 * arrive at ticks; out[i] tells when each was admitted / applied and done.
 * frame_sets = copies of each scene's per-frame arrays (the server uses 2). */
enum { AE_POLICY_REQUEST = 0, AE_POLICY_MOVE = 1, AE_POLICY_CANCEL = 2 };
typedef struct ae_policy_event {
    uint32_t kind;             /* AE_POLICY_REQUEST, AE_POLICY_MOVE, or AE_POLICY_CANCEL:
                                  footprint = index of the request event withdrawn */
    uint32_t scene;
    uint32_t tick;             /* arrival; non-decreasing over the list */
    uint32_t service_ticks;    /* requests: ticks on the GPU once admitted */
    uint64_t footprint;        /* requests: image bytes */
} ae_policy_event;
typedef struct ae_policy_outcome {
    int32_t admit_tick;        /* -1 = never; moves: the tick it was applied or coalesced */
    int32_t done_tick;
    uint32_t version;          /* requests: moves of the scene before it; moves: version after */
    int32_t status;            /* AE_OK, AE_ERR_REJECTED or AE_ERR_CANCELLED */
    uint64_t offset;           /* requests: arena offset; moves: the copy of the per-frame
                                  arrays written, or ~0 when coalesced into a later move */
} ae_policy_outcome;
int ae_serve_policy_simulate(const ae_policy_event *events, uint32_t n, uint64_t arena_bytes,
                             uint32_t max_resident, uint32_t n_scenes, uint32_t frame_sets,
                             uint32_t max_ticks, ae_policy_outcome *out);

/* ------------------------------------------------------------------------ */
/* Test hooks (no counterpart in the reference): failures made on purpose so */
/* the error paths can be exercised without faulting or exhausting a GPU.    */
/* ------------------------------------------------------------------------ */

/* The n-th device allocation of the library from now fails (n = 0: the next
 * one) as if the GPU were out of memory; the ones after it succeed again.
 * n < 0 clears a pending failure.  Process-wide. */
int ae_debug_fail_alloc_after(int64_t n);
/* Device allocations of the library currently live (all contexts, servers
 * and builders of the process): equal before and after a failed call when
 * nothing leaked. */
int64_t ae_debug_live_allocations(void);
/* Why the last ae_create or ae_serve_create on the calling thread returned
 * NULL (AE_ERR_INVALID, AE_ERR_OOM, AE_ERR_CUDA), or AE_OK after a success.
 * Both constructors return a handle as the reference's Renderer::Initialize
 * returns a bool; this gives the failure class. */
int ae_create_status(void);
/* AE_FAULT_TILE_WAIT: the tile-staged extend kernels issue no bulk copy and
 * their bounded wait on the (unarmed) mbarrier phase runs out after a few
 * polls, as a copy that never lands would; no copy is in flight when they
 * give up.  ae_render_frame (wavefront forms) then returns AE_ERR_TIMEOUT;
 * on a server, every unfinished request ends with AE_ERR_TIMEOUT (serving
 * uses the tile-staged extend when extend_threads != 0).  on = 0 turns the
 * fault off. */
/* AE_FAULT_CHECK_LIMITS: the debug walk (AE_VARIANT_PLAIN_CHECKED) checks
 * against capacities and lengths below the true ones (stacks of 2 entries,
 * half of every array), so its checks fire on a valid scene while every access
 * it still makes stays inside the real arrays. */
enum { AE_FAULT_TILE_WAIT = 1, AE_FAULT_CHECK_LIMITS = 2 };
int ae_debug_inject(ae_ctx *ctx, int fault, uint32_t on);
/* The check word of the debug walk (AE_CHECK_* bits set since the last read),
 * then cleared.  Synchronises the context's stream.  No counterpart in the
 * reference (its shaders have no checks). */
int ae_debug_flags(ae_ctx *ctx, uint32_t *flags);
int ae_serve_debug_inject(ae_server *srv, int fault, uint32_t on);

#ifdef __cplusplus
} /* extern "C" */

static_assert(sizeof(ae_object) == 128, "Object_GPU stride");
static_assert(offsetof(ae_object, radius) == 28, "Object_GPU layout");
static_assert(offsetof(ae_object, rotation) == 76, "Object_GPU layout");
static_assert(offsetof(ae_object, density) == 80, "Object_GPU layout");
static_assert(offsetof(ae_object, emission) == 84, "Object_GPU layout");
static_assert(offsetof(ae_object, textureTint) == 92, "Object_GPU layout");
static_assert(offsetof(ae_object, r) == 96, "Object_GPU layout");
static_assert(offsetof(ae_object, fuzz) == 108, "Object_GPU layout");
static_assert(offsetof(ae_object, textureID) == 124, "Object_GPU layout");
static_assert(sizeof(ae_instance) == 48, "MeshInstance_GPU stride");
static_assert(sizeof(ae_bvh_node) == 48, "BVHNode_GPU stride");
static_assert(sizeof(ae_vertex) == 32, "Vertex_GPU stride");
static_assert(offsetof(ae_config, exposure) == 124, "Config layout");
static_assert(offsetof(ae_config, debugView) == 128, "Config layout");
static_assert(offsetof(ae_config, jitter_y) == 144, "Config layout");
static_assert(offsetof(ae_config, displayOnly) == 148, "Config layout");
static_assert(offsetof(ae_config, traceScale) == 152, "Config layout");
static_assert(offsetof(ae_config, frameIndex) == 156, "Config layout");
static_assert(offsetof(ae_config, historyCap) == 168, "Config layout");
static_assert(offsetof(ae_config, prevViewProj) == 176, "Config layout");
static_assert(sizeof(ae_config) == 240, "Config size");
static_assert(sizeof(ae_ray) == 32, "ray record");
static_assert(sizeof(ae_hit) == 20, "hit record");
static_assert(sizeof(ae_serve_settings) == 56, "serve settings");
static_assert(sizeof(ae_serve_request) == 280, "serve request");
static_assert(sizeof(ae_serve_result) == 64, "serve result");
static_assert(sizeof(ae_serve_stats) == 136, "serve stats");
static_assert(sizeof(ae_policy_event) == 24, "policy event");
static_assert(sizeof(ae_policy_outcome) == 24, "policy outcome");
#endif

#endif /* AE_B200_H */
