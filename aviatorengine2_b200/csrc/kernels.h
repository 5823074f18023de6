// kernels.h - host-visible launchers and per-frame parameter blocks.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/ae_b200.h"
#include "ae_math.h"

namespace ae {

struct DevScene;
struct Checks;

// Everything the frame kernels derive from Config once per frame (the camera
// basis of hybrid:1347-1361), computed on the host with the same intrinsics
// the shader uses per invocation.
struct FrameParams {
    uint32_t width, height, batch, spp, depth, display_only, frame_index;
    float exposure, defocus_angle;
    f3 source, pixel0, pixel_u, pixel_v, defocus_u, defocus_v, sky;
    f3 cam_u, cam_v, cam_w;
};

FrameParams make_frame_params(const ae_config &c);

// watertight: the watertight triangle test in the same walk (AE_VARIANT_PLAIN_WT).
cudaError_t launch_closest_plain(const DevScene &S, const ae_ray *rays, uint32_t n, ae_hit *hits, cudaStream_t st,
                                 bool watertight = false);
cudaError_t launch_closest_checked(const DevScene &S, const Checks &C, const ae_ray *rays, uint32_t n, ae_hit *hits,
                                   cudaStream_t st);
cudaError_t launch_count_plain(const DevScene &S, const ae_ray *rays, uint32_t n, unsigned long long *totals,
                               cudaStream_t st);
cudaError_t launch_count_paths(const DevScene &S, const FrameParams &F, unsigned long long *totals, cudaStream_t st);
cudaError_t launch_render_plain(const DevScene &S, const FrameParams &F, float4 *accum, uchar4 *display,
                                float4 *frame, cudaStream_t st);

}  // namespace ae
