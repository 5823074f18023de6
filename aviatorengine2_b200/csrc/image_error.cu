// image_error.cu - error of a rendered image against a reference image,
// reduced on the GPU in FP64.  This is the only FP64 arithmetic on the
// device: it scores FP32 renders against the FP64 CPU oracle.
//
// Two passes keep the result independent of scheduling: each block reduces a
// fixed stripe of pixels in a fixed tree order into one partial per block,
// then a single block adds the partials in block order.
#include <cuda_runtime.h>

#include <vector>

#include "context.h"

namespace ae {
namespace {

constexpr int kErrThreads = 256;
constexpr int kErrBlocks = 592;  // 4 per SM on a 148-SM B200

struct ErrPartial {
    double rel, abs, sq, max;
};

__device__ ErrPartial block_reduce(ErrPartial v) {
    __shared__ ErrPartial sh[kErrThreads / 32];
    for (int off = 16; off > 0; off >>= 1) {
        v.rel += __shfl_down_sync(0xffffffffu, v.rel, off);
        v.abs += __shfl_down_sync(0xffffffffu, v.abs, off);
        v.sq += __shfl_down_sync(0xffffffffu, v.sq, off);
        v.max = fmax(v.max, __shfl_down_sync(0xffffffffu, v.max, off));
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    if (warp == 0) {
        v = lane < kErrThreads / 32 ? sh[lane] : ErrPartial{0.0, 0.0, 0.0, 0.0};
        for (int off = 16; off > 0; off >>= 1) {
            v.rel += __shfl_down_sync(0xffffffffu, v.rel, off);
            v.abs += __shfl_down_sync(0xffffffffu, v.abs, off);
            v.sq += __shfl_down_sync(0xffffffffu, v.sq, off);
            v.max = fmax(v.max, __shfl_down_sync(0xffffffffu, v.max, off));
        }
    }
    return v;
}

// Pixel p of the comparison is image pixel p, or (xy[2p], xy[2p+1]) when a
// pixel list is given (coordinates checked on the host).
__global__ void __launch_bounds__(kErrThreads) k_image_error(const float4 *__restrict__ img,
                                                             const double *__restrict__ ref, size_t n, double eps,
                                                             const uint32_t *__restrict__ xy, uint32_t width,
                                                             ErrPartial *partials) {
    ErrPartial acc{0.0, 0.0, 0.0, 0.0};
    for (size_t p = size_t(blockIdx.x) * kErrThreads + threadIdx.x; p < n; p += size_t(gridDim.x) * kErrThreads) {
        const float4 x = img[xy ? size_t(xy[2 * p + 1]) * width + xy[2 * p] : p];
        const double xs[3] = {double(x.x), double(x.y), double(x.z)};
        for (int k = 0; k < 3; k++) {
            const double r = ref[4 * p + k];
            const double e = fabs(xs[k] - r);
            acc.rel += e / (fabs(r) + eps);
            acc.abs += e;
            acc.sq += e * e;
            acc.max = fmax(acc.max, e);
        }
    }
    const ErrPartial b = block_reduce(acc);
    if (threadIdx.x == 0) partials[blockIdx.x] = b;
}

__global__ void __launch_bounds__(kErrThreads) k_image_error_final(const ErrPartial *partials, int n_partials,
                                                                   double count, double *out) {
    ErrPartial acc{0.0, 0.0, 0.0, 0.0};
    for (int i = threadIdx.x; i < n_partials; i += kErrThreads) {
        const ErrPartial p = partials[i];
        acc.rel += p.rel;
        acc.abs += p.abs;
        acc.sq += p.sq;
        acc.max = fmax(acc.max, p.max);
    }
    const ErrPartial t = block_reduce(acc);
    if (threadIdx.x == 0) {
        out[0] = t.rel / count;
        out[1] = t.abs / count;
        out[2] = t.max;
        out[3] = sqrt(t.sq / count);
    }
}

}  // namespace
}  // namespace ae

using namespace ae;

static int image_error(ae_ctx *ctx, int which, const uint32_t *xy, uint32_t n_px, const double *reference,
                       double eps, double *out4) {
    Ctx *c = reinterpret_cast<Ctx *>(ctx);
    if (!c) return AE_ERR_INVALID;
    if (!reference || !out4) return c->fail(AE_ERR_INVALID, "null reference or output");
    if (!(eps >= 0.0)) return c->fail(AE_ERR_INVALID, "eps must be non-negative");
    const float4 *img = nullptr;
    if (which == AE_IMAGE_ACCUM) img = c->accum.ptr;
    else if (which == AE_IMAGE_FRAME) img = c->frame.ptr;
    else return c->fail(AE_ERR_INVALID, "image error compares AE_IMAGE_ACCUM or AE_IMAGE_FRAME");
    const uint32_t W = c->settings.width, H = c->settings.height;
    const size_t n = xy ? size_t(n_px) : size_t(W) * H;
    if (!img || size_t(W) * H == 0) return c->fail(AE_ERR_STATE, "no image yet");
    if (xy) {
        if (n_px == 0) return c->fail(AE_ERR_INVALID, "empty pixel list");
        for (uint32_t i = 0; i < n_px; i++)
            if (xy[2 * i] >= W || xy[2 * i + 1] >= H)
                return c->fail(AE_ERR_INVALID, "pixel %u (%u, %u) outside the %ux%u image", i, xy[2 * i], xy[2 * i + 1],
                               W, H);
    }
    int rc = c->cuda(cudaSetDevice(c->settings.device), "cudaSetDevice");
    if (rc) return rc;
    // Scratch for the reference copy, the pixel list, the partials and the result.
    const size_t ref_bytes = n * 4 * sizeof(double);
    const size_t xy_bytes = xy ? ((n * 2 * sizeof(uint32_t) + 15) / 16) * 16 : 0;
    const size_t part_bytes = kErrBlocks * sizeof(ErrPartial);
    void *scratch = nullptr;
    if (dev_alloc(&scratch, ref_bytes + xy_bytes + part_bytes + 4 * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        return c->fail(AE_ERR_OOM, "image error scratch");
    }
    double *d_ref = static_cast<double *>(scratch);
    uint32_t *d_xy = xy ? reinterpret_cast<uint32_t *>(static_cast<char *>(scratch) + ref_bytes) : nullptr;
    ErrPartial *d_part = reinterpret_cast<ErrPartial *>(static_cast<char *>(scratch) + ref_bytes + xy_bytes);
    double *d_out = reinterpret_cast<double *>(static_cast<char *>(scratch) + ref_bytes + xy_bytes + part_bytes);
    rc = c->cuda(cudaMemcpyAsync(d_ref, reference, ref_bytes, cudaMemcpyHostToDevice, c->stream), "upload reference");
    if (!rc && xy)
        rc = c->cuda(cudaMemcpyAsync(d_xy, xy, n * 2 * sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream),
                     "upload pixel list");
    if (!rc) {
        k_image_error<<<kErrBlocks, kErrThreads, 0, c->stream>>>(img, d_ref, n, eps, d_xy, W, d_part);
        k_image_error_final<<<1, kErrThreads, 0, c->stream>>>(d_part, kErrBlocks, double(n) * 3.0, d_out);
        c->launches += 2;
        rc = c->cuda(cudaGetLastError(), "image error launch");
    }
    if (!rc) rc = c->cuda(cudaMemcpyAsync(out4, d_out, 4 * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "copy");
    if (!rc) rc = c->cuda(cudaStreamSynchronize(c->stream), "image error");
    dev_free(scratch);
    return rc;
}

extern "C" int ae_image_error(ae_ctx *ctx, int which, const double *reference, double eps, double *out4) {
    return image_error(ctx, which, nullptr, 0, reference, eps, out4);
}

extern "C" int ae_image_error_pixels(ae_ctx *ctx, int which, const uint32_t *xy, uint32_t n_px,
                                     const double *reference, double eps, double *out4) {
    if (ctx && !xy) return reinterpret_cast<Ctx *>(ctx)->fail(AE_ERR_INVALID, "null pixel list");
    return image_error(ctx, which, xy, n_px, reference, eps, out4);
}
