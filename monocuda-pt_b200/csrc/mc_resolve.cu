// mc_resolve.cu - resolve and output encoding of an accumulation buffer, once
// per image: resolve_kernel (PT:3092-3100) with toneMapChannel and
// linearToSrgb (PT:3060-3090), computeAutoExposure / logLuminanceSumKernel
// (PT:3101-3132), and the 8-bit encoding of main() (PT:4363-4380), fused in
// one pass over the buffer.
//
// Compiled with --use_fast_math like the reference: the per-pixel arithmetic
// (division by the sample count, powf in linearToSrgb, logf of the luminance)
// is written as the reference writes it, so the compiler emits the same
// approximations. The log-luminance sum differs on purpose: the reference adds
// FP32 warp sums with atomics in whatever order they arrive; here each block
// sums in FP64 and every block of the resolve pass adds the block sums in the
// same fixed order, so the exposure is the same on every run.
//
// Bound: HBM. Per pixel 12 B read, plus 12 B (float outputs) or 3 B (8-bit)
// written; an automatic exposure reads the buffer twice.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "mc_internal.h"

namespace mc {
namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ float linear_to_srgb(float v) {  // PT:3060-3070
    v = fmaxf(v, 0.0f);
    float s;
    if (v <= 0.0031308f) s = 12.92f * v;
    else s = 1.055f * powf(v, 1.0f / 2.4f) - 0.055f;
    return s;
}

__device__ __forceinline__ float tone_map(float v, int op) {  // PT:3074-3089
    v = fmaxf(v, 0.f);
    switch (op) {
        case MC_TONEMAP_REINHARD: return v / (1.f + v);
        case MC_TONEMAP_ACES: {
            float m = (v * (2.51f * v + 0.03f)) / (v * (2.43f * v + 0.59f) + 0.14f);
            return fminf(fmaxf(m, 0.0f), 1.0f);
        }
        default: return v;
    }
}

// PT:4370-4378: NaN shield, clamp to [0,1], 255.99 scale, truncation.
__device__ __forceinline__ unsigned char to_byte(float c) {
    float f = isfinite(c) ? fminf(fmaxf(c, 0.0f), 1.0f) : 0.0f;
    return (unsigned char)(255.99f * f);
}

__device__ double block_sum(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kThreads / 32; w++) t += sh[w];
    __syncthreads();
    return t;  // valid in thread 0
}

// ln(1e-4 + luminance) of every pixel's average (PT:3103-3111), summed per block.
__global__ void __launch_bounds__(kThreads) k_log_luminance(const float* __restrict__ accum, long long pixels,
                                                            int samples, double* __restrict__ partial) {
    __shared__ double sh[kThreads / 32];
    const float delta = 1e-4f;
    double acc = 0.0;
    for (long long p = (long long)blockIdx.x * kThreads + threadIdx.x; p < pixels; p += (long long)gridDim.x * kThreads) {
        const float fs = float(samples);
        const float rx = accum[3 * p] / fs, ry = accum[3 * p + 1] / fs, rz = accum[3 * p + 2] / fs;
        const float lum = 0.2126f * rx + 0.7152f * ry + 0.0722f * rz;
        acc += (double)logf(delta + (isfinite(lum) ? fmaxf(lum, 0.0f) : 0.0f));
    }
    const double t = block_sum(acc, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = t;
}

// fmt: MC_IMAGE_RGB8 / RGB_F32 / PFM. The exposure is `exposure`, or, when
// nparts > 0, 0.18 / exp(sum of the partials / pixels) (PT:3121-3132).
__global__ void __launch_bounds__(kThreads) k_resolve(const float* __restrict__ accum, int W, int H, int samples,
                                                      int fmt, int tonemap, float exposure,
                                                      const double* __restrict__ partial, int nparts,
                                                      void* __restrict__ out, float* __restrict__ chosen) {
    __shared__ double sh[kThreads / 32];
    __shared__ float sExposure;
    const long long pixels = (long long)W * H;
    if (nparts > 0) {
        // identical in every block: each thread sums a fixed stride of the
        // partials, then the fixed warp/block tree
        double v = 0.0;
        for (int i = threadIdx.x; i < nparts; i += kThreads) v += partial[i];
        const double t = block_sum(v, sh);
        if (threadIdx.x == 0) sExposure = (float)(0.18 / exp(t / (double)pixels));
    } else if (threadIdx.x == 0) {
        sExposure = exposure;
    }
    __syncthreads();
    const float e = sExposure;
    if (blockIdx.x == 0 && threadIdx.x == 0 && chosen) *chosen = e;
    const float fs = float(samples);
    for (long long p = (long long)blockIdx.x * kThreads + threadIdx.x; p < pixels; p += (long long)gridDim.x * kThreads) {
        // PT:3098: accumBuffer[pixel] / float(samplesSoFar) * exposure
        const float ax = accum[3 * p] / fs * e, ay = accum[3 * p + 1] / fs * e, az = accum[3 * p + 2] / fs * e;
        if (fmt == MC_IMAGE_PFM) {
            const long long y = p / W, x = p - y * W;
            float* o = (float*)out + 3 * ((H - 1 - y) * (long long)W + x);
            o[0] = ax; o[1] = ay; o[2] = az;
            continue;
        }
        const float r = linear_to_srgb(tone_map(ax, tonemap));
        const float g = linear_to_srgb(tone_map(ay, tonemap));
        const float b = linear_to_srgb(tone_map(az, tonemap));
        if (fmt == MC_IMAGE_RGB_F32) {
            float* o = (float*)out + 3 * p;
            o[0] = r; o[1] = g; o[2] = b;
        } else {
            unsigned char* o = (unsigned char*)out + 3 * p;
            o[0] = to_byte(r); o[1] = to_byte(g); o[2] = to_byte(b);
        }
    }
}

}  // namespace
}  // namespace mc

extern "C" mc_status mc_image_encode(mc_context* ctx, const float* accum, int32_t width, int32_t height, int32_t samples,
                                     const mc_image_options* opts, void* out, int64_t* bytes, float* chosen_exposure) {
    using namespace mc;
    if (!ctx || !accum || !opts || !bytes || width <= 0 || height <= 0 || samples <= 0)
        return set_error(MC_ERR_INVALID, "mc_image_encode: bad arguments");
    const int fmt = opts->format;
    if (fmt < MC_IMAGE_RGB8 || fmt > MC_IMAGE_PNG) return set_error(MC_ERR_INVALID, "mc_image_encode: unknown format %d", fmt);
    if (opts->tonemap < MC_TONEMAP_NONE || opts->tonemap > MC_TONEMAP_ACES)
        return set_error(MC_ERR_INVALID, "mc_image_encode: unknown tone map %d", opts->tonemap);
    if ((fmt == MC_IMAGE_PNG || fmt == MC_IMAGE_PFM) && opts->device_output)
        return set_error(MC_ERR_INVALID, "mc_image_encode: PNG and PFM files are written to host memory only");
    const long long pixels = (long long)width * height;
    const size_t rgb8 = (size_t)pixels * 3, f32 = (size_t)pixels * 12;
    char header[64];
    int hlen = 0;
    if (fmt == MC_IMAGE_PFM) hlen = std::snprintf(header, sizeof(header), "PF\n%d %d\n-1.0\n", width, height);
    int64_t pngBytes = 0;
    if (fmt == MC_IMAGE_PNG) {
        mc_status s = mc_png_encode(nullptr, width, height, nullptr, &pngBytes);
        if (s != MC_OK) return s;
    }
    const size_t payload = fmt == MC_IMAGE_RGB8 || fmt == MC_IMAGE_PNG ? rgb8 : f32;
    const int64_t total = fmt == MC_IMAGE_PNG ? pngBytes : (int64_t)(payload + hlen);
    if (!out) {
        *bytes = total;
        return MC_OK;
    }
    if (*bytes < total) return set_error(MC_ERR_INVALID, "mc_image_encode: output holds %lld bytes, %lld needed",
                                         (long long)*bytes, (long long)total);
    const int kind = fmt == MC_IMAGE_PNG ? MC_IMAGE_RGB8 : fmt;
    const int grid = (int)std::max(1ll, std::min((pixels + kThreads - 1) / kThreads, (long long)ctx->sm_count * 8));
    // scratch: block partials, the chosen exposure, then (host output) the payload
    const size_t partBytes = (size_t)grid * sizeof(double) + 16;
    const bool staged = !opts->device_output;
    mc_status st = devbuf_reserve(ctx->scratch[4], partBytes + (staged ? payload : 0));
    if (st != MC_OK) return st;
    double* partial = (double*)ctx->scratch[4].ptr;
    float* dChosen = (float*)((char*)ctx->scratch[4].ptr + (size_t)grid * sizeof(double));
    void* dOut = staged ? (void*)((char*)ctx->scratch[4].ptr + partBytes) : out;
    if (!staged && ((uintptr_t)out & 3u) && kind == MC_IMAGE_RGB_F32)
        return set_error(MC_ERR_INVALID, "mc_image_encode: a float output must be 4-byte aligned");
    const bool autoExposure = !(opts->exposure > 0.f);
    if (autoExposure) k_log_luminance<<<grid, kThreads, 0, ctx->stream>>>(accum, pixels, samples, partial);
    k_resolve<<<grid, kThreads, 0, ctx->stream>>>(accum, width, height, samples, kind, opts->tonemap, opts->exposure,
                                                   partial, autoExposure ? grid : 0, dOut, dChosen);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error((int)e, "mc_image_encode launch", __FILE__, __LINE__);
    float chosen = opts->exposure;
    e = cudaMemcpyAsync(&chosen, dChosen, sizeof(float), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess && staged) {
        if (fmt == MC_IMAGE_PNG) {
            std::vector<uint8_t> px(rgb8);
            e = cudaMemcpyAsync(px.data(), dOut, rgb8, cudaMemcpyDeviceToHost, ctx->stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
            if (e == cudaSuccess) {
                int64_t nb = *bytes;
                st = mc_png_encode(px.data(), width, height, (uint8_t*)out, &nb);
                if (st != MC_OK) return st;
            }
        } else {
            if (fmt == MC_IMAGE_PFM) std::memcpy(out, header, (size_t)hlen);
            e = cudaMemcpyAsync((char*)out + hlen, dOut, payload, cudaMemcpyDeviceToHost, ctx->stream);
        }
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_error((int)e, "mc_image_encode", __FILE__, __LINE__);
    *bytes = total;
    if (chosen_exposure) *chosen_exposure = chosen;
    return MC_OK;
}

extern "C" mc_status mc_image_encode_host(mc_context* ctx, const float* accum_host, int32_t width, int32_t height,
                                          int32_t samples, const mc_image_options* opts, void* out, int64_t* bytes,
                                          float* chosen_exposure) {
    using namespace mc;
    if (!ctx || !accum_host || !opts || width <= 0 || height <= 0)
        return set_error(MC_ERR_INVALID, "mc_image_encode_host: bad arguments");
    if (opts->device_output) return set_error(MC_ERR_INVALID, "mc_image_encode_host: the output goes to host memory");
    const size_t n = (size_t)width * height * 3 * sizeof(float);
    mc_status st = devbuf_reserve(ctx->scratch[3], n);
    if (st != MC_OK) return st;
    if (out) {  // a size query needs no upload
        st = upload_host(ctx, ctx->scratch[3].ptr, accum_host, n);
        if (st != MC_OK) return st;
    }
    return mc_image_encode(ctx, (const float*)ctx->scratch[3].ptr, width, height, samples, opts, out, bytes,
                           chosen_exposure);
}
