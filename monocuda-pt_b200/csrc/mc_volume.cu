// mc_volume.cu - dense density grids for heterogeneous media: upload, the fog
// sphere of createFogSphereGrid (src/volume_io.cpp:53-64), and a sampling
// entry point that reads the grid exactly as the render kernels do.
//
// Compiled with --use_fast_math like mc_render.cu; the sampler is floors,
// subtractions, multiplies and fused multiply-adds, so its values do not
// depend on that flag.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "mc_internal.h"
#include "mc_volume.cuh"

#define MC_CUDA(call)                                                                      \
    do {                                                                                   \
        cudaError_t e__ = (call);                                                          \
        if (e__ != cudaSuccess) return mc::cuda_error((int)e__, #call, __FILE__, __LINE__); \
    } while (0)

namespace mc {
namespace {

__global__ void k_volume_density(const mc_volume_grid* g, const float* pts, int n, float* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = volume_density(g, V3(pts[3 * (size_t)i], pts[3 * (size_t)i + 1], pts[3 * (size_t)i + 2]));
}

bool finite3(const float* v) { return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]); }

}  // namespace
}  // namespace mc

extern "C" {

mc_status mc_volume_grid_create(mc_context* ctx, const float* density_host, int32_t nx, int32_t ny, int32_t nz,
                                const float origin[3], float voxel_size, const mc_volume_grid** d_grid,
                                mc_volume_grid* header) {
    using namespace mc;
    if (!ctx || !density_host || !origin || !d_grid || nx < 1 || ny < 1 || nz < 1 || !(voxel_size > 0.0f) ||
        !std::isfinite(voxel_size) || !finite3(origin))
        return set_error(MC_ERR_INVALID, "mc_volume_grid_create: bad arguments");
    const long long count = (long long)nx * ny * nz;
    if (count > (1ll << 34)) return set_error(MC_ERR_INVALID, "mc_volume_grid_create: grid too large");
    float maximum = 0.0f;
    for (long long i = 0; i < count; i++) {
        const float v = density_host[i];
        if (!(v >= 0.0f) || !std::isfinite(v))
            return set_error(MC_ERR_INVALID, "mc_volume_grid_create: density %lld is negative or not finite", i);
        maximum = std::max(maximum, v);
    }
    // the majorant of delta tracking; the reference refuses grids without one (volume_io.cpp:19-24)
    if (!(maximum > 0.0f)) return set_error(MC_ERR_INVALID, "mc_volume_grid_create: the grid's maximum density is 0");
    mc_volume_grid h;
    std::memset(&h, 0, sizeof(h));
    for (int a = 0; a < 3; a++) h.origin[a] = origin[a];
    h.voxel_size = voxel_size;
    h.inv_voxel_size = 1.0f / voxel_size;
    h.dims[0] = nx; h.dims[1] = ny; h.dims[2] = nz;
    h.maximum_density = maximum;
    const int n3[3] = {nx, ny, nz};
    for (int a = 0; a < 3; a++) {
        h.world_min[a] = origin[a];
        h.world_max[a] = origin[a] + voxel_size * (float)(n3[a] - 1);
    }
    char* dev = nullptr;
    const size_t bytes = kVolumeHeaderBytes + (size_t)count * sizeof(float);
    if (cudaMalloc(&dev, bytes) != cudaSuccess) {
        cudaGetLastError();
        return set_error(MC_ERR_OOM, "mc_volume_grid_create: device allocation of %zu bytes failed", bytes);
    }
    cudaError_t e = cudaMemcpyAsync(dev, &h, sizeof(h), cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    mc_status st = MC_OK;
    if (e != cudaSuccess) st = cuda_error((int)e, "cudaMemcpyAsync", __FILE__, __LINE__);
    else st = upload_host(ctx, dev + kVolumeHeaderBytes, density_host, (size_t)count * sizeof(float));
    if (st != MC_OK) {
        cudaFree(dev);
        return st;
    }
    *d_grid = reinterpret_cast<const mc_volume_grid*>(dev);
    if (header) *header = h;
    return MC_OK;
}

mc_status mc_volume_grid_destroy(const mc_volume_grid* d_grid) {
    if (d_grid) cudaFree(const_cast<mc_volume_grid*>(d_grid));
    return MC_OK;
}

mc_status mc_volume_fog_sphere(float radius, float voxel_size, float half_width, float* density_host, int32_t dims[3],
                               float origin[3]) {
    using namespace mc;
    if (!dims || !origin || !(radius > 0.0f) || !(voxel_size > 0.0f) || !(half_width > 0.0f) || !std::isfinite(radius) ||
        !std::isfinite(voxel_size) || !std::isfinite(half_width))
        return set_error(MC_ERR_INVALID, "mc_volume_fog_sphere: bad arguments");
    const double r = radius, h = voxel_size, band = (double)half_width * h;
    const double halfCount = std::ceil(r / h) + 1.0;
    if (halfCount > 2048.0) return set_error(MC_ERR_INVALID, "mc_volume_fog_sphere: more than 4097 voxels per axis");
    const int half = (int)halfCount;
    const int n = 2 * half + 1;
    for (int a = 0; a < 3; a++) {
        dims[a] = n;
        origin[a] = (float)(-half * h);
    }
    if (!density_host) return MC_OK;
    for (int k = 0; k < n; k++) {
        const double z = (k - half) * h;
        for (int j = 0; j < n; j++) {
            const double y = (j - half) * h;
            for (int i = 0; i < n; i++) {
                const double x = (i - half) * h;
                const double v = (r - std::sqrt(x * x + y * y + z * z)) / band;
                density_host[i + (size_t)n * (j + (size_t)n * k)] = (float)std::min(1.0, std::max(0.0, v));
            }
        }
    }
    return MC_OK;
}

mc_status mc_volume_density(mc_context* ctx, const mc_volume_grid* d_grid, const float* d_points, int32_t n,
                            float* d_out) {
    using namespace mc;
    if (!ctx || !d_grid || n < 0 || (n > 0 && (!d_points || !d_out)))
        return set_error(MC_ERR_INVALID, "mc_volume_density: bad arguments");
    if (n == 0) return MC_OK;
    const int blocks = std::min((n + 255) / 256, ctx->sm_count * 8);
    k_volume_density<<<blocks, 256, 0, ctx->stream>>>(d_grid, d_points, n, d_out);
    MC_CUDA(cudaGetLastError());
    MC_CUDA(cudaStreamSynchronize(ctx->stream));
    return MC_OK;
}

}  // extern "C"
