// Test-infrastructure stand-in, see nanovdb/NanoVDB.h in this directory: the
// order-1 (trilinear) sampler over the dense grid. Each interpolation step is
// a + w * (b - a) as one fused multiply-add, along z, then y, then x, with the
// 8 voxels around floor(x) (0 outside the grid).
#pragma once
#include <nanovdb/NanoVDB.h>
namespace nanovdb { namespace math {
template <int Order>
struct DenseSampler;

template <>
struct DenseSampler<1> {
    const FloatGrid* grid;
    __host__ __device__ static float lerp(float a, float b, float w) { return fmaf(w, b - a, a); }
    __host__ __device__ float operator()(const Vec3f& x) const {
        const float fx = floorf(x[0]), fy = floorf(x[1]), fz = floorf(x[2]);
        // every voxel outside (or a NaN coordinate): the value is 0
        if (!(fx >= -1.0f && fx <= (float)(grid->dims[0] - 1) && fy >= -1.0f && fy <= (float)(grid->dims[1] - 1) &&
              fz >= -1.0f && fz <= (float)(grid->dims[2] - 1)))
            return 0.0f;
        const int i = (int)fx, j = (int)fy, k = (int)fz;
        const float u = x[0] - fx, v = x[1] - fy, w = x[2] - fz;
        const float z00 = lerp(grid->voxel(i, j, k), grid->voxel(i, j, k + 1), w);
        const float z01 = lerp(grid->voxel(i, j + 1, k), grid->voxel(i, j + 1, k + 1), w);
        const float z10 = lerp(grid->voxel(i + 1, j, k), grid->voxel(i + 1, j, k + 1), w);
        const float z11 = lerp(grid->voxel(i + 1, j + 1, k), grid->voxel(i + 1, j + 1, k + 1), w);
        return lerp(lerp(z00, z01, v), lerp(z10, z11, v), u);
    }
};

template <int Order, typename AccessorT>
__host__ __device__ DenseSampler<Order> createSampler(const AccessorT& accessor) {
    return DenseSampler<Order>{accessor.grid};
}
}}  // namespace nanovdb::math
