// Compile-only stand-in, see nanovdb/NanoVDB.h in this directory.
#pragma once
#include <nanovdb/NanoVDB.h>
namespace nanovdb { namespace math {
template <int Order>
struct ZeroSampler {
    __host__ __device__ float operator()(const Vec3f&) const { return 0.0f; }
};
template <int Order, typename AccessorT>
__host__ __device__ ZeroSampler<Order> createSampler(const AccessorT&) { return ZeroSampler<Order>{}; }
}}  // namespace nanovdb::math
