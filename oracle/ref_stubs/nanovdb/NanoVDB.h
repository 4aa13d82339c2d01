// Compile-only stand-in for nanovdb (openvdb v12.0.1, nanovdb/ subtree), which
// the reference fetches at configure time and which is absent here. It declares
// the few names src/path_tracer.cu uses in sampleVolumeDensity
// (path_tracer.cu:784-789). No scene here carries a density grid, so these
// bodies never run; they return zero density.
#pragma once
namespace nanovdb {
struct Vec3f {
    float v[3];
    __host__ __device__ Vec3f(float a, float b, float c) { v[0] = a; v[1] = b; v[2] = c; }
};
struct FloatAccessor {};
struct FloatTree {
    __host__ __device__ FloatAccessor getAccessor() const { return FloatAccessor{}; }
};
struct FloatGrid {
    FloatTree mTree;
    __host__ __device__ Vec3f worldToIndexF(const Vec3f& p) const { return p; }
    __host__ __device__ const FloatTree& tree() const { return mTree; }
};
}  // namespace nanovdb
