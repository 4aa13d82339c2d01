// Test-infrastructure stand-in for nanovdb (openvdb v12.0.1, nanovdb/ subtree),
// which the reference fetches at configure time and which is absent here. It
// gives the names src/path_tracer.cu uses in sampleVolumeDensity
// (path_tracer.cu:784-789) a working meaning over a DENSE grid, so that the
// reference's own delta and ratio tracking (path_tracer.cu:796-838) can run on
// the same grids as the render library under test:
//   - a FloatGrid is a 64-byte header (the library's mc_volume_grid layout:
//     origin, voxel size, 1 / voxel size, dims, maximum, bounds) followed by
//     dims[0] * dims[1] * dims[2] floats, x fastest; value 0 outside;
//   - worldToIndexF maps p to (p - origin) * (1 / voxel size), voxel (i,j,k)
//     sitting at index point (i,j,k), as NanoVDB's index space does for a grid
//     with a uniform scale and no rotation;
//   - the order-1 sampler (math/SampleFromVoxels.h) is NanoVDB's trilinear
//     reading: the 8 voxels around floor(x), interpolated along z, y, then x.
// NanoVDB's sparse tree and its file format are not reproduced.
#pragma once
namespace nanovdb {
struct Vec3f {
    float v[3];
    __host__ __device__ Vec3f(float a, float b, float c) { v[0] = a; v[1] = b; v[2] = c; }
    __host__ __device__ float operator[](int i) const { return v[i]; }
};

struct FloatGrid;

struct FloatAccessor {
    const FloatGrid* grid;
};

// The tree sits at the grid's address; it only hands out accessors.
struct FloatTree {
    __host__ __device__ FloatAccessor getAccessor() const {
        return FloatAccessor{reinterpret_cast<const FloatGrid*>(this)};
    }
};

struct FloatGrid {
    float origin[3];
    float voxelSize;
    float inverseVoxelSize;
    int dims[3];
    float maximum;
    float worldMinimum[3];
    float worldMaximum[3];
    int reserved;

    __host__ __device__ Vec3f worldToIndexF(const Vec3f& p) const {
        return Vec3f((p.v[0] - origin[0]) * inverseVoxelSize, (p.v[1] - origin[1]) * inverseVoxelSize,
                     (p.v[2] - origin[2]) * inverseVoxelSize);
    }
    __host__ __device__ const FloatTree& tree() const { return *reinterpret_cast<const FloatTree*>(this); }
    __host__ __device__ float voxel(int i, int j, int k) const {
        if (i < 0 || j < 0 || k < 0 || i >= dims[0] || j >= dims[1] || k >= dims[2]) return 0.0f;
        const float* values = reinterpret_cast<const float*>(reinterpret_cast<const char*>(this) + 64);
        return values[i + (long long)dims[0] * (j + (long long)dims[1] * k)];
    }
};
static_assert(sizeof(FloatGrid) == 64, "the voxels follow a 64-byte header");
}  // namespace nanovdb
