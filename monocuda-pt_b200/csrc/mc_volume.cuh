// mc_volume.cuh - heterogeneous media: the dense density grid, its trilinear
// sample, and the two trackers of PT:784-838.
//
// The reference reads a NanoVDB FloatGrid (PT:784-789: worldToIndexF, then
// nanovdb::math::createSampler<1>, a trilinear sampler with background 0).
// mc_volume_grid is a dense stand-in with the same reading: index point
// (p - origin) * inv_voxel_size, the 8 voxels around its floor, interpolated
// along z, then y, then x. Delta tracking (free flight) and ratio tracking
// (transmittance) follow PT:796-815 and PT:817-838 step for step, so that
// they draw the same random numbers in the same order as the reference.
#pragma once

#include "mc_math.cuh"

namespace mc {

constexpr int kVolumeHeaderBytes = 64;
static_assert(sizeof(mc_volume_grid) == kVolumeHeaderBytes, "the voxels follow the 64-byte header");

MC_D const float* volume_voxels(const mc_volume_grid* g) {
    return reinterpret_cast<const float*>(reinterpret_cast<const char*>(g) + kVolumeHeaderBytes);
}

MC_D float volume_lerp(float a, float b, float w) { return fmaf(w, b - a, a); }

// Grid value at world point p (0 outside the voxels).
MC_D float volume_density(const mc_volume_grid* g, const V3& p) {
    const float inv = g->inv_voxel_size;
    const float x = (p.x - g->origin[0]) * inv;
    const float y = (p.y - g->origin[1]) * inv;
    const float z = (p.z - g->origin[2]) * inv;
    const int nx = g->dims[0], ny = g->dims[1], nz = g->dims[2];
    const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
    // all 8 voxels outside (or a NaN coordinate): every term is 0
    if (!(fx >= -1.0f && fx <= (float)(nx - 1) && fy >= -1.0f && fy <= (float)(ny - 1) && fz >= -1.0f &&
          fz <= (float)(nz - 1)))
        return 0.0f;
    const int i = (int)fx, j = (int)fy, k = (int)fz;
    const float u = x - fx, v = y - fy, w = z - fz;
    const float* vox = volume_voxels(g);
    auto at = [&](int a, int b, int c) -> float {
        if (a < 0 || b < 0 || c < 0 || a >= nx || b >= ny || c >= nz) return 0.0f;
        return __ldg(vox + a + (long long)nx * (b + (long long)ny * c));
    };
    const float c00 = volume_lerp(at(i, j, k), at(i, j, k + 1), w);
    const float c01 = volume_lerp(at(i, j + 1, k), at(i, j + 1, k + 1), w);
    const float c10 = volume_lerp(at(i + 1, j, k), at(i + 1, j, k + 1), w);
    const float c11 = volume_lerp(at(i + 1, j + 1, k), at(i + 1, j + 1, k + 1), w);
    return volume_lerp(volume_lerp(c00, c01, v), volume_lerp(c10, c11, v), u);
}

// PT:796-815 delta tracking: the distance of the first real collision along
// o + d t, or maxDistance when the ray leaves the medium without one.
template <class Rng>
MC_D float volume_free_flight(const mc_volume_grid* g, float extinctionScale, float gridMax, const V3& o, const V3& d,
                              float maxDistance, Rng& rng) {
    const float majorant = extinctionScale * gridMax;
    if (!(majorant > 0.0f)) return maxDistance;
    float t = 0.0f;
    for (int step = 0; step < 8192; step++) {
        t -= logf(1.0f - rng.uniform()) / majorant;
        if (t >= maxDistance) return maxDistance;
        const float density = volume_density(g, o + d * t);
        if (rng.uniform() < density / gridMax) return t;
    }
    return maxDistance;
}

// PT:817-838 ratio tracking: the transmittance of the segment o + d t, t in
// [0, length), as the product of (1 - density / majorant) at the tentative
// collisions; 0 once it falls below 1e-4.
template <class Rng>
MC_D float volume_transmittance(const mc_volume_grid* g, float extinctionScale, float gridMax, const V3& o, const V3& d,
                                float length, Rng& rng) {
    const float majorant = extinctionScale * gridMax;
    if (!(majorant > 0.0f)) return 1.0f;
    float T = 1.0f;
    float t = 0.0f;
    for (int step = 0; step < 8192; step++) {
        t -= logf(1.0f - rng.uniform()) / majorant;
        if (t >= length) break;
        const float density = volume_density(g, o + d * t);
        T = T * (1.0f - density / gridMax);
        if (T < 1e-4f) return 0.0f;
    }
    return T;
}

}  // namespace mc
