// mc_shade.cuh - materials, environment map, light and camera sampling.
// Every function restates the reference function it cites (path_tracer.cu),
// keeping its operation order and its order of random draws.
#pragma once
#include "mc_math.cuh"
#include "mc_abi.h"

namespace mc {

MC_D V3 v3(const mc_vec3& v) { return V3(v.x, v.y, v.z); }

// PT:216-234 sampleTexture
MC_D V3 sample_texture(const mc_texture& t, float u, float v) {
    switch (t.type) {
        case MC_TEX_SOLID: return v3(t.color_a);
        case MC_TEX_CHECKER: {
            int cu = (int)floorf(u * t.scale);
            int cv = (int)floorf(v * t.scale);
            bool even = ((cu + cv) & 1) == 0;
            return even ? v3(t.color_a) : v3(t.color_b);
        }
        case MC_TEX_IMAGE: {
            float4 texel = tex2D<float4>((cudaTextureObject_t)t.image, u, 1.0f - v);
            return V3(texel.x, texel.y, texel.z);
        }
        default: return V3(1.f, 0.f, 1.f);
    }
}

// PT:408-412 environmentUv
MC_D V2 env_uv(const mc_env_map& env, const V3& d) {
    float u = atan2f(d.z, d.x) / (2.0f * MC_PI) + 0.5f + env.rotation / (2.0f * MC_PI);
    float v = acosf(fminf(fmaxf(d.y, -1.0f), 1.0f)) / MC_PI;
    return V2(u - floorf(u), v);
}

// PT:414-419 environmentDirection
MC_D V3 env_direction(const mc_env_map& env, float u, float v) {
    float phi = (u - 0.5f) * 2.0f * MC_PI - env.rotation;
    float theta = v * MC_PI;
    float sinTheta = sinf(theta);
    return V3(cosf(phi) * sinTheta, cosf(theta), sinf(phi) * sinTheta);
}

// PT:421-426 environmentRadiance
MC_D V3 env_radiance(const mc_env_map& env, const V3& d, const V3& fallback) {
    if (!env.enabled) return fallback;
    V2 uv = env_uv(env, d.normalize());
    float4 texel = tex2D<float4>((cudaTextureObject_t)env.texture, uv.x, uv.y);
    return V3(texel.x, texel.y, texel.z) * env.intensity;
}

// PT:428-431 environmentSelectionProbability
MC_D float env_selection_probability(const mc_env_map& env, int lightCount) {
    if (!env.enabled || env.total_weight <= 0.0f) return 0.0f;
    return (lightCount > 0) ? 0.5f : 1.0f;
}

// PT:433-442 findCdfInterval
MC_D int find_cdf_interval(const float* cdf, int count, float value) {
    int low = 0, high = count - 1;
    while (low < high) {
        int mid = (low + high) >> 1;
        if (cdf[mid + 1] <= value) low = mid + 1;
        else high = mid;
    }
    return low;
}

// PT:444-449 environmentTexelPdf
MC_D float env_texel_pdf(const mc_env_map& env, int row, int col, float sinTheta) {
    if (sinTheta < 1e-6f) return 0.0f;
    const float* cdf = env.col_cdf + (size_t)row * (env.width + 1);
    float w = cdf[col + 1] - cdf[col];
    return w * env.width * env.height / (env.total_weight * 2.0f * MC_PI * MC_PI * sinTheta);
}

// PT:451-457 environmentDirectionPdf
MC_D float env_direction_pdf(const mc_env_map& env, const V3& d) {
    V3 u = d.normalize();
    V2 uv = env_uv(env, u);
    int col = min((int)(uv.x * env.width), env.width - 1);
    int row = min((int)(uv.y * env.height), env.height - 1);
    return env_texel_pdf(env, row, col, sqrtf(fmaxf(1.0f - u.y * u.y, 0.0f)));
}

// PT:459-467 sampleEnvironmentDirection (CDF inversion; four draws)
template <class Rng>
MC_D V3 env_sample(const mc_env_map& env, Rng& rng, float& pdf) {
    int row = find_cdf_interval(env.row_cdf, env.height, rng.uniform() * env.total_weight);
    const float* cdf = env.col_cdf + (size_t)row * (env.width + 1);
    int col = find_cdf_interval(cdf, env.width, rng.uniform() * cdf[env.width]);
    float u = (col + rng.uniform()) / env.width;
    float v = (row + rng.uniform()) / env.height;
    pdf = env_texel_pdf(env, row, col, sinf(v * MC_PI));
    return env_direction(env, u, v);
}

// Environment direction from the map's alias table (MC_ENV_SAMPLE_ALIAS):
// texel i = floor(u0 * n), kept when u1 < its threshold, else its alias; then
// the point inside the texel and the density as in env_sample. Four draws,
// one table read instead of two binary searches; the same texel distribution
// w / total_weight as the CDFs (Walker/Vose alias method). alias: int2 per
// texel (threshold as float bits, alias index).
template <class Rng>
MC_D V3 env_sample_alias(const mc_env_map& env, const int2* __restrict__ alias, Rng& rng, float& pdf) {
    const int n = env.width * env.height;
    int i = min((int)(rng.uniform() * (float)n), n - 1);
    const int2 e = __ldg(alias + i);
    if (!(rng.uniform() < __int_as_float(e.x))) i = e.y;
    const int row = i / env.width;
    const int col = i - row * env.width;
    float u = (col + rng.uniform()) / env.width;
    float v = (row + rng.uniform()) / env.height;
    pdf = env_texel_pdf(env, row, col, sinf(v * MC_PI));
    return env_direction(env, u, v);
}

// PT:498-509 random_unit_vector (rejection in the cube)
template <class Rng>
MC_D V3 random_unit_vector(Rng& rng) {
    while (true) {
        float x = rng.uniform() * 2.f - 1.f;
        float y = rng.uniform() * 2.f - 1.f;
        float z = rng.uniform() * 2.f - 1.f;
        V3 p(x, y, z);
        if (p.length_squared() < 1.0f) return p.normalize();
    }
}

// PT:511-518
template <class Rng>
MC_D V3 lambertian_scatter(const V3& n, Rng& rng) {
    V3 r = n + random_unit_vector(rng);
    if (r.length_squared() < 1e-8f) return n;
    return r.normalize();
}

// PT:520-522
MC_D V3 specular_scatter(const V3& in, const V3& n) { return in.normalize().reflect(n); }

// PT:524-539
template <class Rng>
MC_D V3 dielectric_scatter(const V3& in, const V3& n, float eta, Rng& rng) {
    V3 unit = in.normalize();
    float cosTheta = fminf((-unit).dot(n), 1.0f);
    float sinTheta = sqrtf(1.0f - cosTheta * cosTheta);
    bool cannot = (eta * sinTheta) > 1.0f;
    float reflectProbability = cannot ? 1.0f : schlick(cosTheta, eta);
    if (rng.uniform() < reflectProbability) return unit.reflect(n);
    return refract(unit, n, eta);
}

// PT:541-551
template <class Rng>
MC_D V3 isotropic_scatter(Rng& rng) {
    float u1 = rng.uniform();
    float u2 = rng.uniform();
    float z = 1.0f - 2.0f * u1;
    float r = sqrtf(fmaxf(0.0f, 1.0f - z * z));
    float phi = 2.0f * MC_PI * u2;
    return V3(r * cosf(phi), r * sinf(phi), z);
}

// PT:556-578 Henyey-Greenstein by CDF inversion around the incoming direction
template <class Rng>
MC_D V3 hg_scatter(const V3& in, float g, Rng& rng) {
    if (fabsf(g) < 1e-3f) return isotropic_scatter(rng);
    float u1 = rng.uniform();
    float u2 = rng.uniform();
    float sq = (1.0f - g * g) / (1.0f + g - 2.0f * g * u1);
    float cosTheta = (1.0f + g * g - sq * sq) / (2.0f * g);
    cosTheta = fminf(fmaxf(cosTheta, -1.0f), 1.0f);
    float sinTheta = sqrtf(fmaxf(0.0f, 1.0f - cosTheta * cosTheta));
    float phi = 2.0f * MC_PI * u2;
    V3 forward = in.normalize();
    V3 helper = (fabsf(forward.x) > 0.9f) ? V3(0.f, 1.f, 0.f) : V3(1.f, 0.f, 0.f);
    V3 tangent = helper.cross(forward).normalize();
    V3 bitangent = forward.cross(tangent);
    return tangent * (sinTheta * cosf(phi)) + bitangent * (sinTheta * sinf(phi)) + forward * cosTheta;
}

// PT:744-755 sample_triangle
template <class Rng>
MC_D V3 sample_triangle(const V3& v0, const V3& v1, const V3& v2, Rng& rng) {
    float r1 = rng.uniform();
    float r2 = rng.uniform();
    float s = sqrtf(r1);
    float w0 = 1.0f - s;
    float w1 = r2 * s;
    float w2 = 1.0f - w0 - w1;
    return v0 * w0 + v1 * w1 + v2 * w2;
}

// PT:1633-1642 random_in_unit_disk
template <class Rng>
MC_D V3 random_in_unit_disk(Rng& rng) {
    while (true) {
        float x = rng.uniform() * 2.f - 1.f;
        float y = rng.uniform() * 2.f - 1.f;
        V3 p(x, y, 0.0f);
        if (p.length_squared() < 1.0f) return p;
    }
}

// PT:1648-1658 Camera::getRay (pixel centre, no jitter; lens sample, then time)
template <class Rng>
MC_D void camera_ray(const mc_camera& cam, int px, int py, Rng& rng, V3& origin, V3& dir, float& time) {
    V3 pixelCenter = v3(cam.pixel00) + (v3(cam.pixel_delta_u) * float(px)) + (v3(cam.pixel_delta_v) * float(py));
    V3 lens = random_in_unit_disk(rng) * cam.lens_radius;
    V3 offset = v3(cam.u) * lens.x + v3(cam.v) * lens.y;
    origin = v3(cam.center) + offset;
    time = rng.uniform();
    dir = (pixelCenter - origin).normalize();
}

}  // namespace mc
