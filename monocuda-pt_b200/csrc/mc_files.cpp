// mc_files.cpp - host file readers of the command-line driver: PFM
// environment maps (the rules of loadPfmAsRgba32f, src/path_tracer.cu:335-368)
// and dense density-grid files for --volume.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "mc_internal.h"

namespace {

struct File {
    FILE* f;
    explicit File(const char* path, const char* mode) : f(std::fopen(path, mode)) {}
    ~File() {
        if (f) std::fclose(f);
    }
};

}  // namespace

extern "C" {

mc_status mc_pfm_read(const char* path, int32_t* width, int32_t* height, float* rgba) {
    if (!path || !width || !height) return mc::set_error(MC_ERR_INVALID, "mc_pfm_read: null argument");
    File file(path, "rb");
    if (!file.f) return mc::set_error(MC_ERR_NOT_FOUND, "mc_pfm_read: cannot open '%s'", path);
    // header: magic, width, height, scale as whitespace-separated fields, then one byte
    char magic[3] = {0, 0, 0};
    int w = 0, h = 0;
    float scale = 0.0f;
    if (std::fscanf(file.f, "%2s %d %d %f", magic, &w, &h, &scale) != 4 || std::strcmp(magic, "PF") != 0 || w <= 0 ||
        h <= 0 || std::fgetc(file.f) == EOF)
        return mc::set_error(MC_ERR_INVALID, "mc_pfm_read: '%s' is not a colour PFM", path);
    if (scale > 0.0f) return mc::set_error(MC_ERR_INVALID, "mc_pfm_read: '%s' is big-endian (not supported)", path);
    if ((long long)w * h > (1ll << 30)) return mc::set_error(MC_ERR_INVALID, "mc_pfm_read: '%s' is too large", path);
    std::vector<float> rgb((size_t)w * h * 3);
    if (std::fread(rgb.data(), sizeof(float), rgb.size(), file.f) != rgb.size())
        return mc::set_error(MC_ERR_INVALID, "mc_pfm_read: '%s' holds fewer than %d x %d pixels", path, w, h);
    if (rgba) {
        for (int y = 0; y < h; y++) {
            const float* src = rgb.data() + (size_t)(h - 1 - y) * w * 3;  // bottom row first in the file
            float* dst = rgba + (size_t)y * w * 4;
            for (int x = 0; x < w; x++) {
                dst[4 * x + 0] = src[3 * x + 0];
                dst[4 * x + 1] = src[3 * x + 1];
                dst[4 * x + 2] = src[3 * x + 2];
                dst[4 * x + 3] = 1.0f;
            }
        }
    }
    *width = w;
    *height = h;
    return MC_OK;
}

mc_status mc_volume_file_read(const char* path, int32_t dims[3], float origin[3], float* voxel_size,
                              float* density_host) {
    if (!path || !dims || !origin || !voxel_size) return mc::set_error(MC_ERR_INVALID, "mc_volume_file_read: null argument");
    File file(path, "rb");
    if (!file.f) return mc::set_error(MC_ERR_NOT_FOUND, "mc_volume_file_read: cannot open '%s'", path);
    char magic[6] = {0};
    int n[3] = {0, 0, 0};
    float v = 0.0f, o[3] = {0.0f, 0.0f, 0.0f};
    if (std::fscanf(file.f, "%5s %d %d %d %f %f %f %f", magic, &n[0], &n[1], &n[2], &v, &o[0], &o[1], &o[2]) != 8 ||
        std::strcmp(magic, "MCVOL") != 0 || std::fgetc(file.f) != '\n')
        return mc::set_error(MC_ERR_INVALID, "mc_volume_file_read: '%s' has no MCVOL header line", path);
    if (n[0] < 1 || n[1] < 1 || n[2] < 1 || !(v > 0.0f) || !std::isfinite(v) || !std::isfinite(o[0]) ||
        !std::isfinite(o[1]) || !std::isfinite(o[2]))
        return mc::set_error(MC_ERR_INVALID, "mc_volume_file_read: '%s' has a bad header", path);
    const long long count = (long long)n[0] * n[1] * n[2];
    if (count > (1ll << 34)) return mc::set_error(MC_ERR_INVALID, "mc_volume_file_read: '%s' is too large", path);
    for (int a = 0; a < 3; a++) {
        dims[a] = n[a];
        origin[a] = o[a];
    }
    *voxel_size = v;
    if (!density_host) return MC_OK;
    if (std::fread(density_host, sizeof(float), (size_t)count, file.f) != (size_t)count)
        return mc::set_error(MC_ERR_INVALID, "mc_volume_file_read: '%s' holds fewer than %lld values", path, count);
    return MC_OK;
}

mc_status mc_volume_file_write(const char* path, const int32_t dims[3], const float origin[3], float voxel_size,
                               const float* density_host) {
    if (!path || !dims || !origin || !density_host || dims[0] < 1 || dims[1] < 1 || dims[2] < 1 || !(voxel_size > 0.0f))
        return mc::set_error(MC_ERR_INVALID, "mc_volume_file_write: bad arguments");
    File file(path, "wb");
    if (!file.f) return mc::set_error(MC_ERR_NOT_FOUND, "mc_volume_file_write: cannot create '%s'", path);
    const size_t count = (size_t)dims[0] * dims[1] * dims[2];
    // %.9g reads back to the same float
    bool ok = std::fprintf(file.f, "MCVOL %d %d %d %.9g %.9g %.9g %.9g\n", dims[0], dims[1], dims[2], (double)voxel_size,
                           (double)origin[0], (double)origin[1], (double)origin[2]) > 0 &&
              std::fwrite(density_host, sizeof(float), count, file.f) == count;
    if (!ok) return mc::set_error(MC_ERR_INVALID, "mc_volume_file_write: writing '%s' failed", path);
    return MC_OK;
}

}  // extern "C"
