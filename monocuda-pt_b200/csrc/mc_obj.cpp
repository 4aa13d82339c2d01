// mc_obj.cpp - OBJ/MTL loading (loadObject PT:2644-2859, loadMtlFile
// PT:2614-2680, the OBJ index helpers PT:2529-2592) and the PPM reader for
// the images its materials use (loadPpmAsRgba8 PT:236-294; the textures are
// made by mc_image_texture_create). Host code: it produces the AoS triangles
// that scene ingestion (mc_scene_ingest_host) and the BVH build take next.
//
// Compiled with -ffp-contract=off: positions, normals and their transforms are
// computed with the reference's host operations in the reference's order, so
// the triangles are bit-identical. Lines are tokenised with the same stream
// extraction the reference uses, so malformed lines read the same way (a
// failed number extraction yields 0).
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#include "mc_abi.h"
#include "mc_host_scene.h"
#include "mc_internal.h"

using namespace mc_host;

namespace {

struct HV2 {
    float u = 0.f, v = 0.f;
};

struct Corner {
    int pos, uv, nrm;  // -1 = missing
};

struct Face {
    Corner c[3];
    int material = -1;  // -1 = the caller's fallback material
};

struct MaterialLibrary {
    std::vector<mc_material> materials;
    std::map<std::string, int> byName;
};

// OBJ indices start at 1; negative ones count back from the end of the list.
int resolve_index(int raw, int count) {
    if (raw > 0) return raw - 1;
    if (raw < 0) return count + raw;
    return -1;
}

// "7", "7/3", "7/3/5", "7//5"
Corner parse_corner(const std::string& tok, int np, int nt, int nn) {
    int raw[3] = {0, 0, 0};
    size_t start = 0;
    for (int part = 0; part < 3; part++) {
        const size_t slash = tok.find('/', start);
        const std::string piece = tok.substr(start, slash == std::string::npos ? std::string::npos : slash - start);
        if (!piece.empty()) raw[part] = std::atoi(piece.c_str());
        if (slash == std::string::npos) break;
        start = slash + 1;
    }
    return Corner{resolve_index(raw[0], np), resolve_index(raw[1], nt), resolve_index(raw[2], nn)};
}

std::string directory_of(const std::string& path) {
    const size_t s = path.find_last_of("/\\");
    return s == std::string::npos ? "." : path.substr(0, s);
}

// Texture paths use '/', and the image is read from a .ppm beside it
// ("textures\\wall.png" -> "textures/wall.ppm").
std::string ppm_path_of(std::string p) {
    for (char& ch : p)
        if (ch == '\\') ch = '/';
    const size_t dot = p.find_last_of('.'), slash = p.find_last_of('/');
    if (dot != std::string::npos && (slash == std::string::npos || dot > slash)) p = p.substr(0, dot);
    return p + ".ppm";
}

// PT:236-257: the next decimal integer of a PPM header, skipping whitespace
// and '#' comments; the character after the number is consumed.
bool ppm_int(FILE* f, int& value) {
    if (std::feof(f) || std::ferror(f)) return false;
    int ch = std::fgetc(f);
    while (ch != EOF) {
        if (ch == '#') {
            while (ch != '\n' && ch != EOF) ch = std::fgetc(f);
        } else if (std::isspace(ch)) {
            ch = std::fgetc(f);
        } else {
            break;
        }
    }
    if (ch == EOF || !std::isdigit(ch)) return false;
    value = 0;
    while (ch != EOF && std::isdigit(ch)) {
        value = value * 10 + (ch - '0');
        ch = std::fgetc(f);
    }
    return true;
}

struct Textures {
    bool enabled = false;
    std::map<std::string, uint64_t> cache;  // by .ppm path; 0 = could not be loaded
    std::vector<uint64_t> created;
};

uint64_t load_texture(Textures& tx, const std::string& ppmPath) {
    auto it = tx.cache.find(ppmPath);
    if (it != tx.cache.end()) return it->second;
    uint64_t handle = 0;
    int w = 0, h = 0;
    if (mc_ppm_read(ppmPath.c_str(), &w, &h, nullptr) == MC_OK && w > 0 && h > 0) {
        std::vector<uint8_t> rgba((size_t)w * h * 4);
        if (mc_ppm_read(ppmPath.c_str(), &w, &h, rgba.data()) == MC_OK &&
            mc_image_texture_create(rgba.data(), w, h, &handle) == MC_OK && handle)
            tx.created.push_back(handle);
        else
            handle = 0;
    }
    tx.cache[ppmPath] = handle;
    return handle;
}

// PT:2614-2680: newmtl / Kd / Ke / map_Kd. A material with a positive Ke
// component is emissive; otherwise lambertian, with the map_Kd image when it
// loads (the flat Kd colour and one missing texture counted when not).
bool load_mtl(const std::string& path, const std::string& dir, MaterialLibrary& lib, Textures& tx, int& missing) {
    std::ifstream file(path);
    if (!file.is_open()) return false;
    std::string name, texture;
    HV color(0.8f, 0.8f, 0.8f), emission(0.f, 0.f, 0.f);
    bool open = false;
    auto finish = [&]() {
        if (!open) return;
        mc_material m = make_lambertian(color);
        const bool emits = std::fmax(emission.x, std::fmax(emission.y, emission.z)) > 0.f;
        if (emits) {
            m = make_emissive(emission);
        } else if (!texture.empty()) {
            uint64_t handle = tx.enabled ? load_texture(tx, dir + "/" + ppm_path_of(texture)) : 0;
            if (handle) {
                m = base_material(MC_MAT_LAMBERTIAN);  // make_image_texture (PT:318-320)
                m.albedo.type = MC_TEX_IMAGE;
                m.albedo.color_a = mc_vec3{1, 1, 1};
                m.albedo.color_b = mc_vec3{0, 0, 0};
                m.albedo.scale = 1.f;
                m.albedo.image = handle;
            } else {
                missing++;
            }
        }
        lib.byName[name] = (int)lib.materials.size();
        lib.materials.push_back(m);
        open = false;
    };
    std::string line;
    while (std::getline(file, line)) {
        std::istringstream ls(line);
        std::string key;
        ls >> key;
        if (key == "newmtl") {
            finish();
            ls >> name;
            color = HV(0.8f, 0.8f, 0.8f);
            emission = HV(0.f, 0.f, 0.f);
            texture.clear();
            open = true;
        } else if (key == "Kd" && open) {
            float r, g, b;
            ls >> r >> g >> b;
            color = HV(r, g, b);
        } else if (key == "Ke" && open) {
            float r, g, b;
            ls >> r >> g >> b;
            emission = HV(r, g, b);
        } else if (key == "map_Kd" && open) {
            ls >> texture;
        }
    }
    finish();
    return true;
}

}  // namespace

extern "C" {

mc_status mc_ppm_read(const char* path, int32_t* width, int32_t* height, uint8_t* rgba) {
    if (!path || !width || !height) return mc::set_error(MC_ERR_INVALID, "mc_ppm_read: null argument");
    FILE* f = std::fopen(path, "rb");
    if (!f) return mc::set_error(MC_ERR_NOT_FOUND, "mc_ppm_read: cannot open '%s'", path);
    int w = 0, h = 0, maxv = 0;
    bool ok = std::fgetc(f) == 'P' && std::fgetc(f) == '6' && ppm_int(f, w) && ppm_int(f, h) && ppm_int(f, maxv) &&
              maxv == 255 && !std::feof(f) && !std::ferror(f) && w > 0 && h > 0;
    if (ok && rgba) {
        std::vector<uint8_t> rgb((size_t)w * h * 3);
        ok = std::fread(rgb.data(), 1, rgb.size(), f) == rgb.size();
        if (ok)
            for (size_t p = 0; p < (size_t)w * h; p++) {
                rgba[4 * p] = rgb[3 * p];
                rgba[4 * p + 1] = rgb[3 * p + 1];
                rgba[4 * p + 2] = rgb[3 * p + 2];
                rgba[4 * p + 3] = 255;
            }
    }
    std::fclose(f);
    if (!ok) return mc::set_error(MC_ERR_INVALID, "mc_ppm_read: '%s' is not a binary 8-bit PPM", path);
    *width = w;
    *height = h;
    return MC_OK;
}

mc_status mc_obj_load(const char* path, const mc_material* fallback, mc_vec3 translation, float scale, float rotation_y,
                      int32_t load_textures, mc_scene_host* scene, mc_obj_info* info) {
    if (!path || !fallback || !scene) return mc::set_error(MC_ERR_INVALID, "mc_obj_load: null argument");
    if (info) std::memset(info, 0, sizeof(*info));
    std::ifstream file(path);
    if (!file.is_open()) return mc::set_error(MC_ERR_NOT_FOUND, "mc_obj_load: cannot open '%s'", path);
    const std::string dir = directory_of(path);
    std::vector<HV> positions, normals;
    std::vector<HV2> uvs;
    std::vector<Face> faces;
    MaterialLibrary lib;
    Textures tx;
    tx.enabled = load_textures != 0;
    int missing = 0, current = -1;
    std::set<std::string> unknown;
    std::string line;
    while (std::getline(file, line)) {
        std::istringstream ls(line);
        std::string key;
        ls >> key;
        if (key == "v") {
            float x, y, z;
            ls >> x >> y >> z;
            positions.push_back(HV(x, y, z));
        } else if (key == "vt") {
            float u, v;
            ls >> u >> v;
            uvs.push_back(HV2{u, v});
        } else if (key == "vn") {
            float x, y, z;
            ls >> x >> y >> z;
            normals.push_back(HV(x, y, z));
        } else if (key == "mtllib") {
            std::string name;
            while (ls >> name) load_mtl(dir + '/' + name, dir, lib, tx, missing);
        } else if (key == "usemtl") {
            std::string name;
            ls >> name;
            auto it = lib.byName.find(name);
            if (it != lib.byName.end()) current = it->second;
            else current = lib.materials.size() == 1 ? 0 : -1;  // PT:2719-2727
            if (it == lib.byName.end()) unknown.insert(name);
        } else if (key == "f") {
            std::vector<Corner> corners;
            std::string tok;
            while (ls >> tok)
                corners.push_back(parse_corner(tok, (int)positions.size(), (int)uvs.size(), (int)normals.size()));
            for (size_t k = 1; k + 1 < corners.size(); k++) {  // fan (0, k, k + 1)
                Face f;
                f.c[0] = corners[0];
                f.c[1] = corners[k];
                f.c[2] = corners[k + 1];
                f.material = current;
                faces.push_back(f);
            }
        }
    }
    if (info) {
        info->materials = (int32_t)lib.materials.size();
        info->textures_missing = missing;
        info->unknown_materials = (int32_t)unknown.size();
    }
    auto keep_textures = [&]() {
        if (!info) {
            for (uint64_t t : tx.created) mc_image_texture_destroy(t);
            return;
        }
        info->textures_loaded = (int32_t)tx.created.size();
        info->textures = tx.created.empty() ? nullptr : (uint64_t*)std::malloc(tx.created.size() * sizeof(uint64_t));
        if (info->textures) std::memcpy(info->textures, tx.created.data(), tx.created.size() * sizeof(uint64_t));
    };
    if (positions.empty() || faces.empty()) {
        keep_textures();
        return mc::set_error(MC_ERR_INVALID, "mc_obj_load: '%s' has no vertices or no faces", path);
    }

    // PT:2758-2776: centre on x/z, lowest point at y = 0, largest side 1, then
    // scale, rotation about y and translation of the bottom centre
    HV lo = positions[0], hi = positions[0];
    for (size_t i = 1; i < positions.size(); i++) {
        lo = HV(std::fmin(lo.x, positions[i].x), std::fmin(lo.y, positions[i].y), std::fmin(lo.z, positions[i].z));
        hi = HV(std::fmax(hi.x, positions[i].x), std::fmax(hi.y, positions[i].y), std::fmax(hi.z, positions[i].z));
    }
    const HV size = hi - lo;
    const float largest = std::fmax(size.x, std::fmax(size.y, size.z));
    const HV bottom((lo.x + hi.x) * 0.5f, lo.y, (lo.z + hi.z) * 0.5f);
    const float c = cosf(rotation_y), s = sinf(rotation_y);
    const HV t(translation);
    std::vector<HV> xf(positions.size());
    for (size_t i = 0; i < positions.size(); i++) {
        const HV q = (positions[i] - bottom) * (scale / largest);
        xf[i] = HV(q.x * c + q.z * s, q.y, -q.x * s + q.z * c) + t;
    }
    // PT:2777-2790: without vn, area-weighted vertex normals
    std::vector<HV> avg;
    const int np = (int)positions.size();
    if (normals.empty()) {
        avg.assign(positions.size(), HV(0.f, 0.f, 0.f));
        for (const Face& f : faces) {
            const int i0 = f.c[0].pos, i1 = f.c[1].pos, i2 = f.c[2].pos;
            if (i0 < 0 || i1 < 0 || i2 < 0 || i0 >= np || i1 >= np || i2 >= np) continue;
            const HV w = (xf[i1] - xf[i0]).cross(xf[i2] - xf[i0]);
            avg[i0] = avg[i0] + w;
            avg[i1] = avg[i1] + w;
            avg[i2] = avg[i2] + w;
        }
    }
    std::vector<mc_triangle> out;
    out.reserve(faces.size());
    int skipped = 0;
    for (const Face& f : faces) {
        bool valid = true;
        for (int k = 0; k < 3; k++)
            if (f.c[k].pos < 0 || f.c[k].pos >= np) valid = false;
        if (!valid) {
            skipped++;
            continue;
        }
        const HV v0 = xf[f.c[0].pos], v1 = xf[f.c[1].pos], v2 = xf[f.c[2].pos];
        if ((v1 - v0).cross(v2 - v0).length() < 1e-9f) {  // zero area: the normal would be NaN
            skipped++;
            continue;
        }
        const mc_material m = f.material >= 0 && f.material < (int)lib.materials.size() ? lib.materials[f.material] : *fallback;
        mc_triangle tri = make_triangle(v0, v1, v2, m);
        mc_vec2* uvt[3] = {&tri.uv0, &tri.uv1, &tri.uv2};
        mc_vec3* nt[3] = {&tri.n0, &tri.n1, &tri.n2};
        for (int k = 0; k < 3; k++) {
            const int ui = f.c[k].uv;
            if (ui >= 0 && ui < (int)uvs.size()) *uvt[k] = mc_vec2{uvs[ui].u, uvs[ui].v};
        }
        for (int k = 0; k < 3; k++) {
            const int ni = f.c[k].nrm;
            if (ni >= 0 && ni < (int)normals.size() && normals[ni].length_squared() > 0.0f) {
                const HV n = normals[ni];
                *nt[k] = HV(n.x * c + n.z * s, n.y, -n.x * s + n.z * c).normalize();
            } else if (!avg.empty()) {
                const HV& a = avg[f.c[k].pos];
                if (a.length_squared() > 0.0f) *nt[k] = a.normalize();
            }
        }
        out.push_back(tri);
    }
    if (!out.empty()) {
        const size_t total = (size_t)scene->triangle_count + out.size();
        mc_triangle* grown = (mc_triangle*)std::realloc(scene->triangles, total * sizeof(mc_triangle));
        if (!grown) {
            keep_textures();
            return mc::set_error(MC_ERR_OOM, "mc_obj_load: host allocation failed");
        }
        std::memcpy(grown + scene->triangle_count, out.data(), out.size() * sizeof(mc_triangle));
        scene->triangles = grown;
        scene->triangle_count = (int32_t)total;
    }
    if (info) {
        info->triangles_added = (int32_t)out.size();
        info->faces_skipped = skipped;
    }
    keep_textures();
    if (out.empty()) return mc::set_error(MC_ERR_INVALID, "mc_obj_load: '%s' gave no triangles", path);
    return MC_OK;
}

mc_status mc_obj_info_free(mc_obj_info* info) {
    if (!info) return MC_OK;
    std::free(info->textures);
    info->textures = nullptr;
    return MC_OK;
}

}  // extern "C"
