// Compile-only stand-in for minipbrt (vilya/minipbrt @a6f9dad), which the
// reference fetches at configure time and which is absent here. It declares
// only the names src/path_tracer.cu touches in its pbrt importer
// (path_tracer.cu:1989-2483). Loader::load always fails, so the importer is
// never reached; none of the synthetic scenes use pbrt input.
#pragma once
#include <cstdint>
#include <cstddef>
#include <vector>

namespace minipbrt {

static constexpr uint32_t kInvalidIndex = 0xFFFFFFFFu;

struct Transform { float start[4][4]; float end[4][4]; };

enum class ShapeType { TriangleMesh, Sphere, Other };
struct Shape {
    virtual ~Shape() {}
    virtual ShapeType type() const { return ShapeType::Other; }
    Transform shapeToWorld;
    uint32_t areaLight = kInvalidIndex, insideMedium = kInvalidIndex, material = kInvalidIndex, object = kInvalidIndex;
};
struct TriangleMesh : Shape {
    ShapeType type() const override { return ShapeType::TriangleMesh; }
    int* indices = nullptr; uint32_t num_indices = 0, num_vertices = 0;
    float* P = nullptr; float* N = nullptr; float* uv = nullptr;
};
struct Sphere : Shape { ShapeType type() const override { return ShapeType::Sphere; } float radius = 1.f; };

struct Instance { Transform instanceToWorld; uint32_t object = kInvalidIndex, areaLight = kInvalidIndex; };
struct Object { Transform objectToInstance; uint32_t firstShape = 0, numShapes = 0; };

struct ColorTex { float value[3] = {0, 0, 0}; uint32_t texture = kInvalidIndex; };
struct FloatTex { float value = 0.f; uint32_t texture = kInvalidIndex; };

enum class TextureType { ImageMap, Constant, Scale, Other };
struct Texture { virtual ~Texture() {} virtual TextureType type() const { return TextureType::Other; } };
struct ImageMapTexture : Texture { TextureType type() const override { return TextureType::ImageMap; } char* filename = nullptr; };
struct ConstantTexture : Texture { TextureType type() const override { return TextureType::Constant; } float value[3] = {0, 0, 0}; };
struct ScaleTexture : Texture { TextureType type() const override { return TextureType::Scale; } ColorTex tex1, tex2; };

enum class MaterialType { Matte, Plastic, Substrate, Uber, Disney, Glass, Mirror, Metal, Mix, None, Other };
struct Material { virtual ~Material() {} virtual MaterialType type() const { return MaterialType::Other; } char* name = nullptr; };
struct MatteMaterial : Material { ColorTex Kd; };
struct PlasticMaterial : Material { ColorTex Kd; };
struct SubstrateMaterial : Material { ColorTex Kd; };
struct UberMaterial : Material { ColorTex Kd; };
struct DisneyMaterial : Material { ColorTex color; };
struct GlassMaterial : Material { FloatTex eta; };
struct MirrorMaterial : Material { ColorTex Kr; };
struct MetalMaterial : Material { ColorTex eta, k; FloatTex uroughness; };
struct MixMaterial : Material { uint32_t namedmaterial1 = kInvalidIndex; };

struct Medium { float sigma_a[3] = {0, 0, 0}, sigma_s[3] = {0, 0, 0}; float scale = 1.f, g = 0.f; };

struct AreaLight { virtual ~AreaLight() {} };
struct DiffuseAreaLight : AreaLight { float L[3] = {0, 0, 0}; float scale[3] = {1, 1, 1}; };

enum class LightType { Infinite, Distant, Point, Spot, Other };
struct Light {
    virtual ~Light() {}
    virtual LightType type() const { return LightType::Other; }
    Transform lightToWorld; float scale[3] = {1, 1, 1};
};
struct InfiniteLight : Light { float L[3] = {0, 0, 0}; char* mapname = nullptr; };
struct DistantLight : Light { float from[3] = {0, 0, 0}, to[3] = {0, 0, 1}, L[3] = {0, 0, 0}; };
struct PointLight : Light { float from[3] = {0, 0, 0}, I[3] = {0, 0, 0}; };
struct SpotLight : Light { float from[3] = {0, 0, 0}, I[3] = {0, 0, 0}; };

enum class FilmType { Image, Other };
struct Film { virtual ~Film() {} virtual FilmType type() const { return FilmType::Other; } void get_resolution(int& w, int& h) const { w = 0; h = 0; } };

enum class CameraType { Perspective, Other };
struct Camera { virtual ~Camera() {} virtual CameraType type() const { return CameraType::Other; } Transform cameraToWorld; };
struct PerspectiveCamera : Camera { float fov = 90.f; };

struct Scene {
    std::vector<Shape*> shapes;
    std::vector<Instance*> instances;
    std::vector<Object*> objects;
    std::vector<Texture*> textures;
    std::vector<Material*> materials;
    std::vector<AreaLight*> areaLights;
    std::vector<Medium*> mediums;
    std::vector<Light*> lights;
    Film* film = nullptr;
    Camera* camera = nullptr;
    bool load_all_ply_meshes(bool) { return false; }
    bool all_to_triangle_mesh(bool) { return false; }
};

struct Error {
    const char* message() const { return "pbrt input is not available in this build"; }
    bool has_line_and_column() const { return false; }
    int64_t line() const { return 0; }
    int64_t column() const { return 0; }
};

struct Loader {
    bool load(const char*) { return false; }
    const Error* error() const { static Error e; return &e; }
    Scene* borrow_scene() { return nullptr; }
};

}  // namespace minipbrt
