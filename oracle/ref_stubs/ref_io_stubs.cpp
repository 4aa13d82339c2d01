// Compile-only stand-ins for the reference's stb/tinyexr/nanovdb I/O helpers
// (src/image_io.cpp, src/volume_io.cpp), whose third-party sources are absent
// here. Declarations come from the reference's own headers. Loading always
// fails; saving reports success without writing. The oracle harness never
// reads or writes image files: scenes and environment maps are passed in as
// arrays.
#include "image_io.h"
#include "volume_io.h"

bool loadImageRgba8(const char*, int& w, int& h, std::vector<unsigned char>& px) { w = h = 0; px.clear(); return false; }
bool loadImageRgbaFloat(const char*, int& w, int& h, std::vector<float>& px) { w = h = 0; px.clear(); return false; }
bool saveImageRgb8Png(const char*, int, int, const std::vector<unsigned char>&) { return true; }
bool loadNanoVdbGrid(const char*, VolumeGrid&) { return false; }
bool createFogSphereGrid(float, float, VolumeGrid&) { return false; }
