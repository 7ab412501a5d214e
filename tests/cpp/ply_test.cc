// The C++ ingest drop-in PlyHelper (include/phaser_gpu.hpp) on a generated
// Ouster-style PLY: values narrowed through double to float as the reference's
// tinyply + point cloud do.  Host only.  Built and run by tests/test_cpp_ply.py
// with the file path as argument.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <stdexcept>
#include <string>

#include "phaser_gpu.hpp"

namespace {
template <typename T>
void put_le(std::ofstream& f, T v) {
  unsigned char b[sizeof(T)];
  std::memcpy(b, &v, sizeof(T));
  const uint16_t one = 1;
  unsigned char lo;
  std::memcpy(&lo, &one, 1);
  if (lo != 1)  // big-endian host: write little-endian bytes
    for (size_t i = 0; i < sizeof(T) / 2; ++i) std::swap(b[i], b[sizeof(T) - 1 - i]);
  f.write(reinterpret_cast<const char*>(b), sizeof(T));
}

float x_of(int i) { return 0.5f * (float)i - 1.0f; }
float y_of(int i) { return 0.25f * (float)i; }
float z_of(int i) { return -0.125f * (float)i + 1e-3f; }
float in_of(int i) { return 100.0f + (float)i / 3.0f; }
uint16_t refl_of(int i) { return (uint16_t)(1000 + 37 * i); }
uint16_t noise_of(int i) { return (uint16_t)(7 * i); }
uint32_t range_of(int i) { return 4000000000u - 3u * (uint32_t)i; }  // above 2^24: rounds in float
}  // namespace

int main(int argc, char** argv) {
  using namespace phaser_gpu;
  if (argc < 2) return 9;
  const std::string path = argv[1];
  const int n = 6;
  {
    std::ofstream f(path, std::ios::binary);
    f << "ply\nformat binary_little_endian 1.0\ncomment ouster-like\nelement vertex " << n << "\n"
      << "property float x\nproperty float y\nproperty float z\nproperty float intensity\n"
      << "property uint t\nproperty ushort reflectivity\nproperty uchar ring\nproperty ushort noise\n"
      << "property uint range\nend_header\n";
    for (int i = 0; i < n; ++i) {
      put_le(f, x_of(i));
      put_le(f, y_of(i));
      put_le(f, z_of(i));
      put_le(f, in_of(i));
      put_le(f, (uint32_t)(10 * i));
      put_le(f, refl_of(i));
      put_le(f, (uint8_t)i);
      put_le(f, noise_of(i));
      put_le(f, range_of(i));
    }
  }
  const PlyPointCloud pc = PlyHelper().readPlyFromFile(path);
  if (pc.size() != (size_t)n || pc.reflectivity.size() != (size_t)n || pc.ambient.size() != (size_t)n ||
      pc.range.size() != (size_t)n)
    return 1;
  for (int i = 0; i < n; ++i) {
    const float* p = &pc.xyzi[4 * i];
    if (p[0] != x_of(i) || p[1] != y_of(i) || p[2] != z_of(i) || p[3] != in_of(i)) return 2;
    if (pc.reflectivity[i] != (float)(double)refl_of(i) || pc.ambient[i] != (float)(double)noise_of(i) ||
        pc.range[i] != (float)(double)range_of(i))
      return 3;
  }
  std::printf("ply_fields %zu\n", pc.size());
  // renamed fields (the --phaser_ply_*_str flags): an absent one stays empty
  const PlyPointCloud pc2 = PlyHelper("intensity", "no_such_field", "noise", "range").readPlyFromFile(path);
  if (!pc2.reflectivity.empty() || pc2.ambient.size() != (size_t)n) return 4;
  const CloudView v = pc2.view();
  if (v.n_points != (uint32_t)n || v.reflectivity != nullptr || v.ambient != pc2.ambient.data()) return 5;
  std::printf("ply_renamed ok\n");
  try {
    PlyHelper().readPlyFromFile(path + ".missing");
    return 6;
  } catch (const std::runtime_error&) {
    std::printf("ply_missing_rejected\n");
  }
  std::printf("ok\n");
  return 0;
}
