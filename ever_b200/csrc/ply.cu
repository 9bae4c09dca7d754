// Scene loader for trained ellipsoid scenes stored as binary PLY (host code).
//
// Reference: splinetracers/fast_ellipsoid_splinetracer/ply_file_loader.cc:196-293
// (ReadSceneFromFile) and :166-193 (NormalizeSceneData). The file holds, per vertex, 62
// little-endian floats: mean (3), normal (3, skipped), 48 spherical-harmonic values in
// file order (read as 16 coefficients x 3 channels, as the reference reads them), opacity
// (1), scale (3) and rotation (4). Values are converted as the reference converts them:
//   quaternion  q / (q . q)                 (the reference divides by the squared length)
//   scale       min(softplus(s) + 3e-4, 25), softplus(x) = x for x > 5
//   density     max(0, -log(max(1 - 0.99 sigmoid(o), 1e-10))) / (2 min(scale))
// The reference's optional Morton pre-sort is not applied (it is unused there, and
// ever_scene_build sorts the ellipsoids on the device).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "internal.cuh"

namespace {

constexpr int kPlyFloats = 62;

struct PlyHeader {
  int64_t count = 0;
  size_t data_offset = 0;
};

bool next_line(const std::string& s, size_t& pos, std::string& line) {
  if (pos >= s.size()) return false;
  size_t e = s.find('\n', pos);
  if (e == std::string::npos) e = s.size();
  line = s.substr(pos, e - pos);
  if (!line.empty() && line.back() == '\r') line.pop_back();
  pos = e + 1;
  return true;
}

std::vector<std::string> split(const std::string& line) {
  std::vector<std::string> parts;
  std::istringstream in(line);
  std::string w;
  while (in >> w) parts.push_back(w);
  return parts;
}

// Parses the header; returns an error message or "" on success.
std::string parse_header(const std::string& s, PlyHeader& h) {
  size_t pos = 0;
  std::string line;
  if (!next_line(s, pos, line) || line != "ply") return "expected the file to start with a \"ply\" line";
  if (!next_line(s, pos, line) || line != "format binary_little_endian 1.0")
    return "expected \"format binary_little_endian 1.0\"";
  if (!next_line(s, pos, line)) return "truncated header";
  auto p = split(line);
  if (p.size() != 3 || p[0] != "element" || p[1] != "vertex") return "expected \"element vertex <count>\"";
  char* end = nullptr;
  const long long n = std::strtoll(p[2].c_str(), &end, 10);
  if (*end != '\0' || n < 0 || n >= (1ll << 30)) return "bad vertex count";
  int props = 0;
  for (;;) {
    if (!next_line(s, pos, line)) return "header has no end_header line";
    if (line == "end_header") break;
    p = split(line);
    if (p.size() != 3 || p[0] != "property") return "expected \"property <type> <name>\" lines";
    if (p[1] != "float" && p[1] != "float32") return "every property must be a float";
    ++props;
  }
  if (props != kPlyFloats) return "expected 62 float properties per vertex (mean, normal, 48 SH, opacity, scale, rotation)";
  h.count = n;
  h.data_offset = pos;
  if (s.size() - pos < size_t(n) * kPlyFloats * sizeof(float)) return "vertex data is truncated";
  return "";
}

bool read_file(const char* path, std::string& out) {
  std::ifstream f(path, std::ios::binary);
  if (!f) return false;
  std::ostringstream b;
  b << f.rdbuf();
  out = b.str();
  return true;
}

float softplus_ref(float x) { return x > 5 ? x : std::log(1 + std::exp(x)); }
float sigmoid_ref(float x) { return 1.0f / (1 + std::exp(-x)); }

}  // namespace

extern "C" {

int64_t ever_ply_count(const char* path) {
  if (!path) {
    ever::set_last_error(EVER_ERR_INVALID, "ever_ply_count: null path");
    return -1;
  }
  std::string s;
  if (!read_file(path, s)) {
    ever::set_last_error(EVER_ERR_INVALID, "ever_ply_count: cannot open the file");
    return -1;
  }
  PlyHeader h;
  const std::string err = parse_header(s, h);
  if (!err.empty()) {
    ever::set_last_error(EVER_ERR_INVALID, ("ever_ply_count: " + err).c_str());
    return -1;
  }
  return h.count;
}

int ever_ply_read(const char* path, int64_t capacity, float* mean, float* scale, float* quat, float* density,
                  float* features) {
  if (!path || !mean || !scale || !quat || !density || !features)
    return ever::set_last_error(EVER_ERR_INVALID, "ever_ply_read: null pointer");
  std::string s;
  if (!read_file(path, s)) return ever::set_last_error(EVER_ERR_INVALID, "ever_ply_read: cannot open the file");
  PlyHeader h;
  const std::string err = parse_header(s, h);
  if (!err.empty()) return ever::set_last_error(EVER_ERR_INVALID, ("ever_ply_read: " + err).c_str());
  if (h.count > capacity) return ever::set_last_error(EVER_ERR_INVALID, "ever_ply_read: buffers hold fewer vertices");
  const char* data = s.data() + h.data_offset;
  for (int64_t i = 0; i < h.count; ++i) {
    float v[kPlyFloats];
    std::memcpy(v, data + size_t(i) * kPlyFloats * sizeof(float), sizeof(v));
    for (int a = 0; a < 3; ++a) mean[3 * i + a] = v[a];
    for (int k = 0; k < 48; ++k) features[48 * i + k] = v[6 + k];
    const float opacity = v[54];
    float len = 0;
    for (int q = 0; q < 4; ++q) len += v[58 + q] * v[58 + q];
    for (int q = 0; q < 4; ++q) quat[4 * i + q] = v[58 + q] / len;
    float norm = 9999;
    for (int a = 0; a < 3; ++a) {
      const float sc = float(std::min(softplus_ref(v[55 + a]) + 3 * 1e-4, 25.0));
      scale[3 * i + a] = sc;
      norm = std::min(2 * sc, norm);
    }
    const float alpha = float(0.99 * sigmoid_ref(opacity));
    const float inv_op = float(std::fmax(0, -std::log(std::fmax(1 - alpha, 1e-10))));
    density[i] = inv_op / norm;
  }
  return EVER_OK;
}

}  // extern "C"
