// sc_ply.cpp — Inria 3DGS PLY in/out (crates/nano-splat/src/ply.rs:17-256)
// together with SplatBuffer::{from,to}_gaussians (splat_store.rs:60-94).
//
// Writer: binary_little_endian 1.0, the fixed field order x y z nx ny nz
// f_dc_0..2 f_rest_0..44 opacity scale_0..2 rot_0..3 (62 floats per vertex);
// normals are written as +Y like to_gaussians does.
// Reader: properties are matched by name; only `property float` and
// binary_little_endian are accepted; missing normals and missing f_rest_k
// read as absent / 0; any other missing field is an error.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/splat_cuda.h"

namespace {

struct FileCloser {
  FILE* f;
  ~FileCloser() { if (f) std::fclose(f); }
};

std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && (s[a] == ' ' || s[a] == '\t' || s[a] == '\r' || s[a] == '\n')) ++a;
  while (b > a && (s[b - 1] == ' ' || s[b - 1] == '\t' || s[b - 1] == '\r' || s[b - 1] == '\n')) --b;
  return s.substr(a, b - a);
}

bool starts_with(const std::string& s, const char* p) { return s.rfind(p, 0) == 0; }

}  // namespace

extern "C" sc_status sc_write_ply(const char* path, const sc_host_splats* s) {
  if (!path || !s) return SC_ERR_INVALID_ARG;
  if (s->n && (!s->positions || !s->rotations || !s->scales || !s->opacities || !s->sh_dc || !s->sh_rest))
    return SC_ERR_INVALID_ARG;
  FileCloser fc{std::fopen(path, "wb")};
  if (!fc.f) return SC_ERR_IO;
  std::string h = "ply\nformat binary_little_endian 1.0\nelement vertex " + std::to_string(s->n) + "\n";
  for (const char* p : {"x", "y", "z", "nx", "ny", "nz", "f_dc_0", "f_dc_1", "f_dc_2"})
    h += std::string("property float ") + p + "\n";
  for (int i = 0; i < 45; ++i) h += "property float f_rest_" + std::to_string(i) + "\n";
  h += "property float opacity\n";
  for (int i = 0; i < 3; ++i) h += "property float scale_" + std::to_string(i) + "\n";
  for (int i = 0; i < 4; ++i) h += "property float rot_" + std::to_string(i) + "\n";
  h += "end_header\n";
  if (std::fwrite(h.data(), 1, h.size(), fc.f) != h.size()) return SC_ERR_IO;
  std::vector<float> buf;
  const uint32_t chunk = 4096;
  buf.resize((size_t)chunk * 62);
  for (uint32_t i0 = 0; i0 < s->n; i0 += chunk) {
    const uint32_t cnt = std::min<uint32_t>(chunk, s->n - i0);
    for (uint32_t q = 0; q < cnt; ++q) {
      const size_t i = (size_t)i0 + q;
      float* r = buf.data() + (size_t)q * 62;
      r[0] = s->positions[3 * i]; r[1] = s->positions[3 * i + 1]; r[2] = s->positions[3 * i + 2];
      r[3] = 0.0f; r[4] = 1.0f; r[5] = 0.0f;
      r[6] = s->sh_dc[3 * i]; r[7] = s->sh_dc[3 * i + 1]; r[8] = s->sh_dc[3 * i + 2];
      std::memcpy(r + 9, s->sh_rest + 45 * i, 45 * 4);
      r[54] = s->opacities[i];
      r[55] = s->scales[3 * i]; r[56] = s->scales[3 * i + 1]; r[57] = s->scales[3 * i + 2];
      std::memcpy(r + 58, s->rotations + 4 * i, 16);
    }
    if (std::fwrite(buf.data(), 4, (size_t)cnt * 62, fc.f) != (size_t)cnt * 62) return SC_ERR_IO;
  }
  return SC_OK;
}

extern "C" sc_status sc_read_ply(const char* path, sc_host_splats* dst, uint32_t* n_out) {
  if (!path) return SC_ERR_INVALID_ARG;
  FileCloser fc{std::fopen(path, "rb")};
  if (!fc.f) return SC_ERR_IO;
  char line[1024];
  if (!std::fgets(line, sizeof line, fc.f) || trim(line) != "ply") return SC_ERR_FORMAT;
  bool ble = false;
  unsigned long long count = 0;
  std::vector<std::string> props;
  for (;;) {
    if (!std::fgets(line, sizeof line, fc.f)) return SC_ERR_FORMAT;  // unterminated header
    const std::string t = trim(line);
    if (t.empty() || starts_with(t, "comment ")) continue;
    if (t == "end_header") break;
    if (starts_with(t, "format ")) { ble = starts_with(t.substr(7), "binary_little_endian"); continue; }
    if (starts_with(t, "element vertex ")) {
      char* end = nullptr;
      const std::string num = trim(t.substr(15));
      count = std::strtoull(num.c_str(), &end, 10);
      if (num.empty() || (end && *end)) return SC_ERR_FORMAT;
      continue;
    }
    if (starts_with(t, "property float ")) { props.push_back(trim(t.substr(15))); continue; }
    if (starts_with(t, "element ")) continue;
    if (starts_with(t, "property ")) return SC_ERR_FORMAT;  // only `property float` is supported
  }
  if (!ble) return SC_ERR_FORMAT;
  if (count > 0xFFFFFFFFull) return SC_ERR_FORMAT;
  auto idx = [&](const std::string& nm) -> int {
    for (size_t i = 0; i < props.size(); ++i)
      if (props[i] == nm) return (int)i;
    return -1;
  };
  static const char* req[] = {"x", "y", "z", "f_dc_0", "f_dc_1", "f_dc_2", "opacity", "scale_0", "scale_1",
                              "scale_2", "rot_0", "rot_1", "rot_2", "rot_3"};
  int ri[14];
  for (int k = 0; k < 14; ++k) {
    ri[k] = idx(req[k]);
    if (ri[k] < 0) return SC_ERR_FORMAT;  // missing required property
  }
  int rest[45];
  for (int k = 0; k < 45; ++k) rest[k] = idx("f_rest_" + std::to_string(k));
  if (n_out) *n_out = (uint32_t)count;
  if (!dst) return SC_OK;
  if (dst->n < count) return SC_ERR_CAPACITY;
  if (count && (!dst->positions || !dst->rotations || !dst->scales || !dst->opacities || !dst->sh_dc || !dst->sh_rest))
    return SC_ERR_INVALID_ARG;
  const size_t nprop = props.size();
  std::vector<float> rec(nprop);
  for (unsigned long long i = 0; i < count; ++i) {
    if (std::fread(rec.data(), 4, nprop, fc.f) != nprop) return SC_ERR_IO;
    for (int c = 0; c < 3; ++c) dst->positions[3 * i + c] = rec[ri[c]];
    for (int c = 0; c < 3; ++c) dst->sh_dc[3 * i + c] = rec[ri[3 + c]];
    dst->opacities[i] = rec[ri[6]];
    for (int c = 0; c < 3; ++c) dst->scales[3 * i + c] = rec[ri[7 + c]];
    for (int c = 0; c < 4; ++c) dst->rotations[4 * i + c] = rec[ri[10 + c]];
    for (int c = 0; c < 45; ++c) dst->sh_rest[45 * i + c] = rest[c] >= 0 ? rec[rest[c]] : 0.0f;
  }
  dst->n = (uint32_t)count;
  return SC_OK;
}
