// Volume files: VolumeRender(string path) (core/volume.cu:835-911).
//
// Formats, as the reference reads them:
//  * <path>.bin (checked first): int32 resolution r, then r^3 fp32 densities,
//    index (x*r + y)*r + z. Written by the reference (and here) as a cache
//    after a text or .vox file is read; convert.py writes the same layout.
//  * *.txt: the resolution r, then r^3 densities as whitespace-separated
//    decimal numbers, same index order.
//  * *.vox: a 256^3 grid; lines starting with 'w', 'h' or 'd' are header
//    lines, every other line holds 64 integers 0..255 that become densities
//    value * 64 / 255, consecutive in index order.
// Parsing is host code over the whole file in memory (no iostreams).
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "mr_internal.h"

namespace mr {

static bool read_file(const std::string& path, std::vector<char>* out) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) return false;
  fseek(f, 0, SEEK_END);
  long n = ftell(f);
  fseek(f, 0, SEEK_SET);
  if (n < 0) {
    fclose(f);
    return false;
  }
  out->resize((size_t)n + 1);
  size_t got = n ? fread(out->data(), 1, (size_t)n, f) : 0;
  fclose(f);
  (*out)[got] = 0;
  out->resize(got + 1);
  return got == (size_t)n;
}

static bool ends_with(const std::string& s, const char* suf) {
  size_t n = std::strlen(suf);
  return s.size() >= n && s.compare(s.size() - n, n, suf) == 0;
}

constexpr int kMaxFileRes = 1024;

// Parses `path` (resolved as the reference resolves it) into `data`.
static int parse_volume(const std::string& path, int* res, std::vector<float>* data, bool* from_bin) {
  std::vector<char> buf;
  *from_bin = false;
  if (read_file(path + ".bin", &buf)) {
    const size_t bytes = buf.size() - 1;
    if (bytes < 4) return set_error(MR_ERR_ARG, "%s.bin: truncated header", path.c_str());
    int32_t r;
    std::memcpy(&r, buf.data(), 4);
    if (r <= 0 || r > kMaxFileRes) return set_error(MR_ERR_ARG, "%s.bin: resolution %d out of range", path.c_str(), r);
    const size_t n = (size_t)r * r * r;
    if (bytes < 4 + n * 4)
      return set_error(MR_ERR_ARG, "%s.bin: %zu data bytes for resolution %d (need %zu)", path.c_str(), bytes - 4, r,
                       n * 4);
    data->resize(n);
    std::memcpy(data->data(), buf.data() + 4, n * 4);
    *res = r;
    *from_bin = true;
    return MR_OK;
  }
  if (ends_with(path, "txt")) {
    if (!read_file(path, &buf)) return set_error(MR_ERR_ARG, "%s: cannot read", path.c_str());
    char* p = buf.data();
    char* end = nullptr;
    errno = 0;
    long r = std::strtol(p, &end, 10);
    if (end == p || r <= 0 || r > kMaxFileRes) return set_error(MR_ERR_ARG, "%s: bad resolution", path.c_str());
    p = end;
    const size_t n = (size_t)r * r * r;
    data->assign(n, 0.0f);
    for (size_t i = 0; i < n; ++i) {
      float v = std::strtof(p, &end);
      if (end == p) return set_error(MR_ERR_ARG, "%s: %zu of %zu values", path.c_str(), i, n);
      (*data)[i] = v;
      p = end;
    }
    *res = (int)r;
    return MR_OK;
  }
  if (ends_with(path, "vox")) {
    if (!read_file(path, &buf)) return set_error(MR_ERR_ARG, "%s: cannot read", path.c_str());
    const int r = 256;
    const size_t n = (size_t)r * r * r;
    data->assign(n, 0.0f);
    const float inv = 64.0f / 255.0f;
    size_t i = 0;
    char* p = buf.data();
    while (*p && i < n) {
      char* eol = std::strchr(p, '\n');
      char* next = eol ? eol + 1 : p + std::strlen(p);
      if (eol) *eol = 0;
      if (*p != 'w' && *p != 'h' && *p != 'd') {
        // a data line: 64 integers (the reference reads 64 per line)
        char* q = p;
        int vals[64];
        int k = 0;
        for (; k < 64; ++k) {
          char* e = nullptr;
          long v = std::strtol(q, &e, 10);
          if (e == q) break;
          vals[k] = (int)v;
          q = e;
        }
        if (k == 64) {
          for (int j = 0; j < 64 && i + j < n; ++j) (*data)[i + j] = (float)vals[j] * inv;
          i += 64;
        } else if (k > 0) {
          return set_error(MR_ERR_ARG, "%s: a data line holds %d values, expected 64", path.c_str(), k);
        }
      }
      p = next;
    }
    *res = r;
    return MR_OK;
  }
  return set_error(MR_ERR_ARG, "%s: no %s.bin and not a .txt or .vox file", path.c_str(), path.c_str());
}

}  // namespace mr

using namespace mr;

extern "C" int mr_volume_file_read(const char* path, float* host_out, size_t capacity, int32_t* resolution) {
  clear_error();
  if (!path || !resolution) return set_error(MR_ERR_ARG, "mr_volume_file_read: NULL argument");
  int r = 0;
  bool from_bin = false;
  std::vector<float> data;
  int rc = parse_volume(path, &r, &data, &from_bin);
  if (rc) return rc;
  *resolution = r;
  if (host_out) {
    if (capacity < data.size())
      return set_error(MR_ERR_ARG, "mr_volume_file_read: %zu floats needed, capacity %zu", data.size(), capacity);
    std::memcpy(host_out, data.data(), data.size() * sizeof(float));
  }
  return MR_OK;
}

extern "C" int mr_volume_load(const char* path, int32_t write_cache, mr_volume** out, void* stream) {
  clear_error();
  if (!path || !out) return set_error(MR_ERR_ARG, "mr_volume_load: NULL argument");
  *out = nullptr;
  int r = 0;
  bool from_bin = false;
  std::vector<float> data;
  int rc = parse_volume(path, &r, &data, &from_bin);
  if (rc) return rc;
  mr_volume* v = nullptr;
  rc = mr_volume_create(r, &v);
  if (rc) return rc;
  rc = mr_volume_set_data(v, data.data(), data.size());
  if (!rc) rc = mr_volume_update(v, stream);
  if (rc) {
    mr_volume_destroy(v);
    return rc;
  }
  if (!from_bin && write_cache) {
    // the reference writes <path>.bin after reading a text or .vox file
    std::string bin = std::string(path) + ".bin";
    FILE* f = fopen(bin.c_str(), "wb");
    if (f) {
      int32_t rr = r;
      bool ok = fwrite(&rr, 4, 1, f) == 1 && fwrite(data.data(), 4, data.size(), f) == data.size();
      fclose(f);
      if (!ok) std::remove(bin.c_str());
    }
  }
  *out = v;
  return MR_OK;
}
