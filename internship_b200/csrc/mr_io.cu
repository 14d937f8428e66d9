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
#include <cmath>
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

// ---- Radiance RGBE (.hdr) images ----------------------------------------------------
// Header lines up to the resolution line "-Y <h> +X <w>" (the reference's
// loader, core/hdr_loader.h:43-104, reads the same two numbers and ignores
// flips); then h scanlines of w pixels, each either flat (4 bytes per pixel)
// or, for 8 <= w <= 32767, in the new run-length form: the bytes 2, 2,
// w >> 8, w & 255, then each of the four components of the scanline as runs
// (count > 128: repeat the next byte count - 128 times) and literal spans
// (count <= 128: that many bytes). A pixel (r, g, b, e) is the colour
// (c + 0.5) * 2^(e - 136) per channel, 0 when e = 0 (the Radiance format).
static int parse_hdr(const std::string& path, int* w_out, int* h_out, std::vector<float>* rgba) {
  std::vector<char> buf;
  if (!read_file(path, &buf)) return set_error(MR_ERR_ARG, "%s: cannot read", path.c_str());
  const size_t size = buf.size() - 1;
  const unsigned char* b = (const unsigned char*)buf.data();
  if (size < 2 || b[0] != '#' || b[1] != '?') return set_error(MR_ERR_ARG, "%s: not a Radiance file", path.c_str());
  size_t pos = 0;
  int w = 0, h = 0;
  bool have_res = false;
  while (pos < size && !have_res) {
    size_t e = pos;
    while (e < size && b[e] != '\n') ++e;
    std::string line((const char*)b + pos, e - pos);
    pos = e + 1;
    if (line.compare(0, 7, "FORMAT=") == 0 && line.find("32-bit_rle_rgbe") == std::string::npos &&
        line.find("32-bit_rle_xyze") == std::string::npos)
      return set_error(MR_ERR_ARG, "%s: unsupported %s", path.c_str(), line.c_str());
    if (!line.empty() && (line[0] == '-' || line[0] == '+')) {
      size_t x = line.find('X'), y = line.find('Y');
      if (x == std::string::npos || y == std::string::npos)
        return set_error(MR_ERR_ARG, "%s: bad resolution line", path.c_str());
      w = std::atoi(line.c_str() + x + 1);
      h = std::atoi(line.c_str() + y + 1);
      have_res = true;
    }
  }
  if (!have_res || w <= 0 || h <= 0 || (long long)w * h > (1ll << 28))
    return set_error(MR_ERR_ARG, "%s: bad or missing resolution", path.c_str());
  rgba->assign((size_t)w * h * 4, 0.0f);
  std::vector<unsigned char> line((size_t)w * 4);
  auto take = [&](size_t n) -> const unsigned char* {
    if (pos + n > size) return nullptr;
    const unsigned char* p = b + pos;
    pos += n;
    return p;
  };
  const bool can_rle = w >= 8 && w <= 0x7fff;
  for (int j = 0; j < h; ++j) {
    const unsigned char* hd = (pos + 4 <= size) ? b + pos : nullptr;
    if (can_rle && hd && hd[0] == 2 && hd[1] == 2 && !(hd[2] & 128)) {
      pos += 4;
      if (((hd[2] << 8) | hd[3]) != w) return set_error(MR_ERR_ARG, "%s: scanline %d length mismatch", path.c_str(), j);
      for (int c = 0; c < 4; ++c) {
        for (int x = 0; x < w;) {
          const unsigned char* n = take(1);
          if (!n) return set_error(MR_ERR_ARG, "%s: truncated scanline %d", path.c_str(), j);
          int cnt = *n;
          if (cnt > 128) {
            cnt &= 127;
            const unsigned char* v = take(1);
            if (!v || cnt == 0 || x + cnt > w) return set_error(MR_ERR_ARG, "%s: bad run in scanline %d", path.c_str(), j);
            for (int k = 0; k < cnt; ++k) line[(size_t)(x++) * 4 + c] = *v;
          } else {
            const unsigned char* v = take((size_t)cnt);
            if (!v || cnt == 0 || x + cnt > w) return set_error(MR_ERR_ARG, "%s: bad span in scanline %d", path.c_str(), j);
            for (int k = 0; k < cnt; ++k) line[(size_t)(x++) * 4 + c] = v[k];
          }
        }
      }
    } else {
      const unsigned char* v = take((size_t)w * 4);
      if (!v) return set_error(MR_ERR_ARG, "%s: truncated scanline %d", path.c_str(), j);
      std::memcpy(line.data(), v, (size_t)w * 4);
    }
    for (int x = 0; x < w; ++x) {
      const unsigned char* q = &line[(size_t)x * 4];
      float* o = &(*rgba)[((size_t)j * w + x) * 4];
      if (q[3]) {
        const float sc = std::ldexp(1.0f, (int)q[3] - 136);
        o[0] = ((float)q[0] + 0.5f) * sc;
        o[1] = ((float)q[1] + 0.5f) * sc;
        o[2] = ((float)q[2] + 0.5f) * sc;
      }
    }
  }
  *w_out = w;
  *h_out = h;
  return MR_OK;
}

}  // namespace mr

using namespace mr;

extern "C" int mr_hdr_read(const char* path, float* host_rgba, size_t capacity, int32_t* width, int32_t* height) {
  clear_error();
  if (!path || !width || !height) return set_error(MR_ERR_ARG, "mr_hdr_read: NULL argument");
  int w = 0, h = 0;
  std::vector<float> px;
  int rc = parse_hdr(path, &w, &h, &px);
  if (rc) return rc;
  *width = w;
  *height = h;
  if (host_rgba) {
    if (capacity < px.size()) return set_error(MR_ERR_ARG, "mr_hdr_read: %zu floats needed", px.size());
    std::memcpy(host_rgba, px.data(), px.size() * sizeof(float));
  }
  return MR_OK;
}

extern "C" int mr_volume_load_hdri(mr_volume* v, const char* path) {
  clear_error();
  if (!v || !path) return set_error(MR_ERR_ARG, "mr_volume_load_hdri: NULL argument");
  int w = 0, h = 0;
  std::vector<float> px;
  int rc = parse_hdr(path, &w, &h, &px);
  if (rc) return rc;
  return mr_volume_set_hdri(v, px.data(), w, h);
}

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
