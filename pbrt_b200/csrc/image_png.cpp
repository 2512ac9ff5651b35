// image_png.cpp — pbrt_write_png: the 8-bit RGBA PNG the reference's renderer writes
// (image_write, src/renderers/mt.rs:152-167, through the `png` crate). The image data is a
// zlib stream of stored (uncompressed) deflate blocks, so any PNG decoder yields exactly the
// given pixels. Host only.
#include <cstdint>
#include <cstdio>
#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/pbrt_b200.h"

namespace {

struct CrcTable {
  uint32_t v[256];
  CrcTable() {
    for (uint32_t n = 0; n < 256; ++n) {  // CRC-32, polynomial 0xEDB88320 (PNG spec, ISO 3309)
      uint32_t c = n;
      for (int k = 0; k < 8; ++k) c = (c & 1u) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
      v[n] = c;
    }
  }
};
const CrcTable crc_table;  // built at load time, read-only afterwards

uint32_t crc(const uint8_t* p, size_t n, uint32_t c = 0xFFFFFFFFu) {
  for (size_t i = 0; i < n; ++i) c = crc_table.v[(c ^ p[i]) & 0xFFu] ^ (c >> 8);
  return c;
}

void put32(std::vector<uint8_t>& v, uint32_t x) {
  v.push_back(uint8_t(x >> 24));
  v.push_back(uint8_t(x >> 16));
  v.push_back(uint8_t(x >> 8));
  v.push_back(uint8_t(x));
}

void chunk(std::vector<uint8_t>& out, const char* type, const std::vector<uint8_t>& data) {
  put32(out, uint32_t(data.size()));
  const size_t start = out.size();
  out.insert(out.end(), type, type + 4);
  out.insert(out.end(), data.begin(), data.end());
  put32(out, crc(out.data() + start, out.size() - start) ^ 0xFFFFFFFFu);
}

}  // namespace

extern "C" int pbrt_write_png(const char* path, const uint8_t* rgba, uint32_t width, uint32_t height) {
  if (!path || !rgba || width == 0 || height == 0) return PBRT_ERR_INVALID_ARGUMENT;
  if (uint64_t(width) * 4 + 1 > 0x7FFFFFFFull || uint64_t(height) > 0x7FFFFFFFull) return PBRT_ERR_INVALID_ARGUMENT;
  // scanlines: filter type 0, then the row's RGBA bytes
  const size_t row = size_t(width) * 4;
  std::vector<uint8_t> raw;
  raw.reserve((row + 1) * height);
  for (uint32_t y = 0; y < height; ++y) {
    raw.push_back(0);
    raw.insert(raw.end(), rgba + y * row, rgba + (y + 1) * row);
  }
  // zlib: header, stored deflate blocks of at most 65535 bytes, Adler-32
  std::vector<uint8_t> z;
  z.reserve(raw.size() + raw.size() / 65535 * 5 + 16);
  z.push_back(0x78);
  z.push_back(0x01);
  size_t pos = 0;
  do {
    const size_t n = std::min<size_t>(65535, raw.size() - pos);
    const bool last = pos + n == raw.size();
    z.push_back(last ? 1 : 0);
    z.push_back(uint8_t(n));
    z.push_back(uint8_t(n >> 8));
    z.push_back(uint8_t(~n));
    z.push_back(uint8_t(~n >> 8));
    z.insert(z.end(), raw.begin() + pos, raw.begin() + pos + n);
    pos += n;
  } while (pos < raw.size());
  uint32_t a = 1, b = 0;
  for (uint8_t c : raw) {
    a = (a + c) % 65521u;
    b = (b + a) % 65521u;
  }
  put32(z, (b << 16) | a);

  std::vector<uint8_t> out = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1A, '\n'};
  std::vector<uint8_t> ihdr;
  put32(ihdr, width);
  put32(ihdr, height);
  ihdr.push_back(8);  // bit depth
  ihdr.push_back(6);  // colour type RGBA
  ihdr.push_back(0);  // deflate
  ihdr.push_back(0);  // adaptive filtering
  ihdr.push_back(0);  // no interlace
  chunk(out, "IHDR", ihdr);
  chunk(out, "IDAT", z);
  chunk(out, "IEND", {});
  FILE* f = std::fopen(path, "wb");
  if (!f) return PBRT_ERR_INVALID_ARGUMENT;
  const size_t w = std::fwrite(out.data(), 1, out.size(), f);
  const int closed = std::fclose(f);
  return (w == out.size() && closed == 0) ? PBRT_OK : PBRT_ERR_INVALID_ARGUMENT;
}
