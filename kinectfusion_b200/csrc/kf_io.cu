// kf_io.cu - the files around the reconstruction loop (host code): the
// PNG depth and colour frames a TUM RGB-D sequence holds (VirtualSensor,
// src/kinectfusion/virtual_sensor.cpp:41-147, decoded by
// image_proc/read_png.cpp), PNG writes of frames, and binary PLY files of
// meshes and raycast point clouds (src/app/frame_output.cpp:76-181).
//
// PNG (ISO/IEC 15948): the chunks are walked and CRC-checked, the IDAT
// stream is inflated with zlib, and the five scanline filters (none, sub,
// up, average, Paeth) are undone row by row.  Depth must be 16-bit
// grayscale and is copied verbatim (the reference's rule); colour accepts
// 8- or 16-bit grayscale, grey+alpha, RGB, RGBA and 8-bit palette images and
// returns RGBA8 pixels packed as R | G << 8 | B << 16 | A << 24.  Interlaced
// (Adam7) images are refused.
#include <zlib.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "kf_internal.h"

namespace kf {
namespace {

const uint8_t kSignature[8] = {137, 80, 78, 71, 13, 10, 26, 10};

uint32_t be32(const uint8_t* p) {
  return (static_cast<uint32_t>(p[0]) << 24) | (static_cast<uint32_t>(p[1]) << 16) |
         (static_cast<uint32_t>(p[2]) << 8) | static_cast<uint32_t>(p[3]);
}

void put32(std::vector<uint8_t>& out, uint32_t v) {
  out.push_back(static_cast<uint8_t>(v >> 24));
  out.push_back(static_cast<uint8_t>(v >> 16));
  out.push_back(static_cast<uint8_t>(v >> 8));
  out.push_back(static_cast<uint8_t>(v));
}

std::vector<uint8_t> read_file(const char* path) {
  FILE* f = std::fopen(path, "rb");
  if (f == nullptr) throw IoError(std::string("Failed to open file: ") + path);
  std::vector<uint8_t> data;
  uint8_t buf[1 << 16];
  size_t n;
  while ((n = std::fread(buf, 1, sizeof(buf), f)) > 0) data.insert(data.end(), buf, buf + n);
  const bool bad = std::ferror(f) != 0;
  std::fclose(f);
  if (bad) throw IoError(std::string("Failed to read file: ") + path);
  return data;
}

void write_file(const char* path, const std::vector<uint8_t>& data) {
  FILE* f = std::fopen(path, "wb");
  if (f == nullptr) throw IoError(std::string("Failed to open output: ") + path);
  const size_t n = std::fwrite(data.data(), 1, data.size(), f);
  const bool bad = std::fclose(f) != 0 || n != data.size();
  if (bad) throw IoError(std::string("Failed to write output: ") + path);
}

struct Png {
  uint32_t width = 0, height = 0;
  int bit_depth = 0, color_type = 0, channels = 0;
  std::vector<uint8_t> palette;  // RGB triples
  std::vector<uint8_t> alpha;    // tRNS of a palette image
  std::vector<uint8_t> pixels;   // unfiltered rows, width * bytes per pixel each
};

int channels_of(int color_type) {
  switch (color_type) {
    case 0: return 1;  // grayscale
    case 2: return 3;  // RGB
    case 3: return 1;  // palette index
    case 4: return 2;  // grey + alpha
    case 6: return 4;  // RGBA
    default: return 0;
  }
}

uint8_t paeth(int a, int b, int c) {
  const int p = a + b - c;
  const int pa = std::abs(p - a), pb = std::abs(p - b), pc = std::abs(p - c);
  if (pa <= pb && pa <= pc) return static_cast<uint8_t>(a);
  if (pb <= pc) return static_cast<uint8_t>(b);
  return static_cast<uint8_t>(c);
}

Png decode(const char* path) {
  const std::vector<uint8_t> file = read_file(path);
  const std::string name(path);
  if (file.size() < 8 || std::memcmp(file.data(), kSignature, 8) != 0) throw IoError("Not a PNG file: " + name);
  Png png;
  std::vector<uint8_t> idat;
  bool have_header = false, ended = false;
  int interlace = 0;
  size_t pos = 8;
  while (pos + 12 <= file.size() && !ended) {
    const uint32_t length = be32(file.data() + pos);
    if (length > file.size() - pos - 12) throw IoError("Truncated PNG chunk: " + name);
    const uint8_t* type = file.data() + pos + 4;
    const uint8_t* data = type + 4;
    const uint32_t crc = be32(data + length);
    if (static_cast<uint32_t>(crc32(0L, type, length + 4)) != crc) throw IoError("PNG chunk CRC mismatch: " + name);
    if (std::memcmp(type, "IHDR", 4) == 0) {
      if (length != 13) throw IoError("Bad PNG header: " + name);
      png.width = be32(data);
      png.height = be32(data + 4);
      png.bit_depth = data[8];
      png.color_type = data[9];
      interlace = data[12];
      if (data[10] != 0 || data[11] != 0) throw IoError("Unknown PNG compression or filter method: " + name);
      have_header = true;
    } else if (std::memcmp(type, "PLTE", 4) == 0) {
      png.palette.assign(data, data + length);
    } else if (std::memcmp(type, "tRNS", 4) == 0) {
      png.alpha.assign(data, data + length);
    } else if (std::memcmp(type, "IDAT", 4) == 0) {
      idat.insert(idat.end(), data, data + length);
    } else if (std::memcmp(type, "IEND", 4) == 0) {
      ended = true;
    }
    pos += 12 + length;
  }
  if (!have_header || !ended) throw IoError("Incomplete PNG file: " + name);
  png.channels = channels_of(png.color_type);
  const bool depth_ok = png.bit_depth == 8 || (png.bit_depth == 16 && png.color_type != 3);
  if (png.channels == 0 || !depth_ok) throw IoError("Unsupported PNG pixel format: " + name);
  if (interlace != 0) throw IoError("Interlaced PNG files are not supported: " + name);
  if (png.width == 0 || png.height == 0 || png.width > (1u << 16) || png.height > (1u << 16)) {
    throw IoError("PNG size out of range: " + name);
  }
  const size_t bpp = static_cast<size_t>(png.channels) * (png.bit_depth / 8);
  const size_t row = static_cast<size_t>(png.width) * bpp;
  std::vector<uint8_t> raw(png.height * (row + 1));
  uLongf raw_len = static_cast<uLongf>(raw.size());
  if (uncompress(raw.data(), &raw_len, idat.data(), static_cast<uLong>(idat.size())) != Z_OK ||
      raw_len != raw.size()) {
    throw IoError("Corrupt PNG image data: " + name);
  }
  png.pixels.resize(png.height * row);
  for (uint32_t y = 0; y < png.height; ++y) {
    const uint8_t filter = raw[y * (row + 1)];
    const uint8_t* in = raw.data() + y * (row + 1) + 1;
    uint8_t* out = png.pixels.data() + y * row;
    const uint8_t* up = y > 0 ? out - row : nullptr;
    for (size_t x = 0; x < row; ++x) {
      const int a = x >= bpp ? out[x - bpp] : 0;
      const int b = up ? up[x] : 0;
      const int c = (up && x >= bpp) ? up[x - bpp] : 0;
      int v = in[x];
      switch (filter) {
        case 0: break;
        case 1: v += a; break;
        case 2: v += b; break;
        case 3: v += (a + b) / 2; break;
        case 4: v += paeth(a, b, c); break;
        default: throw IoError("Bad PNG row filter: " + name);
      }
      out[x] = static_cast<uint8_t>(v);
    }
  }
  return png;
}

// zlib stream of rows that all carry filter `filter` (0 none, 1 sub).
std::vector<uint8_t> encode(uint32_t width, uint32_t height, int bit_depth, int color_type,
                            const std::vector<uint8_t>& rows) {
  const size_t row = rows.size() / height;
  const size_t bpp = static_cast<size_t>(channels_of(color_type)) * (bit_depth / 8);
  std::vector<uint8_t> raw(height * (row + 1));
  for (uint32_t y = 0; y < height; ++y) {
    uint8_t* dst = raw.data() + y * (row + 1);
    const uint8_t* src = rows.data() + y * row;
    dst[0] = 1;  // sub: neighbouring depths or colours differ little
    for (size_t x = 0; x < row; ++x) dst[1 + x] = static_cast<uint8_t>(src[x] - (x >= bpp ? src[x - bpp] : 0));
  }
  uLongf zlen = compressBound(static_cast<uLong>(raw.size()));
  std::vector<uint8_t> z(zlen);
  if (compress2(z.data(), &zlen, raw.data(), static_cast<uLong>(raw.size()), 6) != Z_OK) {
    throw IoError("PNG compression failed");
  }
  z.resize(zlen);
  std::vector<uint8_t> out(kSignature, kSignature + 8);
  auto chunk = [&out](const char* type, const uint8_t* data, size_t length) {
    put32(out, static_cast<uint32_t>(length));
    const size_t start = out.size();
    out.insert(out.end(), type, type + 4);
    out.insert(out.end(), data, data + length);
    put32(out, static_cast<uint32_t>(crc32(0L, out.data() + start, static_cast<uInt>(length + 4))));
  };
  std::vector<uint8_t> ihdr;
  put32(ihdr, width);
  put32(ihdr, height);
  ihdr.push_back(static_cast<uint8_t>(bit_depth));
  ihdr.push_back(static_cast<uint8_t>(color_type));
  ihdr.push_back(0);
  ihdr.push_back(0);
  ihdr.push_back(0);
  chunk("IHDR", ihdr.data(), ihdr.size());
  chunk("IDAT", z.data(), z.size());
  chunk("IEND", nullptr, 0);
  return out;
}

void append_f32(std::string& out, float v) {
  char b[4];
  std::memcpy(b, &v, 4);
  out.append(b, 4);
}

std::string ply_header(uint64_t vertices, uint64_t faces, bool with_faces) {
  std::string h = "ply\nformat binary_little_endian 1.0\nelement vertex " + std::to_string(vertices) +
                  "\nproperty float x\nproperty float y\nproperty float z\n"
                  "property float nx\nproperty float ny\nproperty float nz\n"
                  "property uchar red\nproperty uchar green\nproperty uchar blue\n";
  if (with_faces) {
    h += "element face " + std::to_string(faces) + "\nproperty list uchar uint vertex_indices\n";
  }
  return h + "end_header\n";
}

void write_text_and_binary(const char* path, const std::string& header, const std::string& body) {
  std::vector<uint8_t> data(header.begin(), header.end());
  data.insert(data.end(), body.begin(), body.end());
  write_file(path, data);
}

}  // namespace
}  // namespace kf

using namespace kf;

extern "C" {

kf_status kf_png_info(const char* path, uint32_t* width, uint32_t* height, int32_t* color_type, int32_t* bit_depth) {
  return guarded([&] {
    require(path && width && height, "kf_png_info: null argument");
    const Png png = decode(path);
    *width = png.width;
    *height = png.height;
    if (color_type) *color_type = png.color_type;
    if (bit_depth) *bit_depth = png.bit_depth;
  });
}

kf_status kf_png_read_depth(const char* path, uint16_t* out, uint32_t width, uint32_t height) {
  return guarded([&] {
    require(path && out, "kf_png_read_depth: null argument");
    const Png png = decode(path);
    // read_png<DepthImage> copies verbatim: the file must be 16-bit grayscale
    if (png.color_type != 0 || png.bit_depth != 16) {
      throw IoError(std::string("Expected 16-bit grayscale png: ") + path);
    }
    require(png.width == width && png.height == height, "kf_png_read_depth: image size differs from the buffer");
    const size_t n = static_cast<size_t>(width) * height;
    for (size_t i = 0; i < n; ++i) {
      out[i] = static_cast<uint16_t>((png.pixels[2 * i] << 8) | png.pixels[2 * i + 1]);
    }
  });
}

kf_status kf_png_read_color(const char* path, uint32_t* out, uint32_t width, uint32_t height) {
  return guarded([&] {
    require(path && out, "kf_png_read_color: null argument");
    const Png png = decode(path);
    require(png.width == width && png.height == height, "kf_png_read_color: image size differs from the buffer");
    const size_t n = static_cast<size_t>(width) * height;
    const size_t step = png.bit_depth / 8;  // 16-bit samples keep their high byte
    const size_t bpp = static_cast<size_t>(png.channels) * step;
    for (size_t i = 0; i < n; ++i) {
      const uint8_t* p = png.pixels.data() + i * bpp;
      uint32_t r, g, b, a = 255;
      switch (png.color_type) {
        case 0:
          r = g = b = p[0];
          break;
        case 4:
          r = g = b = p[0];
          a = p[step];
          break;
        case 2:
          r = p[0];
          g = p[step];
          b = p[2 * step];
          break;
        case 6:
          r = p[0];
          g = p[step];
          b = p[2 * step];
          a = p[3 * step];
          break;
        default: {  // palette
          const size_t k = p[0];
          if (3 * k + 2 >= png.palette.size()) throw IoError(std::string("PNG palette index out of range: ") + path);
          r = png.palette[3 * k];
          g = png.palette[3 * k + 1];
          b = png.palette[3 * k + 2];
          if (k < png.alpha.size()) a = png.alpha[k];
        }
      }
      out[i] = r | (g << 8) | (b << 16) | (a << 24);
    }
  });
}

kf_status kf_png_write_depth(const char* path, const uint16_t* depth, uint32_t width, uint32_t height) {
  return guarded([&] {
    require(path && depth && width > 0 && height > 0, "kf_png_write_depth: bad argument");
    std::vector<uint8_t> rows(static_cast<size_t>(width) * height * 2);
    for (size_t i = 0; i < static_cast<size_t>(width) * height; ++i) {
      rows[2 * i] = static_cast<uint8_t>(depth[i] >> 8);
      rows[2 * i + 1] = static_cast<uint8_t>(depth[i]);
    }
    write_file(path, encode(width, height, 16, 0, rows));
  });
}

kf_status kf_png_write_color(const char* path, const uint32_t* rgba, uint32_t width, uint32_t height) {
  return guarded([&] {
    require(path && rgba && width > 0 && height > 0, "kf_png_write_color: bad argument");
    std::vector<uint8_t> rows(static_cast<size_t>(width) * height * 4);
    for (size_t i = 0; i < static_cast<size_t>(width) * height; ++i) {
      for (int c = 0; c < 4; ++c) rows[4 * i + c] = static_cast<uint8_t>(rgba[i] >> (8 * c));
    }
    write_file(path, encode(width, height, 8, 6, rows));
  });
}

kf_status kf_mesh_write_ply(const char* path, const kf_mesh* mesh) {
  return guarded([&] {
    require(path && mesh, "kf_mesh_write_ply: null argument");
    // FrameOutput::write_mesh (frame_output.cpp:127-181): position, normal,
    // colour clamped to [0, 255] as uchar; triangles as uchar 3 + 3 uint
    std::string body;
    body.reserve(mesh->vertex_count * 27 + mesh->triangle_count * 13);
    for (uint64_t i = 0; i < mesh->vertex_count; ++i) {
      for (int c = 0; c < 3; ++c) append_f32(body, mesh->positions[3 * i + c]);
      for (int c = 0; c < 3; ++c) append_f32(body, mesh->normals[3 * i + c]);
      for (int c = 0; c < 3; ++c) {
        const float v = mesh->colors ? mesh->colors[3 * i + c] : 255.0f;
        body.push_back(static_cast<char>(static_cast<uint8_t>(std::clamp(v, 0.0f, 255.0f))));
      }
    }
    for (uint64_t t = 0; t < mesh->triangle_count; ++t) {
      body.push_back(static_cast<char>(3));
      for (int c = 0; c < 3; ++c) {
        char b[4];
        std::memcpy(b, &mesh->triangles[3 * t + c], 4);
        body.append(b, 4);
      }
    }
    write_text_and_binary(path, ply_header(mesh->vertex_count, mesh->triangle_count, true), body);
  });
}

kf_status kf_maps_write_ply(const char* path, const float* points, const float* normals, const uint32_t* colors,
                            uint32_t width, uint32_t height) {
  return guarded([&] {
    require(path && points && normals && colors, "kf_maps_write_ply: null argument");
    // FrameOutput's raycast point cloud (frame_output.cpp:76-117): every
    // pixel with a finite point and normal, colour from its RGBA8 value
    std::string body;
    uint64_t count = 0;
    for (size_t i = 0; i < static_cast<size_t>(width) * height; ++i) {
      const float* p = points + 3 * i;
      const float* n = normals + 3 * i;
      if (!(std::isfinite(p[0]) && std::isfinite(p[1]) && std::isfinite(p[2]) && std::isfinite(n[0]) &&
            std::isfinite(n[1]) && std::isfinite(n[2]))) {
        continue;
      }
      ++count;
      for (int c = 0; c < 3; ++c) append_f32(body, p[c]);
      for (int c = 0; c < 3; ++c) append_f32(body, n[c]);
      for (int c = 0; c < 3; ++c) body.push_back(static_cast<char>(static_cast<uint8_t>(colors[i] >> (8 * c))));
    }
    write_text_and_binary(path, ply_header(count, 0, false), body);
  });
}

}  // extern "C"
