// PNG encoding of 8-bit RGB images (the reference's encode_png,
// src/io/image_io.cpp:45-56), written against zlib: signature, IHDR, one IDAT
// of filter-0 scanlines deflated by zlib, IEND; each chunk CRC-32 protected.
#include <zlib.h>

#include <cstdint>
#include <stdexcept>
#include <vector>

namespace rtg {

namespace {

void put_be32(std::vector<std::uint8_t>& out, std::uint32_t v) {
  out.push_back(static_cast<std::uint8_t>(v >> 24));
  out.push_back(static_cast<std::uint8_t>(v >> 16));
  out.push_back(static_cast<std::uint8_t>(v >> 8));
  out.push_back(static_cast<std::uint8_t>(v));
}

void chunk(std::vector<std::uint8_t>& out, const char type[4], const std::vector<std::uint8_t>& data) {
  put_be32(out, static_cast<std::uint32_t>(data.size()));
  const std::size_t start = out.size();
  out.insert(out.end(), type, type + 4);
  out.insert(out.end(), data.begin(), data.end());
  const uLong crc = crc32(0L, out.data() + start, static_cast<uInt>(out.size() - start));
  put_be32(out, static_cast<std::uint32_t>(crc));
}

}  // namespace

std::vector<std::uint8_t> encode_png(const std::uint8_t* rgb, int width, int height) {
  if (width <= 0 || height <= 0 || !rgb) throw std::invalid_argument("invalid image dimensions");
  const std::size_t row = static_cast<std::size_t>(width) * 3;
  std::vector<std::uint8_t> raw;
  raw.reserve((row + 1) * static_cast<std::size_t>(height));
  for (int y = 0; y < height; ++y) {
    raw.push_back(0);  // filter type: none
    const std::uint8_t* src = rgb + static_cast<std::size_t>(y) * row;
    raw.insert(raw.end(), src, src + row);
  }
  uLongf zlen = compressBound(static_cast<uLong>(raw.size()));
  std::vector<std::uint8_t> z(zlen);
  if (compress2(z.data(), &zlen, raw.data(), static_cast<uLong>(raw.size()), 6) != Z_OK)
    throw std::runtime_error("PNG encoding failed");
  z.resize(zlen);

  std::vector<std::uint8_t> out = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1A, '\n'};
  std::vector<std::uint8_t> ihdr;
  put_be32(ihdr, static_cast<std::uint32_t>(width));
  put_be32(ihdr, static_cast<std::uint32_t>(height));
  ihdr.push_back(8);  // bit depth
  ihdr.push_back(2);  // colour type: truecolour
  ihdr.push_back(0);  // deflate
  ihdr.push_back(0);  // adaptive filtering
  ihdr.push_back(0);  // no interlace
  chunk(out, "IHDR", ihdr);
  chunk(out, "IDAT", z);
  chunk(out, "IEND", {});
  return out;
}

}  // namespace rtg
