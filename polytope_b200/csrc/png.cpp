// png.cpp -- writes RGBA8 pixels as a PNG file (the reference writes its film with lodepng,
// PNGFilm.cpp:50).  The image data is a zlib stream of stored (uncompressed) deflate blocks, so
// the writer needs no compression library; decoders see the same pixels.  PNG chunk CRCs use the
// CRC-32 of ISO 3309 (polynomial 0xEDB88320, reflected), the zlib trailer the Adler-32 of RFC 1950.

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "pt_internal.h"

namespace {

uint32_t crc32_update(uint32_t crc, const uint8_t* p, size_t n) {
    static uint32_t table[256];
    static bool ready = false;
    if (!ready) {
        for (uint32_t i = 0; i < 256; ++i) {
            uint32_t c = i;
            for (int k = 0; k < 8; ++k) c = (c & 1u) ? 0xEDB88320u ^ (c >> 1) : (c >> 1);
            table[i] = c;
        }
        ready = true;
    }
    for (size_t i = 0; i < n; ++i) crc = table[(crc ^ p[i]) & 0xFFu] ^ (crc >> 8);
    return crc;
}

void put_u32_be(std::vector<uint8_t>& v, uint32_t x) {
    v.push_back((uint8_t)(x >> 24));
    v.push_back((uint8_t)(x >> 16));
    v.push_back((uint8_t)(x >> 8));
    v.push_back((uint8_t)x);
}

void put_chunk(std::vector<uint8_t>& out, const char type[4], const std::vector<uint8_t>& data) {
    put_u32_be(out, (uint32_t)data.size());
    const size_t start = out.size();
    out.insert(out.end(), type, type + 4);
    out.insert(out.end(), data.begin(), data.end());
    const uint32_t crc = crc32_update(0xFFFFFFFFu, out.data() + start, out.size() - start) ^ 0xFFFFFFFFu;
    put_u32_be(out, crc);
}

}  // namespace

using namespace pt;

extern "C" int pt_write_png(const char* path, const uint8_t* rgba, uint32_t width, uint32_t height) {
    if (!path || !rgba) return fail(PT_EINVAL, "path or rgba is NULL");
    if (width == 0 || height == 0 || width > (1u << 24) || height > (1u << 24))
        return fail(PT_EINVAL, "image size out of range");
    const size_t row = 4 * (size_t)width;
    // raw scanlines: filter type 0, then the row
    std::vector<uint8_t> raw;
    raw.reserve((row + 1) * height);
    for (uint32_t y = 0; y < height; ++y) {
        raw.push_back(0);
        raw.insert(raw.end(), rgba + y * row, rgba + (y + 1) * row);
    }
    // zlib stream: header (deflate, 32 KiB window, no dictionary, check bits), stored blocks, Adler-32
    std::vector<uint8_t> z;
    z.reserve(raw.size() + raw.size() / 65535 * 5 + 16);
    z.push_back(0x78);
    z.push_back(0x01);
    size_t off = 0;
    do {
        const size_t len = std::min<size_t>(65535, raw.size() - off);
        const bool last = off + len == raw.size();
        z.push_back(last ? 1 : 0);
        z.push_back((uint8_t)len);
        z.push_back((uint8_t)(len >> 8));
        z.push_back((uint8_t)~len);
        z.push_back((uint8_t)(~len >> 8));
        z.insert(z.end(), raw.begin() + off, raw.begin() + off + len);
        off += len;
    } while (off < raw.size());
    uint32_t a = 1, b = 0;
    for (uint8_t c : raw) {
        a = (a + c) % 65521u;
        b = (b + a) % 65521u;
    }
    put_u32_be(z, (b << 16) | a);

    std::vector<uint8_t> png = {0x89, 'P', 'N', 'G', 0x0D, 0x0A, 0x1A, 0x0A};
    std::vector<uint8_t> ihdr;
    put_u32_be(ihdr, width);
    put_u32_be(ihdr, height);
    ihdr.push_back(8);  // bit depth
    ihdr.push_back(6);  // colour type: RGBA
    ihdr.push_back(0);  // compression
    ihdr.push_back(0);  // filter
    ihdr.push_back(0);  // interlace
    put_chunk(png, "IHDR", ihdr);
    put_chunk(png, "IDAT", z);
    put_chunk(png, "IEND", {});

    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(PT_EINVAL, std::string("cannot open ") + path);
    const size_t n = std::fwrite(png.data(), 1, png.size(), f);
    const int closed = std::fclose(f);
    if (n != png.size() || closed != 0) return fail(PT_EINVAL, std::string("cannot write ") + path);
    return PT_OK;
}
