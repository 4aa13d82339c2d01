// mc_image.cpp - host PNG writer for 8-bit RGB pixels (the reference writes its
// image with stb's PNG writer, PT:4381). The pixels go into uncompressed
// ("stored") deflate blocks: a valid PNG whose encoding costs one pass over
// the bytes, for a renderer whose output is read back once per image.
//
// Format (PNG specification, RFC 1950 zlib and RFC 1951 deflate):
//   signature; IHDR (width, height, bit depth 8, colour type 2 = RGB);
//   IDAT = zlib header 0x78 0x01, stored blocks of at most 65535 bytes of the
//   filtered scanlines (filter byte 0 before each row), Adler-32 of those;
//   IEND. Each chunk ends with the CRC-32 (reflected polynomial 0xEDB88320)
//   of its type and data.
#include <cstdint>
#include <cstring>

#include "mc_internal.h"

namespace {

struct Crc32 {
    uint32_t table[256];
    Crc32() {
        for (uint32_t n = 0; n < 256; n++) {
            uint32_t c = n;
            for (int k = 0; k < 8; k++) c = (c & 1u) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
            table[n] = c;
        }
    }
    uint32_t update(uint32_t crc, const uint8_t* p, size_t n) const {
        for (size_t i = 0; i < n; i++) crc = table[(crc ^ p[i]) & 0xFFu] ^ (crc >> 8);
        return crc;
    }
};

const Crc32& crc_table() {
    static const Crc32 t;
    return t;
}

void put_be32(uint8_t* p, uint32_t v) {
    p[0] = (uint8_t)(v >> 24); p[1] = (uint8_t)(v >> 16); p[2] = (uint8_t)(v >> 8); p[3] = (uint8_t)v;
}

constexpr size_t kStoredMax = 65535;

}  // namespace

extern "C" mc_status mc_png_encode(const uint8_t* rgb, int32_t width, int32_t height, uint8_t* out, int64_t* bytes) {
    if (!bytes || width <= 0 || height <= 0) return mc::set_error(MC_ERR_INVALID, "mc_png_encode: bad arguments");
    const size_t row = 1 + (size_t)width * 3;
    const size_t raw = row * (size_t)height;
    if (raw > ((size_t)1 << 40)) return mc::set_error(MC_ERR_INVALID, "mc_png_encode: image too large");
    const size_t blocks = (raw + kStoredMax - 1) / kStoredMax;
    const size_t idat = 2 + blocks * 5 + raw + 4;
    if (idat > 0x7FFFFFFFu) return mc::set_error(MC_ERR_INVALID, "mc_png_encode: image too large for one IDAT chunk");
    const size_t total = 8 + (12 + 13) + (12 + idat) + 12;
    if (!out) {
        *bytes = (int64_t)total;
        return MC_OK;
    }
    if (!rgb) return mc::set_error(MC_ERR_INVALID, "mc_png_encode: null pixels");
    if (*bytes < (int64_t)total) return mc::set_error(MC_ERR_INVALID, "mc_png_encode: output too small");
    const Crc32& crc = crc_table();
    uint8_t* p = out;
    static const uint8_t sig[8] = {0x89, 'P', 'N', 'G', 0x0D, 0x0A, 0x1A, 0x0A};
    std::memcpy(p, sig, 8);
    p += 8;
    // IHDR
    put_be32(p, 13);
    uint8_t* type = p + 4;
    std::memcpy(type, "IHDR", 4);
    put_be32(type + 4, (uint32_t)width);
    put_be32(type + 8, (uint32_t)height);
    type[12] = 8; type[13] = 2; type[14] = 0; type[15] = 0; type[16] = 0;
    put_be32(type + 17, crc.update(0xFFFFFFFFu, type, 17) ^ 0xFFFFFFFFu);
    p = type + 21;
    // IDAT
    put_be32(p, (uint32_t)idat);
    type = p + 4;
    std::memcpy(type, "IDAT", 4);
    uint8_t* d = type + 4;
    *d++ = 0x78;
    *d++ = 0x01;
    uint32_t a = 1, b = 0;  // Adler-32
    size_t done = 0;        // bytes of the filtered scanline stream written
    size_t y = 0, col = 0;  // position in that stream: row y, byte col of the row
    while (done < raw) {
        const size_t len = raw - done < kStoredMax ? raw - done : kStoredMax;
        *d++ = done + len == raw ? 1 : 0;  // BFINAL, BTYPE 00
        d[0] = (uint8_t)len; d[1] = (uint8_t)(len >> 8);
        d[2] = (uint8_t)~len; d[3] = (uint8_t)(~len >> 8);
        d += 4;
        size_t left = len;
        while (left) {
            if (col == 0) {
                *d++ = 0;  // filter type None
                b = (b + a) % 65521u;
                col = 1;
                left--;
                continue;
            }
            size_t take = row - col < left ? row - col : left;
            const uint8_t* src = rgb + y * (size_t)width * 3 + (col - 1);
            std::memcpy(d, src, take);
            for (size_t i = 0; i < take; i++) {
                a += src[i];
                if (a >= 65521u) a -= 65521u;
                b += a;
                if (b >= 65521u) b -= 65521u;
            }
            d += take;
            col += take;
            left -= take;
            if (col == row) {
                col = 0;
                y++;
            }
        }
        done += len;
    }
    put_be32(d, (b << 16) | a);
    d += 4;
    put_be32(d, crc.update(0xFFFFFFFFu, type, 4 + idat) ^ 0xFFFFFFFFu);
    p = d + 4;
    // IEND
    put_be32(p, 0);
    std::memcpy(p + 4, "IEND", 4);
    put_be32(p + 8, crc.update(0xFFFFFFFFu, p + 4, 4) ^ 0xFFFFFFFFu);
    p += 12;
    *bytes = (int64_t)(p - out);
    return MC_OK;
}
