// PNG decoding follows the PNG specification (W3C, Portable Network Graphics, 2nd edition): chunk
// stream, zlib-compressed scanlines, the five per-row filters with the Paeth predictor, and the
// colour types grey, RGB, palette, grey + alpha and RGBA at bit depths 1-16. Inflation is zlib's.
// Binary PPM (P6) and PGM (P5) follow Netpbm's format description. Host code.
#include "image_io.hpp"

#include <zlib.h>

#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iterator>

namespace pt
{
    namespace
    {
        uint32_t be32(const uint8_t* p) { return (uint32_t(p[0]) << 24) | (uint32_t(p[1]) << 16) | (uint32_t(p[2]) << 8) | uint32_t(p[3]); }

        int paeth(int a, int b, int c)
        {
            const int p = a + b - c;
            const int pa = std::abs(p - a), pb = std::abs(p - b), pc = std::abs(p - c);
            if (pa <= pb && pa <= pc) return a;
            return pb <= pc ? b : c;
        }

        bool decode_png(const std::vector<uint8_t>& f, Image8& out, std::string& error)
        {
            static const uint8_t sig[8] = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
            if (f.size() < 8 || std::memcmp(f.data(), sig, 8) != 0) return error = "not a PNG file", false;
            uint32_t w = 0, h = 0;
            int depth = 0, colour = -1, interlace = 0;
            std::vector<uint8_t> idat, palette, paletteAlpha;
            size_t pos = 8;
            bool ended = false;
            while (pos + 12 <= f.size() && !ended)
            {
                const uint32_t len = be32(&f[pos]);
                if (pos + 12 + static_cast<size_t>(len) > f.size()) return error = "truncated PNG chunk", false;
                const uint8_t* type = &f[pos + 4];
                const uint8_t* body = &f[pos + 8];
                const uint32_t crc = be32(&f[pos + 8 + len]);
                if ((crc32(crc32(0L, type, 4), body, len) & 0xFFFFFFFFu) != crc) return error = "PNG chunk CRC mismatch", false;
                if (!std::memcmp(type, "IHDR", 4) && len >= 13)
                {
                    w = be32(body);
                    h = be32(body + 4);
                    depth = body[8];
                    colour = body[9];
                    interlace = body[12];
                }
                else if (!std::memcmp(type, "PLTE", 4)) palette.assign(body, body + len);
                else if (!std::memcmp(type, "tRNS", 4)) paletteAlpha.assign(body, body + len);
                else if (!std::memcmp(type, "IDAT", 4)) idat.insert(idat.end(), body, body + len);
                else if (!std::memcmp(type, "IEND", 4)) ended = true;
                pos += 12 + static_cast<size_t>(len);
            }
            if (w == 0 || h == 0 || w > 32768 || h > 32768) return error = "PNG size missing or above 32768", false;
            if (interlace != 0) return error = "interlaced PNG is not supported", false;
            int samples;
            switch (colour)
            {
                case 0: samples = 1; break;
                case 2: samples = 3; break;
                case 3: samples = 1; break;
                case 4: samples = 2; break;
                case 6: samples = 4; break;
                default: return error = "unknown PNG colour type", false;
            }
            const bool depthOk = depth == 8 || depth == 16 || ((colour == 0 || colour == 3) && (depth == 1 || depth == 2 || depth == 4));
            if (!depthOk) return error = "unsupported PNG bit depth", false;
            if (colour == 3 && palette.size() < 3) return error = "palette PNG without a palette", false;
            const size_t bitsPerPixel = static_cast<size_t>(samples) * depth;
            const size_t rowBytes = (static_cast<size_t>(w) * bitsPerPixel + 7) / 8;
            const size_t bpp = std::max<size_t>(1, bitsPerPixel / 8);  // filter byte distance
            std::vector<uint8_t> raw(static_cast<size_t>(h) * (rowBytes + 1));
            uLongf rawLen = static_cast<uLongf>(raw.size());
            if (uncompress(raw.data(), &rawLen, idat.data(), static_cast<uLong>(idat.size())) != Z_OK || rawLen != raw.size())
                return error = "PNG image data does not inflate to its size", false;
            std::vector<uint8_t> img(static_cast<size_t>(h) * rowBytes), zero(rowBytes, 0);
            for (uint32_t y = 0; y < h; y++)
            {
                const uint8_t filter = raw[y * (rowBytes + 1)];
                const uint8_t* src = &raw[y * (rowBytes + 1) + 1];
                uint8_t* cur = &img[y * rowBytes];
                const uint8_t* prev = y ? &img[(y - 1) * rowBytes] : zero.data();
                for (size_t i = 0; i < rowBytes; i++)
                {
                    const int a = i >= bpp ? cur[i - bpp] : 0, b = prev[i], c = i >= bpp ? prev[i - bpp] : 0;
                    int p;
                    switch (filter)
                    {
                        case 0: p = 0; break;
                        case 1: p = a; break;
                        case 2: p = b; break;
                        case 3: p = (a + b) / 2; break;
                        case 4: p = paeth(a, b, c); break;
                        default: return error = "unknown PNG row filter", false;
                    }
                    cur[i] = static_cast<uint8_t>(src[i] + p);
                }
            }
            // samples to 8 bits (16-bit: the high byte; below 8: scaled to 0..255), then the output layout
            auto sample = [&](uint32_t y, uint32_t x, int s) -> uint32_t
            {
                const uint8_t* row = &img[static_cast<size_t>(y) * rowBytes];
                if (depth == 8) return row[static_cast<size_t>(x) * samples + s];
                if (depth == 16) return row[(static_cast<size_t>(x) * samples + s) * 2];
                const size_t bit = static_cast<size_t>(x) * depth;
                const uint32_t v = (row[bit / 8] >> (8 - depth - bit % 8)) & ((1u << depth) - 1u);
                return v;
            };
            const bool hasAlpha = colour == 4 || colour == 6 || (colour == 3 && !paletteAlpha.empty());
            out.width = w;
            out.height = h;
            out.channels = colour == 0 ? 1u : (hasAlpha ? 4u : 3u);
            out.pixels.assign(static_cast<size_t>(w) * h * out.channels, 0);
            for (uint32_t y = 0; y < h; y++)
                for (uint32_t x = 0; x < w; x++)
                {
                    uint8_t* o = &out.pixels[(static_cast<size_t>(y) * w + x) * out.channels];
                    if (colour == 3)
                    {
                        const uint32_t i = sample(y, x, 0);
                        if (i * 3 + 2 >= palette.size()) return error = "PNG palette index out of range", false;
                        o[0] = palette[i * 3];
                        o[1] = palette[i * 3 + 1];
                        o[2] = palette[i * 3 + 2];
                        if (hasAlpha) o[3] = i < paletteAlpha.size() ? paletteAlpha[i] : 255;
                    }
                    else if (colour == 0)
                        o[0] = static_cast<uint8_t>(depth < 8 ? sample(y, x, 0) * 255u / ((1u << depth) - 1u) : sample(y, x, 0));
                    else if (colour == 4)
                    {
                        o[0] = o[1] = o[2] = static_cast<uint8_t>(sample(y, x, 0));
                        o[3] = static_cast<uint8_t>(sample(y, x, 1));
                    }
                    else
                        for (uint32_t c = 0; c < out.channels; c++) o[c] = static_cast<uint8_t>(sample(y, x, static_cast<int>(c)));
                }
            return true;
        }

        bool decode_pnm(const std::vector<uint8_t>& f, Image8& out, std::string& error)
        {
            if (f.size() < 2 || f[0] != 'P' || (f[1] != '6' && f[1] != '5')) return error = "not a binary PPM/PGM file", false;
            size_t pos = 2;
            uint32_t vals[3] = {0, 0, 0};
            for (int k = 0; k < 3; k++)
            {
                while (pos < f.size() && (std::isspace(f[pos]) || f[pos] == '#'))
                {
                    if (f[pos] == '#')
                        while (pos < f.size() && f[pos] != '\n') pos++;
                    else
                        pos++;
                }
                while (pos < f.size() && std::isdigit(f[pos])) vals[k] = vals[k] * 10 + (f[pos++] - '0');
            }
            pos++;  // one whitespace byte before the raster
            const uint32_t w = vals[0], h = vals[1], maxval = vals[2];
            const uint32_t ch = f[1] == '6' ? 3u : 1u;
            if (w == 0 || h == 0 || w > 32768 || h > 32768 || maxval == 0 || maxval > 255) return error = "unsupported PPM/PGM header", false;
            if (pos + static_cast<size_t>(w) * h * ch > f.size()) return error = "truncated PPM/PGM raster", false;
            out.width = w;
            out.height = h;
            out.channels = ch;
            out.pixels.assign(f.begin() + static_cast<long>(pos), f.begin() + static_cast<long>(pos + static_cast<size_t>(w) * h * ch));
            if (maxval != 255)
                for (auto& v : out.pixels) v = static_cast<uint8_t>(std::min<uint32_t>(255u, v * 255u / maxval));
            return true;
        }
    }

    bool LoadImage8(const std::string& path, Image8& out, std::string& error)
    {
        std::ifstream in(path, std::ios::binary);
        if (!in) return error = "cannot open " + path, false;
        const std::vector<uint8_t> f((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
        bool ok;
        if (f.size() >= 8 && f[0] == 0x89 && f[1] == 'P') ok = decode_png(f, out, error);
        else if (f.size() >= 2 && f[0] == 'P') ok = decode_pnm(f, out, error);
        else return error = path + ": unsupported image format (PNG and binary PPM/PGM are decoded)", false;
        if (!ok) error = path + ": " + error;
        return ok;
    }
}
