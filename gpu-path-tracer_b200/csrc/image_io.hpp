// Texture image files for OBJ/MTL ingest: PNG (8- and 16-bit, every colour type, not interlaced) and
// binary PPM/PGM, decoded to 8-bit channels. Host code.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace pt
{
    struct Image8
    {
        uint32_t width = 0, height = 0, channels = 0;  // channels 1, 3 or 4 (grey + alpha becomes RGBA)
        std::vector<uint8_t> pixels;                   // rows top to bottom, channels interleaved
    };

    // false with a message in `error` when the file cannot be read or its format is not one of the above
    bool LoadImage8(const std::string& path, Image8& out, std::string& error);
}
