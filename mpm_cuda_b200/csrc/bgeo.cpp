// Houdini classic .bgeo particle writer (replaces OutputBego,
// src/utilities/FilesIO.cpp:6-24, which calls Partio::write on a particle set
// whose only attribute is "position", VECTOR of 3 floats).
//
// Layout written (all integers and floats big-endian):
//   int32 magic 'B','g','e','o'   char 'V'   int32 version = 5
//   int32 nPoints, nPrims = 0, nPointGroups = 0, nPrimGroups = 0,
//         nPointAttrib = 0, nVertexAttrib = 0, nPrimAttrib = 0, nDetailAttrib = 0
//   nPoints x float32[4] (x, y, z, w = 1)   -- the implicit point position
//   byte 0x00, byte 0xff                      -- empty "extra" section
// Position is the implicit homogeneous point attribute of the format, so a
// set with only "position" declares no extra point attributes.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

namespace mpm {

static void put_be32(std::vector<unsigned char>& out, uint32_t v) {
    out.push_back((unsigned char)(v >> 24));
    out.push_back((unsigned char)(v >> 16));
    out.push_back((unsigned char)(v >> 8));
    out.push_back((unsigned char)v);
}

static void put_bef(std::vector<unsigned char>& out, float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    put_be32(out, u);
}

// x holds n points of `dim` floats (dim 2 or 3); returns 0 on success
int write_bgeo(const char* path, const float* x, int64_t n, int dim) {
    if (!path || n < 0 || (n > 0 && !x) || (dim != 2 && dim != 3)) return -1;
    if (n > 0x7fffffffLL) return -1;
    std::vector<unsigned char> buf;
    buf.reserve(64 + size_t(n) * 16);
    put_be32(buf, ((uint32_t)'B' << 24) | ((uint32_t)'g' << 16) | ((uint32_t)'e' << 8) | (uint32_t)'o');
    buf.push_back((unsigned char)'V');
    put_be32(buf, 5u);
    put_be32(buf, (uint32_t)n);
    for (int i = 0; i < 7; ++i) put_be32(buf, 0u);
    for (int64_t i = 0; i < n; ++i) {
        put_bef(buf, x[i * dim + 0]);
        put_bef(buf, x[i * dim + 1]);
        put_bef(buf, dim == 3 ? x[i * dim + 2] : 0.f);
        put_bef(buf, 1.f);
    }
    buf.push_back(0x00);
    buf.push_back(0xff);
    FILE* f = std::fopen(path, "wb");
    if (!f) return -1;
    size_t w = std::fwrite(buf.data(), 1, buf.size(), f);
    int rc = std::fclose(f);
    return (w == buf.size() && rc == 0) ? 0 : -1;
}

}  // namespace mpm
