// export.cuh -- .bgeo frame export (GLFWApp::ExportBgeoFile, GLFWApp.cpp:287-405).
//
// The reference writes one Houdini .bgeo (classic "Bgeo" V5 layout, through Partio) per set
// and frame: point attributes position, Cd (3 floats), pscale (1 float) and label (1 int),
// the colour and radius of the set, label 0 for water and 1 for snow.  It fills the int
// label through a float pointer, so the stored int is the bit pattern of 0.0f or 1.0f;
// `float_label` keeps that (the file then matches the reference's byte for byte), 0 writes
// the plain integer.
//
// Layout written here (every number big-endian): int magic 'B''g''e''o', char 'V',
// int version 5, ints nPoints, nPrims 0, nPointGroups 0, nPrimGroups 0, nPointAttrib 3,
// nVertexAttrib 0, nPrimAttrib 0, nAttrib 0; per attribute after position: short name
// length, name, unsigned short count, int type (0 float, 1 int), count zero ints
// (defaults); per point 9 words: x, y, z, w = 1, Cd r g b, pscale, label; then bytes 0x00,
// 0xff.
#pragma once
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace snowb {

static inline void be32(std::vector<unsigned char>& b, uint32_t v)
{
    b.push_back((unsigned char)(v >> 24)); b.push_back((unsigned char)(v >> 16));
    b.push_back((unsigned char)(v >> 8)); b.push_back((unsigned char)v);
}
static inline void be16(std::vector<unsigned char>& b, uint16_t v)
{
    b.push_back((unsigned char)(v >> 8)); b.push_back((unsigned char)v);
}
static inline uint32_t fbits(float f)
{
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}
static void bgeo_attr(std::vector<unsigned char>& b, const char* name, uint16_t count, uint32_t type)
{
    const size_t n = std::strlen(name);
    be16(b, (uint16_t)n);
    b.insert(b.end(), name, name + n);
    be16(b, count);
    be32(b, type);
    for (uint16_t k = 0; k < count; ++k) be32(b, 0u);
}
// Serialise n points (positions as 3 floats each, host memory) and write them to path.
static int bgeo_write(const char* path, const float* pos, uint32_t n, const float rgb[3], float pscale, int label,
                      int float_label, std::string& err)
{
    std::vector<unsigned char> b;
    b.reserve(64 + (size_t)n * 36);
    be32(b, ((((uint32_t)'B' << 8 | 'g') << 8 | 'e') << 8) | 'o');
    b.push_back('V');
    be32(b, 5u);
    const uint32_t head[8] = {n, 0u, 0u, 0u, 3u, 0u, 0u, 0u};
    for (uint32_t v : head) be32(b, v);
    bgeo_attr(b, "Cd", 3, 0u);
    bgeo_attr(b, "pscale", 1, 0u);
    bgeo_attr(b, "label", 1, 1u);
    const uint32_t lab = float_label ? fbits((float)label) : (uint32_t)label;
    for (uint32_t i = 0; i < n; ++i) {
        be32(b, fbits(pos[3ull * i])); be32(b, fbits(pos[3ull * i + 1])); be32(b, fbits(pos[3ull * i + 2]));
        be32(b, fbits(1.f));
        be32(b, fbits(rgb[0])); be32(b, fbits(rgb[1])); be32(b, fbits(rgb[2]));
        be32(b, fbits(pscale));
        be32(b, lab);
    }
    b.push_back(0x00);
    b.push_back(0xff);
    FILE* f = std::fopen(path, "wb");
    if (!f) { err = std::string("cannot open ") + path; return -1; }
    const size_t w = std::fwrite(b.data(), 1, b.size(), f);
    const int c = std::fclose(f);
    if (w != b.size() || c != 0) { err = std::string("short write to ") + path; return -1; }
    return 0;
}

// asynchronous exports: positions are copied into pinned staging on the library's stream,
// and a host thread waits for that copy and writes the file
struct ExportJob {
    std::thread th;
    float* staging = nullptr;
    cudaEvent_t ev = nullptr;
    int rc = 0;
    std::string err;
};
static std::vector<ExportJob*> g_exports;

}  // namespace snowb
