// f16_check.cpp -- host check of the half-precision node encoding
// (HNode4, EncodeHalfNodes in bvh_build.cpp).
//
//   f16_check halves out.bin           every binary16 pattern's value (65536 float32)
//   f16_check round in.bin out.bin     each float32 of in.bin rounded down and up to
//                                      binary16 (2 uint16 per input)
//   f16_check nodes tri.bin            the reference BVH over the triangles (n x 9
//                                      float32), encoded: every decoded child box
//                                      contains its FP32 box, links equal the FP32
//                                      layout's; prints "ok <nodes>"
// Exit status 0 on success.
#include <cstdio>
#include <cstring>
#include <vector>

#include "bvh_build.h"

using namespace rtb200;

static std::vector<float> ReadAll(const char* path)
{
    std::vector<float> v;
    FILE* f = std::fopen(path, "rb");
    if (!f) return v;
    std::fseek(f, 0, SEEK_END);
    const long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    v.resize((size_t)n / 4);
    if (std::fread(v.data(), 4, v.size(), f) != v.size()) v.clear();
    std::fclose(f);
    return v;
}

static bool WriteAll(const char* path, const void* p, size_t bytes)
{
    FILE* f = std::fopen(path, "wb");
    if (!f) return false;
    const bool ok = std::fwrite(p, 1, bytes, f) == bytes;
    std::fclose(f);
    return ok;
}

int main(int argc, char** argv)
{
    if (argc == 3 && !std::strcmp(argv[1], "halves")) {
        std::vector<float> v(65536);
        for (int h = 0; h < 65536; ++h) v[h] = HalfToFloat((uint16_t)h);
        return WriteAll(argv[2], v.data(), v.size() * 4) ? 0 : 1;
    }
    if (argc == 4 && !std::strcmp(argv[1], "round")) {
        const std::vector<float> x = ReadAll(argv[2]);
        std::vector<uint16_t> out(2 * x.size());
        for (size_t i = 0; i < x.size(); ++i) {
            out[2 * i] = FloatToHalfDirected(x[i], -1);
            out[2 * i + 1] = FloatToHalfDirected(x[i], +1);
        }
        return WriteAll(argv[3], out.data(), out.size() * 2) ? 0 : 1;
    }
    if (argc == 3 && !std::strcmp(argv[1], "nodes")) {
        const std::vector<float> tri = ReadAll(argv[2]);
        const int64_t n = (int64_t)(tri.size() / 9);
        BuiltBVH b;
        BuildReferenceBVH(tri.data(), n, 4, b);
        std::vector<HNode4> h;
        std::vector<GpuNode4> f;
        EncodeHalfNodes(b, h);
        EncodeGpuNodes(b, f);
        if (h.size() != f.size()) { std::printf("FAIL node count\n"); return 1; }
        for (size_t i = 0; i < h.size(); ++i)
            for (int c = 0; c < 4; ++c) {
                if (h[i].child[c] != f[i].child[c]) { std::printf("FAIL link %zu %d\n", i, c); return 1; }
                if (f[i].count[c] < 0) {
                    if (!(HalfToFloat(h[i].lox[c]) > HalfToFloat(h[i].hix[c]))) {
                        std::printf("FAIL empty slot %zu %d\n", i, c);
                        return 1;
                    }
                    continue;
                }
                const float lo[3] = {f[i].lox[c], f[i].loy[c], f[i].loz[c]};
                const float hi[3] = {f[i].hix[c], f[i].hiy[c], f[i].hiz[c]};
                const uint16_t hl[3] = {h[i].lox[c], h[i].loy[c], h[i].loz[c]};
                const uint16_t hh[3] = {h[i].hix[c], h[i].hiy[c], h[i].hiz[c]};
                for (int k = 0; k < 3; ++k)
                    if (!(HalfToFloat(hl[k]) <= lo[k] && HalfToFloat(hh[k]) >= hi[k])) {
                        std::printf("FAIL containment %zu %d %d\n", i, c, k);
                        return 1;
                    }
            }
        std::printf("ok %zu\n", h.size());
        return 0;
    }
    std::fprintf(stderr, "usage: f16_check halves|round|nodes ...\n");
    return 2;
}
