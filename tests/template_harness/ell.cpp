// Checks the sliced-ELL in-edge lists of a layer template against its edge
// list: every template edge sits exactly once in its target node's list of
// the right part (interlayer when its target is in the next layer), with its
// source node; every node's entries form a prefix of its slots, in ascending
// edge id (the relaxation's tie order); padding slots hold -1 in both arrays;
// the closing layer's source list follows the reference's dummy-edge rule.
// Usage: ell EX.bin EY.bin nVX conj prune
#include "graph_template.hpp"

#include <cstdio>
#include <cstdlib>
#include <vector>

namespace pgc {
void* host_buffer_alloc(size_t b) { return b ? std::malloc(b) : nullptr; }
void host_buffer_free(void* p) { std::free(p); }
}  // namespace pgc

using namespace pgc;

static std::vector<int> read_ints(const char* path) {
    std::vector<int> v;
    FILE* f = std::fopen(path, "rb");
    if (!f) return v;
    int x;
    while (std::fread(&x, 4, 1, f) == 1) v.push_back(x);
    std::fclose(f);
    return v;
}

int main(int argc, char** argv) {
    if (argc != 6) return 2;
    const std::vector<int> ex = read_ints(argv[1]), ey = read_ints(argv[2]);
    LayerTemplate T;
    const std::string err = build_template(ex.data(), (int64_t)ex.size() / 2, ey.data(), (int64_t)ey.size() / 2,
                                           std::atoll(argv[3]), std::atoi(argv[4]) != 0, std::atoi(argv[5]) != 0, T);
    if (!err.empty()) {
        std::printf("error %s\n", err.c_str());
        return 1;
    }
    long long bad = 0;
    auto fail = [&](const char* what, long long a, long long b) {
        if (++bad <= 10) std::printf("%s (%lld, %lld)\n", what, a, b);
    };
    std::vector<int> seen((size_t)T.eBlock, 0);
    for (int p = 0; p < 2; ++p) {
        if ((long long)T.sp[p].size() != T.nslices + 1 || T.entries[p] != 32LL * T.sp[p][(size_t)T.nslices])
            fail("slot offsets", p, T.entries[p]);
        for (int s = 0; s < T.nslices; ++s)
            for (int lane = 0; lane < 32; ++lane) {
                const long long v = 32LL * s + lane;
                int last = -1;
                bool padding = false;
                for (int j = T.sp[p][(size_t)s]; j < T.sp[p][(size_t)s + 1]; ++j) {
                    const size_t at = (size_t)j * 32 + lane;
                    const int t = T.tedge[p][at], sv = T.src[p][at];
                    if (t < 0) {
                        if (sv != -1) fail("padding with a source", v, sv);
                        padding = true;
                        continue;
                    }
                    if (padding) fail("entry after padding", v, t);
                    if (v >= T.n) fail("entry of a node past the layer", v, t);
                    if (t >= T.eBlock) fail("edge id out of range", v, t);
                    if (t <= last) fail("entries not in ascending edge id", v, t);
                    last = t;
                    ++seen[(size_t)t];
                    if (T.eTrgt[(size_t)t] != v) fail("entry in the wrong node's list", v, t);
                    if (sv != T.eSrc[(size_t)t]) fail("wrong source", v, t);
                    if ((T.eNext[(size_t)t] != 0) != (p == INTER)) fail("wrong part", v, t);
                    if (T.ePos[(size_t)t] != ((int)at | (p << 30))) fail("position not recorded", v, t);
                }
            }
    }
    for (long long t = 0; t < T.eBlock; ++t)
        if (seen[(size_t)t] != 1) fail("edge listed a number of times other than once", t, seen[(size_t)t]);
    // The closing layer's sources: an interlayer edge of block nY-1 reaches
    // the closing layer only when its global source id (nY-1)*n + src is
    // strictly greater than n (cost_time_ratio_solver.cpp:56).  The list is
    // stored only where that drops something, i.e. with two layers.
    if (T.nY == 2) {
        if (T.srcDummy.size() != T.src[INTER].size()) fail("closing-layer list size", (long long)T.srcDummy.size(), 0);
        else
            for (size_t at = 0; at < T.srcDummy.size(); ++at) {
                const int sv = T.src[INTER][at];
                const int want = sv >= 0 && (long long)(T.nY - 1) * T.n + sv > T.n ? sv : -1;
                if (T.srcDummy[at] != want) fail("closing-layer source", (long long)at, T.srcDummy[at]);
            }
    } else if (!T.srcDummy.empty()) {
        fail("closing-layer list stored although nothing is dropped", T.nY, (long long)T.srcDummy.size());
    }
    std::printf("%lld problems (%lld template edges, %d slices)\n", bad, (long long)T.eBlock, T.nslices);
    return bad ? 1 : 0;
}
