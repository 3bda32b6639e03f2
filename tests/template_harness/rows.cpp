// Writes the product space that the host layer template defines: every row
// (product_row, in edge-id order) and the global source and target node of
// every edge, as little-endian int32 arrays one after the other.
// Usage: rows EX.bin EY.bin nVX conj prune out.bin
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
    if (argc != 7) return 2;
    const std::vector<int> ex = read_ints(argv[1]), ey = read_ints(argv[2]);
    const long long nvx = std::atoll(argv[3]);
    const bool conj = std::atoi(argv[4]) != 0, prune = std::atoi(argv[5]) != 0;
    LayerTemplate T;
    const std::string err =
        build_template(ex.data(), (int64_t)ex.size() / 2, ey.data(), (int64_t)ey.size() / 2, nvx, conj, prune, T);
    if (!err.empty()) {
        std::printf("error %s\n", err.c_str());
        return 1;
    }
    const long long edges = (long long)T.nY * T.eBlock;
    const int cols = T.cols();
    std::vector<int> rows((size_t)(edges * cols)), src((size_t)edges), trgt((size_t)edges);
    for (long long e = 0; e < edges; ++e) {
        product_row(T, ey.data(), e, &rows[(size_t)(e * cols)]);
        const long long block = e / T.eBlock, t = e - block * T.eBlock;
        src[(size_t)e] = (int)(block * T.n + T.eSrc[(size_t)t]);
        trgt[(size_t)e] = (int)(((block + T.eNext[(size_t)t]) % T.nY) * T.n + T.eTrgt[(size_t)t]);
    }
    FILE* f = std::fopen(argv[6], "wb");
    if (!f) return 2;
    std::fwrite(rows.data(), 4, rows.size(), f);
    std::fwrite(src.data(), 4, src.size(), f);
    std::fwrite(trgt.data(), 4, trgt.size(), f);
    std::fclose(f);
    std::printf("%lld edges, %d columns\n", edges, cols);
    return 0;
}
