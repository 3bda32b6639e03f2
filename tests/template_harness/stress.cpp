// Builds one layer template many times from several threads at once and
// compares every build with the first: the builder's worker pool serves one
// job at a time (other callers run their loops inline), and its part claims
// carry the job's generation.  Usage: stress EX.bin nVX conj prune nY threads repeats
#include "graph_template.hpp"

#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

namespace pgc {
void* host_buffer_alloc(size_t b) { return b ? std::malloc(b) : nullptr; }
void host_buffer_free(void* p) { std::free(p); }
}  // namespace pgc

using namespace pgc;

template <class V>
static bool same(const V& a, const V& b) {
    return a.size() == b.size() && (a.empty() || std::memcmp(a.data(), b.data(), a.size() * sizeof(a[0])) == 0);
}

static bool equal(const LayerTemplate& a, const LayerTemplate& b) {
    bool ok = a.n == b.n && a.nslices == b.nslices && a.eBlock == b.eBlock && a.entries[0] == b.entries[0] &&
              a.entries[1] == b.entries[1];
    for (int p = 0; p < 2; ++p) ok = ok && same(a.sp[p], b.sp[p]) && same(a.src[p], b.src[p]) && same(a.tedge[p], b.tedge[p]);
    return ok && same(a.srcDummy, b.srcDummy) && same(a.eSrc, b.eSrc) && same(a.eTrgt, b.eTrgt) &&
           same(a.eNext, b.eNext) && same(a.eX, b.eX) && same(a.eY, b.eY) && same(a.ePos, b.ePos);
}

int main(int argc, char** argv) {
    if (argc != 8) return 2;
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    std::vector<int> ex;
    int v;
    while (std::fread(&v, 4, 1, f) == 1) ex.push_back(v);
    std::fclose(f);
    const long long nvx = std::atoll(argv[2]);
    const bool conj = std::atoi(argv[3]) != 0, prune = std::atoi(argv[4]) != 0;
    const int ny = std::atoi(argv[5]), threads = std::atoi(argv[6]), repeats = std::atoi(argv[7]);
    std::vector<int> ey;
    for (int i = 0; i < ny; ++i) {
        ey.push_back(i);
        ey.push_back((i + 1) % ny);
    }
    LayerTemplate ref;
    const std::string err = build_template(ex.data(), (int64_t)ex.size() / 2, ey.data(), ny, nvx, conj, prune, ref);
    if (!err.empty()) {
        std::printf("error %s\n", err.c_str());
        return 1;
    }
    std::atomic<int> bad{0};
    std::vector<std::thread> th;
    for (int t = 0; t < threads; ++t)
        th.emplace_back([&] {
            for (int r = 0; r < repeats; ++r) {
                LayerTemplate T;
                build_template(ex.data(), (int64_t)ex.size() / 2, ey.data(), ny, nvx, conj, prune, T);
                if (!equal(T, ref)) ++bad;
            }
        });
    for (auto& t : th) t.join();
    std::printf("%d of %d builds differ (n %d, eBlock %lld)\n", bad.load(), threads * repeats, ref.n,
                (long long)ref.eBlock);
    return bad.load() ? 1 : 0;
}
