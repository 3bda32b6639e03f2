// Checks the Bellman-Ford team's CTA slice ranges (plan_cta_cuts) against an
// exact search under the same cost model.  A range of slices costs, per part,
// the largest sum any warp gets when the range's slices with rows in that
// part are dealt to the warps round-robin; a slice with r rows costs
// 32 * (ceil(r / rowsPerBatch) + 1), and intralayer rows count only when the
// template has intralayer entries and K > 1.  The objective of a partition
// into at most `blocks` contiguous ranges is
//     max interlayer cost + (K - 1) * max intralayer cost.
// The exact search takes every intralayer cost a range can have as the
// bound, finds by dynamic programming the partition whose ranges all stay
// within it with the smallest interlayer maximum, and keeps the best sum.
// For the planned ranges and for equal slice counts it also checks the
// team's wait lists (cta_wait_lists) against the ones that follow from the
// template's edge list: every template edge joins the CTA that owns its
// target's slice and the one that owns its source's slice, both ways.
// Usage: cuts EX.bin nVX conj prune nY
#include "graph_template.hpp"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <vector>

namespace pgc {
void* host_buffer_alloc(size_t b) { return b ? std::malloc(b) : nullptr; }
void host_buffer_free(void* p) { std::free(p); }
}  // namespace pgc

using namespace pgc;
typedef long long ll;

namespace {

// rows a warp gathers per batch for nk depths (the kernel's batching rule)
int rows_per_batch(int nk) {
    const int g = 20 / nk;
    return g < 1 ? 1 : g > 8 ? 8 : g;
}

struct Model {
    int ns = 0;
    bool intra = false;
    ll reps = 0;
    std::vector<ll> c[2];  // c[p][a * (ns + 1) + b]: cost of range [a, b) in part p

    Model(const LayerTemplate& T, int K, int warps, const int rb[2]) : ns(T.nslices) {
        intra = T.entries[INTRA] > 0 && K > 1;
        reps = intra ? K - 1 : 0;
        for (int p = 0; p < 2; ++p) {
            c[p].assign((size_t)(ns + 1) * (ns + 1), 0);
            for (int a = 0; a < ns; ++a) {
                std::vector<ll> acc((size_t)warps, 0);
                int next = 0;
                ll mx = 0;
                for (int b = a + 1; b <= ns; ++b) {
                    const int rows = T.sp[p][(size_t)b] - T.sp[p][(size_t)b - 1];
                    if (rows > 0 && (p == 0 || intra)) {
                        acc[(size_t)next] += 32LL * ((rows + rb[p] - 1) / rb[p] + 1);
                        mx = std::max(mx, acc[(size_t)next]);
                        next = (next + 1) % warps;
                    }
                    c[p][(size_t)a * (ns + 1) + b] = mx;
                }
            }
        }
    }
    ll cost(int p, int a, int b) const { return a >= b ? 0 : c[p][(size_t)a * (ns + 1) + b]; }

    // objective of the ranges [cut[i], cut[i+1])
    ll objective(const std::vector<int>& cut) const {
        ll mi = 0, mj = 0;
        for (size_t i = 0; i + 1 < cut.size(); ++i) {
            mi = std::max(mi, cost(0, cut[i], cut[i + 1]));
            mj = std::max(mj, cost(1, cut[i], cut[i + 1]));
        }
        return mi + reps * mj;
    }

    // smallest objective over all partitions into at most `blocks` ranges
    ll best(int blocks) const {
        std::vector<ll> bounds{0};
        for (int a = 0; a < ns; ++a)
            for (int b = a + 1; b <= ns; ++b) bounds.push_back(cost(1, a, b));
        std::sort(bounds.begin(), bounds.end());
        bounds.erase(std::unique(bounds.begin(), bounds.end()), bounds.end());
        const ll inf = (ll)1 << 60;
        ll bestObj = inf;
        std::vector<ll> g((size_t)ns + 1), h((size_t)ns + 1);
        for (ll bj : bounds) {
            if (reps * bj >= bestObj) break;
            // g[b]: smallest interlayer maximum covering [0, b) with the ranges so far
            std::fill(g.begin(), g.end(), inf);
            g[0] = 0;
            for (int k = 0; k < blocks; ++k) {
                h = g;  // an empty range changes nothing
                for (int b = 1; b <= ns; ++b)
                    for (int a = 0; a < b; ++a)
                        if (g[(size_t)a] < inf && cost(1, a, b) <= bj)
                            h[(size_t)b] = std::min(h[(size_t)b], std::max(g[(size_t)a], cost(0, a, b)));
                g.swap(h);
            }
            if (g[(size_t)ns] < inf) bestObj = std::min(bestObj, g[(size_t)ns] + reps * bj);
        }
        return bestObj;
    }
};

// wait lists that follow from the template's edges (CSR, ascending)
void edge_wait_lists(const LayerTemplate& T, const std::vector<int>& cut, std::vector<int>& ptr,
                     std::vector<int>& idx) {
    const int blocks = (int)cut.size() - 1;
    std::vector<int> owner((size_t)T.nslices);
    for (int c = 0; c < blocks; ++c)
        for (int s = cut[(size_t)c]; s < cut[(size_t)c + 1]; ++s) owner[(size_t)s] = c;
    std::vector<char> adj((size_t)blocks * blocks, 0);
    for (int64_t t = 0; t < T.eBlock; ++t) {
        const int a = owner[(size_t)(T.eSrc[(size_t)t] >> 5)], b = owner[(size_t)(T.eTrgt[(size_t)t] >> 5)];
        if (a != b) adj[(size_t)a * blocks + b] = adj[(size_t)b * blocks + a] = 1;
    }
    ptr.assign((size_t)blocks + 1, 0);
    idx.clear();
    for (int c = 0; c < blocks; ++c) {
        for (int d = 0; d < blocks; ++d)
            if (adj[(size_t)c * blocks + d]) idx.push_back(d);
        ptr[(size_t)c + 1] = (int)idx.size();
    }
}

bool same_wait_lists(const LayerTemplate& T, const std::vector<int>& cut) {
    std::vector<int> p0, i0, p1, i1;
    cta_wait_lists(T, cut, p0, i0);
    edge_wait_lists(T, cut, p1, i1);
    return p0 == p1 && i0 == i1;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 6) return 2;
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    std::vector<int> ex;
    int v;
    while (std::fread(&v, 4, 1, f) == 1) ex.push_back(v);
    std::fclose(f);
    const long long nvx = std::atoll(argv[2]);
    const bool conj = std::atoi(argv[3]) != 0, prune = std::atoi(argv[4]) != 0;
    const int ny = std::atoi(argv[5]);
    std::vector<int> ey;
    for (int i = 0; i < ny; ++i) {
        ey.push_back(i);
        ey.push_back((i + 1) % ny);
    }
    LayerTemplate T;
    const std::string err = build_template(ex.data(), (int64_t)ex.size() / 2, ey.data(), ny, nvx, conj, prune, T);
    if (!err.empty()) {
        std::printf("error %s\n", err.c_str());
        return 1;
    }
    int cases = 0, bad = 0, badWait = 0;
    for (int K = 1; K <= 6; ++K)
        for (int warps : {1, 2, 3, 20})
            for (int blocks : {1, 2, 3, 5, 8, 13}) {
                const int rb[2] = {K <= 4 ? rows_per_batch(K) : 1, rows_per_batch(1)};
                const std::vector<int> cut = plan_cta_cuts(T, blocks, K, warps, rb);
                const Model m(T, K, warps, rb);
                bool ok = (int)cut.size() == blocks + 1 && cut[0] == 0 && cut[(size_t)blocks] == T.nslices;
                for (int i = 0; ok && i < blocks; ++i) ok = cut[(size_t)i] <= cut[(size_t)i + 1];
                const ll got = ok ? m.objective(cut) : -1, want = m.best(blocks);
                ++cases;
                if (ok && !same_wait_lists(T, cut)) {
                    ++badWait;
                    if (badWait <= 10) std::printf("K=%d warps=%d blocks=%d: wait lists differ\n", K, warps, blocks);
                }
                if (!ok || got != want) {
                    ++bad;
                    if (bad <= 10)
                        std::printf("K=%d warps=%d blocks=%d: planned %lld, best %lld%s\n", K, warps, blocks, got,
                                    want, ok ? "" : " (malformed cuts)");
                }
            }
    // equal slice counts, as many CTAs as slices at most
    for (int blocks : {2, 7, 64, 148}) {
        std::vector<int> cut((size_t)blocks + 1);
        for (int c = 0; c <= blocks; ++c) cut[(size_t)c] = (int)((long long)T.nslices * c / blocks);
        ++cases;
        if (!same_wait_lists(T, cut)) {
            ++badWait;
            std::printf("equal cuts, blocks=%d: wait lists differ\n", blocks);
        }
    }
    std::printf("%d of %d plans differ from the best, %d wait lists differ (slices %d, intralayer entries %lld)\n",
                bad, cases - 4, badWait, T.nslices, (long long)T.entries[INTRA]);
    return bad || badWait ? 1 : 0;
}
