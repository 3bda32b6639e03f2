// Differential check of the branch-and-bound heap (branch_heap.hpp) against
// the oracle's restatement of the reference heap (helper/minheap.cpp:16-277),
// whose slot bookkeeping differs but whose tie rules decide the same pop
// order.  Random operation sequences over few distinct values (so that most
// comparisons are ties) and a small key range (so that pushes of present
// keys and out-of-range keys happen): every result of push / decrease / pop /
// peak / peakKey / getSize / isEmpty must agree.
// Usage: heap seed operations capacity
#include "branch_heap.hpp"
#include "pgc_oracle.cpp"

#include <cstdio>
#include <cstdlib>
#include <random>

int main(int argc, char** argv) {
    if (argc != 4) return 2;
    const unsigned seed = (unsigned)std::atoi(argv[1]);
    const long ops = std::atol(argv[2]), cap = std::atol(argv[3]);
    std::mt19937_64 rng(seed);
    pgc::BranchHeap a(cap);
    orc::MinHeap b(cap);
    long bad = 0, pops = 0, at = 0;
    auto report = [&](const char* what, long i) {
        if (++bad <= 10) std::printf("op %ld: %s differs\n", i, what);
    };
    for (long i = 0; i < ops; ++i) {
        const int kind = (int)(rng() % 10);
        const long key = (long)(rng() % (unsigned long)(cap + 2)) - 1;  // -1 .. cap
        const double value = (double)(rng() % 4) * 0.5;
        if (kind < 4) {
            a.push(value, key);
            b.push(value, key);
        } else if (kind < 6) {
            const double lower = value - 0.5 * (double)(rng() % 3);
            if (a.decrease(key, lower) != b.decrease(key, lower)) report("decrease", i);
        } else if (kind < 9) {
            const auto x = a.pop(), y = b.pop();
            ++pops;
            if (x != y) report("pop", i);
        } else {
            if (a.peak() != b.peak()) report("peak", i);
            if (a.peakKey(key) != b.peakKey(key)) report("peakKey", i);
        }
        if (a.getSize() != b.getSize() || a.isEmpty() != b.isEmpty()) report("size", i);
        at = i;
    }
    // drain
    while (!a.isEmpty() || !b.isEmpty()) {
        const auto x = a.pop(), y = b.pop();
        ++pops;
        if (x != y) {
            report("pop (drain)", at);
            break;
        }
    }
    std::printf("%ld of %ld operations differ (%ld pops)\n", bad, ops, pops);
    return bad ? 1 : 0;
}
