// graph_template.cpp -- builds the layer-invariant in-edge template.
//
// Edge generation order restates product_space.cpp:19-132 (plain graph) and
// conj_product_space.cpp:70-228 (conjugate graph); it has to be identical
// because edge ids, in-edge order (the tie-break order of the relaxation) and
// the rows of the returned matching all follow from it.  Outgoing-edge sets
// of a vertex are taken in ascending edge id (the reference iterates a
// robin_set, whose order is a hash order).
#include "graph_template.hpp"

#include <algorithm>
#include <climits>
#include <atomic>
#include <condition_variable>
#include <mutex>
#include <thread>

namespace pgc {

namespace {

// A pool of host threads that lives for the process: creating and joining
// a thread per part cost about 50 us each, most of a template build's time
// on a 16-core host.  One job runs at a time; a caller that finds the pool
// busy (templates of a batch built by concurrent workers) runs its loop
// itself.
class WorkerPool {
  public:
    static WorkerPool& get() {
        static WorkerPool pool;
        return pool;
    }
    int size() const { return (int)threads_.size() + 1; }
    // Runs f(i) for every i in [0, parts) on the pool and the caller;
    // returns false, having run nothing, when another job holds the pool.
    template <class F>
    bool run(int parts, F& f) {
        std::unique_lock<std::mutex> own(busy_, std::try_to_lock);
        if (!own.owns_lock()) return false;
        Job job;
        {
            std::lock_guard<std::mutex> lk(m_);
            job.call = [](void* ctx, int i) { (*static_cast<F*>(ctx))(i); };
            job.ctx = &f;
            job.parts = parts;
            job.gen = ++gen_;
            job_ = job;
            remaining_ = parts;
            // parts are claimed from (generation, next index): a thread still
            // holding an older job's snapshot can claim nothing of this one
            next_.store((uint64_t)job.gen << 32);
        }
        cv_.notify_all();
        work(job);
        std::unique_lock<std::mutex> lk(m_);
        done_.wait(lk, [&] { return remaining_ == 0; });
        return true;
    }

  private:
    struct Job {
        void (*call)(void*, int) = nullptr;
        void* ctx = nullptr;
        int parts = 0;
        uint32_t gen = 0;
    };
    WorkerPool() {
        const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
        for (int i = 1; i < std::min(hw, 16); ++i) threads_.emplace_back([this] { loop(); });
    }
    ~WorkerPool() {
        {
            std::lock_guard<std::mutex> lk(m_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : threads_) t.join();
    }
    void work(const Job& job) {
        int done = 0;
        uint64_t v = next_.load();
        for (;;) {
            if ((uint32_t)(v >> 32) != job.gen) break;
            const int i = (int)(uint32_t)v;
            if (i >= job.parts) break;
            if (!next_.compare_exchange_weak(v, v + 1)) continue;
            job.call(job.ctx, i);
            ++done;
            v = next_.load();
        }
        if (done) {
            std::lock_guard<std::mutex> lk(m_);
            remaining_ -= done;
            if (remaining_ == 0) done_.notify_all();
        }
    }
    void loop() {
        uint32_t seen = 0;
        for (;;) {
            Job job;
            {
                std::unique_lock<std::mutex> lk(m_);
                cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
                job = job_;
            }
            work(job);
        }
    }
    std::vector<std::thread> threads_;
    std::mutex busy_, m_;
    std::condition_variable cv_, done_;
    Job job_;
    int remaining_ = 0;
    std::atomic<uint64_t> next_{0};
    uint32_t gen_ = 0;
    bool stop_ = false;
};

// Runs f(begin, end) over [0, n) split across the host's cores, in parts of
// at least `grain` items.
template <class F>
void parallel_for(int64_t n, F f, int64_t grain = 2048) {
    WorkerPool& pool = WorkerPool::get();
    const int64_t parts = std::max<int64_t>(1, std::min<int64_t>(pool.size(), n / grain));
    if (parts <= 1) {
        f((int64_t)0, n);
        return;
    }
    auto part = [&](int i) { f(n * i / parts, n * (i + 1) / parts); };
    if (!pool.run((int)parts, part)) f((int64_t)0, n);
}

struct EdgeOut {
    int src, trgt;
    int8_t next;
    int x0, x1, x2;
    int8_t y;
};

// Writes template edges from position `at` on; the arrays are sized once
// for the known count.
struct Emitter {
    LayerTemplate& T;
    size_t at = 0;
    Emitter(LayerTemplate& t, size_t count) : T(t) {
        T.eSrc.resize(count);
        T.eTrgt.resize(count);
        T.eNext.resize(count);
        T.eX.resize(3 * count);
        T.eY.resize(count);
    }
    Emitter(LayerTemplate& t, size_t count, size_t from) : T(t), at(from) { (void)count; }
    void operator()(const EdgeOut& e) {
        T.eSrc[at] = e.src;
        T.eTrgt[at] = e.trgt;
        T.eNext[at] = e.next;
        T.eX[3 * at] = e.x0;
        T.eX[3 * at + 1] = e.x1;
        T.eX[3 * at + 2] = e.x2;
        T.eY[at] = e.y;
        ++at;
    }
};

void build_plain(const int* EX, int64_t nEX, LayerTemplate& T) {
    Emitter emit(T, (size_t)(nEX * (T.prune ? 1 : 2) + T.nvx));
    for (int64_t j = 0; j < nEX; ++j) {
        const int a = EX[2 * j], b = EX[2 * j + 1];
        if (!T.prune) emit({a, b, 0, a, b, 0, Y_SS});
        emit({a, b, 1, a, b, 0, Y_SM});
    }
    for (int x = 0; x < T.nvx; ++x) emit({x, x, 1, x, x, 0, Y_SM});
}

void build_conj(const int* EX, int64_t nEX, LayerTemplate& T) {
    // outgoing edges of every vertex in ascending edge id (CSR)
    std::vector<int> outPtr((size_t)T.nvx + 1, 0), out((size_t)nEX);
    for (int64_t e = 0; e < nEX; ++e) ++outPtr[(size_t)EX[2 * e] + 1];
    for (int v = 0; v < T.nvx; ++v) outPtr[(size_t)v + 1] += outPtr[(size_t)v];
    {
        std::vector<int> fill(outPtr.begin(), outPtr.end() - 1);
        for (int64_t e = 0; e < nEX; ++e) out[(size_t)fill[(size_t)EX[2 * e]]++] = (int)e;
    }
    // turns (j, it): edge it leaves the head of edge j and does not return to
    // its tail.  Every edge j emits a fixed number of template edges per
    // turn, so the offsets of all j are known up front and ranges of j are
    // written in parallel.
    std::vector<int64_t> turns((size_t)nEX + 1, 0);
    parallel_for(nEX, [&](int64_t j0, int64_t j1) {
        for (int64_t j = j0; j < j1; ++j) {
            const int s3 = EX[2 * j], m3 = EX[2 * j + 1];
            int c = 0;
            for (int q = outPtr[(size_t)m3]; q < outPtr[(size_t)m3 + 1]; ++q)
                if (EX[2 * out[(size_t)q] + 1] != s3) ++c;
            turns[(size_t)j + 1] = c;
        }
    });
    for (int64_t j = 0; j < nEX; ++j) turns[(size_t)j + 1] += turns[(size_t)j];
    const int64_t allTurns = turns[(size_t)nEX];
    const int perA = T.prune ? 0 : 2, perB = T.prune ? 2 : 3;
    const size_t count = (size_t)((perA + perB) * allTurns + 2 * nEX);
    Emitter sized(T, count);
    const int off2d = (int)nEX;
    const int off3d = T.prune ? off2d : 2 * (int)nEX;
    const size_t baseB = (size_t)(perA * allTurns);
    parallel_for(nEX, [&](int64_t j0, int64_t j1) {
        Emitter emitA(T, count, (size_t)(perA * turns[(size_t)j0]));
        Emitter emitB(T, count, baseB + (size_t)(perB * turns[(size_t)j0] + 2 * j0));
        for (int j = (int)j0; j < (int)j1; ++j) {
            const int s3 = EX[2 * j], m3 = EX[2 * j + 1];
            for (int q = outPtr[(size_t)m3]; q < outPtr[(size_t)m3 + 1]; ++q) {
                const int it = out[(size_t)q];
                const int t3 = EX[2 * it + 1];
                if (t3 == s3) continue;
                if (!T.prune) {
                    emitA({off2d + j, off2d + it, 0, s3, m3, t3, Y_SSS});
                    emitA({off2d + j, it, 0, s3, m3, t3, Y_SSM});
                }
                emitB({j, it, 1, s3, m3, t3, Y_SMT});
                if (!T.prune) emitB({j, off2d + it, 1, s3, m3, t3, Y_SMM});
                emitB({off3d + j, it, 1, m3, m3, t3, Y_SMT});
            }
            emitB({j, off3d + j, 1, s3, m3, m3, Y_SMT});
            emitB({off3d + j, off3d + j, 1, m3, m3, m3, Y_SMT});
        }
    });
}

void build_sell(LayerTemplate& T) {
    T.nslices = (T.n + 31) / 32;
    const int64_t n = T.n, nt = T.eBlock;
    // In-edges of every (part, target) in ascending template edge id: one
    // stable counting sort on the key part * n + target, in parallel.  Chunk
    // c of the edge range counts its keys, the counts give each chunk its
    // start inside every key's list, and each chunk places its edges in
    // order.
    const int64_t nk = 2 * n;
    const int chunks = (int)std::max<int64_t>(1, std::min<int64_t>(WorkerPool::get().size(), nt / 65536));
    auto key = [&](int64_t t) { return (int64_t)(T.eNext[(size_t)t] ? INTER : INTRA) * n + T.eTrgt[(size_t)t]; };
    auto range = [&](int64_t c, int64_t& t0, int64_t& t1) {
        t0 = nt * c / chunks;
        t1 = nt * (c + 1) / chunks;
    };
    std::vector<RawVec<int>> cnt((size_t)chunks);
    parallel_for(chunks, [&](int64_t c0, int64_t c1) {
        for (int64_t c = c0; c < c1; ++c) {
            RawVec<int>& h = cnt[(size_t)c];
            h.assign((size_t)nk, 0);
            int64_t t0, t1;
            range(c, t0, t1);
            for (int64_t t = t0; t < t1; ++t) ++h[(size_t)key(t)];
        }
    }, 1);
    RawVec<int> ptr((size_t)nk + 1);  // start of key k's list
    parallel_for(nk, [&](int64_t k0, int64_t k1) {
        for (int64_t k = k0; k < k1; ++k) {
            int d = 0;
            for (int c = 0; c < chunks; ++c) d += cnt[(size_t)c][(size_t)k];
            ptr[(size_t)k + 1] = d;
        }
    });
    ptr[0] = 0;
    for (int64_t k = 0; k < nk; ++k) ptr[(size_t)k + 1] += ptr[(size_t)k];
    parallel_for(nk, [&](int64_t k0, int64_t k1) {
        for (int64_t k = k0; k < k1; ++k) {
            int at = ptr[(size_t)k];
            for (int c = 0; c < chunks; ++c) {
                const int m = cnt[(size_t)c][(size_t)k];
                cnt[(size_t)c][(size_t)k] = at;
                at += m;
            }
        }
    });
    RawVec<int> list((size_t)nt);
    parallel_for(chunks, [&](int64_t c0, int64_t c1) {
        for (int64_t c = c0; c < c1; ++c) {
            RawVec<int>& at = cnt[(size_t)c];
            int64_t t0, t1;
            range(c, t0, t1);
            for (int64_t t = t0; t < t1; ++t) list[(size_t)at[(size_t)key(t)]++] = (int)t;
        }
    }, 1);
    // slot offsets: a slice is as wide as its largest in-degree
    for (int p = 0; p < 2; ++p) {
        const int* pp = ptr.data() + (size_t)p * n;
        RawVec<int>& sp = T.sp[p];
        sp.resize((size_t)T.nslices + 1);
        sp[0] = 0;
        for (int s = 0; s < T.nslices; ++s) {
            int w = 0;
            for (int i = 0; i < 32; ++i) {
                const int64_t v = 32LL * s + i;
                if (v < n) w = std::max(w, pp[v + 1] - pp[v]);
            }
            sp[(size_t)s + 1] = sp[(size_t)s] + w;
        }
        T.entries[p] = (int64_t)sp.back() * 32;
        T.src[p].resize((size_t)T.entries[p]);
        T.tedge[p].resize((size_t)T.entries[p]);
    }
    T.ePos.resize((size_t)nt);  // every template edge is placed in its part below
    parallel_for(2LL * T.nslices, [&](int64_t q0, int64_t q1) {
        for (int64_t q = q0; q < q1; ++q) {
            const int p = (int)(q / T.nslices);
            const int64_t s = q - (int64_t)p * T.nslices;
            const int* pp = ptr.data() + (size_t)p * n;
            const RawVec<int>& sp = T.sp[p];
            const size_t r0 = (size_t)sp[(size_t)s] * 32, r1 = (size_t)sp[(size_t)s + 1] * 32;
            std::fill(T.src[p].begin() + r0, T.src[p].begin() + r1, -1);
            std::fill(T.tedge[p].begin() + r0, T.tedge[p].begin() + r1, -1);
            for (int i = 0; i < 32; ++i) {
                const int64_t v = 32 * s + i;
                if (v >= n) continue;
                for (int j = 0; j < pp[v + 1] - pp[v]; ++j) {
                    const int t = list[(size_t)(pp[v] + j)];
                    const size_t at = r0 + (size_t)j * 32 + (size_t)i;
                    T.src[p][at] = T.eSrc[(size_t)t];
                    T.tedge[p][at] = t;
                    T.ePos[(size_t)t] = (int)at | (p << 30);
                }
            }
        }
    }, 64);
    // The closing layer takes the INTER edges of block nY-1 whose global
    // source id is strictly greater than n (cost_time_ratio_solver.cpp:56);
    // with two layers that drops the edges leaving node 0 of layer 1.  With
    // more layers the list equals the INTER one and is not stored.
    if (T.nY == 2) {
        T.srcDummy = T.src[INTER];
        for (auto& s : T.srcDummy)
            if (s == 0) s = -1;
    }
}

}  // namespace

void host_parallel_for(int64_t n, int64_t grain, const std::function<void(int64_t, int64_t)>& f) {
    parallel_for(n, [&](int64_t a, int64_t b) { f(a, b); }, grain);
}

std::string build_template(const int* EX, int64_t nEX, const int* EY, int64_t nEY, int64_t nVX, bool conj,
                           bool prune, LayerTemplate& T) {
    if (nEX < 1) return "EX must have at least one row";
    if (nEY < 2) return "EY must have at least two rows (one product layer per Y edge)";
    int mx = -1;
    for (int64_t i = 0; i < 2 * nEX; ++i) {
        if (EX[i] < 0 || EX[i] >= nVX) return "EX refers to a vertex outside VX";
        mx = std::max(mx, EX[i]);
    }
    for (int64_t i = 0; i < 2 * nEY; ++i)
        if (EY[i] < 0) return "EY holds a negative vertex index";
    T = LayerTemplate();
    T.conj = conj;
    T.prune = prune;
    T.nvx = mx + 1;
    T.nY = (int)nEY;
    if (!conj && T.nvx != nVX)
        return "the plain product graph needs every vertex of VX to appear in EX (|VX| == max(EX)+1)";
    if (conj) {
        if (3 * nEX > INT_MAX / 4) return "EX too large";
        T.n = (int)(3 * nEX);
        build_conj(EX, nEX, T);
    } else {
        T.n = (int)nVX;
        build_plain(EX, nEX, T);
    }
    T.eBlock = (int64_t)T.eSrc.size();
    build_sell(T);
    (void)EY;
    return "";
}

void product_row(const LayerTemplate& T, const int* EY, int64_t e, int* out) {
    const int64_t b = e / T.eBlock, t = e % T.eBlock;
    const int s2 = EY[2 * b], m2 = EY[2 * b + 1];
    const int t2 = EY[2 * ((b + 1) % T.nY) + 1];
    const int* x = &T.eX[(size_t)(3 * t)];
    switch (T.eY[(size_t)t]) {
        case Y_SS: out[0] = s2; out[1] = s2; break;
        case Y_SM: out[0] = s2; out[1] = m2; break;
        case Y_SSS: out[0] = s2; out[1] = s2; out[2] = s2; break;
        case Y_SSM: out[0] = s2; out[1] = s2; out[2] = m2; break;
        case Y_SMT: out[0] = s2; out[1] = m2; out[2] = t2; break;
        case Y_SMM: out[0] = s2; out[1] = m2; out[2] = m2; break;
    }
    if (T.conj) {
        out[3] = x[0]; out[4] = x[1]; out[5] = x[2];
    } else {
        out[2] = x[0]; out[3] = x[1];
    }
}

// Contiguous slice ranges for `blocks` CTAs of `warps` warps with balanced
// step times.  A warp relaxes the CTA's slices that have rows in the step's
// part, round-robin, and one slice of one step costs it about (gather
// batches + 1) memory latencies, with rowsPerBatch[p] rows per batch in
// part p: the batches of its rows and the epilogue
// (the winner's record, the stores).  Slices without rows are visited only
// by two steps per sweep and cost nothing here.
// Steps are coupled across the team by the hand-offs, so a layer costs the
// slowest warp of any CTA in the interlayer step plus K - 1 times the
// slowest in an intralayer step (those run only when the layer has
// intralayer edges).  The cuts therefore bound the two kinds separately:
// for bounds (bi, bj) CTAs are filled greedily while their slowest warps
// stay within both -- optimal for the pair, since a range's costs never grow
// when it shrinks -- and the pair with the smallest bi + (K - 1) bj that
// fits in `blocks` CTAs is kept (bj in steps of one latency, bi by binary
// search).  Costs are in 1/32 of a latency.
std::vector<int> plan_cta_cuts(const LayerTemplate& T, int blocks, int K, int warps, const int rowsPerBatch[2]) {
    const int ns = T.nslices;
    std::vector<int> cut((size_t)blocks + 1, ns);
    cut[0] = 0;
    if (blocks <= 1 || ns == 0) return cut;
    warps = std::max(1, warps);
    const bool intra = T.entries[INTRA] > 0 && K > 1;
    const int rb[2] = {std::max(1, rowsPerBatch[0]), std::max(1, rowsPerBatch[1])};
    std::vector<long long> w[2];
    long long lo[2] = {0, 0}, hi[2] = {0, 0};
    for (int p = 0; p < 2; ++p) {
        w[p].resize((size_t)ns);
        for (int s = 0; s < ns; ++s) {
            const int rows = T.sp[p][(size_t)s + 1] - T.sp[p][(size_t)s];
            w[p][(size_t)s] = (p == 1 && !intra) || rows == 0 ? 0 : 32LL * ((rows + rb[p] - 1) / rb[p] + 1);
            lo[p] = std::max(lo[p], w[p][(size_t)s]);
            hi[p] += w[p][(size_t)s];
        }
    }
    std::vector<long long> acc[2] = {std::vector<long long>((size_t)warps), std::vector<long long>((size_t)warps)};
    // fills CTAs greedily under (bi, bj); returns the CTAs used (cuts in c
    // when given).  A CTA's warps take its slices with rows in a part
    // round-robin (a0, a1: the warp that gets the next one); slices without
    // rows cost nothing.
    auto fill = [&](long long bi, long long bj, std::vector<int>* c) -> int {
        int used = 1, start = 0, a0 = 0, a1 = 0;
        long long* acc0 = acc[0].data();
        long long* acc1 = acc[1].data();
        std::fill(acc0, acc0 + warps, 0);
        std::fill(acc1, acc1 + warps, 0);
        const long long* w0 = w[0].data();
        const long long* w1 = w[1].data();
        for (int s = 0; s < ns; ++s) {
            const long long x0 = w0[s], x1 = w1[s];
            if (s > start && ((x0 && acc0[a0] + x0 > bi) || (x1 && acc1[a1] + x1 > bj))) {
                if (c && used < blocks) (*c)[(size_t)used] = s;
                if (++used > blocks && !c) return used;
                start = s;
                a0 = a1 = 0;
                std::fill(acc0, acc0 + warps, 0);
                std::fill(acc1, acc1 + warps, 0);
            }
            if (x0) {
                acc0[a0] += x0;
                if (++a0 == warps) a0 = 0;
            }
            if (x1) {
                acc1[a1] += x1;
                if (++a1 == warps) a1 = 0;
            }
        }
        return used;
    };
    const long long reps = intra ? K - 1 : 0;
    // the smallest intralayer bound that fits at all, then up from there
    long long j0 = lo[1], j1 = hi[1];
    while (j0 < j1) {
        const long long mid = j0 + (j1 - j0) / 2;
        if (fill(hi[0], mid, nullptr) <= blocks) j1 = mid;
        else j0 = mid + 1;
    }
    long long bestI = -1, bestJ = -1, bestCost = 0;
    for (long long bj = j0, tries = 0; tries < 64; bj += 32, ++tries) {
        if (bestI >= 0 && reps * bj >= bestCost) break;
        if (bj > hi[1]) bj = hi[1];
        if (fill(hi[0], bj, nullptr) <= blocks) {
            long long a = lo[0], b = hi[0];
            while (a < b) {
                const long long mid = a + (b - a) / 2;
                if (fill(mid, bj, nullptr) <= blocks) b = mid;
                else a = mid + 1;
            }
            const long long cost = a + reps * bj;
            if (bestI < 0 || cost < bestCost) {
                bestI = a;
                bestJ = bj;
                bestCost = cost;
            }
        }
        if (bj >= hi[1] || !intra) break;
    }
    const int used = fill(bestI, bestJ, &cut);
    // CTAs past the last range keep empty ranges at the end
    for (int c = used; c < blocks; ++c) cut[(size_t)c] = ns;
    return cut;
}

// Wait lists of the Bellman-Ford team in CSR form (ptr: blocks + 1 offsets,
// idx: CTA ids, ascending per list): CTA c lists every other CTA d joined to
// it by an in-edge of either part, i.e. d owns the slice of a source of one
// of c's in-edges (c reads d's rows) or c owns the slice of a source of one
// of d's (d reads c's rows, so d must be done before c overwrites them).
// CTA c owns the slices [cut[c], cut[c+1]).  The product graph repeats one
// layer template, so one pass over the template covers every layer; the
// closing layer's sources are a subset of the interlayer ones.
void cta_wait_lists(const LayerTemplate& T, const std::vector<int>& cut, std::vector<int>& ptr, std::vector<int>& idx) {
    const int blocks = (int)cut.size() - 1;
    std::vector<int> owner((size_t)T.nslices);
    for (int c = 0; c < blocks; ++c)
        for (int s = cut[(size_t)c]; s < cut[(size_t)c + 1]; ++s) owner[(size_t)s] = c;
    // the CTA pairs joined by an in-edge, in parallel over slices (each part
    // of the range marks its own matrix; the matrices are OR-ed)
    std::vector<unsigned char> adj((size_t)blocks * blocks, 0);
    std::mutex adjMu;
    host_parallel_for(T.nslices, 256, [&](int64_t s0, int64_t s1) {
        std::vector<unsigned char> mine((size_t)blocks * blocks, 0);
        for (int p = 0; p < 2; ++p) {
            for (int64_t s = s0; s < s1; ++s) {
                const int ct = owner[(size_t)s];
                int last = ct;
                for (int j = T.sp[p][(size_t)s]; j < T.sp[p][(size_t)s + 1]; ++j)
                    for (int lane = 0; lane < 32; ++lane) {
                        const int sv = T.src[p][(size_t)j * 32 + lane];
                        if (sv < 0) continue;
                        const int cs = owner[(size_t)(sv >> 5)];
                        if (cs == ct || cs == last) continue;
                        last = cs;
                        mine[(size_t)ct * blocks + cs] = 1;
                        mine[(size_t)cs * blocks + ct] = 1;
                    }
            }
        }
        std::lock_guard<std::mutex> lock(adjMu);
        for (size_t i = 0; i < adj.size(); ++i) adj[i] |= mine[i];
    });
    ptr.assign((size_t)blocks + 1, 0);
    idx.clear();
    for (int c = 0; c < blocks; ++c) {
        for (int d = 0; d < blocks; ++d)
            if (adj[(size_t)c * blocks + d]) idx.push_back(d);
        ptr[(size_t)c + 1] = (int)idx.size();
    }
}

}  // namespace pgc
