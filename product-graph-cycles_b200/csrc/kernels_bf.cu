// kernels_bf.cu -- layered Bellman-Ford sweeps of the cycle solvers on sm_100a.
//
// One launch runs one Bellman-Ford call of the reference
// (mooreBellmanFordSubroutineCPU, cost_time_ratio_solver.cpp:251-542, and
// dijkstra_solver.cpp:203-388) from its set-up to its verdict, so the host
// sees one launch per call instead of one per (layer, depth).
//
// Semantics kept exactly (the result must equal the reference's):
//  * the DP table keeps the reference's row layout: layer l writes parity
//    l % 2 at depths 0..K-1; layer 0 does not reset its depth >= 1 rows; the
//    wrap reads row numLayers % 2 (a row index, as in the reference);
//  * relaxation is pull-based: node v of (layer, depth) takes the FIRST
//    minimum over its in-edges in ascending edge id (and, for interlayer
//    edges, over source depths 0..K-1), with strict '<' against the running
//    value and against the upper bound;  w = c - lambda*t and every sum are
//    rounded double operations (no fused multiply-add);
//  * predecessors are written only on improvement, so stale entries evolve as
//    in the reference.
//
// Work split of one (layer, depth) step: every CTA owns a range of node
// slices (32 nodes each) balanced by in-edge entries.  Phase A: the CTA's
// threads take the in-edge entries of a chunk of slices independently --
// source index, cost and time, then the source's DP record -- and leave each
// entry's best candidate in shared memory, so a whole chunk costs two memory
// latencies however large the in-degree.  Phase B: one thread per node folds
// its entries in edge order (the reference's tie-break) and writes the node.
//
// Cycle detection: the reference walks predecessors from every negative
// start node in ascending order of its value until a start node repeats.
// Here each DP record also carries its path's origin (the layer-0 start node
// it leaves from) and its length in predecessor steps, so one "lap" of the
// walk (layer-0 node -> next layer-0 node) is a table lookup.  Each candidate
// is decided with Brent's cycle-finding algorithm on that lap function; the
// candidate with the smallest (value, index) whose walk repeats within the
// reference's step limit wins.  When a lap cannot be derived from the
// current sweep (a stale predecessor), that candidate is re-walked literally:
// all such candidates at once, each by cycle finding on the predecessor
// function, advanced a bounded number of loads per round between team
// barriers.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <map>
#include <mutex>
#include <set>
#include <tuple>

#include "device_common.cuh"

namespace pgc {

namespace {

struct Team {
    int cta, ncta;
    unsigned* cnt;
    unsigned* gen;
    int* err;
    unsigned spin;  // polls of a wait before it gives up
    __device__ long long thread() const { return (long long)cta * blockDim.x + threadIdx.x; }
    __device__ long long nthreads() const { return (long long)ncta * blockDim.x; }
};

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned atom_add_acq_rel_u32(unsigned* p, unsigned v) {
    unsigned old;
    asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Team barrier that also ORs one flag over the team.  One CTA:
// __syncthreads_or.  Several CTAs (cooperative launch, all resident): after
// the CTA-wide barrier, thread 0 adds 1 (+ 1 << 16 if its CTA's flag is set)
// to a global counter with acquire-release semantics (cumulative over the
// CTA's writes).  The last arrival resets the counter and publishes the next
// generation with the team's flag in bit 0 (release store); the others poll
// the generation with acquire loads -- briefly spinning, then backing off --
// for a bounded number of iterations.  A CTA whose wait runs out raises the
// error word and gets ok = false; every other waiter checks the error word
// while polling and gives up too, so every CTA ends within a bounded time.
__device__ int team_sync_or(const Team& t, int flag, bool& ok) {
    __shared__ int s_flag, s_ok;
    const int any = __syncthreads_or(flag);
    if (threadIdx.x == 0) {
        int res = any, good = 1;
        if (t.ncta > 1) {
            const unsigned g = ld_acquire_u32(t.gen);
            const unsigned add = 1u + (any ? (1u << 16) : 0u);
            const unsigned old = atom_add_acq_rel_u32(t.cnt, add);
            if ((old & 0xffffu) == (unsigned)t.ncta - 1) {
                res = ((old + add) >> 16) != 0;
                atomicExch(t.cnt, 0u);
                st_release_u32(t.gen, (((g >> 1) + 1) << 1) | (unsigned)res);
            } else {
                unsigned spins = 0, cur;
                while ((cur = ld_acquire_u32(t.gen)) == g) {
                    ++spins;
                    if (spins > t.spin || ((spins & 63u) == 0 && *(volatile int*)t.err)) {
                        atomicExch(t.err, 1);
                        good = 0;
                        break;
                    }
                    if (spins > 4096) __nanosleep(64);
                }
                res = (int)(cur & 1u);
            }
        }
        s_flag = res;
        s_ok = good;
    }
    __syncthreads();
    ok = s_ok != 0;
    return s_flag;
}

__device__ __forceinline__ bool team_sync(const Team& t) {
    bool ok;
    team_sync_or(t, 0, ok);
    return ok;
}

// Lexicographic (value, index) key.
struct Key {
    double v;
    int i;
};
__device__ __forceinline__ bool key_less(const Key& a, const Key& b) {
    return a.v < b.v || (a.v == b.v && a.i < b.i);
}
__device__ __forceinline__ Key warp_min(Key k) {
    for (int o = 16; o > 0; o >>= 1) {
        Key x;
        x.v = __shfl_xor_sync(0xffffffffu, k.v, o);
        x.i = __shfl_xor_sync(0xffffffffu, k.i, o);
        if (key_less(x, k)) k = x;
    }
    return k;
}
// Block-wide minimum; result valid in every thread.  `slot` names one of the
// shared scratch sets so that two reductions in a row do not collide.
__device__ Key block_min(Key k, int slot) {
    __shared__ double sv[2][32];
    __shared__ int si[2][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    k = warp_min(k);
    if (lane == 0) { sv[slot][w] = k.v; si[slot][w] = k.i; }
    __syncthreads();
    Key r{kInfD, 0x7fffffff};
    if (w == 0) {
        if (lane < nw) { r.v = sv[slot][lane]; r.i = si[slot][lane]; }
        r = warp_min(r);
        if (lane == 0) { sv[slot][0] = r.v; si[slot][0] = r.i; }
    }
    __syncthreads();
    r.v = sv[slot][0];
    r.i = si[slot][0];
    __syncthreads();
    return r;
}

__device__ __forceinline__ int original_index(int n, int K, int e) {
    // cost_time_ratio_solver.cpp:240-250
    const int per = n * K;
    const int layer = e / per;
    const int rem = e - layer * per;
    const int depth = rem / n;
    return rem - depth * n + layer * n;
}

// DP record of node v at depth k in the parity row starting at rowBase =
// parity * n * Kp.  Its value lives in p.dv at rowBase + v * Kp + k (a
// node's depths side by side: one vector load gathers them); its path origin
// and length live in p.doh at rowBase + k * n + v (depth-major: the stores
// of a warp's 32 consecutive nodes are 256 contiguous bytes, where the
// node-major index would spread them over 32 sectors; they are read one at
// a time).  Loads come from shared memory when the whole team is one CTA
// that keeps its tables there (S), else through L2 (other CTAs write the
// records during the launch, so L1 must not serve stale lines).
template <bool S>
__device__ __forceinline__ double ldV(const BfParams& p, size_t r) {
    if constexpr (S) return p.dv[r];
    else return __ldcg(p.dv + r);
}
__device__ __forceinline__ size_t oh_index(const BfParams& p, size_t rowBase, int v, int k) {
    return rowBase + (size_t)k * p.n + v;
}
template <bool S>
__device__ __forceinline__ int2 ldOH(const BfParams& p, size_t rowBase, int v, int k) {
    if constexpr (S) return p.doh[oh_index(p, rowBase, v, k)];
    else return __ldcg(p.doh + oh_index(p, rowBase, v, k));
}
__device__ __forceinline__ void stE(const BfParams& p, size_t rowBase, int v, int k, double val, int o, int h) {
    p.dv[rowBase + (size_t)v * p.Kp + k] = val;
    p.doh[oh_index(p, rowBase, v, k)] = make_int2(o, h);
}

// The NK values of consecutive depths starting at `rec` (a node's row of
// Kp values: 16-byte aligned for Kp = 2, 32-byte aligned for Kp = 4) in one
// vector load: 8, 16 or 32 bytes, one sector of L2 per source.  NK = 3 reads
// the row's fourth value too and ignores it.
template <bool S, int NK>
__device__ __forceinline__ void ld_row(const double* rec, double (&d)[NK]) {
    if constexpr (NK == 1) {
        d[0] = S ? rec[0] : __ldcg(rec);
    } else if constexpr (NK == 2) {
        const double2 x = S ? *reinterpret_cast<const double2*>(rec) : __ldcg(reinterpret_cast<const double2*>(rec));
        d[0] = x.x;
        d[1] = x.y;
    } else {
        static_assert(NK <= 4, "a node row holds at most four depths here");
        double a, b, c, e;
        if constexpr (S) {
            const double2 x = reinterpret_cast<const double2*>(rec)[0], y = reinterpret_cast<const double2*>(rec)[1];
            a = x.x; b = x.y; c = y.x; e = y.y;
        } else {
            asm volatile("ld.global.cg.v4.f64 {%0, %1, %2, %3}, [%4];"
                         : "=d"(a), "=d"(b), "=d"(c), "=d"(e)
                         : "l"(rec)
                         : "memory");
        }
        d[0] = a;
        d[1] = b;
        d[2] = c;
        if constexpr (NK == 4) d[3] = e;
        else (void)e;
    }
}

// ---------------------------------------------------------------------------
// Step staging.  The in-edge streams a CTA reads in one step -- source
// indices, costs and times of the rows of its slices -- are contiguous and do
// not depend on the DP values, so the CTA copies the next step's streams
// into shared memory with bulk asynchronous copies (TMA, no multicast) while
// the current step runs and hands off.  Two buffers alternate; each has an
// mbarrier that completes when its copies have landed.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_addr(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
// One bounded wait for the phase with the given parity; true when it completed.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, unsigned limit) {
    for (unsigned spins = 0; spins < limit; ++spins) {
        unsigned done;
        asm volatile(
            "{\n\t.reg .pred P;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, P;\n\t}"
            : "=r"(done)
            : "r"(smem_addr(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
// Global -> shared bulk copy (16-byte aligned addresses, size a multiple of 16).
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// Brings [src, src + bytes) into L2 (16-byte aligned, a multiple of 16).
__device__ __forceinline__ void bulk_prefetch_l2(const void* src, unsigned bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

// Shared-memory state of a CTA: its slices' row offsets per part (staged
// once per launch) and the two step buffers.
struct Stage {
    const int* splInter;         // sp[s0 + i] of the interlayer part, i = 0..s1-s0
    const int* splIntra;         // same for the intralayer part
    const int* actInter;         // the CTA's slices (s - s0) with interlayer rows
    const int* actIntra;         // ... with intralayer rows
    int nActInter, nActIntra;
    char* buf0;
    char* buf1;
    unsigned long long* bar;     // [2]
    int rowCap;                  // rows one buffer holds
    bool srcOnly;                // buffers hold the source indices only; costs and times are read in place
    unsigned phase;              // bit b: parity of buffer b's next completion
    unsigned pending;            // bit b: copies issued into buffer b, not yet waited for
    int costBytes, timeBytes;    // bytes per entry of the cost and time streams
    unsigned spin;               // polls of a copy wait before it gives up
    __device__ const int* spl(int part) const { return part ? splIntra : splInter; }
    __device__ const int* act(int part) const { return part ? actIntra : actInter; }
    __device__ int nAct(int part) const { return part ? nActIntra : nActInter; }
    __device__ char* buf(int b) const { return b ? buf1 : buf0; }
};

struct StepRef {
    int l, k;
};
__device__ __forceinline__ bool step_empty(const BfParams& p, int l, int k) { return l == p.nY && k > 0; }

// Stage step (l, k) into buffer b.  Every thread keeps the same bookkeeping;
// thread 0 issues the copies.
__device__ void stage_issue(const BfParams& p, Stage& st, int s0, int s1, int b, int l, int k) {
    if (st.rowCap == 0 || step_empty(p, l, k)) return;
    const int* spl = st.spl(k == 0 ? 0 : 1);
    const int r0 = spl[0], r1 = spl[s1 - s0];
    if (r1 <= r0) return;
    st.pending |= 1u << b;
    if (threadIdx.x != 0) return;
    const size_t e0 = (size_t)r0 * 32, cnt = (size_t)(r1 - r0) * 32;
    const int* src = k == 0 ? (l == p.nY ? p.srcDummy : p.srcInter) : p.srcIntra;
    const size_t base = (size_t)l * (size_t)p.layerStride + (k == 0 ? 0 : (size_t)p.interEntries);
    char* dst = st.buf(b);
    const unsigned bs = (unsigned)(cnt * 4), bc = (unsigned)(cnt * st.costBytes), bt = (unsigned)(cnt * st.timeBytes);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (st.srcOnly) {
        // the costs and times are read in place during the step; bring them
        // into L2 meanwhile, so those reads overlap the gathers at L2 latency
        mbar_expect(st.bar + b, bs);
        bulk_load(dst, src + e0, bs, st.bar + b);
        bulk_prefetch_l2((const char*)p.cost + (base + e0) * st.costBytes, bc);
        if (bt) bulk_prefetch_l2((const char*)p.time + (base + e0) * st.timeBytes, bt);
        return;
    }
    mbar_expect(st.bar + b, bs + bc + bt);
    bulk_load(dst, src + e0, bs, st.bar + b);
    bulk_load(dst + (size_t)st.rowCap * 32 * 4, (const char*)p.cost + (base + e0) * st.costBytes, bc, st.bar + b);
    if (bt)
        bulk_load(dst + (size_t)st.rowCap * 32 * (4 + st.costBytes), (const char*)p.time + (base + e0) * st.timeBytes,
                  bt, st.bar + b);
}

// Wait for buffer b if copies were issued into it (every thread).
__device__ __forceinline__ bool stage_wait(Stage& st, int b) {
    if (!((st.pending >> b) & 1u)) return true;
    const bool ok = mbar_wait(st.bar + b, (st.phase >> b) & 1u, st.spin);
    st.phase ^= 1u << b;
    st.pending &= ~(1u << b);
    return ok;
}

// Before the CTA exits: no copy may still be writing its shared memory.
__device__ __forceinline__ void stage_drain(Stage& st) {
    stage_wait(st, 0);
    stage_wait(st, 1);
}

// ---------------------------------------------------------------------------
// One (layer, depth) step of the sweep over the CTA's slices [s0, s1), with
// the step's streams staged in buffer `sb`.
//
// A warp owns a slice of 32 target nodes (lane = node).  The slice's in-edge
// rows are visited in the reference's order -- ascending edge, then source
// depth -- in batches of up to min(kGather / NK, 8) rows (NK source depths
// per edge, a compile-time constant of the step kind); the last batch has
// exactly the rows that remain.  First every source value of the batch is
// gathered (independent loads), then the batch is folded into the running
// first minimum, so a batch costs one memory latency.  The fold keeps only
// thr = min(best, upper bound) and the position of the last improvement: a
// candidate is taken iff cand < thr, which is the reference's
// (cand < best && cand < ub), and an unreached source (+inf) can never pass
// it.  The winner's origin and path length are read once per node after the
// fold.  Returns whether this thread improved a node.
// ---------------------------------------------------------------------------

struct StepView {
    const int* src;     // source index per entry, from the step's first row
    const void* cost;
    const char* time;
    const double* srcv; // DP values of the source layer (its record 0)
    size_t sbase;       // record index of the source layer's record 0
    int Kp, kofs, nk;
    double lam, tconst;
};

template <class CT, int TK>
__device__ __forceinline__ double edge_weight(const StepView& v, int q) {
    double t = v.tconst;
    if (TK == 1) t = (double)reinterpret_cast<const float*>(v.time)[q];
    else if (TK == 2) t = reinterpret_cast<const double*>(v.time)[q];
    return __dsub_rn((double)reinterpret_cast<const CT*>(v.cost)[q], __dmul_rn(v.lam, t));
}

// Rows [row, j1) of one slice for lane `lane`; NK > 0 source depths per edge
// known at compile time, NK == 0: v.nk depths, one gather at a time.
// One batch of exactly NR rows starting at `row`: every source value is
// gathered first, then the batch is folded in edge order.  `win` records the
// position of the last improvement (row * 8 + depth); thr is its value.
// TREE: the batch's candidates are reduced as a balanced tree of (value,
// position) minima instead of one sequential compare chain (the batched
// kernel, whose register budget holds the extra live values; the
// single-graph kernel's 96-register budget does not).
template <class CT, int TK, bool S, int NK, int NR, bool TREE>
__device__ __forceinline__ void fold_batch(const StepView& v, int lane, int row, double& thr, int& win) {
    int sv[NR];
    double d[NR][NK];
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        sv[r] = v.src[(row + r) * 32 + lane];
        if (sv[r] >= 0) {
            ld_row<S, NK>(v.srcv + (size_t)sv[r] * v.Kp + v.kofs, d[r]);
        } else {
#pragma unroll
            for (int kk = 0; kk < NK; ++kk) d[r][kk] = kInfD;
        }
    }
    if constexpr (!TREE) {
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            if (sv[r] < 0) continue;
            const double w = edge_weight<CT, TK>(v, (row + r) * 32 + lane);
#pragma unroll
            for (int kk = 0; kk < NK; ++kk) {
                const double cand = __dadd_rn(d[r][kk], w);
                if (cand < thr) { thr = cand; win = ((row + r) << 3) | kk; }
            }
        }
    } else {
        // The candidates in edge order (row, then depth), reduced so that
        // the left -- earlier -- candidate wins ties: the first minimum,
        // which is what the sequential scan `cand < thr` ends with.  A NaN
        // candidate, which that scan never takes, enters as +inf; neither
        // is ever below thr.
        constexpr int N = NR * NK;
        double cv[N];
        int ci[N];
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            const double w = sv[r] >= 0 ? edge_weight<CT, TK>(v, (row + r) * 32 + lane) : 0.0;
#pragma unroll
            for (int kk = 0; kk < NK; ++kk) {
                double c = kInfD;
                if (sv[r] >= 0) {
                    c = __dadd_rn(d[r][kk], w);
                    if (c != c) c = kInfD;
                }
                cv[r * NK + kk] = c;
                ci[r * NK + kk] = r * NK + kk;
            }
        }
#pragma unroll
        for (int s = 1; s < N; s <<= 1) {
#pragma unroll
            for (int i = 0; i + s < N; i += 2 * s) {
                if (cv[i + s] < cv[i]) {
                    cv[i] = cv[i + s];
                    ci[i] = ci[i + s];
                }
            }
        }
        if (cv[0] < thr) {
            thr = cv[0];
            win = ((row + ci[0] / NK) << 3) | (ci[0] % NK);
        }
    }
}

// The last nr (1 <= nr <= NR) rows as one batch of exactly nr rows.  The row
// count is the slice's, the same in every lane, so no lane runs row slots
// that do not exist.
template <class CT, int TK, bool S, int NK, int NR, bool TREE>
__device__ __forceinline__ void fold_tail(const StepView& v, int lane, int row, int nr, double& thr, int& win) {
    if constexpr (NR <= 1) {
        fold_batch<CT, TK, S, NK, 1, TREE>(v, lane, row, thr, win);
    } else {
        if (nr == NR) fold_batch<CT, TK, S, NK, NR, TREE>(v, lane, row, thr, win);
        else fold_tail<CT, TK, S, NK, NR - 1, TREE>(v, lane, row, nr, thr, win);
    }
}

// Rows [row, j1) of one slice for lane `lane`.  Returns the position of the
// winning candidate -- row * 8 + depth for NK > 0, row * nk + depth for the
// run-time depth count (NK == 0) -- or -1; thr holds its value.
template <class CT, int TK, bool S, int NK, bool TREE>
__device__ __forceinline__ int fold_rows(const StepView& v, int lane, int row, int j1, double& thr) {
    int win = -1;
    if constexpr (NK > 0) {
        constexpr int RB = bf_rows_per_batch(NK);
        for (; j1 - row >= RB; row += RB) fold_batch<CT, TK, S, NK, RB, TREE>(v, lane, row, thr, win);
        if (row < j1) fold_tail<CT, TK, S, NK, RB, TREE>(v, lane, row, j1 - row, thr, win);
    } else {
        for (; row < j1; ++row) {
            const int sv = v.src[row * 32 + lane];
            if (sv < 0) continue;
            const double w = edge_weight<CT, TK>(v, row * 32 + lane);
            const double* rec = v.srcv + (size_t)sv * v.Kp + v.kofs;
            for (int kk = 0; kk < v.nk; ++kk) {
                const double cand = __dadd_rn(S ? rec[kk] : __ldcg(rec + kk), w);
                if (cand < thr) { thr = cand; win = row * v.nk + kk; }
            }
        }
    }
    return win;
}

template <class CT, int TK, bool S, int NK, bool TREE>
__device__ bool relax_slices(const BfParams& p, const StepView& sv, const int* spl, const int* act, int nAct, int s0,
                             int s1, int l, int k) {
    const int n = p.n, K = p.K, Kp = p.Kp;
    const size_t cur = (size_t)(l & 1) * n * Kp;
    const bool empty = step_empty(p, l, k);
    const int r0 = spl[0];
    int* predRow = p.pred + (size_t)l * n * K + (size_t)k * n;
    const int srcLayer = k == 0 ? l - 1 : l;
    const int lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    const double ub = p.ub;
    bool any = false;
    // A slice without rows in this step's part only writes (+inf, unknown
    // or end of walk, 0): its nodes are never reached through this part.
    // Their row slots already hold +inf -- from the set-up, or written by an
    // earlier step of the same kind -- except depth 0 of the even layers,
    // whose parity row also holds layer 0's start values: the interlayer
    // step of layer 2 overwrites those.  So that step and the layer-0 steps
    // visit every slice of the CTA; the others only the slices with rows
    // (the origins of a never-reached record are never read).
    const bool all = l == 0 || (l == 2 && k == 0);
    const int count = all ? s1 - s0 : nAct;
    for (int i = (int)(threadIdx.x >> 5); i < count; i += nwarps) {
        const int s = s0 + (all ? i : act[i]);
        const int v = s * 32 + lane;
        const bool valid = v < n;
        const size_t me = cur + (size_t)v * Kp + k;
        double best = (l == 0 && valid) ? ldV<S>(p, me) : kInfD;
        double thr = best < ub ? best : ub;
        int win = -1;
        if (!empty) win = fold_rows<CT, TK, S, NK, TREE>(sv, lane, spl[s - s0] - r0, spl[s + 1 - s0] - r0, thr);
        if (!valid) continue;
        int o = kLapUnknown, h = 0;
        int bs = -1, bk = -1;
        if (win >= 0) {
            const int rw = NK > 0 ? (win >> 3) : win / sv.nk;
            bk = sv.kofs + (NK > 0 ? (win & 7) : win % sv.nk);
            bs = sv.src[rw * 32 + lane];
            best = thr;
        }
        if (bs >= 0) {
            predRow[v] = bs + srcLayer * n * K + bk * n;
            any = true;
            if (srcLayer == 0 && bk == 0) {  // leaves a layer-0 start node
                o = bs;
                h = 1;
            } else {
                const int2 e = ldOH<S>(p, sv.sbase, bs, bk);
                o = e.x;
                h = e.y + 1;
            }
        } else if (l == 0) {
            // Layer 0 keeps an older value and its older predecessor.
            const int pe = __ldcg(predRow + v);
            if (pe < 0) {
                o = kLapEnd;
            } else {
                const int ps = pe - (k - 1) * n;
                if (ps < 0 || ps >= n) {
                    o = kLapUnknown;
                } else if (k - 1 == 0) {
                    o = ps;
                    h = 1;
                } else {
                    const int2 e = ldOH<S>(p, cur, ps, k - 1);
                    o = e.x;
                    h = e.y + 1;
                }
            }
        }
        stE(p, cur, v, k, best, o, h);
    }
    return any;
}

template <class CT, int TK, bool S, bool TREE>
__device__ bool relax_step(const BfParams& p, const Stage& st, int sb, int s0, int s1, int l, int k) {
    const int n = p.n, K = p.K, Kp = p.Kp;
    const bool inter = (k == 0);
    const int part = inter ? 0 : 1;
    const int* spl = st.spl(part);
    const int r0 = spl[0];
    StepView v;
    // the step's streams from row r0 on: staged in shared memory; or the
    // source indices staged and the costs and times read in place
    // (srcOnly); or all read in place when no buffer fits (rowCap == 0)
    if (st.rowCap > 0 && !st.srcOnly) {
        char* b = st.buf(sb);
        v.src = reinterpret_cast<const int*>(b);
        v.cost = b + (size_t)st.rowCap * 32 * 4;
        v.time = b + (size_t)st.rowCap * 32 * (4 + sizeof(CT));
    } else {
        const size_t off = (size_t)l * (size_t)p.layerStride + (inter ? 0 : (size_t)p.interEntries) + (size_t)r0 * 32;
        v.src = st.rowCap > 0 ? reinterpret_cast<const int*>(st.buf(sb))
                              : (inter ? (l == p.nY ? p.srcDummy : p.srcInter) : p.srcIntra) + (size_t)r0 * 32;
        v.cost = reinterpret_cast<const CT*>(p.cost) + off;
        v.time = TK == 0 ? nullptr : reinterpret_cast<const char*>(p.time) + off * st.timeBytes;
    }
    v.sbase = (size_t)((inter ? l - 1 : l) & 1) * n * Kp;
    v.srcv = p.dv + v.sbase;
    v.Kp = Kp;
    v.kofs = inter ? 0 : k - 1;
    v.nk = inter ? K : 1;
    v.lam = p.lambda;
    v.tconst = p.tconst;
    const int* act = st.act(part);
    const int na = st.nAct(part);
    if (!inter) return relax_slices<CT, TK, S, 1, TREE>(p, v, spl, act, na, s0, s1, l, k);
    switch (K) {
        case 1: return relax_slices<CT, TK, S, 1, TREE>(p, v, spl, act, na, s0, s1, l, k);
        case 2: return relax_slices<CT, TK, S, 2, TREE>(p, v, spl, act, na, s0, s1, l, k);
        case 3: return relax_slices<CT, TK, S, 3, TREE>(p, v, spl, act, na, s0, s1, l, k);
        case 4: return relax_slices<CT, TK, S, 4, TREE>(p, v, spl, act, na, s0, s1, l, k);
        default: return relax_slices<CT, TK, S, 0, TREE>(p, v, spl, act, na, s0, s1, l, k);
    }
}

// Dataflow hand-off between steps of a multi-CTA team.  Step `step` of this
// CTA is complete; publish it, then wait until every CTA on this CTA's wait
// list (the owners of the sources it reads and the readers of the rows it
// overwrites next) has completed it too.  This replaces a grid-wide barrier:
// a CTA waits only for its graph neighbours.  Returns false when a wait ran
// out of iterations or another CTA raised the error word.  The CTA named by
// p.stallCta (a test hook; -1 in every solve) also waits for a word that no
// code writes, so its wait runs out.
__device__ bool step_handoff(const BfParams& p, const Team& t, unsigned step) {
    __syncthreads();  // the CTA's writes of this step are done
    if (threadIdx.x < 32) {
        // release store: with the CTA barrier above it publishes every write
        // of the CTA's threads in this step
        if (threadIdx.x == 0) st_release_u32(p.stepDone + (size_t)t.cta * kStepDoneStride, step);
        __syncwarp();
        const int w0 = __ldg(p.waitPtr + t.cta), w1 = __ldg(p.waitPtr + t.cta + 1);
        const bool stall = t.cta == p.stallCta;
        int good = 1;
        for (int i0 = w0; i0 < w1 + (stall ? 1 : 0) && good; i0 += 32) {
            const int i = i0 + (int)threadIdx.x;
            const unsigned* f = i < w1 ? p.stepDone + (size_t)__ldg(p.waitIdx + i) * kStepDoneStride
                                       : (stall && i == w1) ? &p.ctl->neverSet : nullptr;
            unsigned spins = 0;
            for (;;) {
                const bool ready = f == nullptr || (int)(ld_acquire_u32(f) - step) >= 0;
                if (__all_sync(0xffffffffu, ready)) break;
                ++spins;
                if ((spins & 63u) == 0 && *(volatile int*)t.err) { good = 0; break; }
                if (spins > t.spin) {
                    if (threadIdx.x == 0) atomicExch(t.err, 1);
                    good = 0;
                    break;
                }
                if (spins > 256) __nanosleep(32);
            }
        }
        if (threadIdx.x == 0 && !good) atomicExch(t.err, 1);
    }
    __syncthreads();
    return *(volatile int*)t.err == 0;
}

// Brent's cycle finding on the lap function starting at x0.
// Returns 1 (cycle: first repeated node in *v0, steps in *steps),
// 2 (the walk ends without a repeat) or 3 (undecidable from this sweep).
__device__ int lap_walk(const BfParams& p, int x0, long long limit, int* v0, long long* steps) {
    const int* P = p.lapNext;
    const int* L = p.lapSteps;
    int power = 1, lam = 1;
    int tort = x0;
    int hare = __ldcg(P + x0);
    long long guard = 0;
    const long long guardMax = 4LL * (p.n + 2);
    while (hare != tort) {
        if (hare < 0) return hare == kLapEnd ? 2 : 3;
        if (power == lam) { tort = hare; power <<= 1; lam = 0; }
        hare = __ldcg(P + hare);
        ++lam;
        if (++guard > guardMax) return 3;
    }
    tort = x0;
    hare = x0;
    for (int i = 0; i < lam; ++i) hare = __ldcg(P + hare);
    int mu = 0;
    while (tort != hare) {
        tort = __ldcg(P + tort);
        hare = __ldcg(P + hare);
        if (++mu > p.n + 1) return 3;
    }
    long long S = 0;
    int x = x0;
    for (int i = 0; i < mu + lam; ++i) {
        S += __ldcg(L + x);
        if (S > limit) return 2;
        x = __ldcg(P + x);
    }
    *v0 = tort;
    *steps = S;
    return 1;
}

// The reference's walk from candidate vi (cost_time_ratio_solver.cpp:461-488):
// x_0 = vi, x_(j+1) = pred[x_j]; it stops at the first j in [1, maxLen - 1]
// where x_j is a layer-0 start node (x_j < n) seen before in the walk (vi
// included), and fails when a predecessor leaves the node range (-1
// included) or the limit passes.  Since pred is a function, the walk repeats
// only once it is periodic: with tail mu and cycle length lam, that first
// repeated start node is x_(mu + lam + d), d the offset of the first start
// node on the cycle from x_mu.  So the walk is decided by Brent's cycle
// finding (lam), two pointers lam apart (mu) and a walk round the cycle (d),
// about (3 mu + 5 lam) loads and no visited marks, so every undecided
// candidate walks at once.  A walk advances at most `budget` loads per call
// and keeps its state in p.walks[i]; it returns true once decided, with
// candStat[i] = 1 (candV0[i] = x_j, candSteps[i] = j) or 2.
__device__ void walk_start(const BfParams& p, int i) {
    const long long total = (long long)p.n * (p.nY + 1) * p.K;
    LiteralWalk w{};
    w.phase = 1;
    w.a = i;
    w.b = __ldcg(p.pred + i);
    w.c1 = 1;  // power
    w.c2 = 1;  // lam
    w.c3 = 1;  // position of the hare
    if (w.b < 0 || (long long)w.b >= total) {
        w.phase = 0;
        p.candStat[i] = 2;
    }
    p.walks[i] = w;
}

__device__ bool walk_advance(const BfParams& p, int i, long long budget) {
    LiteralWalk w = p.walks[i];
    if (w.phase == 0) return true;
    const long long total = (long long)p.n * (p.nY + 1) * p.K;
    const long long maxLen = p.numNodes;
    int verdict = 0;  // 1 found, 2 failed
    while (budget > 0 && verdict == 0) {
        if (w.phase == 1) {  // Brent: the cycle length lam (c2); c1 power, c3 hare position
            if (w.a == w.b) {
                w.phase = 2;
                w.c1 = w.c2;  // lam
                w.c2 = w.c2;  // loads left to put the hare lam steps ahead of x_0
                w.a = i;
                w.b = i;
                continue;
            }
            if (w.c1 == w.c2) {
                w.a = w.b;
                w.c1 <<= 1;
                w.c2 = 0;
            }
            w.b = __ldcg(p.pred + w.b);
            --budget;
            ++w.c2;
            ++w.c3;
            // out of range: the walk ends without a repeat; past 3 maxLen loads
            // the tail and cycle exceed maxLen, so no repeat within the limit
            if (w.b < 0 || (long long)w.b >= total || w.c3 > 3 * maxLen + 8) verdict = 2;
        } else if (w.phase == 2) {  // hare lam steps ahead of x_0
            if (w.c2 == 0) {
                w.phase = 3;
                continue;  // c2 now counts the tail length mu
            }
            w.b = __ldcg(p.pred + w.b);
            --budget;
            --w.c2;
        } else if (w.phase == 3) {  // both pointers until they meet at x_mu
            if (w.a == w.b) {
                w.phase = 4;
                w.c3 = 0;  // d
                continue;
            }
            w.a = __ldcg(p.pred + w.a);
            w.b = __ldcg(p.pred + w.b);
            budget -= 2;
            ++w.c2;
        } else {  // round the cycle from x_mu to its first start node
            if (w.a < p.n) {
                const long long j = w.c2 + w.c1 + w.c3;
                if (j <= maxLen - 1) {
                    p.candV0[i] = w.a;
                    p.candSteps[i] = j;
                    verdict = 1;
                } else {
                    verdict = 2;
                }
            } else if (w.c3 + 1 >= w.c1) {
                verdict = 2;  // no start node on the cycle: no repeat is ever seen
            } else {
                w.a = __ldcg(p.pred + w.a);
                --budget;
                ++w.c3;
            }
        }
    }
    if (verdict) {
        w.phase = 0;
        p.candStat[i] = verdict;
    }
    p.walks[i] = w;
    return verdict != 0;
}

// Collects the cycle that closes at v0 (cost_time_ratio_solver.cpp:494-503):
// original node ids in walk order p(v0), p(p(v0)), ..., v0.
__device__ int extract_cycle(const BfParams& p, int v0, long long cLength) {
    const long long total = (long long)p.n * (p.nY + 1) * p.K;
    int pr = __ldcg(p.pred + v0);
    int len = 0;
    if (pr < 0 || pr >= total) return BF_ERR_WALK;
    p.cycleBuf[len++] = original_index(p.n, p.K, pr);
    for (long long kk = cLength - 1; kk > 0; --kk) {
        pr = __ldcg(p.pred + pr);
        if (pr < 0 || pr >= total) return BF_ERR_WALK;
        if (len >= p.cycleCap) return BF_ERR_CYCLE_CAP;
        p.cycleBuf[len++] = original_index(p.n, p.K, pr);
        if (pr == v0) break;
    }
    p.ctl->cycleLen = len;
    return BF_FOUND_CYCLE;
}

// The laps of the cycle that closes at v0, for a parallel extract_cycle:
// x_0 = v0, x_(j+1) = lapNext[x_j] until the lap function returns to v0.
// Lap j holds lapSteps[x_j] entries of the cycle buffer from offs[j] on.
// Returns the lap count and the cycle's length in *total, or -1 (unknown
// lap, or longer than the cycle buffer): extract_cycle then walks serially.
__device__ int lap_cycle_list(const BfParams& p, int v0, int* nodes, long long* offs, long long* total) {
    long long off = 0;
    int x = v0;
    for (int j = 0; j < p.n; ++j) {
        nodes[j] = x;
        offs[j] = off;
        off += __ldcg(p.lapSteps + x);
        x = __ldcg(p.lapNext + x);
        if (x < 0 || off > p.cycleCap) return -1;
        if (x == v0) {
            *total = off;
            return j + 1;
        }
    }
    return -1;
}

// Lap j of a parallel extract_cycle: len predecessor steps from x, written
// from cycleBuf[off] on.  The lap must stay off layer-0 start nodes until its
// last step, which must reach xNext; otherwise (or when a predecessor leaves
// the node range) it returns non-zero and the serial walk decides.
__device__ int walk_lap(const BfParams& p, int x, int xNext, long long off, long long len) {
    const long long total = (long long)p.n * (p.nY + 1) * p.K;
    int pr = x;
    for (long long s = 0; s < len; ++s) {
        pr = __ldcg(p.pred + pr);
        if (pr < 0 || pr >= total) return 1;
        if (pr < p.n && s + 1 < len) return 2;
        p.cycleBuf[off + s] = original_index(p.n, p.K, pr);
    }
    return pr == xNext ? 0 : 2;
}

// Upper-bound path (cost_time_ratio_solver.cpp:370-397): from the closing
// copy of the start node back to the start node.
__device__ int extract_ub_path(const BfParams& p, int start) {
    const int n = p.n, K = p.K;
    const long long total = (long long)n * (p.nY + 1) * K;
    const long long maxLength = (long long)p.nY * K;
    const long long firstV = start + (long long)n * p.nY * K;
    int len = 0;
    p.cycleBuf[len++] = original_index(n, K, (int)firstV);
    int pr = __ldcg(p.pred + firstV);
    p.cycleBuf[len++] = (pr >= 0 && pr < total) ? original_index(n, K, pr) : -1;
    for (long long kk = maxLength - 1; kk > 0; --kk) {
        if (pr == -1) break;
        if (pr < 0 || pr >= total) return BF_ERR_WALK;
        pr = __ldcg(p.pred + pr);
        if (len >= p.cycleCap) return BF_ERR_CYCLE_CAP;
        p.cycleBuf[len++] = (pr >= 0 && pr < total) ? original_index(n, K, pr) : -1;
        if (pr == start) break;
    }
    p.ctl->cycleLen = len;
    return BF_UB_DONE;
}

// Start vertex of the minimum-cost path that closes at v, by the reference's
// walk (dijkstra_solver.cpp:349-357): follow predecessors from the closing
// copy of v until -1; the last node reached is the start.  Used when the
// closing copy was not reached in this sweep (odd layer counts read their
// lower bound from another row), so its predecessor chain is older.
__device__ int dij_walk_end(const BfParams& p, int v) {
    const int n = p.n, K = p.K;
    const long long total = (long long)n * (p.nY + 1) * K;
    const long long vLast = v + (long long)n * p.nY * K;
    int pr = __ldcg(p.pred + vLast);
    if (pr < 0 || pr >= total) return -1;
    int last = original_index(n, K, pr);
    for (long long kk = (long long)p.nY * K; kk > 0; --kk) {
        pr = __ldcg(p.pred + pr);
        if (pr == -1) break;
        if (pr < 0 || pr >= total) return -1;
        last = original_index(n, K, pr);
    }
    return last;
}

}  // namespace

// ---------------------------------------------------------------------------
// One Bellman-Ford call by a team of CTAs, from its set-up to its verdict in
// p.ctl.  t.cta is the CTA's index in the team: the grid of a single-graph
// launch, or one CTA of a batched launch that solves many graphs.  `smem` is
// the dynamic shared memory after the DP tables: [row offsets and lists of
// slices with rows][two step buffers].
// ---------------------------------------------------------------------------
template <class CT, int TK, bool S, bool TREE = false>
__device__ __forceinline__ void bf_body(const BfParams& p, const Team& t, char* smem) {
    const int n = p.n, K = p.K, Kp = p.Kp;
    const long long tid = t.thread(), nth = t.nthreads();
    const bool isLead = (t.cta == 0 && threadIdx.x == 0);
    const int s0 = __ldg(p.ctaSlice + t.cta), s1 = __ldg(p.ctaSlice + t.cta + 1);
    const bool handoff = t.ncta > 1 && p.flagSync;
    if (handoff && threadIdx.x == 0) p.stepDone[(size_t)t.cta * kStepDoneStride] = 0;
    // shared memory: [row offsets of both parts][slices with rows, per part]
    // [step buffer 0][step buffer 1]
    __shared__ unsigned long long stageBar[2];
    __shared__ int nActive[2];
    Stage st;
    {
        int* spl0 = reinterpret_cast<int*>(smem);
        int* spl1 = spl0 + p.maxCtaSlices + 1;
        int* act0 = spl1 + p.maxCtaSlices + 1;
        int* act1 = act0 + p.maxCtaSlices;
        for (int i = threadIdx.x; i <= s1 - s0; i += blockDim.x) {
            spl0[i] = __ldg(p.spInter + s0 + i);
            spl1[i] = __ldg(p.spIntra + s0 + i);
        }
        __syncthreads();
        if (threadIdx.x < 32) {
            // stream compaction by warp 0: the slices with rows, in order
            const int lane = threadIdx.x;
            for (int part = 0; part < 2; ++part) {
                const int* spl = part ? spl1 : spl0;
                int* act = part ? act1 : act0;
                int base = 0;
                for (int i0 = 0; i0 < s1 - s0; i0 += 32) {
                    const int i = i0 + lane;
                    const bool a = i < s1 - s0 && spl[i + 1] > spl[i];
                    const unsigned m = __ballot_sync(0xffffffffu, a);
                    if (a) act[base + __popc(m & ((1u << lane) - 1u))] = i;
                    base += __popc(m);
                }
                if (lane == 0) nActive[part] = base;
            }
        }
        st.splInter = spl0;
        st.splIntra = spl1;
        st.actInter = act0;
        st.actIntra = act1;
        st.costBytes = sizeof(CT);
        st.timeBytes = TK == 1 ? 4 : TK == 2 ? 8 : 0;
        st.rowCap = p.rowCap;
        st.srcOnly = p.stageSrcOnly != 0;
        st.spin = p.spinLimit;
        const size_t bufBytes =
            bf_stage_buffer_bytes(p.rowCap, st.srcOnly ? 0 : st.costBytes, st.srcOnly ? 0 : st.timeBytes);
        st.buf0 = smem + bf_stage_offset(p.maxCtaSlices);
        st.buf1 = st.buf0 + bufBytes;
        st.bar = stageBar;
        st.phase = 0;
        st.pending = 0;
        if (threadIdx.x == 0) {
            mbar_init(stageBar);
            mbar_init(stageBar + 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __syncthreads();
        st.nActInter = nActive[0];
        st.nActIntra = nActive[1];
    }

    // set-up (cost_time_ratio_solver.cpp:264-287): DP := inf, branch starts := 0
    // (each record is written once, by one thread)
    for (long long r = tid; r < 2LL * n * Kp; r += nth) {
        const long long node = (r / Kp) % n;
        const bool start = r < (long long)n * Kp && r % Kp == 0 && __ldcg(p.branchOf + node) == p.branchId;
        p.dv[r] = start ? 0.0 : kInfD;
        p.doh[r] = make_int2(kLapUnknown, 0);  // every (origin, hops) word, in either layout
    }
    for (long long i = tid; i < n; i += nth) {
        p.bak[i] = kInfD;
        if (__ldcg(p.branchOf + i) == p.branchId) p.pred[i] = -1;
    }
    {
        // branch size and the last branch node (the reference's indexNodeInLayer)
        int last = -1, cnt = 0;
        for (long long i = tid; i < n; i += nth)
            if (__ldcg(p.branchOf + i) == p.branchId) { ++cnt; last = (int)i; }
        Key km{-(double)last, last < 0 ? 0x7fffffff : last};
        if (last < 0) km.v = 1.0;
        km = block_min(km, 0);
        if (threadIdx.x == 0) p.redIdx[t.cta] = km.i;
        for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        __shared__ int scnt;
        if (threadIdx.x == 0) scnt = 0;
        __syncthreads();
        if ((threadIdx.x & 31) == 0) atomicAdd(&scnt, cnt);
        __syncthreads();
        if (threadIdx.x == 0) p.redAux[t.cta] = scnt;
    }
    if (!team_sync(t)) return;
    if (isLead) {
        int total = 0, last = -1;
        for (int c = 0; c < t.ncta; ++c) {
            total += __ldcg(p.redAux + c);
            const int ri = __ldcg(p.redIdx + c);
            if (ri != 0x7fffffff && ri > last) last = ri;
        }
        p.ctl->numInBranch = total;
        p.ctl->indexNodeInLayer = last;
        p.ctl->sweeps = 0;
        p.ctl->status = total == 0 ? BF_ERR_EMPTY_BRANCH : BF_RUNNING;
    }
    if (!team_sync(t)) return;
    if (*(volatile int*)&p.ctl->status != BF_RUNNING) return;

    const int epochBase = p.ctl->epoch;  // read by all before anyone advances it
    if (!team_sync(t)) return;
    const int lastRow = p.nY % 2;
    const int lastPar = lastRow / K, lastDepth = lastRow % K;
    const long long numNodes = p.numNodes;
    int sweep = 0;
    unsigned step = 0;
    // Without intralayer edges (pruned graphs) the depth steps 1..K-1 relax
    // nothing: every record they would write is +inf and stays +inf (layer 0's
    // too: no edge ever reaches its depths >= 1), and the origins they would
    // write are never read (an unreached source never wins).  Only the
    // interlayer step of each layer runs.
    const int kSteps = p.intraEntries == 0 ? 1 : K;
    for (;;) {
        // the first step of the sweep is staged while the backup row is copied
        stage_issue(p, st, s0, s1, 0, kSteps > 1 ? 0 : 1, kSteps > 1 ? 1 : 0);
        for (long long i = tid; i < n; i += nth) p.bak[i] = ldV<S>(p, (size_t)i * Kp);
        if (!team_sync(t)) { stage_drain(st); return; }
        // Layers are relaxed in order; a CTA hands each step off to its
        // graph neighbours only (one team barrier closes the sweep).  The
        // reference stops a sweep at the first layer 1..nY-1 without an
        // improved node; every later layer then stays unreached (all
        // infinite, no predecessor written), so the layers run to the end and
        // the stop is decided from the per-layer stamps after the sweep.
        const int stamp = epochBase + sweep + 1;
        const unsigned long long tRelax = isLead ? clock64() : 0;
        unsigned long long cycRelax = 0, cycHand = 0, cycStage = 0;
        int sb = 0;  // buffer of the current step
        for (int l = 0; l <= p.nY; ++l) {
            for (int k = 0; k < kSteps; ++k) {
                if (l == 0 && k == 0) continue;
                const unsigned long long ta = isLead ? clock64() : 0;
                if (!stage_wait(st, sb)) {
                    atomicExch(t.err, 1);
                    stage_drain(st);
                    return;
                }
                if (isLead) cycStage += clock64() - ta;
                const bool last = l == p.nY && k == kSteps - 1;
                if (!last) stage_issue(p, st, s0, s1, sb ^ 1, k + 1 < kSteps ? l : l + 1, k + 1 < kSteps ? k + 1 : 0);
                const bool any = relax_step<CT, TK, S, TREE>(p, st, sb, s0, s1, l, k);
                if (__any_sync(0xffffffffu, any) && (threadIdx.x & 31) == 0) p.layerFlag[l] = stamp;
                const unsigned long long tb = isLead ? clock64() : 0;
                ++step;
                sb ^= 1;
                const bool ok = (handoff && !last) ? step_handoff(p, t, step) : team_sync(t);
                if (!ok) {
                    stage_drain(st);
                    return;
                }
                if (isLead) {
                    const unsigned long long tc = clock64();
                    cycRelax += tb - ta;
                    cycHand += tc - tb;
                }
            }
        }
        int stopHere = 0;
        for (int l = 1 + (int)threadIdx.x; l < p.nY; l += blockDim.x)
            if (*(volatile int*)(p.layerFlag + l) != stamp) stopHere = 1;
        const bool stop = __syncthreads_or(stopHere) != 0;
        ++sweep;
        const unsigned long long tTail = isLead ? clock64() : 0;
        if (isLead) {
            p.ctl->cycPhaseA += cycRelax;
            p.ctl->cycSync += cycHand;
            p.ctl->cycStage += cycStage;
            p.ctl->cycPhaseB += tTail - tRelax - cycRelax - cycHand;
        }
        if (stop) {
            if (isLead) { p.ctl->status = BF_LAYER_UNREACHED; p.ctl->sweeps = sweep; p.ctl->epoch = epochBase + sweep; }
            return;
        }
        if (p.mode == 1) {
            if (isLead) {
                p.ctl->status = extract_ub_path(p, p.ctl->indexNodeInLayer);
                p.ctl->sweeps = sweep;
                p.ctl->epoch = epochBase + sweep;
            }
            return;
        }
        const size_t lastRowBase = (size_t)lastPar * n * Kp + lastDepth;
        if (p.mode == 2) {
            // minimum-cost verdict: lower bounds of the branch nodes, origin of
            // their closing path, first and first-valid candidates.
            Key first{kInfD, 0x7fffffff}, firstValid{kInfD, 0x7fffffff};
            int anyFinite = 0;
            const size_t dRow = (size_t)(p.nY & 1) * n * Kp;
            for (long long i = tid; i < n; i += nth) {
                if (__ldcg(p.branchOf + i) != p.branchId) { p.lbOut[i] = kInfD; p.originOut[i] = -1; continue; }
                const double lb = ldV<S>(p, lastRowBase + (size_t)i * Kp);
                int o = ldOH<S>(p, dRow, (int)i, 0).x;
                if (o < 0 && !isinf((float)lb)) o = dij_walk_end(p, (int)i);
                p.lbOut[i] = lb;
                p.originOut[i] = o;
                if (!isinf(lb)) anyFinite = 1;
                Key kk{lb, (int)i};
                if (key_less(kk, first)) first = kk;
                if (o == (int)i && !isinf((float)lb) && key_less(kk, firstValid)) firstValid = kk;
            }
            first = block_min(first, 0);
            firstValid = block_min(firstValid, 1);
            anyFinite = __syncthreads_or(anyFinite);
            if (threadIdx.x == 0) {
                p.redVal[2 * t.cta] = first.v;
                p.redIdx[2 * t.cta] = first.i;
                p.redVal[2 * t.cta + 1] = firstValid.v;
                p.redIdx[2 * t.cta + 1] = firstValid.i;
                p.redAux[t.cta] = anyFinite;
            }
            if (!team_sync(t)) return;
            if (isLead) {
                Key f{kInfD, 0x7fffffff}, fv{kInfD, 0x7fffffff};
                int af = 0;
                for (int c = 0; c < t.ncta; ++c) {
                    Key a{__ldcg(p.redVal + 2 * c), __ldcg(p.redIdx + 2 * c)};
                    Key b{__ldcg(p.redVal + 2 * c + 1), __ldcg(p.redIdx + 2 * c + 1)};
                    if (key_less(a, f)) f = a;
                    if (key_less(b, fv)) fv = b;
                    af |= __ldcg(p.redAux + c);
                }
                p.ctl->firstLb = f.v;
                p.ctl->firstV = f.i == 0x7fffffff ? -1 : f.i;
                p.ctl->firstOrigin = f.i == 0x7fffffff ? -1 : __ldcg(p.originOut + f.i);
                p.ctl->validLb = fv.v;
                p.ctl->validV = fv.i == 0x7fffffff ? -1 : fv.i;
                p.ctl->anyFinite = af;
                p.ctl->status = BF_SWEEP_DONE;
                p.ctl->sweeps = sweep;
                p.ctl->epoch = epochBase + sweep;
            }
            return;
        }

        // wrap-around (cost_time_ratio_solver.cpp:399-417) and lap function
        {
            int improved = 0;
            const size_t wRow = (size_t)((p.nY - 1) & 1) * n * Kp;
            const long long layerSpan = (long long)n * K;
            for (long long i = tid; i < n; i += nth) {
                if (__ldcg(p.branchOf + i) == p.branchId) {
                    const double cand = ldV<S>(p, lastRowBase + (size_t)i * Kp);
                    const double b = p.bak[i];
                    double* d0 = p.dv + (size_t)i * Kp;
                    if (cand < b) {
                        improved = 1;
                        *d0 = cand;
                        p.pred[i] = __ldcg(p.pred + (size_t)p.nY * layerSpan + i);
                    } else {
                        *d0 = b;
                    }
                }
                const int pe = p.pred[i];
                int nx = kLapEnd, st = 0;
                if (pe != -1) {
                    const long long lp = pe / layerSpan;
                    const long long rem = pe - lp * layerSpan;
                    const int kp = (int)(rem / n), wv = (int)(rem - (long long)kp * n);
                    if (pe < 0 || lp != p.nY - 1) {
                        nx = kLapUnknown;
                    } else {
                        const int2 w = ldOH<S>(p, wRow, wv, kp);
                        nx = w.x;
                        st = 1 + w.y;
                    }
                }
                p.lapNext[i] = nx;
                p.lapSteps[i] = st;
            }
            bool ok;
            improved = team_sync_or(t, improved, ok);
            if (isLead) atomicAdd(&p.ctl->cycWrap, clock64() - tTail);
            if (!ok) return;
            if (!improved) {
                if (isLead) { p.ctl->status = BF_WRAP_NO_IMPROVE; p.ctl->sweeps = sweep; p.ctl->epoch = epochBase + sweep; }
                return;
            }
        }

        // candidates (cost_time_ratio_solver.cpp:431-489)
        {
            Key bestOk{kInfD, 0x7fffffff}, firstUnknown{kInfD, 0x7fffffff};
            const long long limit = numNodes - 1;
            long long decided = 0;
            for (long long i = tid; i < n; i += nth) {
                int st = 0;
                if (__ldcg(p.branchOf + i) == p.branchId) {
                    const double d0 = ldV<S>(p, (size_t)i * Kp);
                    if (d0 < 0) {
                        int v0 = -1;
                        long long steps = 0;
                        st = p.literalAll ? 3 : lap_walk(p, (int)i, limit, &v0, &steps);
                        p.candV0[i] = v0;
                        p.candSteps[i] = steps;
                        ++decided;
                        Key kk{d0, (int)i};
                        if (st == 1 && key_less(kk, bestOk)) bestOk = kk;
                        if (st == 3 && key_less(kk, firstUnknown)) firstUnknown = kk;
                    }
                }
                p.candStat[i] = st;
            }
            bestOk = block_min(bestOk, 0);
            firstUnknown = block_min(firstUnknown, 1);
            for (int o = 16; o > 0; o >>= 1) decided += __shfl_xor_sync(0xffffffffu, decided, o);
            __shared__ unsigned long long sdec;
            if (threadIdx.x == 0) sdec = 0;
            __syncthreads();
            if ((threadIdx.x & 31) == 0) atomicAdd(&sdec, (unsigned long long)decided);
            __syncthreads();
            if (threadIdx.x == 0) {
                p.redVal[2 * t.cta] = bestOk.v;
                p.redIdx[2 * t.cta] = bestOk.i;
                p.redVal[2 * t.cta + 1] = firstUnknown.v;
                p.redIdx[2 * t.cta + 1] = firstUnknown.i;
                p.redAux64[t.cta] = (long long)sdec;
            }
        }
        __shared__ int sLaps, sBad;
        __shared__ long long sCycLen;
        __shared__ Key sOk, sUnk;
        const unsigned long long tCand = isLead ? clock64() : 0;
        if (!team_sync(t)) return;
        // Every CTA reads the team's best decided candidate and its first
        // undecided one.  Undecided candidates that precede the best decided
        // one are walked literally, all at once, in bounded rounds; then the
        // smallest (value, index) candidate whose walk repeats wins, which is
        // what the reference's walks in ascending order choose.
        if (threadIdx.x == 0) {
            Key ok{kInfD, 0x7fffffff}, unk{kInfD, 0x7fffffff};
            for (int c = 0; c < t.ncta; ++c) {
                Key a{__ldcg(p.redVal + 2 * c), __ldcg(p.redIdx + 2 * c)};
                Key b{__ldcg(p.redVal + 2 * c + 1), __ldcg(p.redIdx + 2 * c + 1)};
                if (key_less(a, ok)) ok = a;
                if (key_less(b, unk)) unk = b;
            }
            sOk = ok;
            sUnk = unk;
        }
        __syncthreads();
        Key ok = sOk;
        const Key unk = sUnk;
        if (unk.i != 0x7fffffff && (ok.i == 0x7fffffff || key_less(unk, ok))) {
            int started = 0;
            for (long long i = tid; i < n; i += nth) {
                if (__ldcg(p.candStat + i) != 3) continue;
                const Key kk{ldV<S>(p, (size_t)i * Kp), (int)i};
                if (!key_less(kk, ok)) {
                    p.candStat[i] = 0;  // follows the best decided candidate: never reached
                    continue;
                }
                walk_start(p, (int)i);
                ++started;
            }
            for (int o = 16; o > 0; o >>= 1) started += __shfl_xor_sync(0xffffffffu, started, o);
            if ((threadIdx.x & 31) == 0 && started) atomicAdd(&p.ctl->fallbackWalks, started);
            for (int round = 0;; ++round) {
                int pending = 0;
                for (long long i = tid; i < n; i += nth)
                    if (__ldcg(p.candStat + i) == 3 && !walk_advance(p, (int)i, kWalkRoundLoads)) pending = 1;
                bool good;
                pending = team_sync_or(t, pending, good);
                if (!good) return;
                if (isLead) p.ctl->walkRounds = round + 1;
                if (!pending) break;
            }
            Key best{kInfD, 0x7fffffff};
            for (long long i = tid; i < n; i += nth) {
                if (__ldcg(p.candStat + i) != 1) continue;
                const Key kk{ldV<S>(p, (size_t)i * Kp), (int)i};
                if (key_less(kk, best)) best = kk;
            }
            best = block_min(best, 0);
            if (threadIdx.x == 0) {
                p.redVal[2 * t.cta] = best.v;
                p.redIdx[2 * t.cta] = best.i;
            }
            if (!team_sync(t)) return;
            if (isLead) {
                ok = Key{kInfD, 0x7fffffff};
                for (int c = 0; c < t.ncta; ++c) {
                    Key a{__ldcg(p.redVal + 2 * c), __ldcg(p.redIdx + 2 * c)};
                    if (key_less(a, ok)) ok = a;
                }
            }
        }
        const unsigned long long tLead = isLead ? clock64() : 0;
        if (isLead) atomicAdd(&p.ctl->cycCand, tLead - tCand);
        int finished = 0;
        if (isLead) {
            long long dec = 0;
            for (int c = 0; c < t.ncta; ++c) dec += __ldcg(p.redAux64 + c);
            p.ctl->candidates += dec;
            int winner = -1, v0 = -1;
            long long steps = 0;
            if (ok.i != 0x7fffffff) {
                winner = ok.i;
                v0 = __ldcg(p.candV0 + winner);
                steps = __ldcg(p.candSteps + winner);
            }
            sLaps = 0;
            if (winner >= 0) {
                p.ctl->v0 = v0;
                p.ctl->cLength = steps;
                p.ctl->candidateVi = winner;
                // A cycle of many laps is one long chain of dependent
                // predecessor loads; its laps are walked side by side by
                // CTA 0 (lap nodes and offsets in the candidate arrays, which
                // are not read again in this launch).
                long long total = 0;
                const int laps = lap_cycle_list(p, v0, p.candV0, p.candSteps, &total);
                if (laps > 0) {
                    sLaps = laps;
                    sCycLen = total;
                } else {
                    p.ctl->status = extract_cycle(p, v0, steps);
                }
            } else if (sweep >= numNodes - 1 || (p.maxSweeps > 0 && sweep >= p.maxSweeps)) {
                p.ctl->status = BF_MAX_SWEEPS;
            }
        }
        if (t.cta == 0) {
            __syncthreads();
            const int laps = sLaps;
            if (laps > 0) {
                if (threadIdx.x == 0) sBad = 0;
                __syncthreads();
                for (int j = (int)threadIdx.x; j < laps; j += blockDim.x) {
                    const long long o0 = __ldcg(p.candSteps + j);
                    const long long o1 = j + 1 < laps ? __ldcg(p.candSteps + j + 1) : sCycLen;
                    const int xn = __ldcg(p.candV0 + (j + 1 < laps ? j + 1 : 0));
                    if (walk_lap(p, __ldcg(p.candV0 + j), xn, o0, o1 - o0) != 0) sBad = 1;
                }
                __syncthreads();
                if (isLead) {
                    if (sBad) {
                        p.ctl->status = extract_cycle(p, p.ctl->v0, p.ctl->cLength);
                    } else {
                        p.ctl->cycleLen = (int)sCycLen;
                        p.ctl->status = BF_FOUND_CYCLE;
                    }
                }
            }
        }
        if (isLead) {
            p.ctl->sweeps = sweep;
            p.ctl->epoch = epochBase + sweep;
            finished = p.ctl->status != BF_RUNNING;
            atomicAdd(&p.ctl->cycLead, clock64() - tLead);
        }
        bool tailOk;
        finished = team_sync_or(t, finished, tailOk);
        if (isLead) atomicAdd(&p.ctl->cycTail, clock64() - tTail);
        if (!tailOk || finished) return;
    }
}

// The Bellman-Ford launch of one graph.  Every CTA of the grid belongs to
// its team.  Dynamic shared memory: [DP tables + backup row, if S][the
// body's stage memory].
template <class CT, int TK, bool S>
__global__ void __launch_bounds__(kBfThreads, 1) bf_kernel(BfParams p) {
    const Team t{(int)blockIdx.x, (int)gridDim.x, &p.ctl->barCount, &p.ctl->barGen, &p.ctl->error, p.spinLimit};
    extern __shared__ double4 smemRaw[];
    char* smem = reinterpret_cast<char*>(smemRaw);
    if constexpr (S) {
        // single-CTA team: the DP records and the backup row live in shared
        // memory for the whole launch (layout as in global memory)
        p.dv = reinterpret_cast<double*>(smem);
        p.doh = reinterpret_cast<int2*>(smem + (size_t)2 * p.n * p.Kp * sizeof(double));
        p.bak = reinterpret_cast<double*>(smem + (size_t)2 * p.n * p.Kp * (sizeof(double) + sizeof(int2)));
        smem += bf_shared_table_bytes(p.n, p.Kp);
    }
    bf_body<CT, TK, S>(p, t, smem);
}

// Minimum-cost path extraction (dijkstra_solver.cpp:349-357): from the
// closing copy of v back to the start node.  Writes original ids in walk
// order; returns the count through ctl->cycleLen.
__global__ void extract_path_kernel(BfParams p, int v) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const int n = p.n, K = p.K;
    const long long total = (long long)n * (p.nY + 1) * K;
    const long long maxLen = (long long)p.nY * K;
    const long long vLast = v + (long long)n * p.nY * K;
    int len = 0;
    int pr = __ldcg(p.pred + vLast);
    if (pr < 0 || pr >= total) { p.ctl->status = BF_ERR_WALK; return; }
    p.cycleBuf[len++] = original_index(n, K, pr);
    for (long long kk = maxLen; kk > 0; --kk) {
        pr = __ldcg(p.pred + pr);
        if (pr == -1) break;
        if (pr < 0 || pr >= total) { p.ctl->status = BF_ERR_WALK; return; }
        if (len >= p.cycleCap) { p.ctl->status = BF_ERR_CYCLE_CAP; return; }
        p.cycleBuf[len++] = original_index(n, K, pr);
    }
    p.ctl->cycleLen = len;
}

// The first in-edge of target T whose source is S (original ids; T >=
// numNodes denotes the closing layer), as computeRatioForCycle's lookup does
// (cost_time_ratio_solver.cpp:103-122): its edge id and the double cost and
// time of that edge.  Returns false when there is none.
__device__ bool lookup_edge(const LookupArgs& a, long long S, long long T, long long* edge, double* c, double* t) {
    if (S < 0 || T < 0) return false;
    const int lt = (int)(T / a.n), v = (int)(T % a.n);
    const int ls = (int)(S / a.n), s = (int)(S % a.n);
    if (lt > a.nY) return false;
    int part;
    const int* src;
    const int* sp;
    const int* ted;
    long long block;
    if (lt == a.nY) {
        if (ls != a.nY - 1) return false;
        part = 0; src = a.srcDummy; sp = a.spInter; ted = a.tedgeInter; block = a.nY - 1;
    } else if (ls == lt) {
        part = 1; src = a.srcIntra; sp = a.spIntra; ted = a.tedgeIntra; block = lt;
    } else if (lt >= 1 && ls == lt - 1) {
        part = 0; src = a.srcInter; sp = a.spInter; ted = a.tedgeInter; block = lt - 1;
    } else {
        return false;
    }
    const int slice = v >> 5, lane = v & 31;
    for (int j = sp[slice]; j < sp[slice + 1]; ++j) {
        const long long e = (long long)j * 32 + lane;
        if (src[e] == s) {
            const long long off = (long long)lt * a.layerStride + (part ? a.interEntries : 0) + e;
            *edge = block * a.eBlock + ted[e];
            *c = a.c32 ? (double)a.c32[off] : a.c64[off];
            *t = a.t32 ? (double)a.t32[off] : a.t64 ? a.t64[off] : a.tconst;
            return true;
        }
    }
    return false;
}

// lookup_edge for each (source, target) pair of a cycle; edge -2 when absent.
__global__ void lookup_pairs_kernel(LookupArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.count) return;
    long long e = -2;
    double c = 0, t = 0;
    if (!lookup_edge(a, a.pairSrc[i], a.pairTrgt[i], &e, &c, &t)) e = -2, c = 0, t = 0;
    a.edgeOut[i] = e;
    a.cOut[i] = c;
    a.tOut[i] = t;
}

// ---------------------------------------------------------------------------
// Batched ratio solves.  Each CTA takes graphs from a queue and runs the
// host driver's ratio solve on the device for each: the initial upper bound
// (cost_time_ratio_solver.cpp:652-707), the Lawler iterations (:558-635)
// with their Bellman-Ford calls as one-CTA teams, and the cycle evaluations
// (computeRatioForCycle, :88-133) in the same double operations and order as
// the host.  The first branch's Lawler result is the solve's result unless
// its cycle wraps (:840-850); then the host takes the graph over with branch
// and bound, and the device's work on it only cost time.
// ---------------------------------------------------------------------------
namespace {

// (int)std::round(x) as x86-64 computes it: out of range or NaN gives INT_MIN.
__device__ __forceinline__ int round_to_int_x86(double x) {
    const double r = round(x);  // half away from zero, as std::round
    if (!(r >= -2147483648.0 && r <= 2147483647.0)) return (int)0x80000000;
    return (int)r;
}
__device__ __forceinline__ double via_float(double x) { return (double)__double2float_rn(x); }

struct CycleSums {
    double ratio, wsum;
};

// computeRatioForCycle's sums over a stored cycle record, one thread, in the
// cycle's order: C += c, T += t, W += c - lambda * t, each a rounded double
// operation.
__device__ CycleSums record_sums(const PairJob& J, int rec, int m, double lambda) {
    const double* c = J.recC[rec];
    const double* t = J.recT[rec];
    double C = 0, T = 0, W = 0;
    for (int i = 0; i < m; ++i) {
        const double ci = __ldcg(c + i), ti = __ldcg(t + i);
        C = __dadd_rn(C, ci);
        T = __dadd_rn(T, ti);
        W = __dadd_rn(W, __dsub_rn(ci, __dmul_rn(lambda, ti)));
    }
    return {__ddiv_rn(C, T), W};
}

// The CTAs that solve one graph together: `all` is the whole team, with
// its own barrier words; `bf` is its first bf.ncta CTAs, the Bellman-Ford
// team the graph was prepared for (a graph with fewer 32-node slices than
// the team has CTAs uses fewer), with the graph's Control barrier words.
// The other CTAs skip the Bellman-Ford calls and wait at the next barrier.
struct SolveTeam {
    Team all, bf;
    __device__ bool lead() const { return all.cta == 0 && threadIdx.x == 0; }
    __device__ bool in_bf() const { return all.cta < bf.ncta; }
};

// A cycle from the Bellman-Ford walk in the cycle buffer (p(v0), ..., v0,
// or the upper-bound path) into record `rec`: the walk reversed, closed with
// the copy of its first node when `close`, and every consecutive pair's edge,
// cost and time (a closing-layer target is its copy: b + numNodes when
// b < n < a, cost_time_ratio_solver.cpp:109-111).  All threads of the team;
// returns the edge count, -1 when an edge is missing, -2 when the record is
// too small, -3 when a team barrier ran out.
__device__ int record_cycle(const PairJob& J, const BfParams& P, const Team& t, int rec, int len, bool close) {
    const int count = len + (close ? 1 : 0);
    if (count > J.cap + 1 || len < 1) return -2;
    int* nodes = J.recNodes[rec];
    const long long nn = P.numNodes;
    const int n = P.n;
    for (long long i = t.thread(); i < len; i += t.nthreads()) nodes[i] = __ldcg(P.cycleBuf + (len - 1 - i));
    if (close && t.cta == 0 && threadIdx.x == 0) nodes[len] = __ldcg(P.cycleBuf + (len - 1)) + (int)nn;
    if (!team_sync(t)) return -3;
    const int m = count - 1;
    int missing = 0;
    for (long long i = t.thread(); i < m; i += t.nthreads()) {
        const int a = __ldcg(nodes + i);
        long long b = __ldcg(nodes + i + 1);
        if (b < n && a > n) b += nn;
        long long e;
        double c, tm;
        if (!lookup_edge(J.lk, a, b, &e, &c, &tm)) {
            missing = 1;
            e = -2, c = 0, tm = 0;
        }
        J.recEdges[rec][i] = e;
        J.recC[rec][i] = c;
        J.recT[rec][i] = tm;
    }
    bool ok;
    const int anyMissing = team_sync_or(t, missing, ok);
    if (!ok) return -3;
    return anyMissing ? -1 : m;
}

// Lawler's outcome of one Bellman-Ford call (the host driver's bellman_ford).
enum Outcome { OUT_FOUND = 0, OUT_NONE = 1, OUT_ZERO = 2 };

template <class CT, int TK>
__device__ __noinline__ void bf_call(const BfParams& P, const Team& t, char* smem) {
    bf_body<CT, TK, false, true>(P, t, smem);
}

// One Bellman-Ford call of the team: the lead publishes the call's state,
// the Bellman-Ford CTAs run it, and every CTA reads its verdict after the
// closing barrier.  False when a team barrier ran out.
template <class CT, int TK>
__device__ bool team_bf_call(PairJob& J, const BfParams& P, const SolveTeam& S, char* smem, bool resetError) {
    if (S.lead()) {
        P.ctl->status = BF_RUNNING;
        if (resetError) P.ctl->error = 0;
    }
    if (!team_sync(S.all)) return false;
    if (S.in_bf()) bf_call<CT, TK>(P, S.bf, smem);
    if (!team_sync(S.all)) return false;
    if (S.lead()) {
        J.bfCalls++;
        J.sweeps += *(volatile int*)&P.ctl->sweeps;
    }
    return true;
}

// The whole ratio solve of one graph by the team.  P is the job's
// Bellman-Ford parameters in each CTA's shared memory.  Work over nodes and
// cycle edges is spread over the team's threads; the sums over a cycle run on
// one thread of every CTA, in the same order, so every CTA takes the same
// branches; only the lead writes the job's outputs.
template <class CT, int TK>
__device__ void pair_solve(PairJob& J, BfParams& P, const SolveTeam& S, char* smem) {
    __shared__ int sState[4];        // [1] the bound search gave up, [3] edges of the last record
    __shared__ double sRatio;
    const Team& t = S.all;
    const bool lead = S.lead();
    const int n = P.n;
    Control* ctl = P.ctl;
    const double tolerance = (double)(float)1e-8;
    const double ubInf = (double)__int_as_float(0x7f800000);
#define PGC_TEAM_FAIL()                                \
    do {                                               \
        if (lead) J.status = PAIR_ERR_WAIT;            \
        return;                                        \
    } while (0)

    // ---- initial upper bound (cost_time_ratio_solver.cpp:652-707) ----
    // the layer-1 node with the lowest float mean in-cost among those with
    // more than three in-edges, first in index order (node 0 if none)
    Key best{kInfD, 0x7fffffff};
    {
        const CT* c1 = reinterpret_cast<const CT*>(P.cost) + P.layerStride;
        for (long long vv = t.thread(); vv < n; vv += t.nthreads()) {
            const int v = (int)vv;
            const int s = v >> 5, lane = v & 31;
            float mean = 0;
            int num = 0;
            for (int j = __ldg(P.spInter + s); j < __ldg(P.spInter + s + 1); ++j) {
                const long long e = (long long)j * 32 + lane;
                if (__ldg(P.srcInter + e) < 0) continue;
                mean = (float)((double)mean + (double)c1[e]);
                ++num;
            }
            for (int j = __ldg(P.spIntra + s); j < __ldg(P.spIntra + s + 1); ++j) {
                const long long e = (long long)j * 32 + lane;
                if (__ldg(P.srcIntra + e) < 0) continue;
                mean = (float)((double)mean + (double)c1[P.interEntries + e]);
                ++num;
            }
            mean = mean / (float)num;
            const Key k{(double)mean, v};
            if (num > 3 && mean < __int_as_float(0x7f800000) && key_less(k, best)) best = k;
        }
        best = block_min(best, 0);
        if (t.ncta > 1) {
            // (value, index) keys are totally ordered: the team's minimum is
            // the one-CTA scan's, however the nodes were split
            if (threadIdx.x == 0) {
                P.redVal[t.cta] = best.v;
                P.redIdx[t.cta] = best.i;
            }
            if (!team_sync(t)) PGC_TEAM_FAIL();
            best = Key{kInfD, 0x7fffffff};
            for (int c = 0; c < t.ncta; ++c) {
                const Key k{__ldcg(P.redVal + c), __ldcg(P.redIdx + c)};
                if (key_less(k, best)) best = k;
            }
        }
    }
    const int startV = best.i == 0x7fffffff ? 0 : best.i;
    for (long long v = t.thread(); v < n; v += t.nthreads()) J.branchOf[v] = v == startV ? 0 : 1;
    if (threadIdx.x == 0) {
        P.mode = 1;
        P.branchId = 0;
        P.lambda = 10;
        P.ub = ubInf;
    }
    if (!team_bf_call<CT, TK>(J, P, S, smem, true)) PGC_TEAM_FAIL();
    if (*(volatile int*)&ctl->error) PGC_TEAM_FAIL();
    {
        const int st = *(volatile int*)&ctl->status;
        if (st == BF_LAYER_UNREACHED) {  // the empty cycle's 0/0 bound: (true, NaN, no rows)
            if (lead) J.status = PAIR_NAN;
            return;
        }
        if (st != BF_UB_DONE) {
            if (lead) {
                J.status = st < 0 ? PAIR_ERR_BF : PAIR_ERR_UB;
                J.bfStatus = st;
            }
            return;
        }
    }
    int neg = 0;
    {
        const int m = record_cycle(J, P, t, neg, *(volatile int*)&ctl->cycleLen, false);
        if (m == -3) PGC_TEAM_FAIL();
        if (m < 0) {
            if (lead) J.status = m == -2 ? PAIR_HOST : PAIR_ERR_EDGE;
            return;
        }
        if (threadIdx.x == 0) {
            sState[3] = m;
            double lambda = 10;
            CycleSums ev = record_sums(J, neg, m, lambda);
            double cycleCost = via_float(ev.wsum);
            int guard = 0, bad = 0;
            while (cycleCost > 0 || isnan(cycleCost)) {
                if (++guard > 4000) {
                    bad = 1;
                    break;
                }
                lambda += lambda;
                ev = record_sums(J, neg, m, lambda);
                cycleCost = via_float(ev.wsum);
            }
            sRatio = via_float(ev.ratio);
            sState[1] = bad;
        }
        __syncthreads();
        if (sState[1]) {
            if (lead) J.status = PAIR_ERR_GUARD;
            return;
        }
    }
    // A NaN or infinite bound: the host's branch-and-bound path (the heap
    // comparison that ends the first branch does not hold then).
    if (!(sRatio < (double)__int_as_float(0x7f800000))) {
        if (lead) J.status = PAIR_HOST;
        return;
    }

    // ---- the first branch: every node starts (cost_time_ratio_solver.cpp:794-829) ----
    for (long long v = t.thread(); v < n; v += t.nthreads()) J.branchOf[v] = 0;
    double currentRatio = sRatio;  // every thread keeps the same copy
    double oldRatio = currentRatio;
    int negEdges = sState[3];
    for (int i = 0;;) {
        if (threadIdx.x == 0) {
            P.mode = 0;
            P.branchId = 0;
            P.lambda = currentRatio;
            P.ub = ubInf;
        }
        if (!team_bf_call<CT, TK>(J, P, S, smem, false)) PGC_TEAM_FAIL();
        if (lead) J.lawlerIters++;
        if (*(volatile int*)&ctl->error) PGC_TEAM_FAIL();
        const int st = *(volatile int*)&ctl->status;
        int outcome;
        if (st == BF_FOUND_CYCLE) {
            const int cand = neg ^ 1;
            const int m = record_cycle(J, P, t, cand, *(volatile int*)&ctl->cycleLen, true);
            if (m == -3) PGC_TEAM_FAIL();
            if (m < 0) {
                if (lead) J.status = m == -2 ? PAIR_HOST : PAIR_ERR_EDGE;
                return;
            }
            if (threadIdx.x == 0) {
                const int integral = round_to_int_x86(record_sums(J, cand, m, currentRatio).wsum);
                int o;
                if (integral < 0) o = OUT_FOUND;
                else if (integral == 0) o = OUT_NONE;
                else o = round_to_int_x86(record_sums(J, neg, negEdges, currentRatio).wsum) == 0 ? OUT_ZERO : OUT_NONE;
                sState[0] = o;
                sState[3] = m;
            }
            __syncthreads();
            outcome = sState[0];
            if (outcome == OUT_FOUND) {
                neg = cand;
                negEdges = sState[3];
            }
        } else if (st == BF_LAYER_UNREACHED || st == BF_WRAP_NO_IMPROVE || st == BF_MAX_SWEEPS) {
            if (threadIdx.x == 0)
                sState[0] = st != BF_MAX_SWEEPS &&
                                    round_to_int_x86(record_sums(J, neg, negEdges, currentRatio).wsum) == 0
                                ? OUT_ZERO
                                : OUT_NONE;
            __syncthreads();
            outcome = sState[0];
        } else {
            if (lead) {
                J.status = PAIR_ERR_BF;
                J.bfStatus = st;
            }
            return;
        }
        if (outcome != OUT_FOUND) break;
        // lawlerSoubroutine's update and stopping rules (:584-597)
        if (threadIdx.x == 0) sRatio = record_sums(J, neg, negEdges, currentRatio).ratio;
        __syncthreads();
        currentRatio = sRatio;
        if (fabs(oldRatio - currentRatio) < tolerance) break;
        if (currentRatio - tolerance > oldRatio) break;
        oldRatio = currentRatio;
        if (i > 1000) break;
        ++i;
    }
    // passes of the cycle through layer 0 (:606-634): more than one, and the
    // branch and bound splits the branch -- the host's part
    if (lead) {
        const int* nodes = J.recNodes[neg];
        int wraps = 0;
        bool left = false;
        for (int i = 0; i <= negEdges; ++i) {
            const int vtx = __ldcg(nodes + i);
            if (left && vtx < n) left = false;
            if (vtx >= n && !left) {
                ++wraps;
                left = true;
            }
        }
        if (wraps > 1 && n > 1) {
            J.status = PAIR_HOST;
        } else {
            const CycleSums fin = record_sums(J, neg, negEdges, currentRatio);
            double T = 0;
            for (int i = 0; i < negEdges; ++i) T += __ldcg(J.recT[neg] + i);
            J.passes = 1;
            J.objective = __double2float_rn(fin.ratio);
            J.nEdges = negEdges;
            J.rec = neg;
            J.adjT = T;
            J.ratio = fin.ratio;
            J.status = PAIR_DONE;
        }
    }
#undef PGC_TEAM_FAIL
}

}  // namespace

// Teams of teamCtas consecutive CTAs take graphs from the queue, largest
// first.  A team's words (teamWords + kTeamWordStride * team, zeroed by the
// caller): barrier counter, generation, error, and the job its lead drew.
// With more than one CTA per team the launch is cooperative, so that every
// CTA of a team is resident.
template <class CT, int TK>
__global__ void __launch_bounds__(kBatchThreads, kBatchBlocksPerSm)
    bf_batch_kernel(PairJob* jobs, int count, int* next, unsigned* teamWords, int teamCtas, unsigned spin) {
    extern __shared__ double4 smemRaw[];
    char* smem = reinterpret_cast<char*>(smemRaw);
    __shared__ BfParams P;
    __shared__ int sJob, sCtas;
    const int cta = (int)(blockIdx.x % (unsigned)teamCtas);
    unsigned* w = teamWords + (size_t)(blockIdx.x / (unsigned)teamCtas) * kTeamWordStride;
    const Team all{cta, teamCtas, w, w + 1, reinterpret_cast<int*>(w + 2), spin};
    const bool lead = cta == 0 && threadIdx.x == 0;
    for (;;) {
        if (lead) w[3] = (unsigned)atomicAdd(next, 1);
        if (!team_sync(all)) return;
        if (threadIdx.x == 0) sJob = (int)__ldcg(w + 3);
        __syncthreads();
        const int j = sJob;
        if (j >= count) return;
        if (threadIdx.x == 0) {
            P = jobs[j].bf;
            sCtas = jobs[j].ctas < 1 ? 1 : jobs[j].ctas > teamCtas ? teamCtas : jobs[j].ctas;
        }
        __syncthreads();
        const SolveTeam S{all, Team{cta, sCtas, &P.ctl->barCount, &P.ctl->barGen, &P.ctl->error, P.spinLimit}};
        const long long c0 = clock64();
        pair_solve<CT, TK>(jobs[j], P, S, smem);
        if (lead) {
            jobs[j].candidates = P.ctl->candidates;
            jobs[j].fallbackWalks = P.ctl->fallbackWalks;
            jobs[j].cycles = clock64() - c0;
        }
        // nobody draws the next job before every CTA has read this one
        if (!team_sync(all)) return;
    }
}

// Host-side launch helpers -------------------------------------------------
static const void* bf_fn(int costIsF32, int timeKind, bool sharedTables) {
    if (sharedTables) {
        if (costIsF32)
            return timeKind == 0 ? (const void*)bf_kernel<float, 0, true>
                                 : timeKind == 1 ? (const void*)bf_kernel<float, 1, true>
                                                 : (const void*)bf_kernel<float, 2, true>;
        return timeKind == 0 ? (const void*)bf_kernel<double, 0, true>
                             : timeKind == 1 ? (const void*)bf_kernel<double, 1, true>
                                             : (const void*)bf_kernel<double, 2, true>;
    }
    if (costIsF32)
        return timeKind == 0 ? (const void*)bf_kernel<float, 0, false>
                             : timeKind == 1 ? (const void*)bf_kernel<float, 1, false>
                                             : (const void*)bf_kernel<float, 2, false>;
    return timeKind == 0 ? (const void*)bf_kernel<double, 0, false>
                         : timeKind == 1 ? (const void*)bf_kernel<double, 1, false>
                                         : (const void*)bf_kernel<double, 2, false>;
}

// The dynamic shared-memory limit is an attribute of the kernel function,
// shared by every host thread: it is always raised to the device's opt-in
// maximum (the same value from every thread, so concurrent solves cannot
// lower it under each other's launches); each launch then requests its own
// size.
static cudaError_t allow_max_dynamic_smem(const void* fn) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    // set once per (function, device): every later launch finds it set
    static std::mutex mu;
    static std::set<std::pair<const void*, int>> done;
    {
        std::lock_guard<std::mutex> lk(mu);
        if (done.count({fn, dev})) return cudaSuccess;
    }
    DeviceInfo info{};
    e = device_info(dev, &info);
    if (e == cudaSuccess) {
        cudaFuncAttributes a{};
        e = cudaFuncGetAttributes(&a, fn);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     info.smemOptin - (int)a.sharedSizeBytes);
    }
    if (e == cudaSuccess) {
        std::lock_guard<std::mutex> lk(mu);
        done.insert({fn, dev});
    }
    return e;
}

// Resident CTAs per SM of `fn` with this block and shared memory, cached.
static cudaError_t max_blocks_per_sm(const void* fn, int threads, size_t smemBytes, int* blocksPerSm) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    static std::mutex mu;
    static std::map<std::tuple<const void*, int, int, size_t>, int> cache;
    const auto key = std::make_tuple(fn, dev, threads, smemBytes);
    {
        std::lock_guard<std::mutex> lk(mu);
        const auto it = cache.find(key);
        if (it != cache.end()) {
            *blocksPerSm = it->second;
            return cudaSuccess;
        }
    }
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocksPerSm, fn, threads, smemBytes);
    if (e == cudaSuccess) {
        std::lock_guard<std::mutex> lk(mu);
        cache[key] = *blocksPerSm;
    }
    return e;
}

cudaError_t launch_bf(const BfParams& p, int costIsF32, int timeKind, int blocks, int threads, bool cooperative,
                      bool sharedTables, size_t smemBytes, cudaStream_t stream) {
    void* args[] = {(void*)&p};
    const void* fn = bf_fn(costIsF32, timeKind, sharedTables);
    const cudaError_t e = allow_max_dynamic_smem(fn);
    if (e != cudaSuccess) return e;
    note_launch();
    if (cooperative) return cudaLaunchCooperativeKernel(fn, dim3(blocks), dim3(threads), args, smemBytes, stream);
    return cudaLaunchKernel(fn, dim3(blocks), dim3(threads), args, smemBytes, stream);
}

cudaError_t bf_max_coop_blocks(int costIsF32, int timeKind, int threads, size_t smemBytes, int* blocksPerSm) {
    const void* fn = bf_fn(costIsF32, timeKind, false);
    const cudaError_t e = allow_max_dynamic_smem(fn);
    if (e != cudaSuccess) return e;
    return max_blocks_per_sm(fn, threads, smemBytes, blocksPerSm);
}

cudaError_t launch_extract_path(const BfParams& p, int v, cudaStream_t stream) {
    note_launch();
    extract_path_kernel<<<1, 32, 0, stream>>>(p, v);
    return cudaGetLastError();
}

static const void* bf_batch_fn(int costIsF32, int timeKind) {
    if (costIsF32)
        return timeKind == 0 ? (const void*)bf_batch_kernel<float, 0>
                             : timeKind == 1 ? (const void*)bf_batch_kernel<float, 1> : (const void*)bf_batch_kernel<float, 2>;
    return timeKind == 0 ? (const void*)bf_batch_kernel<double, 0>
                         : timeKind == 1 ? (const void*)bf_batch_kernel<double, 1> : (const void*)bf_batch_kernel<double, 2>;
}

cudaError_t launch_bf_batch(PairJob* jobs, int count, int* next, unsigned* teamWords, int teamCtas, unsigned spin,
                            int costIsF32, int timeKind, int blocks, int threads, size_t smemBytes,
                            cudaStream_t stream) {
    if (teamCtas < 1 || blocks < teamCtas || blocks % teamCtas != 0) return cudaErrorInvalidValue;
    const void* fn = bf_batch_fn(costIsF32, timeKind);
    const cudaError_t e = allow_max_dynamic_smem(fn);
    if (e != cudaSuccess) return e;
    void* args[] = {(void*)&jobs, (void*)&count, (void*)&next, (void*)&teamWords, (void*)&teamCtas, (void*)&spin};
    note_launch();
    if (teamCtas > 1) return cudaLaunchCooperativeKernel(fn, dim3(blocks), dim3(threads), args, smemBytes, stream);
    return cudaLaunchKernel(fn, dim3(blocks), dim3(threads), args, smemBytes, stream);
}

cudaError_t bf_batch_max_blocks(int costIsF32, int timeKind, int threads, size_t smemBytes, int* blocksPerSm) {
    const void* fn = bf_batch_fn(costIsF32, timeKind);
    const cudaError_t e = allow_max_dynamic_smem(fn);
    if (e != cudaSuccess) return e;
    return max_blocks_per_sm(fn, threads, smemBytes, blocksPerSm);
}

static std::atomic<long long> g_launches{0};
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
long long launch_count() { return g_launches.load(std::memory_order_relaxed); }

cudaError_t device_info(int device, DeviceInfo* out) {
    static std::mutex mu;
    static std::map<int, DeviceInfo> cache;
    {
        std::lock_guard<std::mutex> lk(mu);
        const auto it = cache.find(device);
        if (it != cache.end()) {
            *out = it->second;
            return cudaSuccess;
        }
    }
    DeviceInfo d{};
    cudaError_t e = cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&d.smemOptin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&d.clockKhz, cudaDevAttrClockRate, device);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    cache[device] = d;
    *out = d;
    return cudaSuccess;
}

cudaError_t launch_lookup_pairs(const LookupArgs& a, cudaStream_t stream) {
    if (a.count <= 0) return cudaSuccess;
    note_launch();
    lookup_pairs_kernel<<<(a.count + 127) / 128, 128, 0, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace pgc
