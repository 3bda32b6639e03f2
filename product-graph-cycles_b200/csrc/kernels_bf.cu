// kernels_bf.cu -- layered Bellman-Ford sweeps of the cycle solvers on sm_100a.
//
// One launch runs one Bellman-Ford call of the reference
// (mooreBellmanFordSubroutineCPU, cost_time_ratio_solver.cpp:251-542, and
// dijkstra_solver.cpp:203-388) from its set-up to its verdict, so the host
// only sees one launch per call instead of one per (layer, depth).
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
// Cycle detection: the reference walks predecessors from every negative
// start node in ascending order of its value until a start node repeats.
// Here each stored path also carries its origin (the layer-0 start node it
// leaves from) and its length in predecessor steps, so one "lap" of the walk
// (layer-0 node -> next layer-0 node) is a table lookup.  Each candidate is
// decided with Brent's cycle-finding algorithm on that lap function; the
// candidate with the smallest (value, index) whose walk repeats within the
// reference's step limit wins.  When a lap cannot be derived from the
// current sweep (a stale predecessor), that candidate is re-walked literally.
#include <cuda_runtime.h>

#include <cstdint>

#include "device_common.cuh"

namespace pgc {

namespace {

constexpr unsigned kSpinLimit = 1u << 24;  // ~2 s of polling with 100 ns sleeps

struct Team {
    int cta, ncta;
    unsigned* cnt;
    unsigned* gen;
    int* err;
    __device__ int warp() const { return cta * (int)(blockDim.x >> 5) + (int)(threadIdx.x >> 5); }
    __device__ int nwarps() const { return ncta * (int)(blockDim.x >> 5); }
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
__device__ __forceinline__ void red_add_release_u32(unsigned* p, unsigned v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Team barrier.  One CTA: __syncthreads.  Several CTAs (cooperative launch,
// all resident): after the CTA-wide barrier, thread 0 arrives on a global
// counter with release semantics (cumulative over the CTA's writes); the last
// arrival resets the counter and bumps the generation word with release
// semantics; the others poll the generation with acquire loads, spinning
// briefly and then backing off, for a bounded number of iterations after
// which the error word is raised.  Returns false when the team must stop.
__device__ bool team_sync(const Team& t) {
    __shared__ int s_stop;
    __syncthreads();
    if (threadIdx.x == 0) {
        if (t.ncta > 1) {
            const unsigned g = ld_acquire_u32(t.gen);
            const unsigned arrived = atom_add_acq_rel_u32(t.cnt, 1u);
            if (arrived == (unsigned)t.ncta - 1) {
                atomicExch(t.cnt, 0u);
                red_add_release_u32(t.gen, 1u);
            } else {
                unsigned spins = 0;
                while (ld_acquire_u32(t.gen) == g) {
                    if (++spins > kSpinLimit) {
                        atomicExch(t.err, 1);
                        break;
                    }
                    if (spins > 4096) __nanosleep(64);
                }
            }
        }
        s_stop = *(volatile int*)t.err;
    }
    __syncthreads();
    return s_stop == 0;
}

template <class T>
__device__ __forceinline__ double ld_stream(const T* p) {
    return (double)__ldg(p);
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

// Loads of the distance / origin tables: from shared memory when the whole
// team is one CTA that keeps them there (S), else through L2 (other CTAs
// write them during the launch, so L1 must not serve stale lines).
template <bool S>
__device__ __forceinline__ double ldD(const double* p) {
    if constexpr (S) return *p;
    else return __ldcg(p);
}
template <bool S>
__device__ __forceinline__ double2 ldD2(const double* p) {
    if constexpr (S) return *reinterpret_cast<const double2*>(p);
    else return __ldcg(reinterpret_cast<const double2*>(p));
}
template <bool S>
__device__ __forceinline__ int ldI(const int* p) {
    if constexpr (S) return *p;
    else return __ldcg(p);
}

// ---------------------------------------------------------------------------
// One (layer, depth) step of the sweep.
//
// A warp owns a slice of 32 target nodes (lane = node).  The in-edges of the
// slice are consumed in batches of kBatch slots: first every source index,
// cost and time of the batch is loaded (independent, coalesced 128-byte
// loads), then every source distance (one 16/32-byte vector gather per
// source row), then the batch is folded into the running minimum in edge
// order, so one batch costs about two memory latencies instead of two per
// edge.
// ---------------------------------------------------------------------------
constexpr int kBatch = 4;

template <class CT, int TK, bool S>
__device__ void relax_step(const BfParams& p, const Team& t, int l, int k, int epoch) {
    const int n = p.n, K = p.K, Kp = p.Kp;
    const int par = l & 1;
    double* cur = p.dp + (size_t)par * n * Kp;
    const double* prv = p.dp + (size_t)(par ^ 1) * n * Kp;
    int* corg = p.org + (size_t)par * n * Kp;
    int* chop = p.hops + (size_t)par * n * Kp;
    const int* porg = p.org + (size_t)(par ^ 1) * n * Kp;
    const int* phop = p.hops + (size_t)(par ^ 1) * n * Kp;
    const bool inter = (k == 0);
    const bool empty = (l == p.nY && k > 0);  // the closing layer has no intralayer edges
    const int* sp = inter ? p.spInter : p.spIntra;
    const int* src = inter ? (l == p.nY ? p.srcDummy : p.srcInter) : p.srcIntra;
    const size_t base = (size_t)l * (size_t)p.layerStride + (inter ? 0 : (size_t)p.interEntries);
    const CT* cst = (const CT*)p.cost + base;
    const float* tstF = (TK == 1) ? (const float*)p.time + base : nullptr;
    const double* tstD = (TK == 2) ? (const double*)p.time + base : nullptr;
    int* predRow = p.pred + (size_t)l * n * K + (size_t)k * n;
    const int srcLayer = inter ? l - 1 : l;
    const int nk = inter ? K : 1;            // source depths per edge
    const int kofs = inter ? 0 : k - 1;      // first source depth
    const double* srow = inter ? prv : cur;  // source rows
    const int lane = threadIdx.x & 31;
    const double lam = p.lambda, ub = p.ub;
    bool any = false;
    for (int s = t.warp(); s < p.nslices; s += t.nwarps()) {
        const int v = s * 32 + lane;
        const bool valid = v < n;
        double best = kInfD;
        if (l == 0 && valid) best = ldD<S>(cur + (size_t)v * Kp + k);
        int bs = -1, bk = -1;
        if (!empty) {
            const int j0 = __ldg(sp + s), j1 = __ldg(sp + s + 1);
            if (nk <= 4) {
                for (int jb = j0; jb < j1; jb += kBatch) {
                    int sv[kBatch];
                    double cv[kBatch], tv[kBatch];
#pragma unroll
                    for (int u = 0; u < kBatch; ++u) {
                        sv[u] = -1;
                        cv[u] = 0.0;
                        tv[u] = p.tconst;
                        if (jb + u < j1) {
                            const size_t e = (size_t)(jb + u) * 32 + lane;
                            sv[u] = __ldg(src + e);
                            cv[u] = ld_stream(cst + e);
                            if (TK == 1) tv[u] = (double)__ldg(tstF + e);
                            else if (TK == 2) tv[u] = __ldg(tstD + e);
                        }
                    }
                    double d[kBatch][4];
#pragma unroll
                    for (int u = 0; u < kBatch; ++u) {
                        d[u][0] = d[u][1] = d[u][2] = d[u][3] = kInfD;
                        if (sv[u] >= 0) {
                            const double* r = srow + (size_t)sv[u] * Kp + kofs;
                            if (nk == 1) {
                                d[u][0] = ldD<S>(r);
                            } else {
                                const double2 a = ldD2<S>(r);
                                d[u][0] = a.x;
                                d[u][1] = a.y;
                                if (nk > 2) {
                                    const double2 b = ldD2<S>(r + 2);
                                    d[u][2] = b.x;
                                    d[u][3] = b.y;
                                }
                            }
                        }
                    }
#pragma unroll
                    for (int u = 0; u < kBatch; ++u) {
                        if (sv[u] < 0) continue;
                        const double w = __dsub_rn(cv[u], __dmul_rn(lam, tv[u]));
#pragma unroll
                        for (int kk = 0; kk < 4; ++kk) {
                            if (kk >= nk || isinf(d[u][kk])) continue;
                            const double cand = __dadd_rn(d[u][kk], w);
                            if (cand < best && cand < ub) { best = cand; bs = sv[u]; bk = kofs + kk; }
                        }
                    }
                }
            } else {
                for (int j = j0; j < j1; ++j) {
                    const size_t e = (size_t)j * 32 + lane;
                    const int sv = __ldg(src + e);
                    if (sv < 0) continue;
                    const double c = ld_stream(cst + e);
                    double tt;
                    if (TK == 0) tt = p.tconst;
                    else if (TK == 1) tt = (double)__ldg(tstF + e);
                    else tt = __ldg(tstD + e);
                    const double w = __dsub_rn(c, __dmul_rn(lam, tt));
                    const double* row = srow + (size_t)sv * Kp + kofs;
                    for (int kk = 0; kk < nk; ++kk) {
                        const double dd = ldD<S>(row + kk);
                        if (isinf(dd)) continue;
                        const double cand = __dadd_rn(dd, w);
                        if (cand < best && cand < ub) { best = cand; bs = sv; bk = kofs + kk; }
                    }
                }
            }
        }
        if (valid) {
            cur[(size_t)v * Kp + k] = best;
            int o = kLapUnknown, h = 0;
            int ps = -1, pk = -1;  // source (node, depth) of the stored predecessor
            if (bs >= 0) {
                predRow[v] = bs + srcLayer * n * K + bk * n;
                any = true;
                ps = bs;
                pk = bk;
            } else if (l == 0) {
                // Layer 0 keeps an older value and its older predecessor.
                const int pe = __ldcg(predRow + v);
                if (pe < 0) {
                    o = kLapEnd;
                } else {
                    ps = pe - (k - 1) * n;
                    pk = k - 1;
                    if (ps < 0 || ps >= n) { ps = -1; o = kLapUnknown; }
                }
            }
            if (ps >= 0) {
                if (srcLayer == 0 && pk == 0) {
                    o = ps;
                    h = 1;
                } else {
                    const int* so = (inter && bs >= 0) ? porg : corg;
                    const int* sh = (inter && bs >= 0) ? phop : chop;
                    o = ldI<S>(so + (size_t)ps * Kp + pk);
                    h = ldI<S>(sh + (size_t)ps * Kp + pk) + 1;
                }
            }
            corg[(size_t)v * Kp + k] = o;
            chop[(size_t)v * Kp + k] = h;
        }
    }
    if (__any_sync(0xffffffffu, any) && lane == 0) p.layerFlag[l] = epoch;
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

// The reference's walk (cost_time_ratio_solver.cpp:461-488) for one
// candidate, marking layer-0 start nodes with a walk id instead of clearing
// a boolean column.
__device__ int literal_walk(const BfParams& p, int vi, long long maxLen, int* v0, long long* steps) {
    const int id = ++p.ctl->walkId;
    const int n = p.n;
    const long long total = (long long)n * (p.nY + 1) * p.K;
    int pr = __ldcg(p.pred + vi);
    p.mark[vi] = id;
    long long len = 1;
    for (long long kk = maxLen - 1; kk > 0; --kk) {
        if (pr < n && pr >= 0) {
            if (p.mark[pr] == id) { *v0 = pr; *steps = len; return 1; }
            p.mark[pr] = id;
        }
        if (pr < 0 || pr >= total) return 2;
        pr = __ldcg(p.pred + pr);
        if (pr == -1) return 2;
        ++len;
    }
    return 2;
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
// The Bellman-Ford launch.  Every CTA of the grid belongs to one team.
// ---------------------------------------------------------------------------
template <class CT, int TK, bool S>
__global__ void __launch_bounds__(512) bf_kernel(BfParams p) {
    Team t{(int)blockIdx.x, (int)gridDim.x, &p.ctl->barCount, &p.ctl->barGen, &p.ctl->error};
    const int n = p.n, K = p.K, Kp = p.Kp;
    const long long tid = t.thread(), nth = t.nthreads();
    const bool isLead = (blockIdx.x == 0 && threadIdx.x == 0);
    if constexpr (S) {
        // single-CTA team: distance, backup, origin and hop tables live in
        // shared memory for the whole launch (layout as in global memory)
        extern __shared__ double4 smemRaw[];
        double* sm = reinterpret_cast<double*>(smemRaw);
        p.dp = sm;
        p.bak = sm + 2 * (size_t)n * Kp;
        p.org = reinterpret_cast<int*>(p.bak + n);
        p.hops = p.org + 2 * (size_t)n * Kp;
    }

    // set-up (cost_time_ratio_solver.cpp:264-287): DP := inf, branch starts := 0
    for (long long i = tid; i < 2LL * n * Kp; i += nth) p.dp[i] = kInfD;
    for (long long i = tid; i < n; i += nth) {
        p.bak[i] = kInfD;
        if (p.branchOf[i] == p.branchId) {
            p.dp[(size_t)i * Kp] = 0.0;
            p.pred[i] = -1;
        }
    }
    {
        // branch size and the last branch node (the reference's indexNodeInLayer)
        Key kmax{0, -1};
        int cnt = 0;
        for (long long i = tid; i < n; i += nth)
            if (p.branchOf[i] == p.branchId) { ++cnt; kmax.i = (int)i; }
        Key km{-(double)kmax.i, kmax.i < 0 ? 0x7fffffff : kmax.i};
        km = block_min(km, 0);
        if (threadIdx.x == 0) p.redIdx[blockIdx.x] = km.i;
        for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        __shared__ int scnt;
        if (threadIdx.x == 0) scnt = 0;
        __syncthreads();
        if ((threadIdx.x & 31) == 0) atomicAdd(&scnt, cnt);
        __syncthreads();
        if (threadIdx.x == 0) p.redAux[blockIdx.x] = scnt;
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
    for (;;) {
        const int epoch = epochBase + sweep + 1;
        for (long long i = tid; i < n; i += nth) p.bak[i] = ldD<S>(p.dp + (size_t)i * Kp);
        if (!team_sync(t)) return;
        bool stop = false;
        for (int l = 0; l <= p.nY && !stop; ++l) {
            for (int k = 0; k < K; ++k) {
                if (l == 0 && k == 0) continue;
                relax_step<CT, TK, S>(p, t, l, k, epoch);
                if (!team_sync(t)) return;
            }
            if (l > 0 && l < p.nY && *(volatile int*)&p.layerFlag[l] != epoch) stop = true;
        }
        ++sweep;
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
        if (p.mode == 2) {
            // minimum-cost verdict: lower bounds of the branch nodes, origin of
            // their closing path, first and first-valid candidates.
            Key first{kInfD, 0x7fffffff}, firstValid{kInfD, 0x7fffffff};
            int anyFinite = 0;
            const int* dOrg = p.org + (size_t)(p.nY & 1) * n * Kp;
            for (long long i = tid; i < n; i += nth) {
                if (p.branchOf[i] != p.branchId) { p.lbOut[i] = kInfD; p.originOut[i] = -1; continue; }
                const double lb = ldD<S>(p.dp + (size_t)lastPar * n * Kp + (size_t)i * Kp + lastDepth);
                int o = ldI<S>(dOrg + (size_t)i * Kp);
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
                p.redVal[2 * blockIdx.x] = first.v;
                p.redIdx[2 * blockIdx.x] = first.i;
                p.redVal[2 * blockIdx.x + 1] = firstValid.v;
                p.redIdx[2 * blockIdx.x + 1] = firstValid.i;
                p.redAux[blockIdx.x] = anyFinite;
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
            const int wPar = (p.nY - 1) & 1;
            const int* wOrg = p.org + (size_t)wPar * n * Kp;
            const int* wHop = p.hops + (size_t)wPar * n * Kp;
            const long long layerSpan = (long long)n * K;
            for (long long i = tid; i < n; i += nth) {
                if (p.branchOf[i] == p.branchId) {
                    const double cand = ldD<S>(p.dp + (size_t)lastPar * n * Kp + (size_t)i * Kp + lastDepth);
                    const double b = p.bak[i];
                    if (cand < b) {
                        improved = 1;
                        p.dp[(size_t)i * Kp] = cand;
                        p.pred[i] = __ldcg(p.pred + (size_t)p.nY * layerSpan + i);
                    } else {
                        p.dp[(size_t)i * Kp] = b;
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
                        nx = ldI<S>(wOrg + (size_t)wv * Kp + kp);
                        st = 1 + ldI<S>(wHop + (size_t)wv * Kp + kp);
                    }
                }
                p.lapNext[i] = nx;
                p.lapSteps[i] = st;
            }
            improved = __syncthreads_or(improved);
            if (threadIdx.x == 0) p.redAux[blockIdx.x] = improved;
        }
        if (!team_sync(t)) return;
        {
            int improved = 0;
            for (int c = 0; c < t.ncta; ++c) improved |= *(volatile int*)&p.redAux[c];
            if (!improved) {
                if (isLead) { p.ctl->status = BF_WRAP_NO_IMPROVE; p.ctl->sweeps = sweep; p.ctl->epoch = epochBase + sweep; }
                return;
            }
        }
        // every CTA has read redAux before it is reused below
        if (!team_sync(t)) return;

        // candidates (cost_time_ratio_solver.cpp:431-489)
        {
            Key bestOk{kInfD, 0x7fffffff}, firstUnknown{kInfD, 0x7fffffff};
            const long long limit = numNodes - 1;
            long long decided = 0;
            for (long long i = tid; i < n; i += nth) {
                int st = 0;
                if (p.branchOf[i] == p.branchId) {
                    const double d0 = ldD<S>(p.dp + (size_t)i * Kp);
                    if (d0 < 0) {
                        int v0 = -1;
                        long long steps = 0;
                        st = lap_walk(p, (int)i, limit, &v0, &steps);
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
                p.redVal[2 * blockIdx.x] = bestOk.v;
                p.redIdx[2 * blockIdx.x] = bestOk.i;
                p.redVal[2 * blockIdx.x + 1] = firstUnknown.v;
                p.redIdx[2 * blockIdx.x + 1] = firstUnknown.i;
                p.redAux64[blockIdx.x] = (long long)sdec;
            }
        }
        if (!team_sync(t)) return;
        if (isLead) {
            Key ok{kInfD, 0x7fffffff}, unk{kInfD, 0x7fffffff};
            long long dec = 0;
            for (int c = 0; c < t.ncta; ++c) {
                Key a{__ldcg(p.redVal + 2 * c), __ldcg(p.redIdx + 2 * c)};
                Key b{__ldcg(p.redVal + 2 * c + 1), __ldcg(p.redIdx + 2 * c + 1)};
                if (key_less(a, ok)) ok = a;
                if (key_less(b, unk)) unk = b;
                dec += __ldcg(p.redAux64 + c);
            }
            p.ctl->candidates += dec;
            int winner = -1, v0 = -1;
            long long steps = 0;
            if (ok.i != 0x7fffffff && (unk.i == 0x7fffffff || key_less(ok, unk))) {
                winner = ok.i;
                v0 = __ldcg(p.candV0 + winner);
                steps = __ldcg(p.candSteps + winner);
            } else if (unk.i != 0x7fffffff) {
                // Resolve in ascending (value, index) order; literal walks only
                // for the undecidable candidates.
                Key prev{-kInfD, -1};
                for (;;) {
                    Key next{kInfD, 0x7fffffff};
                    for (int i = 0; i < n; ++i) {
                        const int st = __ldcg(p.candStat + i);
                        if (st == 0) continue;
                        Key kk{ldD<S>(p.dp + (size_t)i * Kp), i};
                        if (key_less(prev, kk) && key_less(kk, next)) next = kk;
                    }
                    if (next.i == 0x7fffffff) break;
                    prev = next;
                    const int st = __ldcg(p.candStat + next.i);
                    if (st == 1) { winner = next.i; v0 = __ldcg(p.candV0 + winner); steps = __ldcg(p.candSteps + winner); break; }
                    if (st == 3) {
                        p.ctl->fallbackWalks++;
                        if (literal_walk(p, next.i, numNodes, &v0, &steps) == 1) { winner = next.i; break; }
                    }
                }
            }
            if (winner >= 0) {
                p.ctl->v0 = v0;
                p.ctl->cLength = steps;
                p.ctl->candidateVi = winner;
                p.ctl->status = extract_cycle(p, v0, steps);
            } else if (sweep >= numNodes - 1 || (p.maxSweeps > 0 && sweep >= p.maxSweeps)) {
                p.ctl->status = BF_MAX_SWEEPS;
            }
            p.ctl->sweeps = sweep;
            p.ctl->epoch = epochBase + sweep;
        }
        if (!team_sync(t)) return;
        if (*(volatile int*)&p.ctl->status != BF_RUNNING) return;
    }
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

// Finds, for each (source, target) pair of original ids, the first in-edge of
// the target whose source matches (computeRatioForCycle's lookup,
// cost_time_ratio_solver.cpp:103-122) and returns its edge id and the double
// cost/time of that edge.  Target ids >= numNodes denote the closing layer.

__global__ void lookup_pairs_kernel(LookupArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.count) return;
    const long long S = a.pairSrc[i], T = a.pairTrgt[i];
    a.edgeOut[i] = -2;
    a.cOut[i] = 0;
    a.tOut[i] = 0;
    if (S < 0 || T < 0) return;
    const int lt = (int)(T / a.n), v = (int)(T % a.n);
    const int ls = (int)(S / a.n), s = (int)(S % a.n);
    if (lt > a.nY) return;
    int part;
    const int* src;
    const int* sp;
    const int* ted;
    long long block;
    if (lt == a.nY) {
        if (ls != a.nY - 1) return;
        part = 0; src = a.srcDummy; sp = a.spInter; ted = a.tedgeInter; block = a.nY - 1;
    } else if (ls == lt) {
        part = 1; src = a.srcIntra; sp = a.spIntra; ted = a.tedgeIntra; block = lt;
    } else if (lt >= 1 && ls == lt - 1) {
        part = 0; src = a.srcInter; sp = a.spInter; ted = a.tedgeInter; block = lt - 1;
    } else {
        return;
    }
    const int slice = v >> 5, lane = v & 31;
    for (int j = sp[slice]; j < sp[slice + 1]; ++j) {
        const long long e = (long long)j * 32 + lane;
        if (src[e] == s) {
            const long long off = (long long)lt * a.layerStride + (part ? a.interEntries : 0) + e;
            a.edgeOut[i] = block * a.eBlock + ted[e];
            a.cOut[i] = a.c64[off];
            a.tOut[i] = a.t64 ? a.t64[off] : a.tconst;
            return;
        }
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

// Bytes of shared memory a single-CTA launch needs to keep the distance,
// backup, origin and hop tables on chip.
size_t bf_shared_table_bytes(int n, int Kp) {
    return (size_t)n * Kp * 2 * sizeof(double) + (size_t)n * sizeof(double) + (size_t)n * Kp * 4 * sizeof(int);
}

cudaError_t launch_bf(const BfParams& p, int costIsF32, int timeKind, int blocks, int threads, bool cooperative,
                      size_t sharedBytes, cudaStream_t stream) {
    void* args[] = {(void*)&p};
    const bool shared = sharedBytes > 0;
    const void* fn = bf_fn(costIsF32, timeKind, shared);
    if (shared) {
        const cudaError_t e =
            cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sharedBytes);
        if (e != cudaSuccess) return e;
    }
    if (cooperative) return cudaLaunchCooperativeKernel(fn, dim3(blocks), dim3(threads), args, sharedBytes, stream);
    return cudaLaunchKernel(fn, dim3(blocks), dim3(threads), args, sharedBytes, stream);
}

cudaError_t bf_max_coop_blocks(int costIsF32, int timeKind, int threads, int* blocksPerSm) {
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocksPerSm, bf_fn(costIsF32, timeKind, false), threads, 0);
}

cudaError_t launch_extract_path(const BfParams& p, int v, cudaStream_t stream) {
    extract_path_kernel<<<1, 32, 0, stream>>>(p, v);
    return cudaGetLastError();
}

cudaError_t launch_lookup_pairs(const LookupArgs& a, cudaStream_t stream) {
    if (a.count <= 0) return cudaSuccess;
    lookup_pairs_kernel<<<(a.count + 127) / 128, 128, 0, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace pgc
