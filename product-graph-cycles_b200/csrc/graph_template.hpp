// graph_template.hpp -- the layer-invariant structure of a cyclic product graph.
//
// Every layer of the reference's product graph has the same topology (only
// the Y indices of its rows change), so the device keeps ONE in-edge list per
// node-within-a-layer and streams per-layer edge costs beside it.
//
// Layout ("sliced ELL", 32 nodes per slice = one warp): for each part
// (INTER = in-edges from the previous layer, INTRA = in-edges from the same
// layer) and each slice s of 32 consecutive target nodes there are
// width(s) slots; slot j of slice s holds, for lane i, the j-th in-edge of
// target node 32*s + i in ascending edge-id order, or -1 past the node's
// in-degree.  Slot j of slice s lives at entries [32*(sp[s]+j), 32*(sp[s]+j)+32).
//
// Edge ids follow the reference's generation order: block b (= the Y edge b)
// holds eBlock consecutive ids; the edge with template offset t in block b
// has id b*eBlock + t.  An INTER slot of layer l holds an edge of block l-1
// (block nY-1 for the closing "dummy" layer l = nY); an INTRA slot of layer l
// holds an edge of block l.
#pragma once
#include <cstdint>
#include <functional>
#include <memory>
#include <new>
#include <string>
#include <utility>
#include <vector>

namespace pgc {

// Host memory for buffers that are copied to the device (pinned where
// possible, from a process-wide cache; defined with the CUDA host code).
void* host_buffer_alloc(size_t bytes);
void host_buffer_free(void* p);

// Allocator of the template arrays and of a handle's inputs: memory from
// host_buffer_alloc, so their uploads are plain DMA, and a resize that leaves
// elements default-initialised (unset for ints): the template builder writes
// every element it sizes, and zeroing tens of MB first was a visible part of
// building a large template.
template <class T>
struct RawAlloc : std::allocator<T> {
    template <class U>
    struct rebind {
        using other = RawAlloc<U>;
    };
    RawAlloc() = default;
    template <class U>
    RawAlloc(const RawAlloc<U>&) noexcept {}
    T* allocate(size_t n) {
        void* p = host_buffer_alloc(n * sizeof(T));
        if (!p && n) throw std::bad_alloc();
        return static_cast<T*>(p);
    }
    void deallocate(T* p, size_t) noexcept { host_buffer_free(p); }
    template <class U>
    void construct(U* p) noexcept {
        ::new ((void*)p) U;
    }
    template <class U, class... A>
    void construct(U* p, A&&... a) {
        ::new ((void*)p) U(std::forward<A>(a)...);
    }
};
template <class T>
using RawVec = std::vector<T, RawAlloc<T>>;

enum Part { INTER = 0, INTRA = 1 };

// How the Y columns of a productspace row are formed from block b:
//   s2 = EY(b,0), m2 = EY(b,1), t2 = EY((b+1) % nY, 1)
enum YPattern : int8_t {
    Y_SS = 0,   // plain intralayer       [s2, s2]
    Y_SM = 1,   // plain interlayer       [s2, m2]
    Y_SSS = 2,  // conj deg2d -> deg2d    [s2, s2, s2]
    Y_SSM = 3,  // conj deg2d -> non-deg  [s2, s2, m2]
    Y_SMT = 4,  // conj interlayer        [s2, m2, t2]
    Y_SMM = 5,  // conj non-deg -> deg2d  [s2, m2, m2]
};

struct LayerTemplate {
    bool conj = false, prune = false;
    int n = 0;          // nodes per layer
    int nvx = 0;        // max(EX) + 1
    int nY = 0;         // number of layers (|EY|)
    int nslices = 0;
    int64_t eBlock = 0; // edges per block
    // sliced-ELL in-edge lists, per part
    RawVec<int> sp[2];             // nslices + 1 slot offsets
    RawVec<int> src[2];            // 32 * slots: local source node or -1
    RawVec<int> tedge[2];          // 32 * slots: template edge offset or -1
    RawVec<int> srcDummy;          // INTER src list of the closing layer; stored for nY == 2 only (else == src[INTER])
    int64_t entries[2] = {0, 0};   // 32 * slots per part
    // per template edge offset (eBlock entries)
    RawVec<int> eSrc, eTrgt;       // local source / target node
    RawVec<int8_t> eNext;          // 1 if the target is in the next layer
    RawVec<int> eX;                // 3 ints per edge: x columns of the row (x2 unused for plain)
    RawVec<int8_t> eY;             // YPattern
    RawVec<int> ePos;              // entry index (part encoded in bit 30) of the edge in its part

    int64_t layerStride() const { return entries[0] + entries[1]; }
    int cols() const { return conj ? 6 : 4; }
};

// Builds the template; returns an empty string or an error message.
std::string build_template(const int* EX, int64_t nEX, const int* EY, int64_t nEY, int64_t nVX, bool conj,
                           bool prune, LayerTemplate& T);

// Runs f(begin, end) over parts of [0, n) of at least `grain` items on the
// process's host worker pool (inline when another job holds the pool).
void host_parallel_for(int64_t n, int64_t grain, const std::function<void(int64_t, int64_t)>& f);

// Contiguous slice ranges [cut[c], cut[c+1]) of `blocks` CTAs of `warps`
// warps for the Bellman-Ford team, balanced on the per-step work of their
// slowest warps; rowsPerBatch[p] = rows a warp gathers per batch in part p.
std::vector<int> plan_cta_cuts(const LayerTemplate& T, int blocks, int K, int warps, const int rowsPerBatch[2]);

// Wait lists of the Bellman-Ford team for the CTA slice ranges `cut`: CTA c
// lists, in ascending order in idx[ptr[c]..ptr[c+1]), every other CTA joined
// to it by an in-edge of the layer template in either direction.
void cta_wait_lists(const LayerTemplate& T, const std::vector<int>& cut, std::vector<int>& ptr, std::vector<int>& idx);

// productspace row of global edge id e (product_space.cpp / conj_product_space.cpp order).
void product_row(const LayerTemplate& T, const int* EY, int64_t e, int* out);

}  // namespace pgc
