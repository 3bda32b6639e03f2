// pgc_host.cpp -- host side of libpgc: the generator facade, the solver
// control loops and the C ABI declared in include/pgc.h.
//
// Division of labour: the device builds the edge costs, rescales them and
// runs every Bellman-Ford call (one launch per call, see kernels_bf.cu);
// the host keeps only the scalar control of the reference's solvers -- the
// Lawler ratio updates, the branch-and-bound heap and the branching rules --
// which touch O(cycle length) or O(nodes per layer) data.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>
#include <atomic>

#include "../../include/pgc.h"
#include "branch_heap.hpp"
#include "device_common.cuh"
#include "graph_template.hpp"

namespace pgc {

namespace {

thread_local std::string g_lastError;

struct Failure : std::runtime_error {
    int code;
    Failure(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define PGC_CUDA(call)                                                                                   \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess)                                                                           \
            throw Failure(PGC_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));             \
    } while (0)

// Process-wide caching allocator for device buffers.  Freed blocks are kept,
// per device, and handed out again to requests of at least half their size,
// so that creating and destroying generators (and re-solving graphs of
// similar size) does not pay cudaMalloc/cudaFree every time.  Every handle
// synchronises its stream before it returns memory here, so a cached block is
// never still in use.  pgc_release_cached_memory() returns the cache to CUDA.
// Pinned host memory for what a handle uploads (its inputs and the layer
// template): copies from it are DMA the host does not stage.  cudaHostAlloc
// is slow, so freed blocks are kept by size and handed out again to requests
// of at least half their size, for the process's lifetime; a handle's
// buffers come back only after its stream has been synchronised.  Pageable
// memory stands in when pinning fails.
class HostPool {
  public:
    static HostPool& get() {
        static HostPool* pool = new HostPool();  // never destroyed: outlives all handles
        return *pool;
    }
    void* allocate(size_t bytes) {
        if (bytes == 0) return nullptr;
        {
            std::lock_guard<std::mutex> lock(mu_);
            auto it = free_.lower_bound(bytes);
            if (it != free_.end() && it->first <= 2 * bytes + (1 << 20)) {
                void* p = it->second;
                sizes_[p] = it->first;
                free_.erase(it);
                return p;
            }
        }
        void* p = nullptr;
        if (cudaHostAlloc(&p, bytes, cudaHostAllocPortable) != cudaSuccess) {
            (void)cudaGetLastError();
            p = std::malloc(bytes);
            if (!p) return nullptr;
            std::lock_guard<std::mutex> lock(mu_);
            pageable_.insert(p);
            return p;
        }
        std::lock_guard<std::mutex> lock(mu_);
        sizes_[p] = bytes;
        return p;
    }
    void deallocate(void* p) {
        if (!p) return;
        std::lock_guard<std::mutex> lock(mu_);
        if (pageable_.erase(p)) {
            std::free(p);
            return;
        }
        auto it = sizes_.find(p);
        if (it == sizes_.end()) return;
        free_.emplace(it->second, p);
        sizes_.erase(it);
    }
    // Unpins and frees the cached blocks (live handles keep theirs).
    void release_cached() {
        std::lock_guard<std::mutex> lock(mu_);
        for (auto& b : free_) cudaFreeHost(b.second);
        free_.clear();
    }

  private:
    std::mutex mu_;
    std::multimap<size_t, void*> free_;
    std::map<void*, size_t> sizes_;
    std::set<void*> pageable_;
};

class DevicePool {
  public:
    static DevicePool& get() {
        static DevicePool* pool = new DevicePool();  // never destroyed: outlives all handles
        return *pool;
    }
    void* allocate(size_t bytes) {
        int dev = 0;
        PGC_CUDA(cudaGetDevice(&dev));
        {
            std::lock_guard<std::mutex> lock(mu_);
            auto& fl = free_[dev];
            auto it = fl.lower_bound(bytes);
            if (it != fl.end() && it->first <= 2 * bytes + (1 << 20)) {
                void* p = it->second;
                sizes_[p] = it->first;
                fl.erase(it);
                return p;
            }
        }
        void* p = nullptr;
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e == cudaErrorMemoryAllocation) {
            (void)cudaGetLastError();
            release_cached();
            e = cudaMalloc(&p, bytes);
        }
        if (e != cudaSuccess) throw Failure(PGC_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
        std::lock_guard<std::mutex> lock(mu_);
        sizes_[p] = bytes;
        devOf_[p] = dev;
        return p;
    }
    void deallocate(void* p) {
        if (!p) return;
        std::lock_guard<std::mutex> lock(mu_);
        auto it = sizes_.find(p);
        if (it == sizes_.end()) return;
        free_[devOf_[p]].emplace(it->second, p);
        sizes_.erase(it);
    }
    void release_cached() {
        std::lock_guard<std::mutex> lock(mu_);
        int cur = 0;
        cudaGetDevice(&cur);
        for (auto& d : free_) {
            cudaSetDevice(d.first);
            for (auto& b : d.second) {
                cudaFree(b.second);
                devOf_.erase(b.second);
            }
            d.second.clear();
        }
        cudaSetDevice(cur);
    }

  private:
    std::mutex mu_;
    std::map<int, std::multimap<size_t, void*>> free_;
    std::map<void*, size_t> sizes_;
    std::map<void*, int> devOf_;
};

template <class T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    ~DBuf() { release(); }
    void release() {
        if (p) DevicePool::get().deallocate(p);
        p = nullptr;
        n = 0;
    }
    void alloc(size_t count) {
        if (count <= n && p) return;
        release();
        if (count == 0) count = 1;
        p = (T*)DevicePool::get().allocate(count * sizeof(T));
        n = count;
    }
    void upload(const T* src, size_t count, cudaStream_t s) {
        alloc(count);
        if (count && src) PGC_CUDA(cudaMemcpyAsync(p, src, count * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    void zero(cudaStream_t s) { PGC_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s)); }
};

enum HoMode { NOMODE = 0, VANILLA, FEATURE, LENGTH, SO3_PLAIN, SO3_ROBUST, PENALISE_DEGENERATE };

// higherOrderDeformationEnergy.cpp:396-412 including its missing "== 0" on
// the last comparison: "penalisedegenerate" maps to VANILLA and any other
// unknown name (the default "") to PENALISE_DEGENERATE.
int string_to_mode(const std::string& s) {
    if (s == "nomode") return NOMODE;
    if (s == "vanilla") return VANILLA;
    if (s == "feature") return FEATURE;
    if (s == "lengthnormalisation") return LENGTH;
    if (s == "plainso3") return SO3_PLAIN;
    if (s == "robustso3") return SO3_ROBUST;
    if (s != "penalisedegenerate") return PENALISE_DEGENERATE;
    return VANILLA;
}

bool ho_supported(int cm, int tm) {
    return (cm == VANILLA && tm == VANILLA) || (cm == VANILLA && tm == LENGTH) || (cm == LENGTH && tm == VANILLA) ||
           (cm == VANILLA && tm == PENALISE_DEGENERATE) || (cm == PENALISE_DEGENERATE && tm == VANILLA) ||
           (cm == FEATURE && tm == SO3_PLAIN) || (cm == FEATURE && tm == SO3_ROBUST) ||
           (cm == SO3_ROBUST && tm == FEATURE) || (cm == SO3_PLAIN && tm == FEATURE);
}

double robust_loss_host(double x, double alpha, double c, double pwr) {
    const double t = std::pow(x / c, pwr);
    const double am2 = std::fabs(alpha - 2);
    return am2 / alpha * (std::pow(t / am2 + 1, 0.5 * alpha) - 1);
}

// (int)std::round(x) as the reference's x86-64 build evaluates it.
int round_to_int(double x) {
    const double r = std::round(x);
    if (!(r >= -2147483648.0 && r <= 2147483647.0)) return INT_MIN;
    return (int)r;
}

int env_int(const char* name, int dflt) {
    const char* v = std::getenv(name);
    if (!v || !*v) return dflt;
    return std::atoi(v);
}

}  // namespace

// The template's and the inputs' allocator (graph_template.hpp).
void* host_buffer_alloc(size_t bytes) { return HostPool::get().allocate(bytes); }
void host_buffer_free(void* p) { HostPool::get().deallocate(p); }

// dst := src[0, count), copied by the host worker pool in 1 MB parts: the
// feature-difference matrix of a large pair is tens of MB, and one thread
// copies about 10 GB/s.
template <class T>
void copy_in(RawVec<T>& dst, const T* src, size_t count) {
    dst.resize(count);
    T* d = dst.data();
    host_parallel_for((int64_t)count, (int64_t)((1 << 20) / sizeof(T)), [&](int64_t a, int64_t b) {
        std::memcpy(d + a, src + a, (size_t)(b - a) * sizeof(T));
    });
}

// A closed walk of the product graph as the reference stores it: original
// node ids (targets in layer 0 that close a lap are written as the closing
// copy numNodes + v only at the end), plus the edge and its cost/time for
// every consecutive pair.
struct CycleRec {
    std::vector<int> nodes;
    std::vector<long long> edges;
    std::vector<double> c, t;
    bool valid() const { return !nodes.empty(); }
};

enum class BfOutcome { NO_NEGATIVE_CYCLE, FOUND_NEGATIVE_CYCLE, ZERO_CYCLE };

struct Stats {
    long long bfCalls = 0, sweeps = 0, candidates = 0, lawlerIters = 0, branches = 0, fallbackWalks = 0;
    double deviceMs = 0;
    long long launches = 0;
    unsigned long long cycA = 0, cycB = 0, cycSync = 0, cycTail = 0;
    unsigned long long cycWrap = 0, cycCand = 0, cycLead = 0;  // parts of cycTail
    unsigned long long cycStage = 0;                           // part of cycA
    long long steps = 0;
    long long ctas = 0, threads = 0, waitEntries = 0;  // team shape of the last launch
};

class Graph {
  public:
    // inputs
    RawVec<double> VX, VY, FD, NX, NY;
    RawVec<int> EX, EY;
    int64_t nvx = 0, nvy = 0, nex = 0, ney = 0;
    bool conj = false, reg = false, prune = false, normalsGiven = false;
    double rlAlpha = 0.7, rlC = 0.6, rlPwr = 4;
    int maxDepth = 4;
    std::string costName = "vanilla", timeName = "";

    int device = 0;
    cudaStream_t stream = nullptr;     // stream all work is issued on
    cudaStream_t ownStream = nullptr;  // the handle's own stream
    bool templateReady = false;        // topology uploaded (it never changes)

    // generated state
    bool generated = false;
    LayerTemplate T;
    int ncols = 1;
    DBuf<int> dSp[2], dSrc[2], dTedge[2], dSrcDummy, dEX, dEY, dESrc, dETrgt, dEXcols;
    DBuf<int8_t> dEYpat, dENext;
    DBuf<double> dVX, dVY, dFD, dNX, dNY;
    DBuf<double4> dQuat;
    DBuf<double> e64[2];
    DBuf<float> e32[2];
    bool f32Valid[2] = {false, false};  // e32 mirrors e64 exactly
    bool f32Known[2] = {false, false};  // e32 state computed since the last energy change

    // solver workspace
    DBuf<double> wDv;
    DBuf<int2> wDoh;
    DBuf<double> wBak, wRedVal, wLb, wCOut, wTOut;
    DBuf<int> wCtaSlice, wWaitPtr, wWaitIdx;
    DBuf<unsigned> wStepDone;
    std::vector<int> ctaCut;   // slice ranges of the uploaded partition
    mutable std::map<std::string, std::vector<int>> cutCache;  // cta_cuts per (blocks, K, warps)
    int cutBlocks = -1, cutK = -1, cutWarps = -1;  // the partition ctaCut was made for
    long long waitEntries = 0;  // wait-list entries over all CTAs of the current partition
    DBuf<int> wPred, wLapNext, wLapSteps, wCandStat, wCandV0, wLayerFlag, wBranch, wCycle,
        wRedIdx, wRedAux, wOrigin, wPairS, wPairT, wCount;
    DBuf<LiteralWalk> wWalks;
    DBuf<long long> wCandSteps, wRedAux64, wEdgeOut;
    DBuf<float> wMean;
    DBuf<Control> wCtl;
    int wsK = -1;
    int ctlEpoch = 0;
    int teamCap = 0;  // most CTAs of a Bellman-Ford launch (0: as many as help)
    // team shape chosen for this graph (pgc_set_team_shape; 0: automatic);
    // the PGC_BF_BLOCKS / PGC_BF_THREADS environment overrides take precedence
    int shapeBlocks = 0, shapeThreads = 0;
    bool workspaceFresh = false;

    // last result
    bool resPasses = false;
    float resObjective = 0;
    int64_t resRows = 0, resCols = 0;
    std::vector<int> resMatching;
    std::vector<long long> resEdges;
    Stats stats;

    // Waiting for the stream: a spin wait by default (lowest latency); while
    // many graphs are solved at once by as many host threads, a blocking
    // wait, so that waiting threads sleep instead of competing for cores.
    bool blockingSync = false;
    cudaEvent_t syncEvent = nullptr;
    cudaEvent_t timeEvents[2] = {nullptr, nullptr};  // around each Bellman-Ford launch
    cudaError_t sync_stream() {
        if (!blockingSync) return cudaStreamSynchronize(stream);
        cudaError_t e = cudaSuccess;
        if (!syncEvent) e = cudaEventCreateWithFlags(&syncEvent, cudaEventBlockingSync | cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventRecord(syncEvent, stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(syncEvent);
        return e;
    }

    // Device -> pageable host copy.  The copy waits for the stream's earlier
    // work inside the driver (a spin); in blocking mode that wait happens on
    // the blocking event first.
    void d2h(void* dst, const void* src, size_t bytes) {
        if (blockingSync) PGC_CUDA(sync_stream());
        PGC_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, stream));
    }

    ~Graph() {
        // device buffers go back to the caching pool: no work may still use them
        if (stream) cudaStreamSynchronize(stream);
        if (syncEvent) cudaEventDestroy(syncEvent);
        for (cudaEvent_t e : timeEvents)
            if (e) cudaEventDestroy(e);
        if (ownStream) cudaStreamDestroy(ownStream);
    }

    long numNodes() const { return (long)T.n * T.nY; }

    // -------------------------------------------------------------------
    void generate();
    void count_top_digits(EnergyArgs& a);
    void upload_template();
    void ensure_generated() {
        if (!generated) generate();
    }
    void energy_changed() {
        f32Known[0] = f32Known[1] = false;
        topHistValid[0] = topHistValid[1] = false;
        e64Stale[0] = e64Stale[1] = false;
    }
    // After a rescale whose values are all exact floats, the float copy is
    // the rescaled column and the double column still holds the values
    // before the rescale: it is rewritten only for a reader that needs it.
    bool e64Stale[2] = {false, false};
    void ensure_e64(int col);
    // First median pass of each column, counted by the energy kernel that
    // wrote it; valid until the column changes.
    DBuf<unsigned long long> topHist[2];
    bool topHistValid[2] = {false, false};
    EnergyArgs energy_args() const;

    // What the adjoint of the last solve needs: the product of the rescale
    // factors applied to each cost column since its costs were last set, the
    // kind of the last result (0 none, 1 ratio, 2 minimum cost) and, for a
    // ratio, the time sum T of its cycle.
    double colScale[2] = {1.0, 1.0};
    int adjKind = 0;
    double adjT = 0;
    double adjLambda = 0;     // the ratio result's C / T in double
    double fdMax = 0;         // maxFd of the ("*", "feature") time column, as the energy used it
    long long fdArgmax = 0;   // the first feat_diff entry holding the maximum
    DBuf<long long> wAdjEdges;
    DBuf<double> wImport;
    // `wait`: finish the stream before returning (batched callers wait once
    // for all graphs instead)
    void backward_feat_diff(double grad, double* gradFd, bool accumulate, bool wait = true);
    void set_cost_vector(const double* in, int64_t rows, int64_t cols);
    void set_feat_diff(const double* fd, int64_t rows, int64_t cols);
    void set_feat_diff_device(const double* fd, int64_t rows, int64_t cols, bool wait = true);
    // After set_feat_diff_device the matrix lives only in dFD; the host copy
    // is read back when a host reader needs it (the feature-time maximum, the
    // CSV export).
    bool fdHostStale = false;
    void ensure_fd_host();

    // -------------------------------------------------------------------
    void solve_ratio(int K);
    void solve_min_cost(int K);
    // Batched ratio solves (pgc_solve_batch): the costs generated and
    // rescaled and a Bellman-Ford team of up to `ctas` CTAs prepared for the
    // device's solve in `job`; then the result taken from the finished job, or the
    // solve finished on the host when the device handed it back.
    void batch_begin(int K, PairJob& job, int threads, int ctas, size_t smemCap, bool regenerate);
    void batch_end(const PairJob& job);
    int batchK = 0;
    size_t batchSmem = 0;  // dynamic shared memory the prepared batch team needs
    size_t batch_smem_bytes() const { return batchSmem; }
    DBuf<int> bRecNodes[2];
    DBuf<long long> bRecEdges[2];
    DBuf<double> bRecC[2], bRecT[2];
    void export_csv();

    // cost export / product space
    void cost_vector(double* out);
    void cost_vector_noalloc(double* out);
    void product_space(int32_t* out);

  private:
    // solver helpers
    struct Run {
        int K, Kp;
        int costF32, timeKind;
        const void* cost;
        const void* time;
        double tconst;
        int blocks, threads;
        bool coop;
        bool sharedTables;  // single CTA keeping its DP records in shared memory
        int flagSync;       // neighbour hand-offs between steps (multi-CTA teams)
        int maxCtaSlices;   // most slices any CTA owns
        int rowCap;         // rows a step buffer holds (0: streams read in place)
        int stageSrcOnly;   // the buffers hold source indices only
        size_t smemBytes;   // dynamic shared memory per CTA
    };
    Run prepare_run(int K, bool ratio);
    // batch mode of prepare_run: a team of up to batchCtas CTAs of
    // batchThreads threads, DP records in global memory, staging only within
    // batchSmemCap bytes
    int batchThreads = 0;
    int batchCtas = 1;
    size_t batchSmemCap = 0;
    void solve_ratio_rescaled(int K);
    void ensure_workspace(int K, int blocks);
    std::vector<int> cta_cuts(int blocks, int K, int warps) const;
    void upload_cta_slices(const std::vector<int>& cut, int K, int warps);
    void upload_branch(const std::vector<int>& branchOf);
    // Every solve starts from an unwritten predecessor table (-1), like the
    // reference's freshly allocated solver state.
    void reset_predecessors() {
        PGC_CUDA(cudaMemsetAsync(wPred.p, 0xff, wPred.n * sizeof(int), stream));
    }
    BfParams params(const Run& r, int mode, int branchId, double lambda, double ub);
    Control launch_bf_call(const Run& r, const BfParams& p);
    std::vector<int> read_cycle_buffer(int len);
    void lookup_pairs(const std::vector<int>& src, const std::vector<int>& trgt, std::vector<long long>& edges,
                      std::vector<double>& c, std::vector<double>& t, double tconst);
    void rescale_columns(double scaling);
    DBuf<MedianState> wMedState;
    DBuf<unsigned long long> wMedHist, wMedCount;
    DBuf<double> wMedBand;
    void ensure_f32(int col);
    void rows_for_edges(const std::vector<long long>& edges);
};

// The product-graph topology depends only on EX, EY and the two graph flags,
// all fixed at construction; it is built and uploaded once.
void Graph::upload_template() {
    const std::string err = build_template(EX.data(), nex, EY.data(), ney, nvx, conj, prune, T);
    if (!err.empty()) throw Failure(PGC_ERR_ARG, err);
    for (int64_t i = 0; i < 2 * ney; ++i)
        if (EY[(size_t)i] >= nvy) throw Failure(PGC_ERR_ARG, "EY refers to a vertex outside VY");
    cudaStream_t s = stream;
    for (int p = 0; p < 2; ++p) {
        dSp[p].upload(T.sp[p].data(), T.sp[p].size(), s);
        dSrc[p].upload(T.src[p].data(), T.src[p].size(), s);
        dTedge[p].upload(T.tedge[p].data(), T.tedge[p].size(), s);
    }
    // The closing layer's source list differs from the interlayer one only
    // with two layers; otherwise the kernels read the interlayer list.
    if (T.nY == 2) dSrcDummy.upload(T.srcDummy.data(), T.srcDummy.size(), s);
    else dSrcDummy.release();
    // Template edge endpoints are read on the device only by the SO(3)
    // energies (frames of the edge's source and target).
    if (conj && reg) {
        dESrc.upload(T.eSrc.data(), T.eSrc.size(), s);
        dETrgt.upload(T.eTrgt.data(), T.eTrgt.size(), s);
        dENext.upload(T.eNext.data(), T.eNext.size(), s);
    } else {
        dESrc.release();
        dETrgt.release();
        dENext.release();
    }
    dEXcols.upload(T.eX.data(), T.eX.size(), s);
    dEYpat.upload(T.eY.data(), T.eY.size(), s);
    dEY.upload(EY.data(), EY.size(), s);
    dEX.upload(EX.data(), EX.size(), s);
    dVX.upload(VX.data(), VX.size(), s);
    dVY.upload(VY.data(), VY.size(), s);
    if (!fdHostStale) dFD.upload(FD.data(), FD.size(), s);  // else dFD already holds it
    templateReady = true;
}

// Graph-dependent fields of the energy kernels' arguments.
EnergyArgs Graph::energy_args() const {
    EnergyArgs a{};
    a.n = T.n;
    a.nY = T.nY;
    a.nvx = (int)nvx;
    a.nvy = (int)nvy;
    a.interEntries = T.entries[INTER];
    a.layerStride = T.layerStride();
    a.total = (long long)(T.nY + 1) * a.layerStride;
    a.tedgeInter = dTedge[INTER].p;
    a.tedgeIntra = dTedge[INTRA].p;
    a.eX = dEXcols.p;
    a.eY = dEYpat.p;
    a.eSrc = dESrc.p;
    a.eTrgt = dETrgt.p;
    a.eNext = dENext.p;
    a.EY = dEY.p;
    a.VX = dVX.p;
    a.VY = dVY.p;
    a.FD = dFD.p;
    return a;
}

// ---------------------------------------------------------------------------
// generate(): product_graph_generators.cpp:21-89
// ---------------------------------------------------------------------------
// Lets the energy kernel count the first median digit of its columns.
void Graph::count_top_digits(EnergyArgs& a) {
    for (int c = 0; c < ncols; ++c) {
        topHist[c].alloc((size_t)1 << kTopDigitBits);
        topHist[c].zero(stream);
    }
    a.hist0 = topHist[0].p;
    a.hist1 = ncols > 1 ? topHist[1].p : nullptr;
}

void Graph::generate() {
    if (conj && !normalsGiven)
        throw Failure(PGC_ERR_STATE, "cannot generate the conjugate product graph without normals (set_normals)");
    cudaStream_t s = stream;
    if (!templateReady) upload_template();
    generated = false;

    const long long stride = T.layerStride();
    const long long total = (long long)(T.nY + 1) * stride;
    EnergyArgs a = energy_args();
    if (!conj) {
        // deformationEnergy.cpp:97-103: two columns only for ("feature", "lengthnormalisation")
        const bool lengthMode = costName == "feature" && timeName == "lengthnormalisation";
        ncols = lengthMode ? 2 : 1;
        a.lengthMode = lengthMode;
        a.lineIntegral = reg || lengthMode;
        e64[0].alloc((size_t)total);
        a.out0 = e64[0].p;
        if (ncols > 1) {
            e64[1].alloc((size_t)total);
            a.out1 = e64[1].p;
        }
        count_top_digits(a);
        PGC_CUDA(launch_plain_energy(a, s, blockingSync));  // batch workers share the device
    } else {
        const int cm = string_to_mode(costName), tm = string_to_mode(timeName);
        if (!ho_supported(cm, tm))
            throw Failure(PGC_ERR_MODE, "cost time mode not supported: (" + costName + ", " + timeName + ")");
        ncols = (tm == NOMODE || tm == VANILLA) ? 1 : 2;
        a.costMode = cm;
        a.timeMode = tm;
        a.rlAlpha = rlAlpha;
        a.rlC = rlC;
        a.rlPwr = rlPwr;
        a.maxSO3 = (double)(float)robust_loss_host(2 * M_PI, rlAlpha, rlC, rlPwr);
        if (tm == FEATURE) {
            ensure_fd_host();
            double m = -std::numeric_limits<double>::infinity();
            long long at = 0;
            for (size_t i = 0; i < FD.size(); ++i)
                if (FD[i] > m) {
                    m = FD[i];
                    at = (long long)i;
                }
            a.maxFd = (double)(float)m;
            fdMax = a.maxFd;
            fdArgmax = at;
        }
        if (reg) {
            dNX.upload(NX.data(), NX.size(), s);
            dNY.upload(NY.data(), NY.size(), s);
            dQuat.alloc((size_t)T.nY * (size_t)nex);
            QuatArgs q{};
            q.nEX = (int)nex;
            q.nY = T.nY;
            q.n = T.n;
            q.prune = prune ? 1 : 0;
            q.EX = dEX.p;
            q.EY = dEY.p;
            q.VX = dVX.p;
            q.VY = dVY.p;
            q.NX = dNX.p;
            q.NY = dNY.p;
            q.out = dQuat.p;
            PGC_CUDA(launch_quaternions(q, s));
            a.quat = dQuat.p;
            a.quatEX = (int)nex;
            a.quatPrune = prune ? 1 : 0;
        }
        e64[0].alloc((size_t)total);
        a.out0 = e64[0].p;
        if (ncols > 1) {
            e64[1].alloc((size_t)total);
            a.out1 = e64[1].p;
        }
        count_top_digits(a);
        PGC_CUDA(launch_ho_energy(a, s));
        dQuat.release();
    }
    PGC_CUDA(sync_stream());
    energy_changed();
    for (int c = 0; c < ncols; ++c) topHistValid[c] = true;
    colScale[0] = colScale[1] = 1.0;
    adjKind = 0;
    generated = true;
}

// ---------------------------------------------------------------------------
// Rescaling: cost_time_ratio_solver.cpp:709-721 with utils::median
// (utils.hpp:196-209).  The k-th value is found by radix selection.
// ---------------------------------------------------------------------------
// Both cost columns' medians and rescales, enqueued whole on the handle's
// stream (launch_median_rescale: radix selection whose state stays on the
// device), then one wait.  The double column is rewritten only when some
// rescaled value is not a float.
void Graph::rescale_columns(double scaling) {
    const long long stride = T.layerStride();
    const long long total = (long long)(T.nY + 1) * stride;
    const long long count = (long long)T.nY * T.eBlock;
    if (count <= 0) throw Failure(PGC_ERR_STATE, "empty product graph");
    wMedState.alloc(2);
    wMedHist.alloc((size_t)1 << kMedianWideBits);
    wMedBand.alloc((size_t)kMedianCompact);
    wMedCount.alloc(1);
    PGC_CUDA(cudaMemsetAsync(wMedHist.p, 0, sizeof(unsigned long long) << kMedianWideBits, stream));
    auto args = [&](int col) {
        SelectArgs a{};
        a.col = e64[col].p;
        a.total = total;
        a.layerStride = stride;
        a.interEntries = T.entries[INTER];
        a.nY = T.nY;
        a.tedgeInter = dTedge[INTER].p;
        a.tedgeIntra = dTedge[INTRA].p;
        return a;
    };
    auto enqueue = [&](int col, bool allPasses) {
        PGC_CUDA(cudaMemsetAsync(wMedCount.p, 0, sizeof(unsigned long long), stream));
        const bool top = topHistValid[col] && !allPasses;
        PGC_CUDA(launch_median_rescale(args(col), top ? topHist[col].p : nullptr, wMedState.p + col, wMedHist.p,
                                       wMedBand.p, wMedCount.p, count, scaling, e32[col].p, 100 * scaling, allPasses,
                                       blockingSync, stream));
        stats.launches += (top ? 1 : 3) + (allPasses ? 10 : 2) + 4;
    };
    for (int col = 0; col < ncols; ++col) {
        ensure_e64(col);
        e32[col].alloc((size_t)total);
        enqueue(col, false);
    }
    MedianState st[2];
    d2h(st, wMedState.p, sizeof(MedianState) * (size_t)ncols);
    PGC_CUDA(sync_stream());
    // a column of few distinct values needs more digit passes: its chain
    // again with every pass (its float copy was not written)
    bool again = false;
    for (int col = 0; col < ncols; ++col) {
        if (st[col].err != 5) continue;
        enqueue(col, true);
        again = true;
    }
    if (again) {
        d2h(st, wMedState.p, sizeof(MedianState) * (size_t)ncols);
        PGC_CUDA(sync_stream());
    }
    bool rewrite = false;
    for (int col = 0; col < ncols; ++col) {
        if (st[col].err) throw Failure(PGC_ERR_INTERNAL, "median selection lost its rank");
        if (st[col].inexact) {
            PGC_CUDA(launch_rescale_f64(args(col), wMedState.p + col, 100 * scaling, stream));
            stats.launches++;
            rewrite = true;
        } else {
            e64Stale[col] = true;
        }
        f32Valid[col] = st[col].inexact == 0;
        f32Known[col] = true;
        topHistValid[col] = false;
        colScale[col] *= st[col].factor;
    }
    if (rewrite) PGC_CUDA(sync_stream());
}

void Graph::ensure_e64(int col) {
    if (!e64Stale[col]) return;
    PGC_CUDA(launch_to_f64(e32[col].p, e64[col].p, T.layerStride(), T.entries[INTER], T.nY, dTedge[INTER].p,
                           dTedge[INTRA].p, stream));
    stats.launches++;
    e64Stale[col] = false;
}

void Graph::ensure_f32(int col) {
    if (f32Known[col]) return;
    ensure_e64(col);
    const long long stride = T.layerStride();
    const long long total = (long long)(T.nY + 1) * stride;
    e32[col].alloc((size_t)total);
    wCount.alloc(1);
    const int one = 1;
    PGC_CUDA(cudaMemcpyAsync(wCount.p, &one, sizeof(int), cudaMemcpyHostToDevice, stream));
    PGC_CUDA(launch_to_f32(e64[col].p, e32[col].p, total, stride, T.entries[INTER], T.nY, dTedge[INTER].p,
                           dTedge[INTRA].p, wCount.p, stream));
    stats.launches++;
    int exact = 0;
    d2h(&exact, wCount.p, sizeof(int));
    PGC_CUDA(sync_stream());
    f32Valid[col] = exact != 0;
    f32Known[col] = true;
}

// ---------------------------------------------------------------------------
// Solver plumbing
// ---------------------------------------------------------------------------
Graph::Run Graph::prepare_run(int K, bool ratio) {
    if (K < 1) throw Failure(PGC_ERR_ARG, "max depth must be >= 1");
    const long long expanded = (long long)T.n * (T.nY + 1) * K;
    if (expanded >= INT_MAX) throw Failure(PGC_ERR_ARG, "product graph too large for 32-bit expanded node ids");
    Run r{};
    r.K = K;
    r.Kp = 1;
    while (r.Kp < K) r.Kp <<= 1;
    ensure_f32(0);
    r.costF32 = f32Valid[0] ? 1 : 0;
    if (!r.costF32) ensure_e64(0);
    r.cost = r.costF32 ? (const void*)e32[0].p : (const void*)e64[0].p;
    if (ratio && ncols > 1) {
        ensure_f32(1);
        r.timeKind = f32Valid[1] ? 1 : 2;
        if (!f32Valid[1]) ensure_e64(1);
        r.time = f32Valid[1] ? (const void*)e32[1].p : (const void*)e64[1].p;
        r.tconst = 0;
    } else {
        r.timeKind = 0;
        r.time = nullptr;
        r.tconst = ratio ? 50000.0 : 0.0;
    }
    // Team shape.  A warp relaxes one slice (32 nodes) per step, so a step
    // costs about one slice's batches of memory latency when every warp has
    // at most one slice.  Small graphs: one CTA that keeps the DP records in
    // shared memory.  Otherwise CTAs of up to kBfThreads threads, one per
    // (threads / 32) slices, up to the number that can be co-resident.  Each
    // CTA stages its next step's streams in two shared-memory buffers; when
    // they cannot fit, it reads the streams in place.
    DeviceInfo info{};
    PGC_CUDA(device_info(device, &info));
    const int sms = info.sms, smemOptin = info.smemOptin;
    const size_t smemCap = (size_t)std::max(0, smemOptin - 1024);  // static shared memory of the kernel
    const int costBytes = r.costF32 ? 4 : 8, timeBytes = r.timeKind == 1 ? 4 : r.timeKind == 2 ? 8 : 0;
    const bool stageOn = env_int("PGC_BF_STAGE", 1) != 0;
    std::vector<int> cut;
    auto stage_need = [&](int blocks, int& maxSl, int& rowCap) -> size_t {
        cut = cta_cuts(blocks, K, r.threads / 32);
        maxSl = 0;
        rowCap = 0;
        for (int c = 0; c < blocks; ++c) {
            const int a = cut[(size_t)c], b = cut[(size_t)c + 1];
            maxSl = std::max(maxSl, b - a);
            for (int p = 0; p < 2; ++p) rowCap = std::max(rowCap, T.sp[p][(size_t)b] - T.sp[p][(size_t)a]);
        }
        rowCap = std::max(rowCap, 1);
        return bf_stage_offset(maxSl) + 2 * bf_stage_buffer_bytes(rowCap, costBytes, timeBytes);
    };
    const size_t tables = bf_shared_table_bytes(T.n, r.Kp);
    if (batchThreads > 0) {
        // a team of the batched launch: up to batchCtas CTAs, none with
        // fewer than one slice; no shared DP tables; the two step buffers
        // only when they fit the launch's shared-memory budget
        r.threads = batchThreads;
        r.blocks = std::max(1, std::min(batchCtas, T.nslices));
        r.coop = false;
        r.sharedTables = false;
        r.flagSync = r.blocks > 1 && env_int("PGC_BF_FLAGS", 1) ? 1 : 0;
        int maxSl = 0, rowCap = 0;
        size_t need = stage_need(r.blocks, maxSl, rowCap);
        r.rowCap = rowCap;
        r.stageSrcOnly = 0;
        if (!stageOn || need > batchSmemCap) {
            const size_t srcOnly = bf_stage_offset(maxSl) + 2 * bf_stage_buffer_bytes(rowCap, 0, 0);
            if (stageOn && srcOnly <= batchSmemCap) {
                r.stageSrcOnly = 1;
                need = srcOnly;
            } else {
                r.rowCap = 0;
                need = bf_stage_offset(maxSl);
            }
        }
        if (need > batchSmemCap) throw Failure(PGC_ERR_ARG, "the graph's slice lists exceed the batch's shared memory");
        r.maxCtaSlices = maxSl;
        r.smemBytes = need;
        // the team's reductions outside the Bellman-Ford calls use every CTA
        ensure_workspace(K, std::max(r.blocks, batchCtas));
        upload_cta_slices(cut, K, r.threads / 32);
        return r;
    }
    int envBlocks = env_int("PGC_BF_BLOCKS", 0), envThreads = env_int("PGC_BF_THREADS", 0);
    if (!envBlocks) envBlocks = shapeBlocks;
    if (!envThreads) envThreads = shapeThreads;
    if (envThreads && (envThreads < 32 || envThreads > kBfThreads || envThreads % 32 != 0))
        throw Failure(PGC_ERR_ARG, "PGC_BF_THREADS must be a multiple of 32 in [32, 640]");
    int maxSl = 0, rowCap = 0;
    int blocks = envBlocks;
    if (blocks <= 0 && T.nslices <= env_int("PGC_BF_SINGLE_CTA_SLICES", 64) &&
        env_int("PGC_BF_SHARED_TABLES", 1) && tables + stage_need(1, maxSl, rowCap) <= smemCap)
        blocks = 1;
    r.threads = envThreads ? envThreads : kBfThreads;
    if (blocks == 1 && !envThreads) r.threads = std::min(kBfThreads, 32 * T.nslices);
    if (blocks <= 0) blocks = (T.nslices + r.threads / 32 - 1) / (r.threads / 32);
    if (teamCap > 0 && !envBlocks) blocks = std::min(blocks, teamCap);
    blocks = std::max(1, std::min(blocks, T.nslices));
    if (blocks == 1 && !envThreads) r.threads = std::min(kBfThreads, 32 * T.nslices);
    r.sharedTables = blocks == 1 && env_int("PGC_BF_SHARED_TABLES", 1) &&
                     tables + bf_stage_offset(T.nslices) <= smemCap;
    if (blocks > 1) {
        int perSm = 0;
        PGC_CUDA(bf_max_coop_blocks(r.costF32, r.timeKind, r.threads, 0, &perSm));
        if (perSm < 1) throw Failure(PGC_ERR_CUDA, "the Bellman-Ford kernel cannot be resident with this block size");
        blocks = std::min(blocks, sms * perSm);
    }
    const size_t fixed = r.sharedTables ? tables : 0;
    size_t need = stage_need(blocks, maxSl, rowCap);
    r.rowCap = rowCap;
    r.stageSrcOnly = 0;
    // PGC_BF_STAGE_SRC: 0 never stage the source indices alone, 1 (default)
    // when the whole streams do not fit, 2 always (tests)
    const int srcMode = env_int("PGC_BF_STAGE_SRC", 1);
    if (!stageOn || fixed + need > smemCap || srcMode == 2) {
        // the source indices alone, the costs and times prefetched to L2
        const size_t srcOnly = bf_stage_offset(maxSl) + 2 * bf_stage_buffer_bytes(rowCap, 0, 0);
        if (stageOn && srcMode && fixed + srcOnly <= smemCap) {
            r.stageSrcOnly = 1;
            need = srcOnly;
        } else {
            r.rowCap = 0;  // read the streams in place
            need = bf_stage_offset(maxSl);
        }
    }
    r.maxCtaSlices = maxSl;
    r.smemBytes = fixed + need;
    if (r.smemBytes > smemCap) throw Failure(PGC_ERR_ARG, "the product graph's DP tables do not fit shared memory");
    if (blocks > 1) {
        int perSm = 0;
        PGC_CUDA(bf_max_coop_blocks(r.costF32, r.timeKind, r.threads, r.smemBytes, &perSm));
        if (perSm < 1) throw Failure(PGC_ERR_CUDA, "the Bellman-Ford kernel cannot be resident with its shared memory");
        if (blocks > sms * perSm) {
            // fewer CTAs fit with this much shared memory: read in place
            blocks = sms * perSm;
            stage_need(blocks, maxSl, rowCap);
            r.rowCap = 0;
            r.stageSrcOnly = 0;
            r.maxCtaSlices = maxSl;
            r.smemBytes = bf_stage_offset(maxSl);
        }
    }
    r.blocks = blocks;
    r.coop = blocks > 1;
    r.flagSync = env_int("PGC_BF_FLAGS", 1) ? 1 : 0;
    ensure_workspace(K, blocks);
    if (cut.size() != (size_t)blocks + 1) stage_need(blocks, maxSl, rowCap);
    upload_cta_slices(cut, K, r.threads / 32);
    return r;
}

// CTA slice ranges of the team (plan_cta_cuts), cached per (blocks, K,
// warps).  A warp gathers bf_rows_per_batch(K) interlayer rows per batch
// (one row when K > 4) and bf_rows_per_batch(1) intralayer rows.
std::vector<int> Graph::cta_cuts(int blocks, int K, int warps) const {
    const std::string key = std::to_string(blocks) + "/" + std::to_string(K) + "/" + std::to_string(warps);
    {
        const auto it = cutCache.find(key);
        if (it != cutCache.end()) return it->second;
    }
    const int rb[2] = {K <= 4 ? bf_rows_per_batch(K) : 1, bf_rows_per_batch(1)};
    std::vector<int> cut = plan_cta_cuts(T, blocks, K, warps, rb);
    cutCache[key] = cut;
    return cut;
}

// Uploads the slice range of every CTA (cta_cuts) and every CTA's wait list
// (cta_wait_lists: the CTAs whose rows it reads through an in-edge, and the
// CTAs that read its rows).
void Graph::upload_cta_slices(const std::vector<int>& cut, int K, int warps) {
    const int blocks = (int)cut.size() - 1;
    if (cutBlocks == blocks && cutK == K && cutWarps == warps && ctaCut == cut) return;
    std::vector<int> ptr, idx;
    cta_wait_lists(T, cut, ptr, idx);
    wCtaSlice.upload(cut.data(), cut.size(), stream);
    wWaitPtr.upload(ptr.data(), ptr.size(), stream);
    if (idx.empty()) idx.push_back(0);  // keep a valid pointer; ptr says the lists are empty
    wWaitIdx.upload(idx.data(), idx.size(), stream);
    waitEntries = ptr.back();
    ctaCut = cut;
    cutBlocks = blocks;
    cutK = K;
    cutWarps = warps;
}

void Graph::ensure_workspace(int K, int blocks) {
    const size_t n = (size_t)T.n;
    int Kp = 1;
    while (Kp < K) Kp <<= 1;
    const size_t expanded = n * (size_t)(T.nY + 1) * (size_t)K;
    if (wsK != K || wPred.n < expanded) {
        wDv.alloc(2 * n * Kp);
        wDoh.alloc(2 * n * Kp);
        wPred.alloc(expanded);
        PGC_CUDA(cudaMemsetAsync(wPred.p, 0xff, expanded * sizeof(int), stream));  // -1
        wsK = K;
    }
    if (wBak.n < n) {
        wBak.alloc(n);
        wLapNext.alloc(n);
        wLapSteps.alloc(n);
        wWalks.alloc(n);
        wCandStat.alloc(n);
        wCandV0.alloc(n);
        wCandSteps.alloc(n);
        wBranch.alloc(n);
        wLb.alloc(n);
        wOrigin.alloc(n);
        wMean.alloc(n);
    }
    if (wLayerFlag.n < (size_t)T.nY + 1) {
        wLayerFlag.alloc((size_t)T.nY + 1);
        wLayerFlag.zero(stream);
        ctlEpoch = 0;
    }
    wCtl.alloc(1);
    wStepDone.alloc((size_t)blocks * kStepDoneStride);
    wRedVal.alloc(2 * (size_t)blocks);
    wRedIdx.alloc(2 * (size_t)blocks);
    wRedAux.alloc((size_t)blocks);
    wRedAux64.alloc((size_t)blocks);
    const size_t cap = std::min<size_t>((size_t)numNodes() + 4, (size_t)1 << 26);
    wCycle.alloc(cap);
}

void Graph::upload_branch(const std::vector<int>& branchOf) {
    PGC_CUDA(cudaMemcpyAsync(wBranch.p, branchOf.data(), branchOf.size() * sizeof(int), cudaMemcpyHostToDevice,
                             stream));
}

BfParams Graph::params(const Run& r, int mode, int branchId, double lambda, double ub) {
    BfParams p{};
    p.n = T.n;
    p.nY = T.nY;
    p.K = r.K;
    p.Kp = r.Kp;
    p.nslices = T.nslices;
    p.numNodes = numNodes();
    p.spInter = dSp[INTER].p;
    p.spIntra = dSp[INTRA].p;
    p.srcInter = dSrc[INTER].p;
    p.srcDummy = dSrcDummy.p ? dSrcDummy.p : dSrc[INTER].p;
    p.srcIntra = dSrc[INTRA].p;
    p.interEntries = T.entries[INTER];
    p.intraEntries = T.entries[INTRA];
    p.layerStride = T.layerStride();
    p.cost = r.cost;
    p.time = r.time;
    p.tconst = r.tconst;
    p.dv = wDv.p;
    p.doh = wDoh.p;
    p.bak = wBak.p;
    p.pred = wPred.p;
    p.ctaSlice = wCtaSlice.p;
    p.waitPtr = wWaitPtr.p;
    p.waitIdx = wWaitIdx.p;
    p.stepDone = wStepDone.p;
    p.flagSync = r.flagSync;
    p.maxCtaSlices = r.maxCtaSlices;
    p.rowCap = r.rowCap;
    p.stageSrcOnly = r.stageSrcOnly;
    p.lapNext = wLapNext.p;
    p.lapSteps = wLapSteps.p;
    p.walks = wWalks.p;
    p.candStat = wCandStat.p;
    p.candV0 = wCandV0.p;
    p.candSteps = wCandSteps.p;
    p.layerFlag = wLayerFlag.p;
    p.branchOf = wBranch.p;
    p.branchId = branchId;
    p.lambda = lambda;
    p.ub = ub;
    p.mode = mode;
    p.maxSweeps = 0;
    // device waits give up after this many polls (PGC_BF_SPIN_LIMIT: tests
    // of the timeout path use a short one); two test hooks, off in every
    // solve: PGC_BF_TEST_STALL_CTA makes that CTA's step hand-off also wait
    // for a word no code writes, and PGC_BF_LITERAL_WALKS=1 decides every
    // candidate by the literal predecessor walk
    p.spinLimit = (unsigned)std::max(1, env_int("PGC_BF_SPIN_LIMIT", (int)kDefaultSpinLimit));
    p.stallCta = env_int("PGC_BF_TEST_STALL_CTA", -1);
    p.literalAll = env_int("PGC_BF_LITERAL_WALKS", 0) ? 1 : 0;
    p.ctl = wCtl.p;
    p.cycleBuf = wCycle.p;
    p.cycleCap = (long long)wCycle.n;
    p.redVal = wRedVal.p;
    p.redIdx = wRedIdx.p;
    p.redAux = wRedAux.p;
    p.redAux64 = wRedAux64.p;
    p.lbOut = wLb.p;
    p.originOut = wOrigin.p;
    return p;
}

Control Graph::launch_bf_call(const Run& r, const BfParams& p) {
    Control c{};
    c.epoch = ctlEpoch;
    PGC_CUDA(cudaMemcpyAsync(wCtl.p, &c, sizeof(Control), cudaMemcpyHostToDevice, stream));
    if (!timeEvents[0]) {
        PGC_CUDA(cudaEventCreate(&timeEvents[0]));
        PGC_CUDA(cudaEventCreate(&timeEvents[1]));
    }
    cudaEvent_t e0 = timeEvents[0], e1 = timeEvents[1];
    PGC_CUDA(cudaEventRecord(e0, stream));
    PGC_CUDA(launch_bf(p, r.costF32, r.timeKind, r.blocks, r.threads, r.coop, r.sharedTables, r.smemBytes, stream));
    PGC_CUDA(cudaEventRecord(e1, stream));
    stats.launches++;
    d2h(&c, wCtl.p, sizeof(Control));
    PGC_CUDA(sync_stream());
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    stats.deviceMs += ms;
    ctlEpoch = c.epoch;
    stats.bfCalls++;
    stats.sweeps += c.sweeps;
    stats.candidates += c.candidates;
    stats.fallbackWalks += c.fallbackWalks;
    stats.cycA += c.cycPhaseA;
    stats.cycB += c.cycPhaseB;
    stats.cycSync += c.cycSync;
    stats.cycTail += c.cycTail;
    stats.cycWrap += c.cycWrap;
    stats.cycCand += c.cycCand;
    stats.cycLead += c.cycLead;
    stats.cycStage += c.cycStage;
    stats.steps += (long long)c.sweeps * ((long long)(T.nY + 1) * (T.entries[INTRA] == 0 ? 1 : r.K) - 1);
    stats.ctas = r.blocks;
    stats.threads = r.threads;
    stats.waitEntries = r.blocks > 1 ? waitEntries : 0;
    if (c.error) {
        // The launch stopped mid-sweep: layers it stamped carry stamps the
        // next launch would issue again.  Clear them, so the handle solves
        // correctly afterwards.
        wLayerFlag.zero(stream);
        ctlEpoch = 0;
        PGC_CUDA(sync_stream());
        throw Failure(PGC_ERR_TIMEOUT,
                      "a wait of the Bellman-Ford kernel (team barrier, step hand-off or staged copy) ran out");
    }
    if (c.status == BF_ERR_EMPTY_BRANCH) throw Failure(PGC_ERR_INTERNAL, "no nodes in branch");
    if (c.status == BF_ERR_CYCLE_CAP) throw Failure(PGC_ERR_INTERNAL, "cycle longer than its buffer");
    if (c.status == BF_ERR_WALK) throw Failure(PGC_ERR_INTERNAL, "predecessor walk left the node range");
    if (c.status == BF_ERR_CHUNK) throw Failure(PGC_ERR_INTERNAL, "a slice exceeds the shared-memory scratch");
    if (c.status == BF_RUNNING) throw Failure(PGC_ERR_INTERNAL, "Bellman-Ford launch ended without a verdict");
    return c;
}

std::vector<int> Graph::read_cycle_buffer(int len) {
    std::vector<int> out((size_t)std::max(0, len));
    if (len > 0)
        d2h(out.data(), wCycle.p, sizeof(int) * (size_t)len);
    PGC_CUDA(sync_stream());
    return out;
}

void Graph::lookup_pairs(const std::vector<int>& src, const std::vector<int>& trgt, std::vector<long long>& edges,
                         std::vector<double>& c, std::vector<double>& t, double tconst) {
    const size_t m = src.size();
    edges.assign(m, -2);
    c.assign(m, 0);
    t.assign(m, 0);
    if (m == 0) return;
    wPairS.upload(src.data(), m, stream);
    wPairT.upload(trgt.data(), m, stream);
    wEdgeOut.alloc(m);
    wCOut.alloc(m);
    wTOut.alloc(m);
    LookupArgs a{};
    a.n = T.n;
    a.nY = T.nY;
    a.numNodes = numNodes();
    a.eBlock = T.eBlock;
    a.spInter = dSp[INTER].p;
    a.spIntra = dSp[INTRA].p;
    a.srcInter = dSrc[INTER].p;
    a.srcDummy = dSrcDummy.p ? dSrcDummy.p : dSrc[INTER].p;
    a.srcIntra = dSrc[INTRA].p;
    a.tedgeInter = dTedge[INTER].p;
    a.tedgeIntra = dTedge[INTRA].p;
    a.interEntries = T.entries[INTER];
    a.layerStride = T.layerStride();
    a.c64 = e64[0].p;
    a.t64 = ncols > 1 ? e64[1].p : nullptr;
    a.c32 = e64Stale[0] ? e32[0].p : nullptr;
    a.t32 = ncols > 1 && e64Stale[1] ? e32[1].p : nullptr;
    a.tconst = tconst;
    a.pairSrc = wPairS.p;
    a.pairTrgt = wPairT.p;
    a.count = (int)m;
    a.edgeOut = wEdgeOut.p;
    a.cOut = wCOut.p;
    a.tOut = wTOut.p;
    PGC_CUDA(launch_lookup_pairs(a, stream));
    stats.launches++;
    d2h(edges.data(), wEdgeOut.p, m * sizeof(long long));
    d2h(c.data(), wCOut.p, m * sizeof(double));
    d2h(t.data(), wTOut.p, m * sizeof(double));
    PGC_CUDA(sync_stream());
}

void Graph::rows_for_edges(const std::vector<long long>& edges) {
    resCols = T.cols();
    resRows = (int64_t)edges.size();
    resMatching.assign((size_t)(resRows * resCols), 0);
    for (size_t i = 0; i < edges.size(); ++i) product_row(T, EY.data(), edges[i], &resMatching[i * (size_t)resCols]);
    resEdges = edges;
}

// ---------------------------------------------------------------------------
// Cost/time-ratio solver (cost_time_ratio_solver.cpp:741-900)
// ---------------------------------------------------------------------------
namespace {

struct RatioEval {
    double ratio, wsum;
};

// computeRatioForCycle (cost_time_ratio_solver.cpp:88-133) over the per-pair
// costs and times of a stored cycle.
RatioEval eval_cycle(const CycleRec& cy, double lambda) {
    double C = 0, Tm = 0, W = 0;
    for (size_t i = 0; i < cy.c.size(); ++i) {
        C += cy.c[i];
        Tm += cy.t[i];
        W += cy.c[i] - lambda * cy.t[i];
    }
    return {C / Tm, W};
}

}  // namespace

void Graph::solve_ratio(int K) {
    ensure_generated();
    stats = Stats();
    const auto wall0 = std::chrono::steady_clock::now();
    const double scaling = 100000.0;
    // In-place rescale of the generator's costs (cost_time_ratio_solver.cpp:875-882).
    rescale_columns(scaling);
    solve_ratio_rescaled(K);
    (void)wall0;
}

// The ratio solve after the rescale: the initial upper bound, then branch
// and bound with Lawler in each branch (cost_time_ratio_solver.cpp:741-864).
void Graph::solve_ratio_rescaled(int K) {
    const double scaling = 100000.0;
    Run r = prepare_run(K, true);
    reset_predecessors();
    const int n = T.n;
    const long long nn = numNodes();
    const double tconst = ncols > 1 ? 0.0 : scaling / 2;
    const double tolerance = (double)(float)1e-8;

    // A cycle from the device walk (p(v0), ..., v0) -> reference order
    // [v0, ..., p(v0), v0 + numNodes], with its edges.
    auto make_cycle = [&](std::vector<int> walk, bool closeWithCopy) {
        CycleRec cy;
        std::reverse(walk.begin(), walk.end());
        if (closeWithCopy) walk.push_back(walk.front() + (int)nn);
        cy.nodes = walk;
        std::vector<int> s, t;
        for (size_t i = 0; i + 1 < walk.size(); ++i) {
            int a = walk[i], b = walk[i + 1];
            if (b < n && a > n) b += (int)nn;  // cost_time_ratio_solver.cpp:109-111
            s.push_back(a);
            t.push_back(b);
        }
        lookup_pairs(s, t, cy.edges, cy.c, cy.t, tconst);
        for (long long e : cy.edges)
            if (e < 0) throw Failure(PGC_ERR_INTERNAL, "cycle edge not found in the product graph");
        return cy;
    };

    std::vector<int> branchOf((size_t)n, 0);
    CycleRec negativeCycle;
    double currentRatio = 0;
    int numNodesInBranch = 0;

    // ---- initial upper bound (cost_time_ratio_solver.cpp:652-707) ----
    {
        std::vector<float> mean((size_t)n);
        std::vector<int> cnt((size_t)n);
        if (e64Stale[0])
            PGC_CUDA(launch_layer1_mean(e32[0].p, T.layerStride(), T.entries[INTER], n, T.nslices, dSp[INTER].p,
                                        dSp[INTRA].p, dSrc[INTER].p, dSrc[INTRA].p, wMean.p, wCandStat.p, stream));
        else
            PGC_CUDA(launch_layer1_mean(e64[0].p, T.layerStride(), T.entries[INTER], n, T.nslices, dSp[INTER].p,
                                        dSp[INTRA].p, dSrc[INTER].p, dSrc[INTRA].p, wMean.p, wCandStat.p, stream));
        stats.launches++;
        d2h(mean.data(), wMean.p, sizeof(float) * n);
        d2h(cnt.data(), wCandStat.p, sizeof(int) * n);
        PGC_CUDA(sync_stream());
        float bestCost = std::numeric_limits<float>::infinity();
        int bestV = 0;
        for (int v = 0; v < n; ++v)
            if (mean[(size_t)v] < bestCost && cnt[(size_t)v] > 3) {
                bestCost = mean[(size_t)v];
                bestV = v;
            }
        std::fill(branchOf.begin(), branchOf.end(), 1);
        branchOf[(size_t)bestV] = 0;
        upload_branch(branchOf);
        currentRatio = 10;
        const double ub = (double)std::numeric_limits<float>::infinity();
        const Control c = launch_bf_call(r, params(r, 1, 0, currentRatio, ub));
        if (c.status == BF_LAYER_UNREACHED) {
            // The sweep from the start node reached no node of some layer: a
            // 2D-degenerate node of a conjugate graph with K = 1, whose
            // out-edges are all intralayer.  The reference then rates its
            // empty cycle (cost_time_ratio_solver.cpp:357-365, :686-697): the
            // bound is 0/0 = NaN, every Bellman-Ford call at lambda = NaN
            // stops at layer 1 on the empty cycle (a zero cycle, :574-577),
            // the branch is pushed and popped as valid (:809-815, :834-838),
            // and the solve returns (true, NaN, no rows) (:855-862).  That
            // result is set here without those launches.  It has no cycle
            // to differentiate.
            stats.lawlerIters = 0;
            resPasses = true;
            resObjective = std::numeric_limits<float>::quiet_NaN();
            rows_for_edges({});
            adjKind = 0;
            adjT = 0;
            return;
        }
        if (c.status != BF_UB_DONE)
            throw Failure(PGC_ERR_INTERNAL, "no closed path through the upper-bound start node");
        numNodesInBranch = c.numInBranch;
        negativeCycle = make_cycle(read_cycle_buffer(c.cycleLen), false);
        RatioEval ev = eval_cycle(negativeCycle, currentRatio);
        double cycleCost = (double)(float)ev.wsum;
        int guard = 0;
        while (cycleCost > 0 || std::isnan(cycleCost)) {
            if (++guard > 4000) throw Failure(PGC_ERR_INTERNAL, "upper-bound ratio search does not terminate");
            currentRatio += currentRatio;
            ev = eval_cycle(negativeCycle, currentRatio);
            cycleCost = (double)(float)ev.wsum;
        }
        currentRatio = (double)(float)ev.ratio;
    }

    // ---- branch and bound (cost_time_ratio_solver.cpp:794-851) ----
    int branchId = 0, maxBranchId = 0;
    double ratioUpperBound = currentRatio;
    double lowerBoundOfCurrentBranch = 0;
    std::vector<int> zeroLayerHits;
    BranchHeap heap(n);
    heap.push(0, branchId);
    std::vector<unsigned char> validLb((size_t)n, 0);
    std::map<int, CycleRec> validCycles;
    std::fill(branchOf.begin(), branchOf.end(), 0);
    upload_branch(branchOf);

    auto bellman_ford = [&](double lambda) -> BfOutcome {
        const Control c = launch_bf_call(r, params(r, 0, branchId, lambda, std::numeric_limits<float>::infinity()));
        numNodesInBranch = c.numInBranch;
        auto old_is_zero = [&]() {
            return round_to_int(eval_cycle(negativeCycle, lambda).wsum) == 0;
        };
        switch (c.status) {
            case BF_LAYER_UNREACHED:
            case BF_WRAP_NO_IMPROVE:
                return old_is_zero() ? BfOutcome::ZERO_CYCLE : BfOutcome::NO_NEGATIVE_CYCLE;
            case BF_MAX_SWEEPS:
                return BfOutcome::NO_NEGATIVE_CYCLE;
            case BF_FOUND_CYCLE: {
                CycleRec cy = make_cycle(read_cycle_buffer(c.cycleLen), true);
                const int integral = round_to_int(eval_cycle(cy, lambda).wsum);
                if (integral < 0) {
                    negativeCycle = std::move(cy);
                    return BfOutcome::FOUND_NEGATIVE_CYCLE;
                }
                if (integral == 0) return BfOutcome::NO_NEGATIVE_CYCLE;
                return old_is_zero() ? BfOutcome::ZERO_CYCLE : BfOutcome::NO_NEGATIVE_CYCLE;
            }
            default:
                throw Failure(PGC_ERR_INTERNAL, "unexpected Bellman-Ford status " + std::to_string(c.status));
        }
    };

    // lawlerSoubroutine (cost_time_ratio_solver.cpp:558-635)
    auto lawler = [&]() -> bool {
        int i = 0;
        const int maxiter = 1000;
        double oldRatio = currentRatio;
        for (;;) {
            const BfOutcome s = bellman_ford(currentRatio);
            stats.lawlerIters++;
            if (s != BfOutcome::FOUND_NEGATIVE_CYCLE) break;
            currentRatio = eval_cycle(negativeCycle, currentRatio).ratio;
            if (std::fabs(oldRatio - currentRatio) < tolerance) break;
            if (currentRatio - tolerance > oldRatio) break;
            oldRatio = currentRatio;
            if (i > maxiter) break;
            ++i;
        }
        lowerBoundOfCurrentBranch = currentRatio;
        int numWraps = 0;
        zeroLayerHits.clear();
        bool entered = true, left = false;
        for (int vtx : negativeCycle.nodes) {
            if (left && vtx < n) { entered = true; left = false; }
            if (entered) { zeroLayerHits.push_back(vtx); entered = false; }
            if (vtx >= n && !left) { ++numWraps; left = true; }
        }
        return numWraps > 1;
    };

    while (!heap.isEmpty()) {
        const auto top = heap.pop();
        branchId = (int)top.second;
        if (validLb[(size_t)branchId]) {
            ratioUpperBound = top.first;
            negativeCycle = validCycles.at(branchId);
            break;
        }
        stats.branches++;
        currentRatio = ratioUpperBound;
        const bool wraps = lawler();
        if (ratioUpperBound < heap.peak() && !wraps) break;
        if (!wraps) {
            // ratioLowerBoundOfCurrentBranch is never assigned in the reference
            // (cost_time_ratio_solver.cpp:835); the branch's final ratio is used.
            heap.push(lowerBoundOfCurrentBranch, branchId);
            validLb[(size_t)branchId] = 1;
            validCycles.emplace(branchId, negativeCycle);
            continue;
        }
        if (numNodesInBranch == 1) continue;
        // branch() (cost_time_ratio_solver.cpp:142-179; the rest is unreachable)
        int offset = 0;
        for (int hit : zeroLayerHits) {
            if (offset > 0) branchOf[(size_t)hit] = maxBranchId + offset;
            ++offset;
        }
        for (int v = 0; v < n; ++v)
            if (branchOf[(size_t)v] == branchId) branchOf[(size_t)v] = maxBranchId;
        maxBranchId += offset;
        for (int hit : zeroLayerHits) heap.push(lowerBoundOfCurrentBranch, branchOf[(size_t)hit]);
        upload_branch(branchOf);
    }

    const RatioEval fin = eval_cycle(negativeCycle, currentRatio);
    resPasses = true;
    resObjective = (float)fin.ratio;
    rows_for_edges(negativeCycle.edges);
    adjKind = 1;
    adjT = 0;
    for (double t : negativeCycle.t) adjT += t;
    adjLambda = fin.ratio;
}

// Host wall time the batch workers spent in batch_begin's phases, summed
// over workers (ns): costs generated, columns rescaled, team prepared.
// Printed by pgc_solve_batch when PGC_BATCH_PHASES is set.
std::atomic<long long> g_batchPhaseNs[3];

void Graph::batch_begin(int K, PairJob& J, int threads, int ctas, size_t smemCap, bool regenerate) {
    const auto t0 = std::chrono::steady_clock::now();
    if (regenerate) generate();
    else ensure_generated();
    if (blockingSync) PGC_CUDA(sync_stream());
    const auto t1 = std::chrono::steady_clock::now();
    stats = Stats();
    batchK = K;
    const double scaling = 100000.0;
    rescale_columns(scaling);
    const auto t2 = std::chrono::steady_clock::now();
    struct PhaseTimer {
        std::chrono::steady_clock::time_point a, b, c;
        ~PhaseTimer() {
            const auto ns = [](auto x, auto y) {
                return (long long)std::chrono::duration_cast<std::chrono::nanoseconds>(y - x).count();
            };
            g_batchPhaseNs[0] += ns(a, b);
            g_batchPhaseNs[1] += ns(b, c);
            g_batchPhaseNs[2] += ns(c, std::chrono::steady_clock::now());
        }
    } phaseTimer{t0, t1, t2};
    batchThreads = threads;
    batchCtas = std::max(1, ctas);
    batchSmemCap = smemCap;
    Run r;
    try {
        r = prepare_run(K, true);
    } catch (...) {
        batchThreads = 0;
        throw;
    }
    batchThreads = 0;
    batchSmem = r.smemBytes;
    reset_predecessors();
    // PGC_BATCH_CYCLE_CAP (tests): a smaller record, so that graphs are
    // handed back to the host
    const long long capMax = std::min<long long>(kBatchCycleCap, std::max(1, env_int("PGC_BATCH_CYCLE_CAP", (int)kBatchCycleCap)));
    const int cap = (int)std::min<long long>(numNodes() + 4, capMax);
    for (int k = 0; k < 2; ++k) {
        bRecNodes[k].alloc((size_t)cap + 1);
        bRecEdges[k].alloc((size_t)cap);
        bRecC[k].alloc((size_t)cap);
        bRecT[k].alloc((size_t)cap);
    }
    J = PairJob{};
    J.bf = params(r, 0, 0, 0.0, std::numeric_limits<float>::infinity());
    J.bf.ctaSlice = wCtaSlice.p;
    J.ctas = r.blocks;
    J.threads = r.threads;
    LookupArgs& a = J.lk;
    a.n = T.n;
    a.nY = T.nY;
    a.numNodes = numNodes();
    a.eBlock = T.eBlock;
    a.spInter = dSp[INTER].p;
    a.spIntra = dSp[INTRA].p;
    a.srcInter = dSrc[INTER].p;
    a.srcDummy = dSrcDummy.p ? dSrcDummy.p : dSrc[INTER].p;
    a.srcIntra = dSrc[INTRA].p;
    a.tedgeInter = dTedge[INTER].p;
    a.tedgeIntra = dTedge[INTRA].p;
    a.interEntries = T.entries[INTER];
    a.layerStride = T.layerStride();
    a.c64 = e64[0].p;
    a.t64 = ncols > 1 ? e64[1].p : nullptr;
    a.c32 = e64Stale[0] ? e32[0].p : nullptr;
    a.t32 = ncols > 1 && e64Stale[1] ? e32[1].p : nullptr;
    a.tconst = ncols > 1 ? 0.0 : scaling / 2;
    J.branchOf = wBranch.p;
    J.tconst = a.tconst;
    for (int k = 0; k < 2; ++k) {
        J.recNodes[k] = bRecNodes[k].p;
        J.recEdges[k] = bRecEdges[k].p;
        J.recC[k] = bRecC[k].p;
        J.recT[k] = bRecT[k].p;
    }
    J.cap = cap;
    J.status = PAIR_PENDING;
    Control c{};
    c.epoch = ctlEpoch;
    PGC_CUDA(cudaMemcpyAsync(wCtl.p, &c, sizeof(Control), cudaMemcpyHostToDevice, stream));
    PGC_CUDA(sync_stream());
}

void Graph::batch_end(const PairJob& J) {
    Control c{};
    d2h(&c, wCtl.p, sizeof(Control));
    PGC_CUDA(sync_stream());
    ctlEpoch = c.epoch;
    stats.bfCalls = J.bfCalls;
    stats.sweeps = J.sweeps;
    stats.lawlerIters = J.lawlerIters;
    stats.candidates = J.candidates;
    stats.fallbackWalks = J.fallbackWalks;
    stats.branches = 1;
    stats.launches += 1;
    // the lead thread's cycle counters, summed over the solve's calls
    stats.cycA = c.cycPhaseA;
    stats.cycB = c.cycPhaseB;
    stats.cycSync = c.cycSync;
    stats.cycTail = c.cycTail;
    stats.cycWrap = c.cycWrap;
    stats.cycCand = c.cycCand;
    stats.cycLead = c.cycLead;
    stats.cycStage = c.cycStage;
    stats.steps = J.sweeps * ((long long)(T.nY + 1) * (T.entries[INTRA] == 0 ? 1 : batchK) - 1);
    {
        DeviceInfo info{};
        if (device_info(device, &info) == cudaSuccess && info.clockKhz > 0)
            stats.deviceMs = (double)J.cycles / info.clockKhz;  // the CTA's time on this graph at the top SM clock
    }
    stats.ctas = J.ctas;
    stats.threads = J.threads;
    switch (J.status) {
        case PAIR_DONE: {
            std::vector<long long> edges((size_t)std::max(0, J.nEdges));
            if (J.nEdges > 0) d2h(edges.data(), bRecEdges[J.rec].p, sizeof(long long) * edges.size());
            PGC_CUDA(sync_stream());
            resPasses = J.passes != 0;
            resObjective = J.objective;
            rows_for_edges(edges);
            adjKind = 1;
            adjT = J.adjT;
            adjLambda = J.ratio;
            return;
        }
        case PAIR_NAN:
            stats.lawlerIters = 0;
            resPasses = true;
            resObjective = std::numeric_limits<float>::quiet_NaN();
            rows_for_edges({});
            adjKind = 0;
            adjT = 0;
            return;
        case PAIR_HOST:
            // branch and bound (or a cycle longer than the device record):
            // the host's solve from the rescaled costs
            stats = Stats();
            solve_ratio_rescaled(batchK);
            return;
        case PAIR_ERR_WAIT:
            wLayerFlag.zero(stream);
            ctlEpoch = 0;
            PGC_CUDA(sync_stream());
            throw Failure(PGC_ERR_TIMEOUT, "a wait of the batched Bellman-Ford solve ran out");
        case PAIR_ERR_UB:
            throw Failure(PGC_ERR_INTERNAL, "no closed path through the upper-bound start node");
        case PAIR_ERR_EDGE:
            throw Failure(PGC_ERR_INTERNAL, "cycle edge not found in the product graph");
        case PAIR_ERR_GUARD:
            throw Failure(PGC_ERR_INTERNAL, "upper-bound ratio search does not terminate");
        case PAIR_ERR_BF:
            if (J.bfStatus == BF_ERR_EMPTY_BRANCH) throw Failure(PGC_ERR_INTERNAL, "no nodes in branch");
            if (J.bfStatus == BF_ERR_CYCLE_CAP) throw Failure(PGC_ERR_INTERNAL, "cycle longer than its buffer");
            if (J.bfStatus == BF_ERR_WALK) throw Failure(PGC_ERR_INTERNAL, "predecessor walk left the node range");
            if (J.bfStatus == BF_ERR_CHUNK) throw Failure(PGC_ERR_INTERNAL, "a slice exceeds the shared-memory scratch");
            if (J.bfStatus == BF_RUNNING) throw Failure(PGC_ERR_INTERNAL, "Bellman-Ford launch ended without a verdict");
            throw Failure(PGC_ERR_INTERNAL, "unexpected Bellman-Ford status " + std::to_string(J.bfStatus));
        default:
            throw Failure(PGC_ERR_INTERNAL, "the batched solve ended without a verdict");
    }
}

// ---------------------------------------------------------------------------
// Minimum-cost solver (dijkstra_solver.cpp:203-579)
// ---------------------------------------------------------------------------
void Graph::solve_min_cost(int K) {
    ensure_generated();
    stats = Stats();
    Run r = prepare_run(K, false);
    reset_predecessors();
    const int n = T.n;
    const long long nn = numNodes();

    // branch graph: the reference's branchGraph when it exists (conjugate
    // graph, conj_product_space.cpp:177-225; plain graph with pruning,
    // product_space.cpp:122-131), else the in-edge sets of layer 0
    // (dijkstra_solver.cpp:93-94).  Entries are used as edge ids
    // (SRCIds(e)), exactly as the reference does (dijkstra_solver.cpp:137-139).
    std::vector<std::vector<long>> bg;
    const bool haveBranchGraph = conj || prune;
    if (haveBranchGraph) {
        std::vector<std::set<long>> sets((size_t)n);
        if (!conj) {
            for (int64_t j = 0; j < nex; ++j) sets[(size_t)EX[2 * j]].insert(EX[2 * j + 1]);
        } else {
            std::vector<std::vector<int>> out((size_t)T.nvx);
            for (int64_t e = 0; e < nex; ++e) out[(size_t)EX[2 * e]].push_back((int)e);
            const long nE = (long)nex;
            for (long j = 0; j < nE; ++j) {
                sets[(size_t)j].insert(j + nE);
                if (!prune) {
                    sets[(size_t)(j + nE)].insert(j + 2 * nE);
                    sets[(size_t)(j + 2 * nE)].insert(j);
                } else {
                    sets[(size_t)(j + nE)].insert(j);
                }
                for (int e : out[(size_t)EX[2 * j]]) {
                    sets[(size_t)j].insert(e);
                    sets[(size_t)(j + nE)].insert(e + nE);
                    if (!prune) sets[(size_t)(j + 2 * nE)].insert(e + 2 * nE);
                }
            }
        }
        bg.resize((size_t)n);
        for (int v = 0; v < n; ++v) bg[(size_t)v].assign(sets[(size_t)v].begin(), sets[(size_t)v].end());
    } else {
        bg.assign((size_t)n, std::vector<long>{-1});
        for (int64_t t = 0; t < T.eBlock; ++t)
            if (!T.eNext[(size_t)t]) bg[(size_t)T.eTrgt[(size_t)t]].push_back((long)t);
    }
    // SRCIds(e) of an edge id (block * eBlock + offset).
    auto src_of = [&](long e) -> long {
        if (e < 0) return -1;
        const long long b = e / T.eBlock, t = e % T.eBlock;
        if (b >= T.nY) return LONG_MAX;
        return (long)(b * n + T.eSrc[(size_t)t]);
    };

    std::vector<int> branchOf((size_t)n, 0);
    upload_branch(branchOf);
    int branchId = 0, maxBranchId = 0, numNodesInBranch = 0;
    double upperBound = std::numeric_limits<double>::infinity();
    double lowerBoundOfCurrentBranch = 0;
    bool upperboundFoundOnFirstTry = false;
    int branchingSrcNode = -1, branchingTargetNode = -1;
    std::vector<int> cycle;  // walk order: [p(vLast), ..., start]
    std::vector<std::pair<double, int>> lowerBounds;

    auto extract = [&](int v) {
        BfParams p = params(r, 2, branchId, 0.0, upperBound);
        Control c{};
        c.epoch = ctlEpoch;
        PGC_CUDA(cudaMemcpyAsync(wCtl.p, &c, sizeof(Control), cudaMemcpyHostToDevice, stream));
        PGC_CUDA(launch_extract_path(p, v, stream));
        stats.launches++;
        d2h(&c, wCtl.p, sizeof(Control));
        PGC_CUDA(sync_stream());
        if (c.status < 0) throw Failure(PGC_ERR_INTERNAL, "minimum-cost path extraction failed");
        return read_cycle_buffer(c.cycleLen);
    };

    // mooreBellmanFordSubroutineCPU (dijkstra_solver.cpp:203-388)
    auto bellman_ford = [&]() -> bool {
        const Control c = launch_bf_call(r, params(r, 2, branchId, 0.0, upperBound));
        numNodesInBranch = c.numInBranch;
        if (c.status == BF_LAYER_UNREACHED) return false;
        if (!c.anyFinite) return false;
        lowerBounds.clear();
        upperboundFoundOnFirstTry = false;
        const float lb1 = (float)c.firstLb;
        if (!std::isinf(lb1)) {
            lowerBoundOfCurrentBranch = lb1;
            if (c.validV == c.firstV) {
                upperboundFoundOnFirstTry = true;
                const float newUb = lb1;
                if (newUb > upperBound) return false;
                if (newUb < upperBound) {
                    upperBound = newUb;
                    cycle = extract(c.firstV);
                }
                return true;
            }
            // The branching pair is the candidate vertex and the start vertex of
            // its path (dijkstra_bnb_subroutine.cu:444-445; the CPU solver's
            // source id at dijkstra_solver.cpp:381 is negative and seeds nothing).
            branchingSrcNode = c.firstV;
            branchingTargetNode = c.firstOrigin;
        }
        if (c.validV >= 0) {
            const float newUb = (float)c.validLb;
            if (newUb < upperBound) {
                upperBound = newUb;
                cycle = extract(c.validV);
            }
        }
        return true;
    };

    // branch (dijkstra_solver.cpp:87-174)
    auto branch = [&](int newId) {
        std::vector<double> lb((size_t)n);
        d2h(lb.data(), wLb.p, sizeof(double) * n);
        PGC_CUDA(sync_stream());
        lowerBounds.clear();
        for (int v = 0; v < n; ++v)
            if (branchOf[(size_t)v] == branchId) lowerBounds.push_back({lb[(size_t)v], v});
        std::sort(lowerBounds.begin(), lowerBounds.end());
        std::vector<double> mark((size_t)n, -1.0);
        BranchHeap h(n);
        for (int i = 0; i < n; ++i) {
            mark[(size_t)i] = -1;
            if (i == branchingSrcNode || i == branchingTargetNode) { mark[(size_t)i] = 1; continue; }
            if (branchOf[(size_t)i] == branchId) h.push(std::numeric_limits<double>::infinity(), i);
        }
        h.push(0.0, branchingSrcNode);
        h.push(0.0, branchingTargetNode);
        if (branchingTargetNode >= 0 && branchingTargetNode < n) branchOf[(size_t)branchingTargetNode] = newId;
        int counter = 0;
        for (const auto& e : lowerBounds) {
            const int v = e.second;
            if (v == branchingSrcNode || v == branchingTargetNode) continue;
            if (branchOf[(size_t)v] != branchId) continue;
            if (counter > std::max(1, numNodesInBranch / 4)) {
                h.push(0.1, v);
                branchOf[(size_t)v] = newId;
            }
            ++counter;
        }
        while (!h.isEmpty()) {
            const auto cur = h.pop();
            const int node = (int)cur.second;
            const float nodeCost = (float)cur.first;
            mark[(size_t)node] = 1.0;
            for (long e : bg[(size_t)node]) {
                if (e == -1) continue;
                const long s = haveBranchGraph ? src_of(e) : src_of(e);
                if (s < 0 || s >= n) continue;
                if (mark[(size_t)s] < 0) {
                    const float oldV = (float)h.peakKey(s);
                    const float newV = nodeCost + 1.0f;
                    if (newV < oldV) {
                        h.decrease(s, newV);
                        branchOf[(size_t)s] = branchOf[(size_t)node];
                    }
                }
            }
        }
        branchingSrcNode = -1;
        branchingTargetNode = -1;
        upload_branch(branchOf);
    };

    BranchHeap heap(n);
    heap.push(0.0, branchId);
    std::vector<unsigned char> validLb((size_t)n, 0);
    std::map<int, std::vector<int>> validCycles;
    while (!heap.isEmpty()) {
        const auto top = heap.pop();
        branchId = (int)top.second;
        if (validLb[(size_t)branchId]) {
            upperBound = top.first;
            cycle = validCycles.at(branchId);
            break;
        }
        stats.branches++;
        if (!bellman_ford()) continue;
        if (upperBound < heap.peak() && upperboundFoundOnFirstTry) break;
        if (upperboundFoundOnFirstTry) {
            heap.push(lowerBoundOfCurrentBranch, branchId);
            validLb[(size_t)branchId] = 1;
            validCycles.emplace(branchId, cycle);
            continue;
        }
        ++maxBranchId;
        if (maxBranchId >= n) throw Failure(PGC_ERR_INTERNAL, "branch id exceeds the node count");
        branch(maxBranchId);
        heap.push(lowerBoundOfCurrentBranch, branchId);
        heap.push(lowerBoundOfCurrentBranch, maxBranchId);
    }
    if (cycle.empty()) throw Failure(PGC_ERR_INTERNAL, "no cycle found");

    // path output (dijkstra_solver.cpp:511-557)
    std::vector<int> cyc = cycle;
    std::reverse(cyc.begin(), cyc.end());
    cyc.push_back(cyc.front() + (int)nn);
    const size_t loopmax = cyc.size();
    std::vector<int> ps, pt;
    std::vector<size_t> pairIndex;
    int loops = 0;
    for (size_t i = 0; i < loopmax; ++i) {
        const int s = cyc[i % loopmax], t = cyc[(i + 1) % loopmax];
        if (t >= nn) ++loops;
        if (t < n && s >= nn && t == s - nn) continue;  // the dummy marker -1 matches first
        ps.push_back(s);
        pt.push_back(t);
    }
    std::vector<long long> edges;
    std::vector<double> cc, tt;
    lookup_pairs(ps, pt, edges, cc, tt, 0.0);
    std::vector<long long> found;
    for (long long e : edges)
        if (e >= 0) found.push_back(e);
    resPasses = loops < 2;
    resObjective = (float)upperBound;
    rows_for_edges(found);
    adjKind = 2;
}

void Graph::cost_vector(double* out) {
    ensure_generated();
    const long long rows = (long long)T.nY * T.eBlock;
    const long long stride = T.layerStride();
    const long long total = (long long)(T.nY + 1) * stride;
    DBuf<double> tmp;
    tmp.alloc((size_t)(rows * ncols));
    for (int c = 0; c < ncols; ++c) ensure_e64(c);
    for (int c = 0; c < ncols; ++c)
        PGC_CUDA(launch_export(e64[c].p, tmp.p, ncols, c, total, stride, T.entries[INTER], T.nY, T.eBlock,
                               dTedge[INTER].p, dTedge[INTRA].p, stream));
    PGC_CUDA(cudaMemcpyAsync(out, tmp.p, sizeof(double) * (size_t)(rows * ncols), cudaMemcpyDeviceToHost, stream));
    PGC_CUDA(sync_stream());
}

// Device address of the no-allocation export scratch on `device` (current).
static double* noalloc_scratch_for(int device) {
    double* p = nullptr;
    const cudaError_t e = noalloc_export_scratch(device, &p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw Failure(PGC_ERR_CUDA, std::string("cudaGetSymbolAddress of the export scratch failed: ") +
                                        cudaGetErrorString(e));
    }
    return p;
}

// cost_vector() through the fixed device scratch: no device allocation, no
// generation.  Every one of the rows x columns values is written by the
// export (each product-graph edge has exactly one stream entry), so nothing
// needs clearing first.
void Graph::cost_vector_noalloc(double* out) {
    if (!generated) throw Failure(PGC_ERR_STATE, "the no-allocation export needs generated edge costs (call generate first)");
    const long long rows = (long long)T.nY * T.eBlock;
    const long long values = rows * ncols;
    if (values > kNoAllocExportValues)
        throw Failure(PGC_ERR_ARG, "cost vector has " + std::to_string(values) +
                                       " values; the no-allocation export holds at most " +
                                       std::to_string(kNoAllocExportValues));
    double* scratch = noalloc_scratch_for(device);
    const long long stride = T.layerStride();
    const long long total = (long long)(T.nY + 1) * stride;
    for (int c = 0; c < ncols; ++c) ensure_e64(c);
    for (int c = 0; c < ncols; ++c)
        PGC_CUDA(launch_export(e64[c].p, scratch, ncols, c, total, stride, T.entries[INTER], T.nY, T.eBlock,
                               dTedge[INTER].p, dTedge[INTRA].p, stream));
    PGC_CUDA(cudaMemcpyAsync(out, scratch, sizeof(double) * (size_t)values, cudaMemcpyDeviceToHost, stream));
    PGC_CUDA(sync_stream());
}

// Adjoint of the last solve's objective with respect to feat_diff (plain
// graph).  Ratio: lambda* = C / T over the cycle's rescaled costs, so
// d lambda* / d c_e = 1[e in cycle] / T; minimum cost: d / d c_e = 1[e in
// cycle].  The rescale is taken with its factor fixed and its rounding passed
// straight through (d c_scaled / d c = product of the factors applied), and
// the energy's adjoint scatters into feat_diff (plain_energy_backward_kernel).
void Graph::backward_feat_diff(double grad, double* gradFd, bool accumulate, bool wait) {
    int cm = 0, tm = 0;
    if (conj) {
        // The conjugate energies read feat_diff once per edge, fd[x2, y2]:
        // in the cost column with slope 1 for ("vanilla", *) and
        // ("feature", *), not at all for the other cost modes.  Their time
        // column reads it only in ("*", "feature"), as max(0, maxFd - fd)
        // (higherOrderDeformationEnergy.cpp:323-327); a ratio's adjoint
        // takes its subgradient (conj_energy_backward_kernel).
        cm = string_to_mode(costName);
        tm = string_to_mode(timeName);
    }
    if (adjKind == 0 || !generated) throw Failure(PGC_ERR_STATE, "no ratio or minimum-cost result to differentiate");
    double coef = grad * colScale[0];
    if (adjKind == 1) coef /= adjT;
    if (!accumulate) PGC_CUDA(cudaMemsetAsync(gradFd, 0, sizeof(double) * (size_t)(nvx * nvy), stream));
    EnergyArgs a = energy_args();
    a.lengthMode = costName == "feature" && timeName == "lengthnormalisation";
    a.lineIntegral = reg || a.lengthMode;
    wAdjEdges.upload(resEdges.data(), resEdges.size(), stream);
    if (!conj) {
        PGC_CUDA(launch_plain_energy_backward(a, wAdjEdges.p, (int)resEdges.size(), T.eBlock, coef, gradFd, stream));
    } else {
        // time part of a ratio: d lambda* / d t_e = -lambda* / T, scaled by
        // the time column's rescale factor, times d t_e / d fd = -1
        const double coefT = (adjKind == 1 && tm == FEATURE && ncols > 1) ? grad * adjLambda * colScale[1] / adjT : 0.0;
        const double coefC = (cm == VANILLA || cm == FEATURE) ? coef : 0.0;
        a.maxFd = fdMax;
        if (coefC != 0.0 || coefT != 0.0)
            PGC_CUDA(launch_conj_energy_backward(a, wAdjEdges.p, (int)resEdges.size(), T.eBlock, coefC, coefT, fdArgmax,
                                                 gradFd, stream));
    }
    stats.launches++;
    if (wait) PGC_CUDA(sync_stream());
}

// The edge costs set directly ([rows x cols] in edge-id order), in place of
// generate(); the next solve uses them as they are (and rescales them).
void Graph::set_cost_vector(const double* in, int64_t rows, int64_t cols) {
    if (!templateReady) upload_template();
    if (rows != (int64_t)T.nY * T.eBlock || cols < 1 || cols > 2)
        throw Failure(PGC_ERR_ARG, "cost vector must be [" + std::to_string((long long)T.nY * T.eBlock) +
                                       " x 1|2], got [" + std::to_string(rows) + " x " + std::to_string(cols) + "]");
    const long long stride = T.layerStride();
    const long long total = (long long)(T.nY + 1) * stride;
    wImport.upload(in, (size_t)(rows * cols), stream);
    ncols = (int)cols;
    for (int c = 0; c < ncols; ++c) {
        e64[c].alloc((size_t)total);
        PGC_CUDA(launch_import(wImport.p, e64[c].p, ncols, c, total, stride, T.entries[INTER], T.nY, T.eBlock,
                               dTedge[INTER].p, dTedge[INTRA].p, stream));
    }
    PGC_CUDA(sync_stream());
    wImport.release();
    energy_changed();
    colScale[0] = colScale[1] = 1.0;
    adjKind = 0;
    generated = true;
}

// A new feature-difference matrix; the next solve regenerates the costs.
void Graph::set_feat_diff(const double* fd, int64_t rows, int64_t cols) {
    if (rows != nvx || cols != nvy) throw Failure(PGC_ERR_ARG, "feat_diff must be |VX| x |VY|");
    copy_in(FD, fd, (size_t)(rows * cols));
    fdHostStale = false;
    if (templateReady) dFD.upload(FD.data(), FD.size(), stream);
    generated = false;
    adjKind = 0;
}

// feat_diff from device memory: one device-to-device copy on the handle's
// stream, finished before returning (the caller may free its buffer then).
void Graph::set_feat_diff_device(const double* fd, int64_t rows, int64_t cols, bool wait) {
    if (rows != nvx || cols != nvy) throw Failure(PGC_ERR_ARG, "feat_diff must be |VX| x |VY|");
    const size_t n = (size_t)(rows * cols);
    dFD.alloc(n);
    PGC_CUDA(cudaMemcpyAsync(dFD.p, fd, n * sizeof(double), cudaMemcpyDeviceToDevice, stream));
    if (wait) PGC_CUDA(sync_stream());
    FD.resize(n);
    fdHostStale = true;
    generated = false;
    adjKind = 0;
}

void Graph::ensure_fd_host() {
    if (!fdHostStale) return;
    d2h(FD.data(), dFD.p, FD.size() * sizeof(double));
    PGC_CUDA(sync_stream());
    fdHostStale = false;
}

void Graph::product_space(int32_t* out) {
    ensure_generated();
    const long long rows = (long long)T.nY * T.eBlock;
    const int cols = T.cols();
    for (long long e = 0; e < rows; ++e) product_row(T, EY.data(), e, out + e * cols);
}

// writeToFile (product_graph_generators.cpp:272-282) with
// utils::writeMatrixToFile (utils.hpp:24-32): full precision, ", " between
// columns, a newline between rows and none after the last row.
void Graph::export_csv() {
    auto writeD = [](const RawVec<double>& m, int64_t rows, int64_t cols, const std::string& name) {
        std::ofstream f(name + ".csv");
        if (!f.is_open()) return;
        f.precision(17);
        for (int64_t i = 0; i < rows; ++i) {
            for (int64_t j = 0; j < cols; ++j) {
                if (j) f << ", ";
                f << m[(size_t)(i * cols + j)];
            }
            if (i + 1 < rows) f << "\n";
        }
    };
    auto writeI = [](const RawVec<int>& m, int64_t rows, int64_t cols, const std::string& name) {
        std::ofstream f(name + ".csv");
        if (!f.is_open()) return;
        for (int64_t i = 0; i < rows; ++i) {
            for (int64_t j = 0; j < cols; ++j) {
                if (j) f << ", ";
                f << m[(size_t)(i * cols + j)];
            }
            if (i + 1 < rows) f << "\n";
        }
    };
    writeD(VX, nvx, 3, "VX");
    writeD(VY, nvy, 3, "VY");
    writeI(EX, nex, 2, "EX");
    writeI(EY, ney, 2, "EY");
    ensure_fd_host();
    writeD(FD, nvx, nvy, "FeatDiffMatrix");
    if (conj) {
        writeD(NX, nvx, 3, "NX");
        writeD(NY, nvy, 3, "NY");
    }
}

}  // namespace pgc

// ===========================================================================
// C ABI
// ===========================================================================
using pgc::Failure;
using pgc::Graph;
using pgc::PairJob;

struct pgc_graph {
    Graph g;
};

namespace {

template <class F>
int guarded(F&& f) {
    try {
        f();
        pgc::g_lastError.clear();
        return PGC_OK;
    } catch (const Failure& e) {
        pgc::g_lastError = e.what();
        // consume a non-sticky runtime error so that it is not reported again
        // by the next launch check
        if (e.code == PGC_ERR_CUDA) (void)cudaGetLastError();
        return e.code;
    } catch (const std::bad_alloc&) {
        pgc::g_lastError = "host allocation failed";
        return PGC_ERR_INTERNAL;
    } catch (const std::exception& e) {
        pgc::g_lastError = e.what();
        return PGC_ERR_INTERNAL;
    }
}

}  // namespace

extern "C" {

int pgc_create(const double* VX, int64_t nvx, const int32_t* EX, int64_t nex, const double* VY, int64_t nvy,
               const int32_t* EY, int64_t ney, const double* feat_diff, int use_conjugate_graph,
               int use_regularising_cost_term, int prune_intralayer, pgc_graph** out) {
    return guarded([&] {
        if (!out) throw Failure(PGC_ERR_ARG, "out is null");
        *out = nullptr;
        if (!VX || !EX || !VY || !EY || !feat_diff) throw Failure(PGC_ERR_ARG, "null input");
        if (nvx < 1 || nex < 1 || nvy < 1 || ney < 1) throw Failure(PGC_ERR_ARG, "empty input");
        std::unique_ptr<pgc_graph> h(new pgc_graph());
        Graph& g = h->g;
        g.nvx = nvx; g.nex = nex; g.nvy = nvy; g.ney = ney;
        g.VX.assign(VX, VX + 3 * nvx);
        g.EX.assign(EX, EX + 2 * nex);
        g.VY.assign(VY, VY + 3 * nvy);
        g.EY.assign(EY, EY + 2 * ney);
        pgc::copy_in(g.FD, feat_diff, (size_t)(nvx * nvy));
        g.conj = use_conjugate_graph != 0;
        g.reg = use_regularising_cost_term != 0;
        g.prune = prune_intralayer != 0;
        PGC_CUDA(cudaGetDevice(&g.device));
        PGC_CUDA(cudaStreamCreateWithFlags(&g.ownStream, cudaStreamNonBlocking));
        g.stream = g.ownStream;
        *out = h.release();
    });
}

void pgc_destroy(pgc_graph* g) { delete g; }

int pgc_set_normals(pgc_graph* h, const double* NX, int64_t rx, int64_t cx, const double* NY, int64_t ry,
                    int64_t cy) {
    return guarded([&] {
        if (!h) throw Failure(PGC_ERR_ARG, "null handle");
        Graph& g = h->g;
        if (rx != g.nvx || cx != 3)
            throw Failure(PGC_ERR_ARG,
                          "normals for shape X do not contain as many entries as expected. Assumed shape = |VX| x 3");
        if (ry != g.nvy || cy != 3)
            throw Failure(PGC_ERR_ARG,
                          "normals for shape Y do not contain as many entries as expected. Assumed shape = |VY| x 3");
        if (!NX || !NY) throw Failure(PGC_ERR_ARG, "null normals");
        g.NX.assign(NX, NX + 3 * rx);
        g.NY.assign(NY, NY + 3 * ry);
        g.normalsGiven = true;
    });
}

int pgc_set_max_depth(pgc_graph* h, int k) {
    return guarded([&] {
        if (!h) throw Failure(PGC_ERR_ARG, "null handle");
        h->g.maxDepth = k;
    });
}

int pgc_set_cost_time_ratio_mode(pgc_graph* h, const char* cost, const char* time) {
    return guarded([&] {
        if (!h) throw Failure(PGC_ERR_ARG, "null handle");
        h->g.costName = cost ? cost : "";
        h->g.timeName = time ? time : "";
    });
}

int pgc_update_robust_loss_params(pgc_graph* h, double alpha, double c, double pwr) {
    return guarded([&] {
        if (!h) throw Failure(PGC_ERR_ARG, "null handle");
        Graph& g = h->g;
        if (!g.conj) return;
        if (g.generated) throw Failure(PGC_ERR_STATE, "cannot update robust loss params after model has been generated");
        g.rlAlpha = alpha;
        g.rlC = c;
        g.rlPwr = pwr;
    });
}

int pgc_set_stream(pgc_graph* h, void* cuda_stream) {
    return guarded([&] {
        if (!h) throw Failure(PGC_ERR_ARG, "null handle");
        Graph& g = h->g;
        PGC_CUDA(cudaStreamSynchronize(g.stream));
        g.stream = cuda_stream ? (cudaStream_t)cuda_stream : g.ownStream;
    });
}

int pgc_generate(pgc_graph* h) {
    return guarded([&] {
        if (!h) throw Failure(PGC_ERR_ARG, "null handle");
        PGC_CUDA(cudaSetDevice(h->g.device));
        h->g.generate();
    });
}

int pgc_cost_vector_shape(pgc_graph* h, int64_t* rows, int64_t* cols) {
    return guarded([&] {
        if (!h) throw Failure(PGC_ERR_ARG, "null handle");
        if (!rows || !cols) throw Failure(PGC_ERR_ARG, "null output");
        PGC_CUDA(cudaSetDevice(h->g.device));
        h->g.ensure_generated();
        *rows = (int64_t)h->g.T.nY * h->g.T.eBlock;
        *cols = h->g.ncols;
    });
}

int pgc_get_cost_vector(pgc_graph* h, double* out) {
    return guarded([&] {
        if (!h) throw Failure(PGC_ERR_ARG, "null handle");
        if (!out) throw Failure(PGC_ERR_ARG, "null output");
        PGC_CUDA(cudaSetDevice(h->g.device));
        h->g.cost_vector(out);
    });
}

int pgc_get_cost_vector_noalloc(pgc_graph* h, double* out) {
    return guarded([&] {
        if (!h || !out) throw pgc::Failure(PGC_ERR_ARG, "null argument");
        PGC_CUDA(cudaSetDevice(h->g.device));
        h->g.cost_vector_noalloc(out);
    });
}

int pgc_product_space_shape(pgc_graph* h, int64_t* rows, int64_t* cols) {
    return guarded([&] {
        if (!h) throw Failure(PGC_ERR_ARG, "null handle");
        if (!rows || !cols) throw Failure(PGC_ERR_ARG, "null output");
        PGC_CUDA(cudaSetDevice(h->g.device));
        h->g.ensure_generated();
        *rows = (int64_t)h->g.T.nY * h->g.T.eBlock;
        *cols = h->g.T.cols();
    });
}

int pgc_get_product_space(pgc_graph* h, int32_t* out) {
    return guarded([&] {
        if (!h) throw Failure(PGC_ERR_ARG, "null handle");
        if (!out) throw Failure(PGC_ERR_ARG, "null output");
        PGC_CUDA(cudaSetDevice(h->g.device));
        h->g.product_space(out);
    });
}

int pgc_solve_with_cost_time_ratio(pgc_graph* h, const char* solver, int max_depth) {
    return guarded([&] {
        if (!h) throw Failure(PGC_ERR_ARG, "null handle");
        Graph& g = h->g;
        const std::string name = solver ? solver : "";
        const int K = max_depth >= 1 ? max_depth : g.maxDepth;
        if (name == "export") {
            g.export_csv();
            g.resPasses = false;
            g.resObjective = -1.0f;
            g.resRows = 4;
            g.resCols = 1;
            g.resMatching.assign(4, 0);
            g.resEdges.clear();
            g.adjKind = 0;
            return;
        }
        if (name != "lawlercpu" && name != "lawlergpu")
            throw Failure(PGC_ERR_SOLVER, "Solver >>" + name + "<< is not implemented");
        PGC_CUDA(cudaSetDevice(g.device));
        g.solve_ratio(K);
    });
}

int pgc_solve_with_minimum_cost(pgc_graph* h, const char* solver, int max_depth) {
    return guarded([&] {
        if (!h) throw Failure(PGC_ERR_ARG, "null handle");
        Graph& g = h->g;
        const std::string name = solver ? solver : "";
        const int K = max_depth >= 1 ? max_depth : g.maxDepth;
        if (name == "export") {
            g.export_csv();
            g.resPasses = false;
            g.resObjective = -1.0f;
            g.resRows = 4;
            g.resCols = 1;
            g.resMatching.assign(4, 0);
            g.resEdges.clear();
            g.adjKind = 0;
            return;
        }
        PGC_CUDA(cudaSetDevice(g.device));
        g.solve_min_cost(K);
    });
}

int pgc_backward_feat_diff(pgc_graph* h, double grad_objective, double* grad_feat_diff, int accumulate) {
    return guarded([&] {
        if (!h || !grad_feat_diff) throw Failure(PGC_ERR_ARG, "null argument");
        PGC_CUDA(cudaSetDevice(h->g.device));
        h->g.backward_feat_diff(grad_objective, grad_feat_diff, accumulate != 0);
    });
}

int pgc_backward_feat_diff_batch(pgc_graph* const* graphs, int64_t count, const double* grad_objectives,
                                 double* const* grad_feat_diffs, int accumulate) {
    return guarded([&] {
        if (count < 0 || (count > 0 && (!graphs || !grad_objectives || !grad_feat_diffs)))
            throw Failure(PGC_ERR_ARG, "null argument");
        for (int64_t i = 0; i < count; ++i)
            if (!graphs[i] || !grad_feat_diffs[i]) throw Failure(PGC_ERR_ARG, "null handle or output of graph " + std::to_string(i));
        // every adjoint enqueued on its graph's stream, then one wait per stream
        for (int64_t i = 0; i < count; ++i) {
            PGC_CUDA(cudaSetDevice(graphs[i]->g.device));
            graphs[i]->g.backward_feat_diff(grad_objectives[i], grad_feat_diffs[i], accumulate != 0, false);
        }
        for (int64_t i = 0; i < count; ++i) {
            PGC_CUDA(cudaSetDevice(graphs[i]->g.device));
            PGC_CUDA(cudaStreamSynchronize(graphs[i]->g.stream));
        }
    });
}

int pgc_set_feat_diff_device_batch(pgc_graph* const* graphs, int64_t count, const double* const* feat_diffs) {
    return guarded([&] {
        if (count < 0 || (count > 0 && (!graphs || !feat_diffs))) throw Failure(PGC_ERR_ARG, "null argument");
        for (int64_t i = 0; i < count; ++i)
            if (!graphs[i] || !feat_diffs[i]) throw Failure(PGC_ERR_ARG, "null handle or input of graph " + std::to_string(i));
        for (int64_t i = 0; i < count; ++i) {
            Graph& g = graphs[i]->g;
            PGC_CUDA(cudaSetDevice(g.device));
            g.set_feat_diff_device(feat_diffs[i], g.nvx, g.nvy, false);
        }
        for (int64_t i = 0; i < count; ++i) {
            PGC_CUDA(cudaSetDevice(graphs[i]->g.device));
            PGC_CUDA(cudaStreamSynchronize(graphs[i]->g.stream));
        }
    });
}

int pgc_set_cost_vector(pgc_graph* h, const double* costs, int64_t rows, int64_t cols) {
    return guarded([&] {
        if (!h || !costs) throw Failure(PGC_ERR_ARG, "null argument");
        PGC_CUDA(cudaSetDevice(h->g.device));
        h->g.set_cost_vector(costs, rows, cols);
    });
}

int pgc_set_feat_diff(pgc_graph* h, const double* feat_diff, int64_t rows, int64_t cols) {
    return guarded([&] {
        if (!h || !feat_diff) throw Failure(PGC_ERR_ARG, "null argument");
        PGC_CUDA(cudaSetDevice(h->g.device));
        h->g.set_feat_diff(feat_diff, rows, cols);
    });
}

int pgc_set_feat_diff_device(pgc_graph* h, const double* feat_diff, int64_t rows, int64_t cols) {
    return guarded([&] {
        if (!h || !feat_diff) throw Failure(PGC_ERR_ARG, "null argument");
        PGC_CUDA(cudaSetDevice(h->g.device));
        h->g.set_feat_diff_device(feat_diff, rows, cols);
    });
}

int pgc_set_team_cap(pgc_graph* h, int max_ctas) {
    return guarded([&] {
        if (!h) throw Failure(PGC_ERR_ARG, "null handle");
        if (max_ctas < 0) throw Failure(PGC_ERR_ARG, "max_ctas must be >= 0");
        h->g.teamCap = max_ctas;
    });
}

int pgc_set_team_shape(pgc_graph* h, int ctas, int threads_per_cta) {
    return guarded([&] {
        if (!h) throw Failure(PGC_ERR_ARG, "null handle");
        if (ctas < 0) throw Failure(PGC_ERR_ARG, "ctas must be >= 0");
        if (threads_per_cta && (threads_per_cta < 32 || threads_per_cta > pgc::kBfThreads || threads_per_cta % 32 != 0))
            throw Failure(PGC_ERR_ARG, "threads per CTA must be 0 or a multiple of 32 in [32, 640]");
        h->g.shapeBlocks = ctas;
        h->g.shapeThreads = threads_per_cta;
    });
}

namespace {
// Phases of the calling thread's last pgc_solve_batch (pgc_batch_profile).
thread_local double g_batchProfile[8] = {0, 0, 0, 0, 0, 0, 0, 0};
double ms_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}
}  // namespace

int pgc_kernel_launches(int64_t* out) {
    return guarded([&] {
        if (!out) throw Failure(PGC_ERR_ARG, "null output");
        *out = pgc::launch_count();
    });
}

int pgc_batch_profile(double* out8) {
    return guarded([&] {
        if (!out8) throw Failure(PGC_ERR_ARG, "null output");
        for (int i = 0; i < 8; ++i) out8[i] = g_batchProfile[i];
    });
}

int pgc_solve_batch(pgc_graph* const* graphs, int64_t count, const char* solver, int max_depth, int ctas_per_graph,
                    int workers, int regenerate, int* status) {
    return guarded([&] {
        for (double& x : g_batchProfile) x = 0;
        const auto tStart = std::chrono::steady_clock::now();
        if (count < 0 || (count > 0 && (!graphs || !status))) throw Failure(PGC_ERR_ARG, "null argument");
        const std::string name = solver ? solver : "";
        const bool ratio = name == "lawlercpu" || name == "lawlergpu";
        if (workers <= 0) workers = 64;
        workers = (int)std::max<int64_t>(1, std::min<int64_t>(workers, count));
        std::vector<std::string> errors((size_t)count);
        // Runs f(i) for every graph on the worker threads; a graph whose
        // status is already a failure is skipped.
        auto for_each_graph = [&](auto&& f) {
            std::atomic<int64_t> next{0};
            auto work = [&] {
                for (;;) {
                    const int64_t i = next.fetch_add(1);
                    if (i >= count) return;
                    if (status[i] != PGC_OK) continue;
                    status[i] = f(i);
                    if (status[i] != PGC_OK) errors[(size_t)i] = pgc_last_error();
                }
            };
            std::vector<std::thread> pool;
            for (int w = 1; w < workers; ++w) pool.emplace_back(work);
            work();
            for (auto& t : pool) t.join();
        };
        for (int64_t i = 0; i < count; ++i) status[i] = graphs[i] ? PGC_OK : PGC_ERR_ARG;
        int dev = 0;
        PGC_CUDA(cudaGetDevice(&dev));
        pgc::DeviceInfo info{};
        PGC_CUDA(pgc::device_info(dev, &info));
        const int sms = info.sms;
        if (ratio && pgc::env_int("PGC_BATCH_STREAMS", 0) == 0) {
            // One launch solves every graph: its CTAs take the graphs from a
            // queue, largest first, and run each whole ratio solve on the
            // device.  The costs are generated and rescaled per graph by the
            // workers first; graphs whose first branch's cycle wraps are
            // finished on the host afterwards, with branch and bound.
            const int threads = pgc::kBatchThreads;
            const size_t smemCap = (size_t)std::max(0, info.smemOptin / pgc::kBatchBlocksPerSm - 2048);
            // CTAs per team (PGC_BATCH_TEAM, default 8): a team relaxes a
            // graph's steps side by side, so more CTAs per graph shorten each
            // solve; fewer overlap more graphs' latencies
            int team = ctas_per_graph > 0 ? ctas_per_graph : pgc::env_int("PGC_BATCH_TEAM", 8);
            team = std::max(1, std::min(team, sms * pgc::kBatchBlocksPerSm));
            const unsigned spin = (unsigned)std::max(1, pgc::env_int("PGC_BF_SPIN_LIMIT", (int)pgc::kDefaultSpinLimit));
            std::vector<PairJob> jobs((size_t)count);
            std::vector<int> costF32((size_t)count, 0), timeKind((size_t)count, 0);
            std::vector<size_t> smemNeed((size_t)count, 0);
            std::vector<double> work((size_t)count, 0);
            for_each_graph([&](int64_t i) {
                pgc_graph* h = graphs[i];
                return guarded([&] {
                    Graph& g = h->g;
                    if (g.device != dev) throw Failure(PGC_ERR_ARG, "a batch's graphs must live on the current device");
                    const int K = max_depth >= 1 ? max_depth : g.maxDepth;
                    g.blockingSync = true;
                    try {
                        g.batch_begin(K, jobs[(size_t)i], threads, team, smemCap, regenerate != 0);
                    } catch (...) {
                        g.blockingSync = false;
                        throw;
                    }
                    g.blockingSync = false;
                    costF32[(size_t)i] = jobs[(size_t)i].bf.cost == (const void*)g.e32[0].p ? 1 : 0;
                    timeKind[(size_t)i] = jobs[(size_t)i].bf.time == nullptr ? 0
                                          : jobs[(size_t)i].bf.time == (const void*)g.e32[1].p ? 1 : 2;
                    smemNeed[(size_t)i] = jobs[(size_t)i].bf.maxCtaSlices >= 0 ? g.batch_smem_bytes() : 0;
                    work[(size_t)i] = (double)g.T.layerStride() * g.T.nY * K;
                });
            });
            g_batchProfile[0] = ms_since(tStart);
            if (std::getenv("PGC_BATCH_PHASES")) {
                std::fprintf(stderr, "[pgc] batch preparation, summed over %d workers: generate %.1f ms, rescale %.1f ms, "
                             "team %.1f ms; wall %.1f ms\n", workers, pgc::g_batchPhaseNs[0].exchange(0) * 1e-6,
                             pgc::g_batchPhaseNs[1].exchange(0) * 1e-6, pgc::g_batchPhaseNs[2].exchange(0) * 1e-6,
                             g_batchProfile[0]);
            }
            const auto tKernel = std::chrono::steady_clock::now();
            // one launch per (cost type, time kind) group, largest graphs first
            pgc::DBuf<PairJob> dJobs;
            pgc::DBuf<int> dNext;
            pgc::DBuf<unsigned> dTeamWords;
            cudaStream_t bs = nullptr;
            PGC_CUDA(cudaStreamCreateWithFlags(&bs, cudaStreamNonBlocking));
            struct StreamGuard {
                cudaStream_t s;
                ~StreamGuard() { if (s) cudaStreamDestroy(s); }
            } guard{bs};
            std::vector<int64_t> order;
            for (int64_t i = 0; i < count; ++i)
                if (status[i] == PGC_OK) order.push_back(i);
            std::stable_sort(order.begin(), order.end(), [&](int64_t x, int64_t y) {
                const int gx = costF32[(size_t)x] * 3 + timeKind[(size_t)x], gy = costF32[(size_t)y] * 3 + timeKind[(size_t)y];
                if (gx != gy) return gx < gy;
                return work[(size_t)x] > work[(size_t)y];
            });
            std::vector<PairJob> packed(order.size());
            for (size_t k = 0; k < order.size(); ++k) packed[k] = jobs[(size_t)order[k]];
            if (!packed.empty()) {
                dJobs.alloc(packed.size());
                dNext.alloc(8);
                // words of at most 32 teams per SM, allocated once: a group's
                // launch may still run when the next group's words are zeroed
                // behind it on the stream
                const size_t maxTeams = (size_t)sms * 32;
                dTeamWords.alloc(maxTeams * pgc::kTeamWordStride);
                PGC_CUDA(cudaMemcpyAsync(dJobs.p, packed.data(), sizeof(PairJob) * packed.size(),
                                         cudaMemcpyHostToDevice, bs));
                PGC_CUDA(cudaMemsetAsync(dNext.p, 0, 8 * sizeof(int), bs));
                for (size_t k0 = 0, grp = 0; k0 < order.size(); ++grp) {
                    size_t k1 = k0;
                    size_t smem = 0;
                    const int cf = costF32[(size_t)order[k0]], tk = timeKind[(size_t)order[k0]];
                    while (k1 < order.size() && costF32[(size_t)order[k1]] == cf && timeKind[(size_t)order[k1]] == tk)
                        smem = std::max(smem, smemNeed[(size_t)order[k1++]]);
                    int perSm = 0;
                    PGC_CUDA(pgc::bf_batch_max_blocks(cf, tk, threads, smem, &perSm));
                    if (perSm < 1) throw Failure(PGC_ERR_CUDA, "the batched solve kernel cannot be resident");
                    // whole teams, all resident (the launch is cooperative
                    // when a team has more than one CTA)
                    const int g = std::min(team, sms * perSm);
                    const int teams = (int)std::min<size_t>({k1 - k0, (size_t)(sms * perSm / g), maxTeams});
                    const int blocks = teams * g;
                    PGC_CUDA(cudaMemsetAsync(dTeamWords.p, 0, (size_t)teams * pgc::kTeamWordStride * sizeof(unsigned), bs));
                    g_batchProfile[5] += blocks;
                    g_batchProfile[6] = threads;
                    g_batchProfile[7] = std::max(g_batchProfile[7], (double)smem);
                    PGC_CUDA(pgc::launch_bf_batch(dJobs.p + k0, (int)(k1 - k0), dNext.p + grp % 8, dTeamWords.p, g,
                                                  spin, cf, tk, blocks, threads, smem, bs));
                    k0 = k1;
                }
                PGC_CUDA(cudaMemcpyAsync(packed.data(), dJobs.p, sizeof(PairJob) * packed.size(),
                                         cudaMemcpyDeviceToHost, bs));
                PGC_CUDA(cudaStreamSynchronize(bs));
                for (size_t k = 0; k < order.size(); ++k) jobs[(size_t)order[k]] = packed[k];
            }
            g_batchProfile[1] = ms_since(tKernel);
            const auto tEnd = std::chrono::steady_clock::now();
            for (const PairJob& J : jobs) {
                if (J.status == pgc::PAIR_HOST) g_batchProfile[3] += 1;
                if (J.status == pgc::PAIR_DONE || J.status == pgc::PAIR_NAN) g_batchProfile[4] += 1;
            }
            for_each_graph([&](int64_t i) {
                return guarded([&] {
                    Graph& g = graphs[i]->g;
                    g.blockingSync = true;
                    try {
                        g.batch_end(jobs[(size_t)i]);
                    } catch (...) {
                        g.blockingSync = false;
                        throw;
                    }
                    g.blockingSync = false;
                });
            });
            g_batchProfile[2] = ms_since(tEnd);
        } else {
            // each graph on its own stream with a small team: the device runs
            // at most 32 kernels side by side (host work queues), so teams
            // that together cover the SMs keep them all busy
            if (ctas_per_graph <= 0)
                ctas_per_graph = std::max(1, sms / (int)std::max<int64_t>(1, std::min<int64_t>(count, 32)));
            for_each_graph([&](int64_t i) {
                pgc_graph* h = graphs[i];
                const int saved = h->g.teamCap;
                h->g.teamCap = ctas_per_graph;
                h->g.blockingSync = true;
                int rc = regenerate ? pgc_generate(h) : PGC_OK;
                if (rc == PGC_OK)
                    rc = ratio ? pgc_solve_with_cost_time_ratio(h, solver, max_depth)
                               : pgc_solve_with_minimum_cost(h, solver, max_depth);
                h->g.teamCap = saved;
                h->g.blockingSync = false;
                return rc;
            });
        }
        for (int64_t i = 0; i < count; ++i)
            if (status[i] != PGC_OK)
                throw Failure(status[i], "graph " + std::to_string(i) + " of the batch failed: " +
                                             (graphs[i] ? errors[(size_t)i] : std::string("null handle")));
    });
}

int pgc_result(pgc_graph* h, int* passes, float* objective, int64_t* rows, int64_t* cols) {
    return guarded([&] {
        if (!h) throw Failure(PGC_ERR_ARG, "null handle");
        const Graph& g = h->g;
        if (passes) *passes = g.resPasses ? 1 : 0;
        if (objective) *objective = g.resObjective;
        if (rows) *rows = g.resRows;
        if (cols) *cols = g.resCols;
    });
}

int pgc_result_matching(pgc_graph* h, int32_t* out) {
    return guarded([&] {
        if (!h) throw Failure(PGC_ERR_ARG, "null handle");
        const Graph& g = h->g;
        if (!out && !g.resMatching.empty()) throw Failure(PGC_ERR_ARG, "null output");
        if (!g.resMatching.empty()) std::memcpy(out, g.resMatching.data(), sizeof(int32_t) * g.resMatching.size());
    });
}

int pgc_result_cycle_edges(pgc_graph* h, int64_t* out, int64_t capacity, int64_t* count) {
    return guarded([&] {
        if (!h) throw Failure(PGC_ERR_ARG, "null handle");
        const Graph& g = h->g;
        if (!count || (!out && capacity > 0)) throw Failure(PGC_ERR_ARG, "null output");
        *count = (int64_t)g.resEdges.size();
        for (int64_t i = 0; i < *count && i < capacity; ++i) out[i] = g.resEdges[(size_t)i];
    });
}

int pgc_result_profile(pgc_graph* h, int64_t* out8) {
    return guarded([&] {
        if (!h) throw Failure(PGC_ERR_ARG, "null handle");
        if (!out8) throw pgc::Failure(PGC_ERR_ARG, "null output");
        const pgc::Stats& s = h->g.stats;
        out8[0] = (int64_t)s.cycA;
        out8[1] = (int64_t)s.cycB;
        out8[2] = (int64_t)s.cycSync;
        out8[3] = (int64_t)s.cycTail;
        out8[4] = s.steps;
        out8[5] = s.ctas;
        out8[6] = s.threads;
        out8[7] = s.waitEntries;
    });
}

int pgc_result_profile_detail(pgc_graph* h, int64_t* out4) {
    return guarded([&] {
        if (!h) throw Failure(PGC_ERR_ARG, "null handle");
        if (!out4) throw pgc::Failure(PGC_ERR_ARG, "null output");
        const pgc::Stats& s = h->g.stats;
        out4[0] = (int64_t)s.cycStage;
        out4[1] = (int64_t)s.cycWrap;
        out4[2] = (int64_t)s.cycCand;
        out4[3] = (int64_t)s.cycLead;
    });
}

int pgc_result_stats(pgc_graph* h, int64_t* out8) {
    return guarded([&] {
        if (!h) throw Failure(PGC_ERR_ARG, "null handle");
        if (!out8) throw Failure(PGC_ERR_ARG, "null output");
        const pgc::Stats& s = h->g.stats;
        out8[0] = s.bfCalls;
        out8[1] = s.sweeps;
        out8[2] = s.candidates;
        out8[3] = s.lawlerIters;
        out8[4] = s.branches;
        out8[5] = s.fallbackWalks;
        out8[6] = (int64_t)(s.deviceMs * 1000.0);
        out8[7] = s.launches;
    });
}

// utils::normals2d (helper/utils.cpp:93-157).
int pgc_product_graph_sizes(const int32_t* EX, int64_t nex, int64_t nvx, int64_t ney, int conjugate,
                            int prune_intralayer_edges, int64_t* out6) {
    return guarded([&] {
        if (!EX || !out6) throw Failure(PGC_ERR_ARG, "null argument");
        std::vector<int> ey((size_t)(2 * std::max<int64_t>(ney, 0)));
        for (int64_t i = 0; i < ney; ++i) {
            ey[(size_t)(2 * i)] = (int)i;
            ey[(size_t)(2 * i + 1)] = (int)((i + 1) % ney);
        }
        pgc::LayerTemplate T;
        const std::string err = pgc::build_template(EX, nex, ey.data(), ney, nvx, conjugate != 0,
                                                    prune_intralayer_edges != 0, T);
        if (!err.empty()) throw Failure(PGC_ERR_ARG, err);
        int64_t inter = 0;
        for (int64_t t = 0; t < T.eBlock; ++t) inter += T.eNext[(size_t)t] ? 1 : 0;
        out6[0] = T.n;
        out6[1] = T.eBlock;
        out6[2] = inter;
        out6[3] = T.eBlock - inter;
        out6[4] = T.nslices;
        out6[5] = (T.entries[pgc::INTER] + T.entries[pgc::INTRA]) / 32;
    });
}

// utils::normals2d (helper/utils.cpp:93-157) on the device: the curve is
// copied in, curve_normals_kernel computes the normals with the reference's
// operations in its order, and they are copied back.
int pgc_compute_normals_2d(const double* Vin, int64_t nv, const int32_t* E, int64_t ne, double* out) {
    return guarded([&] {
        if (nv < 0 || (nv > 0 && (!Vin || !E || !out))) throw Failure(PGC_ERR_ARG, "null argument");
        if (nv != ne) throw Failure(PGC_ERR_ARG, "V.rows() != E.rows()");
        if (nv > INT_MAX / 3) throw Failure(PGC_ERR_ARG, "curve too long");
        if (nv == 0) return;
        cudaStream_t s = cudaStreamPerThread;
        pgc::DBuf<double> dV, dW, dEn, dEl, dOut;
        pgc::DBuf<int> dE, dBad;
        dV.upload(Vin, (size_t)(3 * nv), s);
        dE.upload(E, (size_t)(2 * ne), s);
        dW.alloc((size_t)(3 * nv));
        dEn.alloc((size_t)(3 * nv));
        dEl.alloc((size_t)nv);
        dOut.alloc((size_t)(3 * nv));
        dBad.alloc(1);
        dBad.zero(s);
        PGC_CUDA(pgc::launch_normals_2d(dV.p, (int)nv, dE.p, dW.p, dEn.p, dEl.p, dOut.p, dBad.p, s));
        int bad = 0;
        PGC_CUDA(cudaMemcpyAsync(&bad, dBad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
        PGC_CUDA(cudaMemcpyAsync(out, dOut.p, sizeof(double) * (size_t)(3 * nv), cudaMemcpyDeviceToHost, s));
        PGC_CUDA(cudaStreamSynchronize(s));
        if (bad == 1) throw Failure(PGC_ERR_ARG, "points dont lie on xy, xz or yz plane");
        if (bad == 2) throw Failure(PGC_ERR_ARG, "E refers to a vertex outside V");
    });
}

// utils::normals3d (helper/utils.cpp:86-90): libigl's per_vertex_normals
// with its default (area) weighting -- per vertex the sum, in face order, of
// its faces' edge cross products (unit normal times twice the area), scaled
// to unit length; on the device (face_normals_kernel .. vertex_normals_kernel).
int pgc_compute_normals_3d(const double* V, int64_t nv, const int32_t* F, int64_t nf, double* out) {
    return guarded([&] {
        if (nv < 0 || nf < 0 || (nv > 0 && (!V || !out)) || (nf > 0 && !F)) throw Failure(PGC_ERR_ARG, "null argument");
        if (nv > INT_MAX / 3 || nf > INT_MAX / 3) throw Failure(PGC_ERR_ARG, "mesh too large");
        if (nv == 0) return;
        cudaStream_t s = cudaStreamPerThread;
        pgc::DBuf<double> dV, dFn, dOut;
        pgc::DBuf<int> dF, dDeg, dOff, dCur, dList, dBad;
        dV.upload(V, (size_t)(3 * nv), s);
        dF.alloc((size_t)std::max<int64_t>(1, 3 * nf));
        if (nf > 0) PGC_CUDA(cudaMemcpyAsync(dF.p, F, sizeof(int) * (size_t)(3 * nf), cudaMemcpyHostToDevice, s));
        dFn.alloc((size_t)std::max<int64_t>(1, 3 * nf));
        dDeg.alloc((size_t)nv);
        dDeg.zero(s);
        dCur.alloc((size_t)nv);
        dCur.zero(s);
        dOff.alloc((size_t)nv + 1);
        dList.alloc((size_t)std::max<int64_t>(1, 3 * nf));
        dOut.alloc((size_t)(3 * nv));
        dBad.alloc(1);
        dBad.zero(s);
        // faces with an index outside V are flagged and left out of every list
        PGC_CUDA(pgc::launch_normals_3d(dV.p, nv, dF.p, nf, dFn.p, dDeg.p, dOff.p, dCur.p, dList.p, dOut.p, dBad.p, s));
        int bad = 0;
        PGC_CUDA(cudaMemcpyAsync(&bad, dBad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
        PGC_CUDA(cudaMemcpyAsync(out, dOut.p, sizeof(double) * (size_t)(3 * nv), cudaMemcpyDeviceToHost, s));
        PGC_CUDA(cudaStreamSynchronize(s));
        if (bad) throw Failure(PGC_ERR_ARG, "F refers to a vertex outside V");
    });
}

int pgc_graph_info(pgc_graph* h, int64_t* out8) {
    return guarded([&] {
        if (!h) throw Failure(PGC_ERR_ARG, "null handle");
        if (!out8) throw Failure(PGC_ERR_ARG, "null output");
        Graph& g = h->g;
        PGC_CUDA(cudaSetDevice(g.device));
        g.ensure_generated();
        int64_t inter = 0, intra = 0;
        for (int64_t t = 0; t < g.T.eBlock; ++t) (g.T.eNext[(size_t)t] ? inter : intra) += 1;
        out8[0] = g.T.n;
        out8[1] = g.T.nY;
        out8[2] = g.T.eBlock;
        out8[3] = inter;
        out8[4] = intra;
        out8[5] = g.T.entries[pgc::INTER];
        out8[6] = g.T.entries[pgc::INTRA];
        out8[7] = g.ncols;
    });
}

int pgc_device_name(pgc_graph* h, char* out, int64_t capacity) {
    return guarded([&] {
        if (!h) throw Failure(PGC_ERR_ARG, "null handle");
        if (!out || capacity < 1) throw Failure(PGC_ERR_ARG, "null or empty output buffer");
        cudaDeviceProp prop{};
        PGC_CUDA(cudaGetDeviceProperties(&prop, h->g.device));
        const size_t len = std::min(std::strlen(prop.name), (size_t)capacity - 1);
        std::memcpy(out, prop.name, len);
        out[len] = '\0';
    });
}

int pgc_release_cached_memory(void) {
    return guarded([&] {
        pgc::DevicePool::get().release_cached();
        pgc::HostPool::get().release_cached();
    });
}

const char* pgc_last_error(void) { return pgc::g_lastError.c_str(); }

const char* pgc_version(void) { return "pgc-b200 0.1.0 (sm_100a)"; }

}  // extern "C"
