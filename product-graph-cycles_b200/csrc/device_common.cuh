// device_common.cuh -- types shared by the sm_100a kernels and the host driver.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace pgc {

constexpr int kWarp = 32;
constexpr double kInfD = __builtin_huge_val();

// Status words written by the Bellman-Ford kernels.
enum BfStatus : int {
    BF_RUNNING = 0,
    BF_FOUND_CYCLE = 1,      // a cycle was detected and extracted (ratio solver)
    BF_LAYER_UNREACHED = 2,  // a layer 1..nY-1 received no finite value
    BF_WRAP_NO_IMPROVE = 3,  // the wrap-around improved no start node
    BF_MAX_SWEEPS = 4,       // numNodes-1 sweeps without a detected cycle
    BF_UB_DONE = 5,          // upper-bound sweep finished, path extracted
    BF_SWEEP_DONE = 6,       // minimum-cost sweep finished
    BF_ERR_EMPTY_BRANCH = -1,
    BF_ERR_BARRIER = -2,     // a grid barrier wait ran out of iterations
    BF_ERR_CYCLE_CAP = -3,   // the extracted cycle does not fit its buffer
    BF_ERR_WALK = -4,        // a predecessor walk left the valid index range
    BF_ERR_CHUNK = -5,       // a slice has more in-edge entries than the scratch holds
};

// Lap-successor codes (see bf kernel): P[v] >= 0 is the next layer-0 node.
constexpr int kLapEnd = -1;      // the walk stops here (predecessor -1)
constexpr int kLapUnknown = -2;  // successor not derivable from this sweep

struct Control {
    int status;
    int error;
    int sweeps;          // sweeps run by the last launch
    int epoch;           // monotone sweep counter (improve flags)
    int numInBranch;
    int indexNodeInLayer;
    int walkRounds;      // rounds of the bounded parallel literal walks (statistics)
    int v0;              // first repeated layer-0 node of the detected cycle
    long long cLength;   // steps the reference's walk needs to detect it
    int cycleLen;        // entries written to the cycle buffer
    int candidateVi;     // candidate whose walk found the cycle
    int fallbackWalks;   // literal walks run because of undecidable shortcuts
    long long candidates;  // candidates decided (for statistics)
    unsigned barCount;
    unsigned barGen;
    // A word no code writes (the host zeroes it before each launch).  The
    // wait-timeout test makes one CTA's step hand-off also wait for it to
    // reach the step number, so that wait runs out.
    unsigned neverSet;
    int pad;
    // SM cycles seen by CTA 0's thread 0 (profiling counters): relaxation,
    // sweep bookkeeping, step hand-offs / barriers, sweep tail
    unsigned long long cycPhaseA, cycPhaseB, cycSync, cycTail;
    // parts of the sweep tail: wrap-around and lap function (up to its team
    // barrier), candidate walks (up to the lead's barrier), the lead's choice
    unsigned long long cycWrap, cycCand, cycLead;
    // part of cycPhaseA spent waiting for the staged streams of a step
    unsigned long long cycStage;
    // minimum-cost outputs
    double firstLb;
    int firstV;
    int firstOrigin;
    double validLb;
    int validV;
    int anyFinite;
};

// State of one bounded literal walk (the reference's predecessor walk from a
// candidate, cost_time_ratio_solver.cpp:461-488), advanced a bounded number
// of predecessor loads per round so that no team barrier waits long.
struct LiteralWalk {
    int phase;        // 0 idle/done, 1 cycle length (Brent), 2 offset hare, 3 tail length, 4 first start node
    int a, b;         // tortoise and hare (expanded node ids)
    int pad;
    long long c1, c2, c3;
};

struct BfParams {
    // graph
    int n, nY, K, Kp, nslices;
    long long numNodes;            // n * nY
    const int* spInter;
    const int* spIntra;
    const int* srcInter;
    const int* srcDummy;
    const int* srcIntra;
    long long interEntries, intraEntries, layerStride;
    const void* cost;              // (nY+1) * layerStride values (float or double)
    const void* time;              // same layout, or nullptr for a constant time
    double tconst;
    // state
    double* dv;                    // [2][n][Kp] path value of every (node, depth) of two layers
    int2* doh;                     // [2][Kp][n] its path's origin (layer-0 start node or kLap* code) and length
    double* bak;                   // [n]
    int* pred;                     // [(nY+1)*K*n], expanded index layer*n*K + k*n + v
    const int* ctaSlice;           // [ncta+1] slice range of every CTA (both parts)
    const int* waitPtr;            // [ncta+1] CSR offsets into waitIdx
    const int* waitIdx;            // CTAs a CTA hands steps off with (its graph neighbours)
    unsigned* stepDone;            // [ncta * kStepDoneStride] last step each CTA completed
    int flagSync;                  // 1: neighbour hand-offs between steps, 0: team barrier
    int maxCtaSlices;              // most slices any CTA owns
    int rowCap;                    // rows (of 32 entries) one step buffer holds
    int stageSrcOnly;              // 1: the buffers hold source indices only (costs, times prefetched to L2)
    int* lapNext;                  // [n]
    int* lapSteps;                 // [n]
    LiteralWalk* walks;            // [n] state of the bounded literal walks
    int* candStat;                 // [n] shortcut verdict per candidate (0 none, 1 cycle, 2 no cycle, 3 undecided)
    int* candV0;                   // [n] first repeated layer-0 node of a candidate's walk
    long long* candSteps;          // [n] predecessor steps that walk needs
    int* layerFlag;                // [nY+1] stamp of the last sweep that improved the layer
    const int* branchOf;
    int branchId;
    double lambda, ub;
    int mode;                      // 0 ratio, 1 ratio upper-bound search, 2 minimum cost
    int maxSweeps;                 // safety cap on sweeps in one launch (0 = unlimited)
    unsigned spinLimit;            // polls of any wait before it gives up and raises the error word
    int stallCta;                  // test hook (-1: none): this CTA's hand-off also waits on ctl->neverSet
    int literalAll;                // test hook: decide every candidate by the literal walk
    Control* ctl;
    int* cycleBuf;                 // original node ids, walk order (reversed on the host)
    long long cycleCap;
    // per-CTA reduction slots
    double* redVal;
    int* redIdx;
    int* redAux;
    long long* redAux64;
    // minimum-cost lower bounds
    double* lbOut;                 // [n] lower bound per node (inf if not in the branch)
    int* originOut;                // [n] origin of the closing path of the node
};

// ---------------------------------------------------------------------------
// Kernel argument blocks and launchers (kernels_energy.cu, kernels_bf.cu).
// ---------------------------------------------------------------------------
struct EnergyArgs {
    int n, nY, nvx, nvy;
    long long interEntries, layerStride, total;  // total = (nY+1) * layerStride
    const int* tedgeInter;
    const int* tedgeIntra;
    const int* eX;       // 3 per template edge
    const int8_t* eY;    // YPattern per template edge
    const int* eSrc;
    const int* eTrgt;
    const int8_t* eNext;
    const int* EY;       // nY x 2
    const double* VX;    // nvx x 3
    const double* VY;    // nvy x 3
    const double* FD;    // nvx x nvy
    const double4* quat; // nY * quatEX distinct frames (w, x, y, z) or nullptr
    int quatEX, quatPrune;  // |EX| and the prune flag: node -> frame map
    // plain graph
    int lengthMode;      // ("feature", "lengthnormalisation"): columns [fd, length]
    int lineIntegral;
    // conjugate graph
    int costMode, timeMode;
    double rlAlpha, rlC, rlPwr;
    double maxSO3, maxFd;  // already rounded through float as in the reference
    double* out0;
    double* out1;        // nullptr for one column
    // histograms of the top kTopDigitBits of the columns' keys (the first
    // median pass), filled when non-null; hist1 only with out1
    unsigned long long* hist0;
    unsigned long long* hist1;
};
// Width of the first digit of the median selection.
constexpr int kTopDigitBits = 12;

struct QuatArgs {
    int nEX, nY, n, prune;
    const int* EX;
    const int* EY;
    const double* VX;
    const double* VY;
    const double* NX;
    const double* NY;
    double4* out;
};

struct SelectArgs {
    const double* col;
    long long total, layerStride, interEntries;
    int nY;
    const int* tedgeInter;
    const int* tedgeIntra;
    unsigned long long* hist;  // 1 << kMedianWideBits counters
};

// State of one column's median selection on the device: the key bits fixed
// so far (prefix under mask), the wanted rank inside the bucket they select
// and its size, the width of the next digit; then the order statistics, the
// median, the rescale factor and whether the float copy is inexact.
struct MedianState {
    unsigned long long prefix, mask;
    long long rank, bucket;
    int shift, bits, done, even;
    int err;                     // 1-4: the selection lost its rank; 5: it needs more digit passes
    int needAbove;               // even count, rank the bucket's largest: xk1 is the smallest key above it
    unsigned long long bucketTop, minAbove;
    double xk, xk1, median, factor;
    int inexact;                 // the rescaled column has a value that is not a float
    int pad;
};
constexpr int kMedianWideBits = 14;          // the second digit's width
constexpr long long kMedianCompact = 1 << 16;  // a bucket this small is selected in one block

struct LookupArgs {
    int n, nY;
    long long numNodes, eBlock;
    const int* spInter;
    const int* spIntra;
    const int* srcInter;
    const int* srcDummy;
    const int* srcIntra;
    const int* tedgeInter;
    const int* tedgeIntra;
    long long interEntries, layerStride;
    const double* c64;
    const double* t64;   // nullptr: constant time
    const float* c32;    // when set: the exact float copies of the rescaled columns, read instead
    const float* t32;
    double tconst;
    const int* pairSrc;
    const int* pairTrgt;
    int count;
    long long* edgeOut;
    double* cOut;
    double* tOut;
};

// One graph of a batched ratio solve (bf_batch_kernel): a CTA takes the job
// from the queue and runs its whole solve on the device -- the initial upper
// bound (cost_time_ratio_solver.cpp:652-707), the Lawler iterations
// (:558-635) and their cycle evaluations (computeRatioForCycle, :88-133) --
// as long as the first branch's cycle does not wrap; otherwise the host
// finishes the solve with branch and bound.
enum PairStatus : int {
    PAIR_PENDING = 0,
    PAIR_DONE = 1,       // result written
    PAIR_NAN = 2,        // the reference's (true, NaN, no rows) result
    PAIR_HOST = 3,       // the solve needs branch and bound (or a longer cycle record): finish on the host
    PAIR_ERR_UB = -1,    // no closed path through the upper-bound start node
    PAIR_ERR_EDGE = -2,  // a cycle edge was not found in the product graph
    PAIR_ERR_BF = -3,    // a Bellman-Ford call ended in an error status (in bfStatus)
    PAIR_ERR_WAIT = -4,  // a device wait ran out
    PAIR_ERR_GUARD = -5, // the upper-bound ratio search did not terminate
};

struct PairJob {
    BfParams bf;           // the graph's Bellman-Ford parameters; mode, branch, lambda, ub set per call
    LookupArgs lk;         // the graph's edge lookup tables (pair arrays unused)
    int* branchOf;         // == bf.branchOf, written by the solve
    double tconst;         // time of every edge when there is no time column
    // two cycle records of capacity `cap`: original node ids (cap + 1), and
    // per edge its id, cost and time
    int* recNodes[2];
    long long* recEdges[2];
    double* recC[2];
    double* recT[2];
    int cap;
    int ctas;              // CTAs of the Bellman-Ford team bf was prepared for
    int threads;           // threads of each of those CTAs
    // outputs
    int status;            // PairStatus
    int bfStatus;          // the failing call's status for PAIR_ERR_BF
    int passes;
    float objective;
    int nEdges;            // edges of the returned cycle, in recEdges[rec]
    int rec;
    double adjT;           // time sum of the returned cycle (the adjoint's T)
    double ratio;          // its ratio C / T in double (the adjoint's lambda*)
    long long cycles;      // SM clock cycles the CTA spent on the graph
    long long bfCalls, sweeps, lawlerIters, candidates, fallbackWalks;
};

constexpr int kStepDoneStride = 8;  // one 32-byte sector per CTA step counter
constexpr int kTeamWordStride = 8;  // words of a batched-solve team (one sector)
// Polls of a device wait before it gives up (~2 s with its back-off).
constexpr unsigned kDefaultSpinLimit = 1u << 24;
// Predecessor loads a literal walk advances per round between team barriers.
constexpr long long kWalkRoundLoads = 4096;
// Most threads per Bellman-Ford CTA: 20 warps fit the kernel's registers
// (about 100 per thread) on one SM without spilling the relaxation loop.
constexpr int kBfThreads = 640;
// Source values a lane gathers before folding them (one batch of rows).
constexpr int kGather = 20;
// Threads of a batched-solve CTA and the CTAs an SM should hold: each CTA
// solves one graph at a time, so CTAs on one SM overlap their latencies.
constexpr int kBatchThreads = 256;
// Capacity of a batched solve's cycle records (edges); a longer cycle hands
// the graph back to the host.
constexpr long long kBatchCycleCap = 1LL << 16;
constexpr int kBatchBlocksPerSm = 2;
// Rows of one gather batch when every row has nk source depths (nk > 0).
__host__ __device__ constexpr int bf_rows_per_batch(int nk) {
    return kGather / nk < 1 ? 1 : kGather / nk > 8 ? 8 : kGather / nk;
}
// Bytes of shared memory a single-CTA launch needs to keep its DP records
// and backup row on chip (128-byte aligned).
__host__ __device__ inline size_t bf_shared_table_bytes(int n, int Kp) {
    const size_t b = (size_t)2 * n * Kp * (sizeof(double) + sizeof(int2)) + (size_t)n * sizeof(double);
    return (b + 127) & ~(size_t)127;
}
// Offset of the first step buffer after the staged row offsets and the
// lists of slices with rows, both per part (128-byte aligned).
__host__ __device__ inline size_t bf_stage_offset(int maxCtaSlices) {
    return ((size_t)(2 * (maxCtaSlices + 1) + 2 * maxCtaSlices) * sizeof(int) + 127) & ~(size_t)127;
}
// Bytes of one step buffer: source index, cost and time of rowCap rows.
__host__ __device__ inline size_t bf_stage_buffer_bytes(int rowCap, int costBytes, int timeBytes) {
    return (size_t)rowCap * 32 * (4 + costBytes + timeBytes);
}
// Attributes of a device that stay fixed while the process runs, queried
// once per device (attribute queries can go to the driver and serialise
// between host threads).
struct DeviceInfo {
    int sms, smemOptin, clockKhz;
};
cudaError_t device_info(int device, DeviceInfo* out);
// Kernel launches the library has issued in this process: every launch
// helper counts its launches.
void note_launch();
long long launch_count();
cudaError_t launch_bf(const BfParams& p, int costIsF32, int timeKind, int blocks, int threads, bool cooperative,
                      bool sharedTables, size_t smemBytes, cudaStream_t stream);
cudaError_t bf_max_coop_blocks(int costIsF32, int timeKind, int threads, size_t smemBytes, int* blocksPerSm);
cudaError_t launch_extract_path(const BfParams& p, int v, cudaStream_t stream);
// Batched ratio solves: `count` jobs taken from a queue (*next, zeroed by the
// caller) by teams of `teamCtas` CTAs (blocks / teamCtas teams) of `threads`
// threads.  teamWords: kTeamWordStride zeroed words per team; spin: polls of
// a team barrier before it gives up.
cudaError_t launch_bf_batch(PairJob* jobs, int count, int* next, unsigned* teamWords, int teamCtas, unsigned spin,
                            int costIsF32, int timeKind, int blocks, int threads, size_t smemBytes,
                            cudaStream_t stream);
cudaError_t bf_batch_max_blocks(int costIsF32, int timeKind, int threads, size_t smemBytes, int* blocksPerSm);
cudaError_t launch_lookup_pairs(const LookupArgs& a, cudaStream_t stream);
// shared: many graphs' passes run side by side (batched solves): a small
// column's pass takes a grid proportional to its entries
cudaError_t launch_plain_energy(const EnergyArgs& a, cudaStream_t s, bool shared = false);
cudaError_t launch_ho_energy(const EnergyArgs& a, cudaStream_t s);
cudaError_t launch_quaternions(const QuatArgs& a, cudaStream_t s);
// Median of a column and its rescale (cost_time_ratio_solver.cpp:709-721),
// enqueued whole on stream s (kernels_energy.cu).
// allPasses: every digit pass that 64 key bits can need (else the first two;
// a column that needs more comes back with err 5).
cudaError_t launch_median_rescale(const SelectArgs& a, unsigned long long* topHist, MedianState* st,
                                  unsigned long long* hist, double* band, unsigned long long* count, long long nValues,
                                  double scaling, float* col32, double clip, bool allPasses, bool shared,
                                  cudaStream_t s);
cudaError_t launch_rescale_f64(const SelectArgs& a, MedianState* st, double clip, cudaStream_t s);
cudaError_t launch_to_f64(const float* col32, double* col, long long layerStride, long long interEntries, int nY,
                          const int* ti, const int* tr, cudaStream_t s);
cudaError_t launch_to_f32(const double* col, float* col32, long long total, long long layerStride,
                          long long interEntries, int nY, const int* ti, const int* tr, int* exact, cudaStream_t s);
cudaError_t launch_export(const double* col, double* out, int cols, int c, long long total, long long layerStride,
                          long long interEntries, int nY, long long eBlock, const int* ti, const int* tr,
                          cudaStream_t s);
// Most values (rows x columns) the no-allocation cost export holds: 2^21
// doubles, 16 MiB of device memory fixed at module load.
constexpr long long kNoAllocExportValues = 1LL << 21;
// Device address of the no-allocation export scratch on `device` (which must
// be current); taken with cudaGetSymbolAddress on the first call, then cached.
cudaError_t noalloc_export_scratch(int device, double** ptr);
cudaError_t launch_plain_energy_backward(const EnergyArgs& a, const long long* edges, int count, long long eBlock,
                                        double coef, double* grad, cudaStream_t s);
cudaError_t launch_conj_energy_backward(const EnergyArgs& a, const long long* edges, int count, long long eBlock,
                                       double coef, double coefT, long long argmax, double* grad, cudaStream_t s);
cudaError_t launch_import(const double* in, double* col, int cols, int c, long long total, long long layerStride,
                          long long interEntries, int nY, long long eBlock, const int* ti, const int* tr,
                          cudaStream_t s);
cudaError_t launch_normals_3d(const double* V, long long nv, const int* F, long long nf, double* fn, int* deg,
                              int* off, int* cursor, int* list, double* out, int* bad, cudaStream_t s);
cudaError_t launch_normals_2d(const double* Vin, int nv, const int* E, double* V, double* en, double* el, double* out,
                              int* bad, cudaStream_t s);
cudaError_t launch_layer1_mean(const double* cost, long long layerStride, long long interEntries, int n, int nslices,
                               const int* spI, const int* spA, const int* srcI, const int* srcA, float* meanOut,
                               int* countOut, cudaStream_t s);
cudaError_t launch_layer1_mean(const float* cost, long long layerStride, long long interEntries, int n, int nslices,
                               const int* spI, const int* spA, const int* srcI, const int* srcA, float* meanOut,
                               int* countOut, cudaStream_t s);

}  // namespace pgc
