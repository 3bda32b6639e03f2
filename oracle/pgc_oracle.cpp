// pgc_oracle.cpp -- CPU restatement of the reference's cycle-search path.
//
// TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA
// product is compared against; only tests/, __graft_entry__.smoke() and the
// cpu_baseline leg of bench.py may load it.  It is never linked into, or
// called by, the product library.
//
// Parity status: UNPINNED against the reference binary.  The reference cannot
// be compiled in this environment (every translation unit includes Eigen, and
// Eigen, robin-map and libigl are fetched by CMake at configure time; none are
// on disk), and the reference ships no golden vectors or tests.  This
// restatement is pinned instead against exhaustive brute-force enumeration of
// cycles on toy product graphs (tests/golden/, tests/test_oracle_*.py).
//
// Every routine cites the reference file:line whose behaviour it restates.
// Deliberate, documented deviations from the reference (all of them only
// touch behaviour that the reference leaves undefined or order-dependent):
//   * robin_set iteration order is replaced by ascending insertion order
//     (ascending edge id for in-edge sets, ascending value for vertex sets);
//   * std::sort of equal lower bounds is replaced by a sort on
//     (value, vertex index);
//   * the uninitialised ratioLowerBoundOfCurrentBranch
//     (cost_time_ratio_solver.cpp:835) is taken to be the branch's final ratio;
//   * for the pruned conjugate graph the node count is n * |EY| instead of
//     max(SRC)+1 (the latter drops the isolated last third of the last layer
//     and makes the reference read outside its arrays);
//   * pow(x, 2) in line integrals is written x*x;
//   * the 3x3 SVD of the SO(3) frame alignment is a one-sided Jacobi SVD
//     written from the mathematics (Eigen's JacobiSVD is not available).
// Compile with -ffp-contract=off so that c - lambda*t is never fused,
// matching the reference's x86-64 (SSE2) build.

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <limits>
#include <map>
#include <set>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

using i64 = long long;
static const double kInf = std::numeric_limits<double>::infinity();

static int thread_count() {
#ifdef _OPENMP
    int n = 0;
#pragma omp parallel reduction(+ : n)
    n += 1;
    return n;
#else
    return 1;
#endif
}
static inline int thread_id() {
#ifdef _OPENMP
    return omp_get_thread_num();
#else
    return 0;
#endif
}

// (int)std::round(x) as compiled for x86-64: out-of-range or NaN gives INT_MIN.
static int round_to_int(double x) {
    double r = std::round(x);
    if (!(r >= -2147483648.0 && r <= 2147483647.0)) return INT_MIN;
    return (int)r;
}

struct DMat {  // row-major dense double matrix
    i64 rows = 0, cols = 0;
    std::vector<double> v;
    DMat() {}
    DMat(i64 r, i64 c, double fill = 0.0) : rows(r), cols(c), v((size_t)(r * c), fill) {}
    double& operator()(i64 r, i64 c) { return v[(size_t)(r * cols + c)]; }
    double operator()(i64 r, i64 c) const { return v[(size_t)(r * cols + c)]; }
};
struct IMat {  // row-major dense int32 matrix
    i64 rows = 0, cols = 0;
    std::vector<int> v;
    IMat() {}
    IMat(i64 r, i64 c, int fill = 0) : rows(r), cols(c), v((size_t)(r * c), fill) {}
    int& operator()(i64 r, i64 c) { return v[(size_t)(r * cols + c)]; }
    int operator()(i64 r, i64 c) const { return v[(size_t)(r * cols + c)]; }
};

// ---------------------------------------------------------------------------
// Indexed binary min-heap.  Restates helper/minheap.cpp:16-277: keys are
// small integers, values are doubles; push ignores a key that is present or
// out of range; ties are resolved exactly as there (sift-up moves past an
// equal parent, sift-down prefers the right child on equality and moves past
// an equal child).  Pop order on equal values decides which branch-and-bound
// branch is explored next, so these rules are kept.
// ---------------------------------------------------------------------------
class MinHeap {
  public:
    explicit MinHeap(long cap) : slot_(cap, {-1.0, -1}), where_(cap, -1), cap_(cap) {}
    bool isEmpty() const { return size_ == 0; }
    long getSize() const { return size_; }
    double peak() const { return size_ == 0 ? kInf : slot_[0].first; }
    double peakKey(long key) const {
        if (key < 0 || key >= cap_ || where_[key] == -1) return -1.0;
        return slot_[where_[key]].first;
    }
    void push(double value, long key) {
        if (key < 0 || key >= cap_ || where_[key] != -1 || size_ == cap_) return;
        slot_[firstFree_] = {value, key};
        where_[key] = firstFree_;
        siftUp(firstFree_);
        ++size_;
        if (firstFree_ == lastUsed_ + 1) ++lastUsed_;
        if (size_ == cap_) { firstFree_ = size_ + 1; return; }
        while (slot_[firstFree_].second > -1) ++firstFree_;
    }
    bool decrease(long key, double value) {
        if (key < 0 || key >= cap_) return false;
        long at = where_[key];
        if (at != -1 && value < slot_[at].first) {
            slot_[at].first = value;
            siftUp(at);
            return slot_[at].first != value;
        }
        return false;
    }
    std::pair<double, long> pop() {
        if (size_ == 0) return {-1.0, -1};
        std::pair<double, long> top = slot_[0];
        slot_[0].first = kInf;
        swapSlots(0, lastUsed_);
        slot_[lastUsed_] = {-1.0, -1};
        where_[top.second] = -1;
        long landed = siftDown(0);
        if (lastUsed_ < firstFree_) firstFree_ = lastUsed_;
        while (lastUsed_ >= 0 && slot_[lastUsed_].second == -1) --lastUsed_;
        if (landed > lastUsed_) lastUsed_ = landed;
        --size_;
        return top;
    }

  private:
    void swapSlots(long a, long b) {
        if (a == b || a < 0 || b < 0 || a >= cap_ || b >= cap_ || slot_[a].second == -1 ||
            slot_[b].second == -1)
            return;
        std::swap(slot_[a], slot_[b]);
        where_[slot_[a].second] = a;
        where_[slot_[b].second] = b;
    }
    long siftUp(long i) {
        if (i < 0 || i >= cap_) return -1;
        while (i > 0) {
            long up = (i - 1) / 2;
            if (!(slot_[up].first >= slot_[i].first)) break;
            std::swap(slot_[up], slot_[i]);
            where_[slot_[i].second] = i;
            where_[slot_[up].second] = up;
            i = up;
        }
        return i;
    }
    long siftDown(long i) {
        if (i < 0 || i >= cap_) return -1;
        for (;;) {
            long l = 2 * i + 1, r = 2 * i + 2;
            bool lOk = l < cap_ && slot_[l].second != -1 && slot_[l].first <= slot_[i].first;
            bool rOk = r < cap_ && slot_[r].second != -1 && slot_[r].first <= slot_[i].first;
            long go = -1;
            if (lOk && rOk) go = (slot_[r].first <= slot_[l].first) ? r : l;
            else if (lOk) go = l;
            else if (rOk) go = r;
            if (go < 0) break;
            std::swap(slot_[go], slot_[i]);
            where_[slot_[i].second] = i;
            where_[slot_[go].second] = go;
            i = go;
        }
        return i;
    }
    std::vector<std::pair<double, long>> slot_;
    std::vector<long> where_;
    long cap_, size_ = 0, firstFree_ = 0, lastUsed_ = -1;
};

// ---------------------------------------------------------------------------
// Product graphs
// ---------------------------------------------------------------------------
struct ProductGraph {
    IMat ps;                   // E x 4 (plain) or E x 6 (conjugate)
    std::vector<int> src, trgt;
    std::vector<std::vector<long>> branchGraph;  // empty when not produced
};

static std::vector<std::vector<long>> to_sorted(const std::vector<std::set<long>>& s) {
    std::vector<std::vector<long>> out(s.size());
    for (size_t i = 0; i < s.size(); ++i) out[i].assign(s[i].begin(), s[i].end());
    return out;
}

// product_space.cpp:19-132.  Per Y-edge i: for every row j of EX an
// intralayer edge (unless pruned) then an interlayer edge, then one vertical
// edge per X vertex.  Node id = layer * |VX| + x.
static ProductGraph plain_product_graph(const IMat& EX, const IMat& EY, bool prune) {
    int nvx = 0;
    for (int x : EX.v) nvx = std::max(nvx, x + 1);
    const i64 nEX = EX.rows, nEY = EY.rows;
    ProductGraph g;
    const i64 perLayer = (prune ? 0 : nEX) + nEX + nvx;
    g.ps = IMat(nEY * perLayer, 4);
    g.src.resize((size_t)(nEY * perLayer));
    g.trgt.resize((size_t)(nEY * perLayer));
    i64 e = 0;
    for (i64 i = 0; i < nEY; ++i) {
        const i64 next = (i + 1) % nEY;
        for (i64 j = 0; j < nEX; ++j) {
            if (!prune) {
                g.ps(e, 0) = EY(i, 0); g.ps(e, 1) = EY(i, 0); g.ps(e, 2) = EX(j, 0); g.ps(e, 3) = EX(j, 1);
                g.src[e] = (int)(i * nvx + EX(j, 0));
                g.trgt[e] = (int)(i * nvx + EX(j, 1));
                ++e;
            }
            g.ps(e, 0) = EY(i, 0); g.ps(e, 1) = EY(i, 1); g.ps(e, 2) = EX(j, 0); g.ps(e, 3) = EX(j, 1);
            g.src[e] = (int)(i * nvx + EX(j, 0));
            g.trgt[e] = (int)(next * nvx + EX(j, 1));
            ++e;
        }
        for (i64 x = 0; x < nvx; ++x) {
            g.ps(e, 0) = EY(i, 0); g.ps(e, 1) = EY(i, 1); g.ps(e, 2) = (int)x; g.ps(e, 3) = (int)x;
            g.src[e] = (int)(i * nvx + x);
            g.trgt[e] = (int)(next * nvx + x);
            ++e;
        }
    }
    if (prune) {  // product_space.cpp:122-131: a vertex -> vertex adjacency
        std::vector<std::set<long>> bg((size_t)nvx);
        for (i64 j = 0; j < nEX; ++j) bg[EX(j, 0)].insert(EX(j, 1));
        g.branchGraph = to_sorted(bg);
    }
    return g;
}

// conj_product_space.cpp:16-228.  Nodes are product edges: per layer
// [non-degenerate | degenerate-2d | degenerate-3d] x |EX| (the last two
// coincide at offset |EX| when pruned).  Outgoing-edge sets of a vertex are
// iterated in ascending edge id.
static ProductGraph conj_product_graph(const IMat& EX, const IMat& EY, bool prune) {
    int nvx = 0;
    for (int x : EX.v) nvx = std::max(nvx, x + 1);
    const int nEX = (int)EX.rows;
    const i64 nEY = EY.rows;
    std::vector<std::vector<int>> out((size_t)nvx);
    for (int e = 0; e < nEX; ++e) out[EX(e, 0)].push_back(e);
    const int n = 3 * nEX;
    const int off2d = nEX;
    const int off3d = prune ? off2d : 2 * nEX;
    ProductGraph g;
    std::vector<int> rows;
    rows.reserve(1024);
    auto add = [&](int a, int b, int c, int d, int e2, int f, int s, int t) {
        rows.push_back(a); rows.push_back(b); rows.push_back(c);
        rows.push_back(d); rows.push_back(e2); rows.push_back(f);
        g.src.push_back(s);
        g.trgt.push_back(t);
    };
    for (i64 i = 0; i < nEY; ++i) {
        const int nxt = (int)((i + 1) % nEY);
        const int cur0 = (int)(i * n), nxt0 = nxt * n;
        const int s2 = EY(i, 0), m2 = EY(i, 1), t2 = EY(nxt, 1);
        if (!prune) {
            for (int j = 0; j < nEX; ++j) {
                const int s3 = EX(j, 0), m3 = EX(j, 1);
                for (int it : out[m3]) {
                    const int t3 = EX(it, 1);
                    if (t3 == s3) continue;
                    add(s2, s2, s2, s3, m3, t3, cur0 + off2d + j, cur0 + off2d + it);
                    add(s2, s2, m2, s3, m3, t3, cur0 + off2d + j, cur0 + it);
                }
            }
        }
        for (int j = 0; j < nEX; ++j) {
            const int s3 = EX(j, 0), m3 = EX(j, 1);
            for (int it : out[m3]) {
                const int t3 = EX(it, 1);
                if (t3 == s3) continue;
                add(s2, m2, t2, s3, m3, t3, cur0 + j, nxt0 + it);
                if (!prune) add(s2, m2, m2, s3, m3, t3, cur0 + j, nxt0 + off2d + it);
                add(s2, m2, t2, m3, m3, t3, cur0 + off3d + j, nxt0 + it);
            }
            add(s2, m2, t2, s3, m3, m3, cur0 + j, nxt0 + off3d + j);
            add(s2, m2, t2, m3, m3, m3, cur0 + off3d + j, nxt0 + off3d + j);
        }
    }
    g.ps.rows = (i64)g.src.size();
    g.ps.cols = 6;
    g.ps.v = std::move(rows);
    // conj_product_space.cpp:177-225
    std::vector<std::set<long>> bg((size_t)n);
    for (int j = 0; j < nEX; ++j) {
        bg[j].insert(j + nEX);
        if (!prune) {
            bg[j + nEX].insert(j + 2 * nEX);
            bg[j + 2 * nEX].insert(j);
        } else {
            bg[j + nEX].insert(j);
        }
        for (int pass = 0; pass < 2; ++pass) {  // the reference walks out(EX(j,0)) twice
            for (int e : out[EX(j, 0)]) {
                bg[j].insert(e);
                bg[j + nEX].insert(e + nEX);
                if (!prune) bg[j + 2 * nEX].insert(e + 2 * nEX);
            }
        }
    }
    g.branchGraph = to_sorted(bg);
    return g;
}

// ---------------------------------------------------------------------------
// Energies
// ---------------------------------------------------------------------------
enum HoMode { NOMODE, VANILLA, FEATURE, LENGTH, SO3_PLAIN, SO3_ROBUST, PENALISE_DEGENERATE };

// higherOrderDeformationEnergy.cpp:396-412, including its missing "== 0" on
// the last comparison: "penalisedegenerate" maps to VANILLA and every other
// unknown string (the default "") maps to PENALISE_DEGENERATE.
static HoMode string_to_mode(const std::string& s) {
    if (s == "nomode") return NOMODE;
    if (s == "vanilla") return VANILLA;
    if (s == "feature") return FEATURE;
    if (s == "lengthnormalisation") return LENGTH;
    if (s == "plainso3") return SO3_PLAIN;
    if (s == "robustso3") return SO3_ROBUST;
    if (s != "penalisedegenerate") return PENALISE_DEGENERATE;
    return VANILLA;
}

// deformationEnergy.cpp:11-78 and :97-103.
static DMat plain_energy(const DMat& VX, const DMat& VY, const IMat& ps, const DMat& FD, bool reg,
                         const std::string& cost, const std::string& time) {
    const bool lengthMode = (cost == "feature" && time == "lengthnormalisation");
    const bool lineIntegral = reg || lengthMode;
    DMat E(ps.rows, lengthMode ? 2 : 1, 0.0);
#pragma omp parallel for
    for (i64 i = 0; i < ps.rows; ++i) {
        const long y0 = ps(i, 0), y1 = ps(i, 1), x0 = ps(i, 2), x1 = ps(i, 3);
        if (y0 == -1) { E(i, 0) = 999999999.9; continue; }
        double li = 1.0;
        if (lineIntegral) {
            li = 0.0;
            for (int j = 0; j < 3; ++j) {
                const double dy = VY(y0, j) - VY(y1, j);
                li += dy * dy;
                const double dx = VX(x0, j) - VX(x1, j);
                li += dx * dx;
            }
            li = std::sqrt(li);
        }
        const double fd = FD(x0, y0) + FD(x1, y1);
        if (!lengthMode) {
            E(i, 0) = 0.5 * fd * li;
        } else {
            E(i, 0) = fd;
            E(i, 1) = li;
        }
    }
    return E;
}

struct Quat { double w, x, y, z; };

static void normalized3(const double in[3], double out[3]) {
    const double sq = in[0] * in[0] + in[1] * in[1] + in[2] * in[2];
    if (sq > 0.0) {
        const double nrm = std::sqrt(sq);
        for (int i = 0; i < 3; ++i) out[i] = in[i] / nrm;
    } else {
        for (int i = 0; i < 3; ++i) out[i] = in[i];
    }
}
static void cross3(const double a[3], const double b[3], double o[3]) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}
static double det3(const double m[3][3]) {
    return m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) -
           m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
           m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
}

// One-sided (Hestenes) Jacobi SVD of a 3x3 matrix A = U diag(s) V^T with the
// singular values sorted in decreasing order.
static void svd3(const double A[3][3], double U[3][3], double s[3], double V[3][3]) {
    double W[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) { W[i][j] = A[i][j]; V[i][j] = (i == j) ? 1.0 : 0.0; }
    for (int sweep = 0; sweep < 60; ++sweep) {
        double off = 0.0;
        for (int p = 0; p < 2; ++p)
            for (int q = p + 1; q < 3; ++q) {
                double a = 0, b = 0, c = 0;
                for (int i = 0; i < 3; ++i) { a += W[i][p] * W[i][p]; b += W[i][q] * W[i][q]; c += W[i][p] * W[i][q]; }
                if (std::fabs(c) <= 1e-300) continue;
                off = std::max(off, std::fabs(c) / std::sqrt(a * b + 1e-300));
                const double zeta = (b - a) / (2.0 * c);
                const double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
                const double cs = 1.0 / std::sqrt(1.0 + t * t), sn = cs * t;
                for (int i = 0; i < 3; ++i) {
                    const double wp = W[i][p], wq = W[i][q];
                    W[i][p] = cs * wp - sn * wq;
                    W[i][q] = sn * wp + cs * wq;
                    const double vp = V[i][p], vq = V[i][q];
                    V[i][p] = cs * vp - sn * vq;
                    V[i][q] = sn * vp + cs * vq;
                }
            }
        if (off < 1e-15) break;
    }
    int order[3] = {0, 1, 2};
    double nrm[3];
    for (int j = 0; j < 3; ++j) nrm[j] = std::sqrt(W[0][j] * W[0][j] + W[1][j] * W[1][j] + W[2][j] * W[2][j]);
    std::sort(order, order + 3, [&](int a, int b) { return nrm[a] > nrm[b]; });
    double Vs[3][3], Ws[3][3];
    for (int k = 0; k < 3; ++k) {
        s[k] = nrm[order[k]];
        for (int i = 0; i < 3; ++i) { Vs[i][k] = V[i][order[k]]; Ws[i][k] = W[i][order[k]]; }
    }
    for (int k = 0; k < 3; ++k)
        for (int i = 0; i < 3; ++i) V[i][k] = Vs[i][k];
    // U columns: normalised W columns; rank-deficient columns completed by cross products.
    double u0[3], u1[3], u2[3];
    double c0[3] = {Ws[0][0], Ws[1][0], Ws[2][0]}, c1[3] = {Ws[0][1], Ws[1][1], Ws[2][1]},
           c2[3] = {Ws[0][2], Ws[1][2], Ws[2][2]};
    const double tiny = 1e-14 * (s[0] > 0 ? s[0] : 1.0);
    if (s[0] > tiny) normalized3(c0, u0); else { u0[0] = 1; u0[1] = 0; u0[2] = 0; }
    if (s[1] > tiny) normalized3(c1, u1);
    else {
        double e[3] = {std::fabs(u0[0]) < 0.9 ? 1.0 : 0.0, std::fabs(u0[0]) < 0.9 ? 0.0 : 1.0, 0.0};
        double t[3];
        cross3(u0, e, t);
        normalized3(t, u1);
    }
    if (s[2] > tiny) normalized3(c2, u2);
    else {
        double t[3];
        cross3(u0, u1, t);
        normalized3(t, u2);
    }
    for (int i = 0; i < 3; ++i) { U[i][0] = u0[i]; U[i][1] = u1[i]; U[i][2] = u2[i]; }
}

// Quaternion of a rotation matrix (Shepperd's method).
static Quat quat_from_rot(const double R[3][3]) {
    Quat q;
    const double tr = R[0][0] + R[1][1] + R[2][2];
    if (tr > 0) {
        double t = std::sqrt(tr + 1.0);
        q.w = 0.5 * t;
        t = 0.5 / t;
        q.x = (R[2][1] - R[1][2]) * t;
        q.y = (R[0][2] - R[2][0]) * t;
        q.z = (R[1][0] - R[0][1]) * t;
    } else {
        int i = 0;
        if (R[1][1] > R[0][0]) i = 1;
        if (R[2][2] > R[i][i]) i = 2;
        const int j = (i + 1) % 3, k = (j + 1) % 3;
        double t = std::sqrt(R[i][i] - R[j][j] - R[k][k] + 1.0);
        double v[3];
        v[i] = 0.5 * t;
        t = 0.5 / t;
        q.w = (R[k][j] - R[j][k]) * t;
        v[j] = (R[j][i] + R[i][j]) * t;
        v[k] = (R[k][i] + R[i][k]) * t;
        q.x = v[0]; q.y = v[1]; q.z = v[2];
    }
    return q;
}

// higherOrderDeformationEnergy.cpp:16-53: rows of X and Y are the normalised
// frames [n, e, c]; the rotation is U diag(1,1,det(UV^T)) V^T from the SVD of
// X^T Y.
static Quat frame_rotation(const double v2[3], const double n2[3], const double c2[3], const double v3[3],
                           const double n3[3], const double c3[3]) {
    double X[3][3], Y[3][3];
    normalized3(n2, X[0]); normalized3(v2, X[1]); normalized3(c2, X[2]);
    normalized3(n3, Y[0]); normalized3(v3, Y[1]); normalized3(c3, Y[2]);
    double M[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double acc = 0;
            for (int r = 0; r < 3; ++r) acc += X[r][i] * Y[r][j];
            M[i][j] = acc;
        }
    double U[3][3], s[3], V[3][3];
    svd3(M, U, s, V);
    double UVt[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double acc = 0;
            for (int r = 0; r < 3; ++r) acc += U[i][r] * V[j][r];
            UVt[i][j] = acc;
        }
    const double d = det3(UVt);
    double R[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            R[i][j] = U[i][0] * V[j][0] + U[i][1] * V[j][1] + d * U[i][2] * V[j][2];
    return quat_from_rot(R);
}

// higherOrderDeformationEnergy.cpp:65-77
static double so3_distance(const Quat& a, const Quat& b) {
    double ip = std::fabs(a.w * b.w + (a.x * b.x + a.y * b.y + a.z * b.z));
    if (ip > 1) ip = 1;
    if (ip < -1) ip = -1;
    if (std::isnan(ip)) return 0;
    return 2 * std::acos(ip);
}

struct RobustLoss {
    double alpha, c, pwr;
    // higherOrderDeformationEnergy.cpp:55-63 (Barron's general robust loss)
    double operator()(double x) const {
        const double t = std::pow(x / c, pwr);
        const double am2 = std::fabs(alpha - 2);
        return am2 / alpha * (std::pow(t / am2 + 1, 0.5 * alpha) - 1);
    }
};

// higherOrderDeformationEnergy.cpp:95-134 (USE_MATLAB_CONVENTION): one
// quaternion per product node, index = layer * 3|EX| + node.
static std::vector<Quat> node_quaternions(const DMat& VX, const IMat& EX, const DMat& NX, const DMat& VY,
                                          const IMat& EY, const DMat& NY, bool prune) {
    const i64 nEX = EX.rows, nEY = EY.rows, n = 3 * nEX;
    std::vector<Quat> q((size_t)(n * nEY));
    auto frame2d = [&](i64 i, double e[3], double nn[3], double c[3]) {
        for (int k = 0; k < 3; ++k) {
            e[k] = VY(EY(i, 1), k) - VY(EY(i, 0), k);
            nn[k] = NY(EY(i, 0), k);
        }
        cross3(e, nn, c);
    };
#pragma omp parallel for
    for (i64 i = 0; i < nEY; ++i) {
        double e2[3], n2[3], c2[3], e2p[3], n2p[3], c2p[3];
        frame2d(i, e2, n2, c2);
        frame2d((i + nEY - 1) % nEY, e2p, n2p, c2p);
        for (i64 j = 0; j < n; ++j) {
            const i64 ed = j - (j / nEX) * nEX;
            double e3[3], n3[3], c3[3];
            for (int k = 0; k < 3; ++k) {
                e3[k] = VX(EX(ed, 1), k) - VX(EX(ed, 0), k);
                n3[k] = (NX(EX(ed, 0), k) + NX(EX(ed, 1), k)) / 2;
            }
            cross3(e3, n3, c3);
            Quat r;
            if (j < nEX) r = frame_rotation(e2, n2, c2, e3, n3, c3);
            else if (j < 2 * nEX && !prune) r = frame_rotation(e2p, n2p, c2p, e3, n3, c3);
            else r = frame_rotation(e2, n2, c2, e3, n3, c3);
            q[(size_t)(i * n + j)] = r;
        }
    }
    return q;
}

// higherOrderDeformationEnergy.cpp:209-339.  Unsupported (cost, time) pairs
// throw.  For (lengthnormalisation|penalisedegenerate-as-cost, vanilla) the
// reference also writes a second column into a one-column matrix; that write
// is out of bounds there and is dropped here.
static DMat ho_energy(const DMat& VX, const IMat& EX, const DMat& NX, const DMat& VY, const IMat& EY,
                      const DMat& NY, const ProductGraph& g, const DMat& FD, bool useSO3, const RobustLoss& rl,
                      bool prune, const std::string& costName, const std::string& timeName) {
    const HoMode cm = string_to_mode(costName), tm = string_to_mode(timeName);
    const bool supported = (cm == VANILLA && tm == VANILLA) || (cm == VANILLA && tm == LENGTH) ||
                           (cm == LENGTH && tm == VANILLA) || (cm == VANILLA && tm == PENALISE_DEGENERATE) ||
                           (cm == PENALISE_DEGENERATE && tm == VANILLA) || (cm == FEATURE && tm == SO3_PLAIN) ||
                           (cm == FEATURE && tm == SO3_ROBUST) || (cm == SO3_ROBUST && tm == FEATURE) ||
                           (cm == SO3_PLAIN && tm == FEATURE);
    if (!supported) throw std::runtime_error("cost time mode not supported");
    const int ncols = (tm == NOMODE || tm == VANILLA) ? 1 : 2;
    const bool needLi = (cm == LENGTH || tm == LENGTH);
    const double twoPi = 2 * M_PI;
    const float maxSO3 = (float)rl(twoPi);
    float maxFd = 0;
    if (tm == FEATURE) {
        double m = -kInf;
        for (double x : FD.v) m = std::max(m, x);
        maxFd = (float)m;
    }
    std::vector<Quat> q;
    if (useSO3) q = node_quaternions(VX, EX, NX, VY, EY, NY, prune);
    DMat E(g.ps.rows, ncols, 0.0);
#pragma omp parallel for
    for (i64 i = 0; i < g.ps.rows; ++i) {
        const long y0 = g.ps(i, 0), y1 = g.ps(i, 1), y2 = g.ps(i, 2);
        const long x0 = g.ps(i, 3), x1 = g.ps(i, 4), x2 = g.ps(i, 5);
        double so3 = 0.0;
        if (useSO3) so3 = so3_distance(q[(size_t)g.src[i]], q[(size_t)g.trgt[i]]);
        const double fd = FD(x2, y2);
        double li = 0;
        if (needLi) {
            for (int j = 0; j < 3; ++j) {
                const double dy = VY(y0, j) - VY(y1, j);
                li += dy * dy;
                const double dx = VX(x0, j) - VX(x1, j);
                li += dx * dx;
            }
            li = std::sqrt(li);
        }
        const bool degenerate = (y2 == y1 || x2 == x1);
        if (cm == VANILLA && tm == VANILLA) {
            E(i, 0) = rl(so3) + fd;
        } else if (cm == VANILLA && tm == LENGTH) {
            E(i, 0) = rl(so3) + fd;
            E(i, 1) = li;
        } else if (cm == LENGTH && tm == VANILLA) {
            E(i, 0) = li;
        } else if (cm == VANILLA && tm == PENALISE_DEGENERATE) {
            E(i, 0) = rl(so3) + fd;
            E(i, 1) = degenerate ? 0.1 : 1;
        } else if (cm == PENALISE_DEGENERATE && tm == VANILLA) {
            E(i, 0) = degenerate ? 0.1 : 1;
        } else if (cm == FEATURE && tm == SO3_PLAIN) {
            E(i, 0) = fd;
            E(i, 1) = std::max(0.0, twoPi - so3);
        } else if (cm == FEATURE && tm == SO3_ROBUST) {
            E(i, 0) = fd;
            E(i, 1) = std::max(0.0, (double)maxSO3 - rl(so3));
        } else if (cm == SO3_ROBUST && tm == FEATURE) {
            E(i, 0) = rl(so3);
            E(i, 1) = std::max(0.0, (double)maxFd - fd);
        } else {  // SO3_PLAIN, FEATURE
            E(i, 0) = so3;
            E(i, 1) = std::max(0.0, (double)maxFd - fd);
        }
    }
    return E;
}

// utils.hpp:196-209: sort a copy; even count -> mean of the two middle values.
static double median_of(std::vector<double> v) {
    std::sort(v.begin(), v.end());
    const size_t n = v.size();
    if (n % 2 == 0) return (v[(n - 2) / 2] + v[(n - 2) / 2 + 1]) / 2.0;
    return v[n / 2];
}

// cost_time_ratio_solver.cpp:709-721, applied in place.
static void rescale_column(DMat& E, int col, double scaling) {
    std::vector<double> c((size_t)E.rows);
    for (i64 i = 0; i < E.rows; ++i) c[(size_t)i] = E(i, col);
    const double med = std::max(median_of(c), 0.001);
    const double factor = scaling / (2.0 * med);
    const double clip = 100 * scaling;
    for (i64 i = 0; i < E.rows; ++i) {
        double x = std::round(factor * E(i, col));
        if (x > clip) x = clip;
        E(i, col) = x;
    }
}

// cost_time_ratio_solver.cpp:42-66 (dijkstra_solver.cpp:41-65 is the same):
// in-edge sets; layer-0 nodes also hold the marker -1; an edge into layer 0
// whose source id is strictly greater than n goes to dummy node numNodes + v.
static std::vector<std::vector<long>> build_in_graph(const std::vector<int>& SRC, const std::vector<int>& TRGT,
                                                     long total, long numNodes, long n) {
    std::vector<std::vector<long>> g((size_t)total);
    for (long v = 0; v < total && v < n; ++v) g[(size_t)v].push_back(-1);
    for (size_t e = 0; e < TRGT.size(); ++e) {
        const long v = TRGT[e];
        if (v < n && SRC[e] > n) {
            g[(size_t)(numNodes + v)].push_back((long)e);
            continue;
        }
        g[(size_t)v].push_back((long)e);
    }
    return g;
}

// ---------------------------------------------------------------------------
// Cost/time-ratio (Lawler) solver, CPU: cost_time_ratio_solver.cpp
// ---------------------------------------------------------------------------
enum BfStatus { CAN_CONTAIN_OPTIMUM, CANNOT_CONTAIN_OPTIMUM, NO_NEGATIVE_CYCLE, FOUND_NEGATIVE_CYCLE, ZERO_CYCLE };

struct SolveStats {
    long long bfCalls = 0, sweeps = 0, candidatesWalked = 0, lawlerIters = 0, branches = 0;
};

struct CtrState {
    long n = 0, numLayers = 0, numNodes = 0;
    int K = 1;
    std::vector<int> branchOf;
    int branchId = 0, maxBranchId = 0, numNodesInBranch = 0;
    std::vector<double> cost, time;
    std::vector<int> pred;
    std::vector<double> dp;  // (2K+1) rows x n
    std::vector<unsigned char> seen;
    std::vector<std::vector<long>> branchGraph, inGraph;
    double lowerBoundOfCurrentBranch = 0, upperBound = 0, ratioLowerBound = 0, ratioUpperBound = 0;
    double currentRatio = 0, tolerance = 0;
    std::vector<int> negativeCycle, upperBoundCycle, zeroLayerHits;
    int branchingSrcNode = -1, branchingTargetNode = -1;
    std::vector<std::pair<double, int>> lowerBounds;
    SolveStats* stats = nullptr;
    double& DP(long r, long v) { return dp[(size_t)(r * n + v)]; }
};

struct CycleEval { double ratio, wsum; IMat rows; std::vector<long> edges; };

// cost_time_ratio_solver.cpp:88-140
static CycleEval ratio_of_cycle(const CtrState& st, const std::vector<int>& cycle, const IMat& ps,
                                const std::vector<int>& SRC, bool writeOutput) {
    double C = 0, T = 0, W = 0;
    CycleEval out;
    if (writeOutput) out.rows = IMat(0, ps.cols);
    for (size_t i = 0; i + 1 < cycle.size(); ++i) {
        const long s = cycle[i];
        long t = cycle[i + 1];
        if (t < st.n && s > st.n) t += st.numNodes;
        long edge = -2;
        for (long e : st.inGraph.at((size_t)t)) {
            if (e != -1 && SRC[(size_t)e] == s) { edge = e; break; }
        }
        if (edge < 0) throw std::runtime_error("cycle edge not found");
        C += st.cost[(size_t)edge];
        T += st.time[(size_t)edge];
        W += st.cost[(size_t)edge] - st.currentRatio * st.time[(size_t)edge];
        out.edges.push_back(edge);
        if (writeOutput) {
            out.rows.rows += 1;
            for (i64 c = 0; c < ps.cols; ++c) out.rows.v.push_back(ps(edge, c));
        }
    }
    out.ratio = C / T;
    out.wsum = W;
    return out;
}

// cost_time_ratio_solver.cpp:240-250
static int original_index(long n, int K, int pred) {
    const long per = n * K;
    const long layer = pred / per;
    const long inLayer = pred - layer * per;
    const long depth = inLayer / n;
    const long vi = inLayer - depth * n;
    return (int)(vi + layer * n);
}

// cost_time_ratio_solver.cpp:251-542
static BfStatus bellman_ford_ctr(CtrState& st, const IMat& ps, const std::vector<int>& SRC, bool searchForZeroCycle,
                                 bool searchForUpperBound) {
    const long n = st.n;
    const int K = st.K;
    const int threads = thread_count();
    if (st.stats) st.stats->bfCalls++;
    std::fill(st.dp.begin(), st.dp.end(), kInf);
    int indexNodeInLayer = -1, numInBranch = 0;
    for (long i = 0; i < n; ++i) {
        if (st.branchOf[(size_t)i] == st.branchId) {
            indexNodeInLayer = (int)i;
            ++numInBranch;
            st.DP(0, i) = 0;
            st.pred[(size_t)i] = -1;
        }
    }
    st.numNodesInBranch = numInBranch;
    if (numInBranch == 0) throw std::runtime_error("no nodes in branch");

    std::vector<unsigned char> improves((size_t)threads, 1);
    bool negativeCycleFound = false;
    int iter = 0;
    const long backupRow = 2 * K;
    while (!negativeCycleFound) {
        if (st.stats) st.stats->sweeps++;
        for (long v = 0; v < n; ++v) st.DP(backupRow, v) = st.DP(0, v);
        for (long layer = 0; layer < st.numLayers + 1; ++layer) {
            const long prevOff = ((layer + 1) % 2) * K, curOff = (layer % 2) * K;
            if (layer != 0) {
                for (long r = curOff; r < curOff + K; ++r)
                    for (long v = 0; v < n; ++v) st.DP(r, v) = kInf;
                std::fill(improves.begin(), improves.end(), 0);
            }
            for (int k = 0; k < K; ++k) {
                if (layer == 0 && k == 0) continue;
#pragma omp parallel for
                for (long vi = 0; vi < n; ++vi) {
                    const int tid = thread_id();
                    const long v = vi + layer * n * K + (long)k * n;
                    const long actual = vi + layer * n;
                    for (long e : st.inGraph[(size_t)actual]) {
                        if (e == -1) continue;
                        const double w = st.cost[(size_t)e] - st.currentRatio * st.time[(size_t)e];
                        const long s = SRC[(size_t)e];
                        const bool intra = (s / n) == layer;
                        if (intra && k != 0) {
                            if (K <= 1) continue;
                            const long sl = s - layer * n;
                            const double d = st.DP(curOff + k - 1, sl);
                            if (std::isinf(d)) continue;
                            const double nv = d + w;
                            if (nv < st.DP(curOff + k, vi) && nv < st.upperBound) {
                                improves[(size_t)tid] = 1;
                                st.pred[(size_t)v] = (int)(sl + layer * n * K + (long)(k - 1) * n);
                                st.DP(curOff + k, vi) = nv;
                            }
                        }
                        if (!intra && k == 0) {
                            for (int kk = 0; kk < K; ++kk) {
                                const long sl = s - (layer - 1) * n;
                                const double d = st.DP(prevOff + kk, sl);
                                if (std::isinf(d)) continue;
                                const double nv = d + w;
                                if (nv < st.DP(curOff, vi) && nv < st.upperBound) {
                                    improves[(size_t)tid] = 1;
                                    st.pred[(size_t)v] = (int)(sl + (layer - 1) * n * K + (long)kk * n);
                                    st.DP(curOff, vi) = nv;
                                }
                            }
                        }
                    }
                }
            }
            bool any = false;
            for (unsigned char b : improves) any = any || b;
            if (!any && layer < st.numLayers && layer > 0) {
                const CycleEval old = ratio_of_cycle(st, st.negativeCycle, ps, SRC, false);
                if (round_to_int(old.wsum) == 0) return ZERO_CYCLE;
                return NO_NEGATIVE_CYCLE;
            }
        }

        if (searchForUpperBound) {
            const long maxLength = st.numLayers * K;
            std::vector<int> cycle;
            const long firstV = indexNodeInLayer + n * st.numLayers * K;
            cycle.push_back(original_index(n, K, (int)firstV));
            int p = st.pred[(size_t)firstV];
            cycle.push_back(original_index(n, K, p));
            for (long kk = maxLength - 1; kk > 0; --kk) {
                if (p == -1) break;
                p = st.pred[(size_t)p];
                cycle.push_back(original_index(n, K, p));
                if (p == indexNodeInLayer) break;
            }
            std::reverse(cycle.begin(), cycle.end());
            st.negativeCycle = cycle;
            const CycleEval ev = ratio_of_cycle(st, cycle, ps, SRC, false);
            const int integral = round_to_int(ev.wsum);
            if (integral == 0) return ZERO_CYCLE;
            if (integral < 0) return FOUND_NEGATIVE_CYCLE;
            return NO_NEGATIVE_CYCLE;
        }

        // wrap: the "last layer" row index is numLayers % 2 (a row, not a
        // depth offset: correct only for even numLayers or K == 1).
        const long lastRow = st.numLayers % 2;
        std::fill(improves.begin(), improves.end(), 0);
#pragma omp parallel for
        for (long vi = 0; vi < n; ++vi) {
            if (st.branchOf[(size_t)vi] != st.branchId) continue;
            const int tid = thread_id();
            const long vLast = n * K * st.numLayers + vi;
            if (st.DP(lastRow, vi) < st.DP(backupRow, vi)) {
                improves[(size_t)tid] = 1;
                st.DP(0, vi) = st.DP(lastRow, vi);
                st.pred[(size_t)vi] = st.pred[(size_t)vLast];
            } else {
                st.DP(0, vi) = st.DP(backupRow, vi);
            }
        }
        bool any = false;
        for (unsigned char b : improves) any = any || b;
        if (!any) {
            const CycleEval old = ratio_of_cycle(st, st.negativeCycle, ps, SRC, false);
            if (round_to_int(old.wsum) == 0) return ZERO_CYCLE;
            return NO_NEGATIVE_CYCLE;
        }

        st.lowerBounds.clear();
        for (long vi = 0; vi < n; ++vi) {
            if (st.branchOf[(size_t)vi] != st.branchId) continue;
            st.lowerBounds.push_back({st.DP(0, vi), (int)vi});
        }
        std::sort(st.lowerBounds.begin(), st.lowerBounds.end());

        volatile bool exists = false;
        int vFirst = -1, cycleLength = -1;
        const long maxCycleLength = st.numNodes;
        const long nlb = (long)st.lowerBounds.size();
#pragma omp parallel for shared(exists)
        for (long li = 0; li < nlb; ++li) {
            const int vi = st.lowerBounds[(size_t)li].second;
            if (st.branchOf[(size_t)vi] != st.branchId) continue;
            if (exists) continue;
            if (!searchForZeroCycle && st.DP(0, vi) >= 0) continue;
            if (searchForZeroCycle && (st.DP(0, vi) <= -st.tolerance || st.DP(0, vi) >= st.tolerance)) continue;
            const int tid = thread_id();
            unsigned char* seen = &st.seen[(size_t)tid * (size_t)n];
            std::memset(seen, 0, (size_t)n);
#pragma omp atomic
            st.stats->candidatesWalked++;
            int p = st.pred[(size_t)vi];
            seen[vi] = 1;
            int len = 1;
            for (long kk = maxCycleLength - 1; kk > 0; --kk) {
                if (p < n && p >= 0) {
                    if (seen[p]) {
#pragma omp critical
                        {
                            exists = true;
                            vFirst = p;
                            cycleLength = len;
                        }
                        break;
                    }
                    seen[p] = 1;
                }
                if (exists) break;
                p = st.pred[(size_t)p];
                if (p == -1) break;
                ++len;
            }
        }

        if (exists) {
            negativeCycleFound = true;
            std::vector<int> cycle;
            int p = st.pred[(size_t)vFirst];
            cycle.push_back(original_index(n, K, p));
            for (long kk = cycleLength - 1; kk > 0; --kk) {
                p = st.pred[(size_t)p];
                cycle.push_back(original_index(n, K, p));
                if (p == vFirst) break;
            }
            std::reverse(cycle.begin(), cycle.end());
            cycle.push_back(cycle.front() + (int)st.numNodes);
            const CycleEval ev = ratio_of_cycle(st, cycle, ps, SRC, false);
            const int integral = round_to_int(ev.wsum);
            if (integral < 0) {
                st.negativeCycle = cycle;
                return FOUND_NEGATIVE_CYCLE;
            } else if (integral == 0) {
                continue;  // leaves the loop (negativeCycleFound is set)
            } else {
                const CycleEval old = ratio_of_cycle(st, st.negativeCycle, ps, SRC, false);
                if (round_to_int(old.wsum) == 0) return ZERO_CYCLE;
                return NO_NEGATIVE_CYCLE;
            }
        }
        ++iter;
        if (iter >= st.numNodes - 1) return NO_NEGATIVE_CYCLE;
    }
    return NO_NEGATIVE_CYCLE;
}

// cost_time_ratio_solver.cpp:558-635
static bool lawler(CtrState& st, const IMat& ps, const std::vector<int>& SRC) {
    int i = 0;
    const int maxiter = 1000;
    double oldRatio = st.currentRatio;
    for (;;) {
        const BfStatus s = bellman_ford_ctr(st, ps, SRC, false, false);
        if (st.stats) st.stats->lawlerIters++;
        if (s == ZERO_CYCLE || s == NO_NEGATIVE_CYCLE) break;
        const CycleEval ev = ratio_of_cycle(st, st.negativeCycle, ps, SRC, false);
        st.currentRatio = ev.ratio;
        if (std::fabs(oldRatio - st.currentRatio) < st.tolerance) break;
        if (st.currentRatio - st.tolerance > oldRatio) break;
        oldRatio = st.currentRatio;
        if (i > maxiter) break;
        ++i;
    }
    st.lowerBoundOfCurrentBranch = st.currentRatio;
    int numWraps = 0;
    st.zeroLayerHits.clear();
    bool entered = true, left = false;
    for (int vtx : st.negativeCycle) {
        if (left && vtx < st.n) { entered = true; left = false; }
        if (entered) { st.zeroLayerHits.push_back(vtx); entered = false; }
        if (vtx >= st.n && !left) { ++numWraps; left = true; }
    }
    return numWraps > 1;
}

// cost_time_ratio_solver.cpp:142-222 -- only the part before the early
// `return` at :179 has an effect; the heap work above it is discarded.
static void branch_ctr(CtrState& st) {
    int offset = 0;
    for (int hit : st.zeroLayerHits) {
        if (offset > 0) st.branchOf[(size_t)hit] = st.maxBranchId + offset;
        ++offset;
    }
    const int counter = 0;
    for (long v = 0; v < st.n; ++v)
        if (st.branchOf[(size_t)v] == st.branchId)
            st.branchOf[(size_t)v] = st.maxBranchId + (int)((counter / st.numNodesInBranch) * offset);
    st.maxBranchId += offset;
}

// cost_time_ratio_solver.cpp:652-707.  The cycle ratio and weight are read
// through a tuple<float, float, ...>, so the start ratio is float-rounded.
static void initial_upper_bound(CtrState& st, const IMat& ps, const std::vector<int>& SRC) {
    float bestCost = std::numeric_limits<float>::infinity();
    int bestV = 0;
    for (long v = 0; v < st.n; ++v) {
        int num = 0;
        float mean = 0;
        for (long e : st.inGraph[(size_t)(v + st.n)]) {
            if (e == -1) continue;
            mean = (float)((double)mean + st.cost[(size_t)e]);
            ++num;
        }
        mean = mean / (float)num;
        if (mean < bestCost && num > 3) { bestCost = mean; bestV = (int)v; }
    }
    st.upperBound = (double)std::numeric_limits<float>::infinity();
    st.currentRatio = 10;
    std::fill(st.branchOf.begin(), st.branchOf.end(), 1);
    st.branchOf[(size_t)bestV] = 0;
    st.branchId = 0;
    bellman_ford_ctr(st, ps, SRC, true, true);
    CycleEval ev = ratio_of_cycle(st, st.negativeCycle, ps, SRC, false);
    double cycleCost = (double)(float)ev.wsum;
    int guard = 0;
    while (cycleCost > 0 || std::isnan(cycleCost)) {
        if (++guard > 4000) throw std::runtime_error("upper bound search does not terminate");
        st.currentRatio += st.currentRatio;
        ev = ratio_of_cycle(st, st.negativeCycle, ps, SRC, false);
        cycleCost = (double)(float)ev.wsum;
    }
    st.currentRatio = (double)(float)ev.ratio;
    std::fill(st.branchOf.begin(), st.branchOf.end(), 0);
    st.upperBoundCycle = st.negativeCycle;
}

struct SolveOutput {
    bool passes = false;
    float objective = 0;
    IMat matching;
    std::vector<long> edges;   // edge ids of the returned cycle, in order
    std::vector<int> cycle;    // original node ids
    SolveStats stats;
};

// cost_time_ratio_solver.cpp:741-864 and :868-900
static SolveOutput solve_ctr(const IMat& ps, DMat& energy, const std::vector<int>& SRC, const std::vector<int>& TRGT,
                             long n, int K, const std::vector<std::vector<long>>& branchGraph, long numNodes) {
    const double scaling = 100000.0;
    rescale_column(energy, 0, scaling);
    if (energy.cols > 1) rescale_column(energy, 1, scaling);

    SolveOutput out;
    CtrState st;
    st.stats = &out.stats;
    st.n = n;
    st.K = K;
    st.numNodes = numNodes;
    st.numLayers = numNodes / n;
    const long numTotalNodes = n * (st.numLayers + 1) * K;
    st.pred.assign((size_t)numTotalNodes, -1);
    st.branchOf.assign((size_t)n, 0);
    st.dp.assign((size_t)((2 * K + 1) * n), kInf);
    st.branchGraph = branchGraph;
    st.maxBranchId = 0;
    st.seen.assign((size_t)n * (size_t)thread_count(), 0);
    st.cost.resize((size_t)energy.rows);
    st.time.resize((size_t)energy.rows);
    for (i64 e = 0; e < energy.rows; ++e) {
        st.cost[(size_t)e] = energy(e, 0);
        st.time[(size_t)e] = energy.cols > 1 ? energy(e, 1) : scaling / 2;
    }
    st.tolerance = (double)(float)1e-8;
    st.inGraph = build_in_graph(SRC, TRGT, numNodes + n, numNodes, n);

    initial_upper_bound(st, ps, SRC);

    st.branchId = 0;
    st.ratioLowerBound = 0;
    st.ratioUpperBound = st.currentRatio;
    MinHeap heap(n);
    heap.push(0, st.branchId);
    std::vector<unsigned char> validLb((size_t)n, 0);
    std::map<int, std::vector<int>> validCycles;
    std::fill(st.branchOf.begin(), st.branchOf.end(), 0);
    while (!heap.isEmpty()) {
        const auto top = heap.pop();
        st.branchId = (int)top.second;
        st.ratioLowerBound = top.first;
        if (validLb[(size_t)st.branchId]) {
            st.ratioUpperBound = top.first;
            st.negativeCycle = validCycles.at(st.branchId);
            break;
        }
        out.stats.branches++;
        st.currentRatio = st.ratioUpperBound;
        const bool wraps = lawler(st, ps, SRC);
        if (st.ratioUpperBound < heap.peak() && !wraps) break;
        if (!wraps) {
            heap.push(st.lowerBoundOfCurrentBranch, st.branchId);
            validLb[(size_t)st.branchId] = 1;
            validCycles.emplace(st.branchId, st.negativeCycle);
            continue;
        }
        if (st.numNodesInBranch == 1) continue;
        branch_ctr(st);
        for (int hit : st.zeroLayerHits) heap.push(st.lowerBoundOfCurrentBranch, st.branchOf[(size_t)hit]);
    }
    const CycleEval fin = ratio_of_cycle(st, st.negativeCycle, ps, SRC, true);
    out.passes = true;
    out.objective = (float)fin.ratio;
    out.matching = fin.rows;
    out.edges = fin.edges;
    out.cycle = st.negativeCycle;
    return out;
}

// ---------------------------------------------------------------------------
// Minimum-cost ("dijkstra") solver, CPU: dijkstra_solver.cpp
// ---------------------------------------------------------------------------
struct DijState {
    long n = 0, numLayers = 0, numNodes = 0;
    int K = 1;
    std::vector<int> branchOf;
    int branchId = 0, numNodesInBranch = 0;
    std::vector<double> cost;
    std::vector<int> pred;
    std::vector<double> dp;
    std::vector<std::vector<long>> branchGraph, inGraph;
    double lowerBoundOfCurrentBranch = 0, lowerBound = 0, upperBound = 0;
    std::vector<int> cycle;
    int branchingSrcNode = -1, branchingTargetNode = -1;
    bool upperboundFoundOnFirstTry = false;
    std::vector<std::pair<double, int>> lowerBounds;
    SolveStats* stats = nullptr;
    double& DP(long r, long v) { return dp[(size_t)(r * n + v)]; }
};

// dijkstra_solver.cpp:203-388: one layered sweep from the branch's start set.
static bool bellman_ford_dij(DijState& st, const std::vector<int>& SRC) {
    const long n = st.n;
    const int K = st.K;
    const int threads = thread_count();
    if (st.stats) { st.stats->bfCalls++; st.stats->sweeps++; }
    std::fill(st.dp.begin(), st.dp.end(), kInf);
    int numInBranch = 0;
    for (long i = 0; i < n; ++i) {
        if (st.branchOf[(size_t)i] == st.branchId) {
            ++numInBranch;
            st.DP(0, i) = 0;
            st.pred[(size_t)i] = -1;
        }
    }
    st.numNodesInBranch = numInBranch;
    if (numInBranch == 0) throw std::runtime_error("no nodes in branch");
    std::vector<unsigned char> improves((size_t)threads, 1);
    const long backupRow = 2 * K;
    for (long v = 0; v < n; ++v) st.DP(backupRow, v) = st.DP(0, v);
    for (long layer = 0; layer < st.numLayers + 1; ++layer) {
        const long prevOff = ((layer + 1) % 2) * K, curOff = (layer % 2) * K;
        if (layer != 0) {
            for (long r = curOff; r < curOff + K; ++r)
                for (long v = 0; v < n; ++v) st.DP(r, v) = kInf;
            std::fill(improves.begin(), improves.end(), 0);
        }
        for (int k = 0; k < K; ++k) {
            if (layer == 0 && k == 0) continue;
#pragma omp parallel for
            for (long vi = 0; vi < n; ++vi) {
                const int tid = thread_id();
                const long v = vi + layer * n * K + (long)k * n;
                const long actual = vi + layer * n;
                for (long e : st.inGraph[(size_t)actual]) {
                    if (e == -1) continue;
                    const double w = st.cost[(size_t)e];
                    const long s = SRC[(size_t)e];
                    const bool intra = (s / n) == layer;
                    if (intra && k != 0) {
                        if (K <= 1) continue;
                        const long sl = s - layer * n;
                        const double d = st.DP(curOff + k - 1, sl);
                        if (std::isinf(d)) continue;
                        const double nv = d + w;
                        if (nv < st.DP(curOff + k, vi) && nv < st.upperBound) {
                            improves[(size_t)tid] = 1;
                            st.pred[(size_t)v] = (int)(sl + layer * n * K + (long)(k - 1) * n);
                            st.DP(curOff + k, vi) = nv;
                        }
                    }
                    if (!intra && k == 0) {
                        for (int kk = 0; kk < K; ++kk) {
                            const long sl = s - (layer - 1) * n;
                            const double d = st.DP(prevOff + kk, sl);
                            if (std::isinf(d)) continue;
                            const double nv = d + w;
                            if (nv < st.DP(curOff, vi) && nv < st.upperBound) {
                                improves[(size_t)tid] = 1;
                                st.pred[(size_t)v] = (int)(sl + (layer - 1) * n * K + (long)kk * n);
                                st.DP(curOff, vi) = nv;
                            }
                        }
                    }
                }
            }
        }
        bool any = false;
        for (unsigned char b : improves) any = any || b;
        if (!any && layer < st.numLayers && layer > 0) return false;
    }
    const long lastRow = st.numLayers % 2;
    st.lowerBounds.clear();
    bool anyFinite = false;
    for (long vi = 0; vi < n; ++vi) {
        if (st.branchOf[(size_t)vi] != st.branchId) continue;
        const double lb = st.DP(lastRow, vi);
        st.lowerBounds.push_back({lb, (int)vi});
        if (!std::isinf(lb)) anyFinite = true;
    }
    if (!anyFinite) return false;
    std::sort(st.lowerBounds.begin(), st.lowerBounds.end());

    bool first = true;
    const long maxCycleLength = st.numLayers * K;
    std::vector<int> cycle;
    st.upperboundFoundOnFirstTry = false;
    for (const auto& lbv : st.lowerBounds) {
        const float lb = (float)lbv.first;
        if (std::isinf(lb)) { first = false; continue; }
        const int v = lbv.second;
        const long vLast = v + n * st.numLayers * K;
        cycle.clear();
        if (st.stats) st.stats->candidatesWalked++;
        int p = st.pred[(size_t)vLast];
        cycle.push_back(original_index(n, K, p));
        for (long kk = maxCycleLength; kk > 0; --kk) {
            p = st.pred[(size_t)p];
            if (p == -1) break;
            cycle.push_back(original_index(n, K, p));
        }
        if (first) st.lowerBoundOfCurrentBranch = lb;
        if (v == cycle.back()) {
            if (first) st.upperboundFoundOnFirstTry = true;
            const float newUb = lb;
            if (newUb > st.upperBound && first) return false;
            if (newUb < st.upperBound) {
                st.upperBound = newUb;
                st.cycle = cycle;
            }
            break;
        } else if (first) {
            // dijkstra_solver.cpp:381 takes the source as the last-layer end of
            // the path minus numNodes, a negative id that matches no vertex, so
            // branch_dij() seeds only the new branch and empties the old one.
            // The GPU variant of the reference (dijkstra_bnb_subroutine.cu:444)
            // uses the candidate vertex v; that is followed here.
            st.branchingSrcNode = v;
            st.branchingTargetNode = cycle.back();
        }
        first = false;
    }
    return true;
}

// dijkstra_solver.cpp:87-174
static void branch_dij(DijState& st, const std::vector<int>& SRC, int maxBranchId) {
    const bool useBranchGraph = !st.branchGraph.empty();
    const auto& bg = useBranchGraph ? st.branchGraph : st.inGraph;
    MinHeap heap(st.n);
    for (long i = 0; i < st.n; ++i) {
        st.DP(0, i) = -1;
        if (i == st.branchingSrcNode || i == st.branchingTargetNode) { st.DP(0, i) = 1; continue; }
        if (st.branchOf[(size_t)i] == st.branchId) {
            heap.push(kInf, i);
            st.DP(0, i) = -1;
        }
    }
    heap.push(0.0, st.branchingSrcNode);
    heap.push(0.0, st.branchingTargetNode);
    st.branchOf[(size_t)st.branchingTargetNode] = maxBranchId;
    int counter = 0;
    for (const auto& lbv : st.lowerBounds) {
        const int v = lbv.second;
        if (v == st.branchingSrcNode || v == st.branchingTargetNode) continue;
        if (st.branchOf[(size_t)v] != st.branchId) continue;
        if (counter > std::max(1, st.numNodesInBranch / 4)) {
            heap.push(0.1, v);
            st.branchOf[(size_t)v] = maxBranchId;
        }
        ++counter;
    }
    while (!heap.isEmpty()) {
        const auto cur = heap.pop();
        const int node = (int)cur.second;
        const float nodeCost = (float)cur.first;
        st.DP(0, node) = 1.0;
        for (long e : bg.at((size_t)node)) {
            if (e == -1) continue;
            const int s = SRC[(size_t)e];
            if (st.DP(0, s) < 0) {
                const float oldV = (float)heap.peakKey(s);
                const float newV = nodeCost + 1.0f;
                if (newV < oldV) {
                    heap.decrease(s, newV);
                    st.branchOf[(size_t)s] = st.branchOf[(size_t)node];
                }
            }
        }
    }
    st.branchingSrcNode = -1;
    st.branchingTargetNode = -1;
}

// dijkstra_solver.cpp:407-559 and :563-579
static SolveOutput solve_dij(const IMat& ps, const DMat& energy, const std::vector<int>& SRC,
                             const std::vector<int>& TRGT, long n, int K,
                             const std::vector<std::vector<long>>& branchGraph, long numNodes) {
    SolveOutput out;
    DijState st;
    st.stats = &out.stats;
    st.n = n;
    st.K = K;
    st.numNodes = numNodes;
    st.numLayers = numNodes / n;
    const long numTotalNodes = n * (st.numLayers + 1) * K;
    st.pred.assign((size_t)numTotalNodes, -1);
    st.branchOf.assign((size_t)n, 0);
    st.dp.assign((size_t)((2 * K + 1) * n), kInf);
    st.branchGraph = branchGraph;
    st.upperBound = kInf;
    st.lowerBound = 0;
    st.branchId = 0;
    st.cost.resize((size_t)energy.rows);
    for (i64 e = 0; e < energy.rows; ++e) st.cost[(size_t)e] = energy(e, 0);
    st.inGraph = build_in_graph(SRC, TRGT, numNodes + n, numNodes, n);

    MinHeap heap(n);
    heap.push(0.0, st.branchId);
    int maxBranchId = 0;
    std::vector<unsigned char> validLb((size_t)n, 0);
    std::map<int, std::vector<int>> validCycles;
    while (!heap.isEmpty()) {
        const auto top = heap.pop();
        st.branchId = (int)top.second;
        st.lowerBound = top.first;
        if (validLb[(size_t)st.branchId]) {
            st.upperBound = top.first;
            st.cycle = validCycles.at(st.branchId);
            break;
        }
        out.stats.branches++;
        const bool couldContain = bellman_ford_dij(st, SRC);
        if (!couldContain) continue;
        if (st.upperBound < heap.peak() && st.upperboundFoundOnFirstTry) break;
        if (st.upperboundFoundOnFirstTry) {
            heap.push(st.lowerBoundOfCurrentBranch, st.branchId);
            validLb[(size_t)st.branchId] = 1;
            validCycles.emplace(st.branchId, st.cycle);
            continue;
        }
        ++maxBranchId;
        if (maxBranchId >= n) throw std::runtime_error("branch id exceeds the node count");
        branch_dij(st, SRC, maxBranchId);
        heap.push(st.lowerBoundOfCurrentBranch, st.branchId);
        heap.push(st.lowerBoundOfCurrentBranch, maxBranchId);
    }

    // dijkstra_solver.cpp:511-557
    std::vector<int> cyc = st.cycle;
    const long len = (long)cyc.size();
    std::reverse(cyc.begin(), cyc.end());
    if (cyc.empty()) throw std::runtime_error("no cycle found");
    cyc.push_back(cyc.front() + (int)numNodes);
    const long loopmax = len + 1;
    int loops = 0;
    out.matching = IMat(0, ps.cols);
    for (long i = 0; i < loopmax; ++i) {
        const long s = cyc[(size_t)(i % loopmax)];
        const long t = cyc[(size_t)((i + 1) % loopmax)];
        if (t >= numNodes) ++loops;
        long edge = -2;
        for (long e : st.inGraph.at((size_t)t)) {
            if (e != -1 && SRC[(size_t)e] == s) { edge = e; break; }
            if (e == -1 && t == s - numNodes) { edge = e; break; }
        }
        if (edge == -1) continue;
        if (edge == -2) throw std::runtime_error("cycle edge not found");
        out.matching.rows += 1;
        for (i64 c = 0; c < ps.cols; ++c) out.matching.v.push_back(ps(edge, c));
        out.edges.push_back(edge);
    }
    out.passes = loops < 2;
    out.objective = (float)st.upperBound;
    out.cycle = cyc;
    return out;
}

// ---------------------------------------------------------------------------
// Facade: product_graph_generators.cpp
// ---------------------------------------------------------------------------
struct Generator {
    DMat VX, VY, FD, NX, NY;
    IMat EX, EY;
    bool conj = false, reg = false, prune = false, normalsGiven = false, generated = false;
    double rlAlpha = 0.7, rlC = 0.6, rlPwr = 4;
    int maxDepth = 4;
    std::string costName = "vanilla", timeName = "";
    ProductGraph g;
    DMat energy;
    SolveOutput last;
    std::string error;

    long nodesPerLayer() const {
        if (conj) return 3 * EX.rows;
        return VX.rows;
    }
    long numNodes() const {
        if (conj) return nodesPerLayer() * EY.rows;
        long m = 0;
        for (int s : g.src) m = std::max(m, (long)s + 1);
        return m;
    }
    void generate() {  // product_graph_generators.cpp:21-89
        if (conj) {
            if (!normalsGiven) throw std::runtime_error("normals not set");
            g = conj_product_graph(EX, EY, prune);
            energy = ho_energy(VX, EX, NX, VY, EY, NY, g, FD, reg, RobustLoss{rlAlpha, rlC, rlPwr}, prune, costName,
                               timeName);
        } else {
            g = plain_product_graph(EX, EY, prune);
            if (!prune) g.branchGraph.clear();
            energy = plain_energy(VX, VY, g.ps, FD, reg, costName, timeName);
        }
        generated = true;
    }
    // The energies again on the product graph already built: what a second
    // generate() recomputes when its graph is kept (product_graph_generators.cpp:
    // 44-47, :81-85), and what the device's generate() does with its cached
    // layer template.
    void recompute_energy() {
        if (!generated) {
            generate();
            return;
        }
        if (conj)
            energy = ho_energy(VX, EX, NX, VY, EY, NY, g, FD, reg, RobustLoss{rlAlpha, rlC, rlPwr}, prune, costName,
                               timeName);
        else
            energy = plain_energy(VX, VY, g.ps, FD, reg, costName, timeName);
    }
};

}  // namespace orc

// ---------------------------------------------------------------------------
// C interface used by the tests (ctypes)
// ---------------------------------------------------------------------------
using namespace orc;
static thread_local std::string g_err;

extern "C" {

const char* orc_last_error() { return g_err.c_str(); }

void orc_set_threads(int t) {
#ifdef _OPENMP
    omp_set_num_threads(t > 0 ? t : 1);
#else
    (void)t;
#endif
}

void* orc_create(const double* VX, long long nvx, const int* EX, long long nex, const double* VY, long long nvy,
                 const int* EY, long long ney, const double* FD, int conj, int reg, int prune) {
    Generator* G = new Generator();
    G->VX = DMat(nvx, 3); std::memcpy(G->VX.v.data(), VX, sizeof(double) * nvx * 3);
    G->VY = DMat(nvy, 3); std::memcpy(G->VY.v.data(), VY, sizeof(double) * nvy * 3);
    G->EX = IMat(nex, 2); std::memcpy(G->EX.v.data(), EX, sizeof(int) * nex * 2);
    G->EY = IMat(ney, 2); std::memcpy(G->EY.v.data(), EY, sizeof(int) * ney * 2);
    G->FD = DMat(nvx, nvy); std::memcpy(G->FD.v.data(), FD, sizeof(double) * nvx * nvy);
    G->conj = conj != 0; G->reg = reg != 0; G->prune = prune != 0;
    return G;
}
void orc_destroy(void* h) { delete (Generator*)h; }
int orc_set_normals(void* h, const double* NX, long long nx, const double* NY, long long ny) {
    Generator* G = (Generator*)h;
    if (nx != G->VX.rows || ny != G->VY.rows) return -1;
    G->NX = DMat(nx, 3); std::memcpy(G->NX.v.data(), NX, sizeof(double) * nx * 3);
    G->NY = DMat(ny, 3); std::memcpy(G->NY.v.data(), NY, sizeof(double) * ny * 3);
    G->normalsGiven = true;
    return 0;
}
void orc_set_mode(void* h, const char* cost, const char* time) {
    ((Generator*)h)->costName = cost;
    ((Generator*)h)->timeName = time;
}
void orc_set_max_depth(void* h, int k) { ((Generator*)h)->maxDepth = k; }
void orc_set_robust_loss(void* h, double a, double c, double p) {
    Generator* G = (Generator*)h;
    if (!G->conj || G->generated) return;
    G->rlAlpha = a; G->rlC = c; G->rlPwr = p;
}
int orc_generate(void* h) {
    try { ((Generator*)h)->generate(); return 0; }
    catch (const std::exception& e) { g_err = e.what(); return -1; }
}
int orc_recompute_energy(void* h) {
    try { ((Generator*)h)->recompute_energy(); return 0; }
    catch (const std::exception& e) { g_err = e.what(); return -1; }
}
int orc_ensure_generated(void* h) {
    Generator* G = (Generator*)h;
    if (G->generated) return 0;
    return orc_generate(h);
}
void orc_cost_shape(void* h, long long* rows, long long* cols) {
    *rows = ((Generator*)h)->energy.rows; *cols = ((Generator*)h)->energy.cols;
}
void orc_get_cost(void* h, double* out) {
    const DMat& E = ((Generator*)h)->energy;
    std::memcpy(out, E.v.data(), sizeof(double) * E.v.size());
}
int orc_set_cost(void* h, const double* data, long long rows, long long cols) {
    Generator* G = (Generator*)h;
    if (rows != G->g.ps.rows) return -1;
    G->energy = DMat(rows, cols);
    std::memcpy(G->energy.v.data(), data, sizeof(double) * rows * cols);
    return 0;
}
void orc_ps_shape(void* h, long long* rows, long long* cols) {
    *rows = ((Generator*)h)->g.ps.rows; *cols = ((Generator*)h)->g.ps.cols;
}
void orc_get_ps(void* h, int* out) {
    const IMat& P = ((Generator*)h)->g.ps;
    std::memcpy(out, P.v.data(), sizeof(int) * P.v.size());
}
void orc_get_src_trgt(void* h, int* src, int* trgt) {
    Generator* G = (Generator*)h;
    std::memcpy(src, G->g.src.data(), sizeof(int) * G->g.src.size());
    std::memcpy(trgt, G->g.trgt.data(), sizeof(int) * G->g.trgt.size());
}

// utils::normals2d (helper/utils.cpp:93-157): outward vertex normals of an
// ordered closed curve in a coordinate plane.  The plane is the first
// coordinate column whose sum is below 1e-4 in magnitude; edge normals are
// the edge vectors rotated about z, flipped when the float-rounded test of
// :120-133 finds them pointing inward; a vertex normal is the length-weighted
// sum of the normals of the edges ending and starting at it.  Returns 0, or
// -1 when the points lie in no coordinate plane.
int orc_normals_2d(const double* Vin, long long nv, const int* E, long long ne, double* out) {
    if (nv != ne) return -2;
    std::vector<double> V(Vin, Vin + 3 * nv);
    int zero = -1;
    for (int i = 0; i < 3; ++i) {
        double s = 0;
        for (long long r = 0; r < nv; ++r) s += V[(size_t)(3 * r + i)];
        if (std::fabs(s) < 1e-4) { zero = i; break; }
    }
    if (zero == -1) return -1;
    if (zero != 2) {
        const int order[3] = {zero == 1 ? 0 : 1, 2, zero == 1 ? 1 : 0};
        std::vector<double> W(V.size());
        for (long long r = 0; r < nv; ++r)
            for (int k = 0; k < 3; ++k) W[(size_t)(3 * r + k)] = V[(size_t)(3 * r + order[k])];
        V.swap(W);
    }
    std::vector<double> en((size_t)(3 * ne)), el((size_t)ne);
    for (long long i = 0; i < ne; ++i) {
        const int a = E[2 * i], b = E[2 * i + 1];
        const double ev[3] = {V[(size_t)(3 * a)] - V[(size_t)(3 * b)], V[(size_t)(3 * a + 1)] - V[(size_t)(3 * b + 1)],
                              V[(size_t)(3 * a + 2)] - V[(size_t)(3 * b + 2)]};
        el[(size_t)i] = std::sqrt(ev[0] * ev[0] + ev[1] * ev[1] + ev[2] * ev[2]);
        const double nrm[3] = {ev[1], -ev[0], ev[2]};  // rotation about z
        const double len = std::sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
        for (int k = 0; k < 3; ++k) en[(size_t)(3 * i + k)] = len > 0 ? nrm[k] / len : nrm[k];
    }
    double mx = -INFINITY, mn = INFINITY, my = -INFINITY, mny = INFINITY;
    for (long long r = 0; r < nv; ++r) {
        mx = std::max(mx, V[(size_t)(3 * r)]); mn = std::min(mn, V[(size_t)(3 * r)]);
        my = std::max(my, V[(size_t)(3 * r + 1)]); mny = std::min(mny, V[(size_t)(3 * r + 1)]);
    }
    const float maxX = (float)mx, minX = (float)mn, maxY = (float)my, minY = (float)mny;
    const float mult = (float)(0.1 * std::min(std::fabs(maxX - minX), std::fabs(maxY - minY)));
    double mm = -INFINITY;
    for (long long r = 0; r < nv; ++r) mm = std::max(mm, V[(size_t)(3 * r)] + (double)mult * en[(size_t)(3 * r)]);
    if ((float)mm < maxX)
        for (auto& x : en) x = -x;
    for (long long i = 1; i < nv + 1; ++i) {
        const long long j = i % nv;
        double v[3];
        for (int k = 0; k < 3; ++k)
            v[k] = el[(size_t)(i - 1)] * en[(size_t)(3 * (i - 1) + k)] + el[(size_t)j] * en[(size_t)(3 * j + k)];
        const double len = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        for (int k = 0; k < 3; ++k) out[3 * j + k] = len > 0 ? v[k] / len : v[k];
    }
    return 0;
}

// utils::normals3d (helper/utils.cpp:86-90): libigl per_vertex_normals with
// its default area weighting -- per vertex the sum, in face order, of the
// incident faces' edge cross products (unit normal times twice the area),
// then scaled to unit length.  Returns 0, or -1 for an index outside V.
int orc_normals_3d(const double* V, long long nv, const int* F, long long nf, double* out) {
    for (long long i = 0; i < 3 * nv; ++i) out[i] = 0.0;
    for (long long f = 0; f < nf; ++f) {
        const int a = F[3 * f], b = F[3 * f + 1], c = F[3 * f + 2];
        if (a < 0 || b < 0 || c < 0 || a >= nv || b >= nv || c >= nv) return -1;
        double u[3], w[3];
        for (int k = 0; k < 3; ++k) {
            u[k] = V[3 * b + k] - V[3 * a + k];
            w[k] = V[3 * c + k] - V[3 * a + k];
        }
        const double nrm[3] = {u[1] * w[2] - u[2] * w[1], u[2] * w[0] - u[0] * w[2], u[0] * w[1] - u[1] * w[0]};
        for (int k = 0; k < 3; ++k) {
            out[3 * a + k] += nrm[k];
            out[3 * b + k] += nrm[k];
            out[3 * c + k] += nrm[k];
        }
    }
    for (long long i = 0; i < nv; ++i) {
        const double len = std::sqrt(out[3 * i] * out[3 * i] + out[3 * i + 1] * out[3 * i + 1] +
                                     out[3 * i + 2] * out[3 * i + 2]);
        if (len > 0)
            for (int k = 0; k < 3; ++k) out[3 * i + k] /= len;
    }
    return 0;
}

// which: 0 = cost/time ratio (lawlercpu), 1 = minimum cost (dijkstracpu).
int orc_solve(void* h, int which, int k, int* passes, float* objective) {
    Generator* G = (Generator*)h;
    try {
        if (!G->generated) G->generate();
        const int K = k > 0 ? k : G->maxDepth;
        if (which == 0)
            G->last = solve_ctr(G->g.ps, G->energy, G->g.src, G->g.trgt, G->nodesPerLayer(), K, G->g.branchGraph,
                                G->numNodes());
        else
            G->last = solve_dij(G->g.ps, G->energy, G->g.src, G->g.trgt, G->nodesPerLayer(), K, G->g.branchGraph,
                                G->numNodes());
        *passes = G->last.passes ? 1 : 0;
        *objective = G->last.objective;
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}
void orc_matching_shape(void* h, long long* rows, long long* cols) {
    *rows = ((Generator*)h)->last.matching.rows; *cols = ((Generator*)h)->last.matching.cols;
}
void orc_get_matching(void* h, int* out) {
    const IMat& M = ((Generator*)h)->last.matching;
    std::memcpy(out, M.v.data(), sizeof(int) * M.v.size());
}
long long orc_cycle_edges(void* h, long long* out, long long cap) {
    const auto& E = ((Generator*)h)->last.edges;
    for (size_t i = 0; i < E.size() && (long long)i < cap; ++i) out[i] = E[i];
    return (long long)E.size();
}
void orc_stats(void* h, long long* out5) {
    const SolveStats& s = ((Generator*)h)->last.stats;
    out5[0] = s.bfCalls; out5[1] = s.sweeps; out5[2] = s.candidatesWalked; out5[3] = s.lawlerIters; out5[4] = s.branches;
}

// Phase timings of one ratio solve on the CPU, for the benchmark's CPU
// baseline: out4 = [energy, rescale, in-edge sets, seconds per sweep].  The
// energy is recomputed and rescaled in place; `sweeps` sweeps are run at
// ratio `lambda` by repeated Bellman-Ford calls.
void orc_time_phases(void* h, int k, double lambda, int sweeps, double* out4) {
    Generator* G = (Generator*)h;
    if (!G->generated) G->generate();
    auto now = [] { return std::chrono::steady_clock::now(); };
    auto secs = [](std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
        return std::chrono::duration<double>(b - a).count();
    };
    auto t0 = now();
    if (G->conj)
        G->energy = ho_energy(G->VX, G->EX, G->NX, G->VY, G->EY, G->NY, G->g, G->FD, G->reg,
                              RobustLoss{G->rlAlpha, G->rlC, G->rlPwr}, G->prune, G->costName, G->timeName);
    else
        G->energy = plain_energy(G->VX, G->VY, G->g.ps, G->FD, G->reg, G->costName, G->timeName);
    auto t1 = now();
    rescale_column(G->energy, 0, 100000.0);
    if (G->energy.cols > 1) rescale_column(G->energy, 1, 100000.0);
    auto t2 = now();
    CtrState st;
    SolveStats stats;
    st.stats = &stats;
    st.n = G->nodesPerLayer();
    st.K = k;
    st.numNodes = G->numNodes();
    st.numLayers = st.numNodes / st.n;
    st.inGraph = build_in_graph(G->g.src, G->g.trgt, st.numNodes + st.n, st.numNodes, st.n);
    auto t3 = now();
    st.pred.assign((size_t)(st.n * (st.numLayers + 1) * k), -1);
    st.branchOf.assign((size_t)st.n, 0);
    st.dp.assign((size_t)((2 * k + 1) * st.n), kInf);
    st.seen.assign((size_t)st.n * (size_t)thread_count(), 0);
    st.cost.resize((size_t)G->energy.rows);
    st.time.resize((size_t)G->energy.rows);
    for (i64 e = 0; e < G->energy.rows; ++e) {
        st.cost[(size_t)e] = G->energy(e, 0);
        st.time[(size_t)e] = G->energy.cols > 1 ? G->energy(e, 1) : 50000.0;
    }
    st.currentRatio = lambda;
    st.upperBound = kInf;
    st.tolerance = (double)(float)1e-8;
    auto t4 = now();
    while (stats.sweeps < sweeps) {
        try { bellman_ford_ctr(st, G->g.ps, G->g.src, false, false); }
        catch (const std::exception&) { break; }
    }
    auto t5 = now();
    out4[0] = secs(t0, t1);
    out4[1] = secs(t1, t2);
    out4[2] = secs(t2, t3);
    out4[3] = secs(t4, t5) / (double)std::max<long long>(1, stats.sweeps);
}

// Time `sweeps` Bellman-Ford sweeps of the ratio solver at ratio `lambda` on
// the generated graph (the per-sweep CPU cost used by the benchmark's CPU
// baseline).  Returns seconds.
double orc_time_sweeps(void* h, int k, double lambda, int sweeps) {
    Generator* G = (Generator*)h;
    if (!G->generated) G->generate();
    CtrState st;
    SolveStats stats;
    st.stats = &stats;
    st.n = G->nodesPerLayer();
    st.K = k;
    st.numNodes = G->numNodes();
    st.numLayers = st.numNodes / st.n;
    st.pred.assign((size_t)(st.n * (st.numLayers + 1) * k), -1);
    st.branchOf.assign((size_t)st.n, 0);
    st.dp.assign((size_t)((2 * k + 1) * st.n), kInf);
    st.seen.assign((size_t)st.n * (size_t)thread_count(), 0);
    st.cost.resize((size_t)G->energy.rows);
    st.time.resize((size_t)G->energy.rows);
    for (i64 e = 0; e < G->energy.rows; ++e) {
        st.cost[(size_t)e] = G->energy(e, 0);
        st.time[(size_t)e] = G->energy.cols > 1 ? G->energy(e, 1) : 50000.0;
    }
    st.inGraph = build_in_graph(G->g.src, G->g.trgt, st.numNodes + st.n, st.numNodes, st.n);
    st.currentRatio = lambda;
    st.upperBound = kInf;
    st.tolerance = (double)(float)1e-8;
    // Run whole sweeps through the real routine: each call stops at its first
    // negative cycle or after at most numNodes-1 sweeps, so repeat calls until
    // the requested sweep count is reached.
    auto t0 = std::chrono::steady_clock::now();
    while (stats.sweeps < sweeps) {
        try { bellman_ford_ctr(st, G->g.ps, G->g.src, false, false); }
        catch (const std::exception&) { break; }
    }
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count() / (double)std::max<long long>(1, stats.sweeps) * sweeps;
}

}  // extern "C"
