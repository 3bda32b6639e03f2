// kernels_energy.cu -- edge costs of the product graph, computed on the device
// straight into the per-layer streams that the relaxation reads.
//
// Stream layout: layer l (0..nY) owns layerStride = entries[INTER] +
// entries[INTRA] consecutive values; entry j < entries[INTER] is INTER slot
// entry j (an edge of block l-1), the rest are INTRA entries (edges of block
// l).  Entries that hold no edge are NaN.
//
// Cost formulas restate deformationEnergy.cpp:11-78 (plain graph) and
// higherOrderDeformationEnergy.cpp:209-339 (conjugate graph).  The whole file
// is compiled with --fmad=false so no product is fused into a sum; pure
// arithmetic modes are therefore bit-identical to the CPU formulas.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <map>
#include <mutex>
#include <set>
#include <tuple>

#include "device_common.cuh"

namespace pgc {


enum HoMode { NOMODE = 0, VANILLA, FEATURE, LENGTH, SO3_PLAIN, SO3_ROBUST, PENALISE_DEGENERATE };

__device__ __forceinline__ double line_integral(const EnergyArgs& a, int y0, int y1, int x0, int x1) {
    double li = 0.0;
    for (int j = 0; j < 3; ++j) {
        const double dy = __ldg(a.VY + 3 * y0 + j) - __ldg(a.VY + 3 * y1 + j);
        li = li + dy * dy;
        const double dx = __ldg(a.VX + 3 * x0 + j) - __ldg(a.VX + 3 * x1 + j);
        li = li + dx * dx;
    }
    return sqrt(li);
}

// Visits the per-layer streams in work items of consecutive positions of one
// layer (one division per item, not per entry): f(idx, l, pos, t, inRange)
// for every position; t is the template edge, >= 0 for a real edge (l >= 1
// for interlayer entries, l < nY for intralayer ones).  Positions are visited
// warp-aligned, so every lane of a warp makes the same calls (warp
// collectives inside f are allowed); lanes past the item's end get
// inRange = false.
template <class F>
__device__ __forceinline__ void for_stream_layers(long long layerStride, long long interEntries, int nY,
                                                  const int* ti, const int* tr, F f) {
    // Two positions per thread and round: their template ids are loaded
    // together, and f reads its tables through the read-only path (__ldg), so
    // the compiler may overlap the two positions' table reads with the
    // other's stores.  Positions inside a layer fit 32 bits.
    constexpr int U = 2;
    const int stride = (int)layerStride, inter = (int)interEntries;
    const int chunk = 8 * (int)blockDim.x;  // a multiple of U * blockDim.x
    const int perLayer = (stride + chunk - 1) / chunk;
    const long long items = (long long)perLayer * (nY + 1);
    const int lane = threadIdx.x & 31, step = (int)blockDim.x;
    for (long long it = blockIdx.x; it < items; it += gridDim.x) {
        const int l = (int)(it / perLayer);
        const int p0 = (int)(it - (long long)l * perLayer) * chunk;
        const int p1 = min(p0 + chunk, stride);
        const long long rowBase = (long long)l * layerStride;
        const int* tInter = l >= 1 ? ti : nullptr;
        const int* tIntra = l < nY ? tr - inter : nullptr;
        for (int base = p0 + (int)threadIdx.x; base - lane < p1; base += U * step) {
            int t[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int pos = base + u * step;
                const int* tb = pos < inter ? tInter : tIntra;
                t[u] = (pos < p1 && tb) ? __ldg(tb + pos) : -1;
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int pos = base + u * step;
                if (pos - lane < p1) f(rowBase + pos, l, (long long)pos, t[u], pos < p1);
            }
        }
    }
}

// The same visit for passes that read one column: f(idx, x, valid, inRange)
// with x = col[idx] (0 where !inRange).  Each thread first loads U positions
// (template ids and values) and then calls f on them, so U loads of each
// stream are in flight per thread however much f synchronises; one load at
// a time left a pass at about a quarter of HBM bandwidth.
template <int U, class F>
__device__ __forceinline__ void for_stream_values(const double* col, long long layerStride, long long interEntries,
                                                  int nY, const int* ti, const int* tr, F f) {
    // positions inside a layer fit 32 bits (the streams of one layer are
    // indexed by int slot offsets), which keeps the U-fold unrolled body small
    const int stride = (int)layerStride, inter = (int)interEntries;
    const int chunk = 8 * (int)blockDim.x;  // a multiple of U * blockDim.x
    const int perLayer = (stride + chunk - 1) / chunk;
    const long long items = (long long)perLayer * (nY + 1);
    const int lane = threadIdx.x & 31, step = (int)blockDim.x;
    for (long long it = blockIdx.x; it < items; it += gridDim.x) {
        const int l = (int)(it / perLayer);
        const int p0 = (int)(it - (long long)l * perLayer) * chunk;
        const int p1 = min(p0 + chunk, stride);
        const long long rowBase = (long long)l * layerStride;
        const double* row = col + rowBase;
        const int* tInter = l >= 1 ? ti : nullptr;
        const int* tIntra = l < nY ? tr - inter : nullptr;
        for (int base = p0 + (int)threadIdx.x; base - lane < p1; base += U * step) {
            int t[U];
            double x[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int pos = base + u * step;
                t[u] = -1;
                x[u] = 0.0;
                if (pos < p1) {
                    const int* tb = pos < inter ? tInter : tIntra;
                    if (tb) t[u] = tb[pos];
                    x[u] = row[pos];
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int pos = base + u * step;
                if (pos - lane < p1) f(rowBase + pos, x[u], t[u] >= 0, pos < p1);
            }
        }
    }
}

// Order-preserving 64-bit image of a double (the median selection's keys).
__device__ __forceinline__ unsigned long long order_key(double x) {
    const unsigned long long u = (unsigned long long)__double_as_longlong(x);
    return (u >> 63) ? ~u : (u | 0x8000000000000000ULL);
}

// The energy kernels also count the most significant 12-bit digit of every
// value they write (the first pass of the median selection), when the host
// asks for it: per-thread runs of equal digits, added to shared counters when
// the digit changes, then the block's non-zero counters to the column's
// global histogram.  A column's values share a few exponents, so the runs
// are long.
constexpr int kTopBins = 1 << kTopDigitBits;
struct DigitRun {
    unsigned bin = 0xffffffffu, cnt = 0;
};
__device__ __forceinline__ void count_top_digit(unsigned* sh, DigitRun& r, double x) {
    const unsigned bin = (unsigned)(order_key(x) >> (64 - kTopDigitBits));
    if (bin == r.bin) {
        ++r.cnt;
        return;
    }
    if (r.cnt) atomicAdd(sh + r.bin, r.cnt);
    r.bin = bin;
    r.cnt = 1;
}
__device__ __forceinline__ void top_digit_begin(const EnergyArgs& a, unsigned* sh) {
    if (!a.hist0) return;
    for (int i = threadIdx.x; i < 2 * kTopBins; i += blockDim.x) sh[i] = 0;
    __syncthreads();
}
__device__ __forceinline__ void top_digit_end(const EnergyArgs& a, unsigned* sh, DigitRun& r0, DigitRun& r1) {
    if (!a.hist0) return;
    if (r0.cnt) atomicAdd(sh + r0.bin, r0.cnt);
    if (r1.cnt) atomicAdd(sh + kTopBins + r1.bin, r1.cnt);
    __syncthreads();
    for (int i = threadIdx.x; i < kTopBins; i += blockDim.x) {
        if (sh[i]) atomicAdd(a.hist0 + i, (unsigned long long)sh[i]);
        if (a.hist1 && sh[kTopBins + i]) atomicAdd(a.hist1 + i, (unsigned long long)sh[kTopBins + i]);
    }
}

// Each thread takes U = 4 positions of one layer per round and walks them
// through the entry's chain of dependent reads one level at a time --
// template edge id, then its Y pattern and X columns, then the two feat_diff
// entries -- so each level's U loads are in flight together (one position
// at a time left the kernel at a tenth of HBM bandwidth on small graphs).
// The arithmetic per entry is deformationEnergy.cpp:11-78's, unchanged.
__global__ void plain_energy_kernel(EnergyArgs a) {
    extern __shared__ unsigned int topSh[];  // [2][kTopBins] when a.hist0
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    DigitRun r0, r1;
    top_digit_begin(a, topSh);
    constexpr int U = 4;
    const int stride = (int)a.layerStride, inter = (int)a.interEntries;
    const int chunk = U * (int)blockDim.x;
    const int perLayer = (stride + chunk - 1) / chunk;
    const long long items = (long long)perLayer * (a.nY + 1);
    const int step = (int)blockDim.x;
    for (long long it = blockIdx.x; it < items; it += gridDim.x) {
        const int l = (int)(it / perLayer);
        const int p0 = (int)(it - (long long)l * perLayer) * chunk;
        const long long rowBase = (long long)l * a.layerStride;
        const int* tInter = l >= 1 ? a.tedgeInter : nullptr;
        const int* tIntra = l < a.nY ? a.tedgeIntra - inter : nullptr;
        const int yInter0 = l >= 1 ? __ldg(a.EY + 2 * (l - 1)) : 0, yInter1 = l >= 1 ? __ldg(a.EY + 2 * (l - 1) + 1) : 0;
        const int yIntra0 = l < a.nY ? __ldg(a.EY + 2 * l) : 0, yIntra1 = l < a.nY ? __ldg(a.EY + 2 * l + 1) : 0;
        int t[U], y0[U], y1[U], x0[U], x1[U];
        double f0[U], f1[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int pos = p0 + u * step + (int)threadIdx.x;
            const int* tb = pos < inter ? tInter : tIntra;
            t[u] = (pos < stride && tb) ? __ldg(tb + pos) : -2;  // -2: out of range, -1: empty slot
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int pos = p0 + u * step + (int)threadIdx.x;
            y0[u] = y1[u] = x0[u] = x1[u] = 0;
            if (t[u] >= 0) {
                const bool interPos = pos < inter;
                y0[u] = interPos ? yInter0 : yIntra0;
                y1[u] = __ldg(a.eY + t[u]) == 0 ? y0[u] : (interPos ? yInter1 : yIntra1);
                x0[u] = __ldg(a.eX + 3 * t[u]);
                x1[u] = __ldg(a.eX + 3 * t[u] + 1);
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            f0[u] = f1[u] = 0.0;
            if (t[u] >= 0) {
                f0[u] = __ldg(a.FD + (long long)x0[u] * a.nvy + y0[u]);
                f1[u] = __ldg(a.FD + (long long)x1[u] * a.nvy + y1[u]);
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int pos = p0 + u * step + (int)threadIdx.x;
            if (t[u] == -2 && pos < stride) t[u] = -1;  // a slot of a layer side without edges
            if (pos >= stride) continue;
            const long long idx = rowBase + pos;
            if (t[u] < 0) {
                a.out0[idx] = nan;
                if (a.out1) a.out1[idx] = nan;
                continue;
            }
            const double li = a.lineIntegral ? line_integral(a, y0[u], y1[u], x0[u], x1[u]) : 1.0;
            const double fd = f0[u] + f1[u];
            const double c0 = a.lengthMode ? fd : 0.5 * fd * li;
            a.out0[idx] = c0;
            if (a.lengthMode) a.out1[idx] = li;
            if (a.hist0) {
                count_top_digit(topSh, r0, c0);
                if (a.hist1) count_top_digit(topSh + kTopBins, r1, li);
            }
        }
    }
    top_digit_end(a, topSh, r0, r1);
}

// Adjoint of plain_energy_kernel for the edges of a cycle: scatters
// coef * d(cost)/d(feat_diff) of every listed product edge into grad
// (|VX| x |VY|, row-major).  cost = 0.5 (fd[x0,y0] + fd[x1,y1]) li, or
// fd[x0,y0] + fd[x1,y1] in the ("feature", "lengthnormalisation") mode,
// whose time column li does not depend on feat_diff.  An edge listed twice
// contributes twice.
__global__ void plain_energy_backward_kernel(EnergyArgs a, const long long* edges, int count, long long eBlock,
                                             double coef, double* grad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const long long e = edges[i];
    if (e < 0) return;
    const int b = (int)(e / eBlock), t = (int)(e - (long long)b * eBlock);
    if (b >= a.nY) return;
    const int y0 = a.EY[2 * b];
    const int y1 = a.eY[t] == 0 ? y0 : a.EY[2 * b + 1];
    const int x0 = a.eX[3 * t], x1 = a.eX[3 * t + 1];
    const double li = a.lineIntegral ? line_integral(a, y0, y1, x0, x1) : 1.0;
    const double d = a.lengthMode ? coef : coef * 0.5 * li;
    atomicAdd(grad + (long long)x0 * a.nvy + y0, d);
    atomicAdd(grad + (long long)x1 * a.nvy + y1, d);
}

// Adjoint of ho_energy_kernel's cost column for the edges of a cycle, in the
// modes where that column reads feat_diff once, linearly with slope 1:
// ("vanilla", *) has cost = robust loss + fd[x2, y2], ("feature", *) has
// cost = fd[x2, y2] (higherOrderDeformationEnergy.cpp).  Scatters coef into
// grad[x2, y2] of every listed product edge; an edge listed twice
// contributes twice.
// Every cycle edge e reads fd[x2, y2]: with slope coef in the cost column,
// and, when coefT != 0 (a ratio whose time column is ("*", "feature"):
// t = max(0, maxFd - fd), maxFd the matrix's maximum), with slope -1 in
// the time -- the adjoint there is +coefT at fd[x2, y2] and -coefT at the
// maximum's entry `argmax` (a subgradient: zero where the time is clamped at
// 0, and the two cancel when e reads the maximum itself).
__global__ void conj_energy_backward_kernel(EnergyArgs a, const long long* edges, int count, long long eBlock,
                                            double coef, double coefT, long long argmax, double* grad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const long long e = edges[i];
    if (e < 0) return;
    const int b = (int)(e / eBlock), t = (int)(e - (long long)b * eBlock);
    if (b >= a.nY) return;
    const int s2 = a.EY[2 * b], m2 = a.EY[2 * b + 1], t2 = a.EY[2 * ((b + 1) % a.nY) + 1];
    int y2;
    switch (a.eY[t]) {
        case 2: y2 = s2; break;
        case 3: y2 = m2; break;
        case 4: y2 = t2; break;
        default: y2 = m2; break;
    }
    const int x2 = a.eX[3 * t + 2];
    const long long at = (long long)x2 * a.nvy + y2;
    if (coef != 0.0) atomicAdd(grad + at, coef);
    if (coefT != 0.0 && a.maxFd - __ldg(a.FD + at) > 0.0) {
        atomicAdd(grad + at, coefT);
        atomicAdd(grad + argmax, -coefT);
    }
}

// Inverse of export_kernel: column c of a [rows x cols] edge-ordered matrix
// into the per-layer stream (empty slots get NaN).
__global__ void import_kernel(const double* in, double* col, int cols, int c, long long total, long long layerStride,
                              long long interEntries, int nY, long long eBlock, const int* tedgeInter,
                              const int* tedgeIntra) {
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long l = idx / layerStride;
        const long long pos = idx - l * layerStride;
        long long block;
        int t;
        if (pos < interEntries) {
            t = l < 1 ? -1 : tedgeInter[pos];
            block = l - 1;
        } else {
            t = l >= nY ? -1 : tedgeIntra[pos - interEntries];
            block = l;
        }
        col[idx] = t < 0 ? nan : in[(block * eBlock + t) * cols + c];
    }
}

// ---------------------------------------------------------------------------
// SO(3) frame alignment (higherOrderDeformationEnergy.cpp:16-53, :95-134).
// The reference takes R = U diag(1,1,det(UV^T)) V^T from the SVD of X^T Y.
// The same rotation is the maximiser of tr(R^T M), M = X^T Y, which Horn's
// closed-form method (J. Opt. Soc. Am. A 4(4), 1987) gives directly as the
// eigenvector of the largest eigenvalue of a symmetric 4x4 matrix built from
// S = M^T; the eigenvector is found with cyclic Jacobi rotations.
// ---------------------------------------------------------------------------
__device__ void normalize3(double v[3]) {
    const double sq = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    if (sq > 0.0) {
        const double r = sqrt(sq);
        v[0] /= r; v[1] /= r; v[2] /= r;
    }
}

__device__ double4 frame_quaternion(const double v2[3], const double n2[3], const double v3[3],
                                    const double n3[3]) {
    double X[3][3], Y[3][3];
    // rows [n, e, e x n], each normalised
    double c2[3] = {v2[1] * n2[2] - v2[2] * n2[1], v2[2] * n2[0] - v2[0] * n2[2], v2[0] * n2[1] - v2[1] * n2[0]};
    double c3[3] = {v3[1] * n3[2] - v3[2] * n3[1], v3[2] * n3[0] - v3[0] * n3[2], v3[0] * n3[1] - v3[1] * n3[0]};
    for (int k = 0; k < 3; ++k) {
        X[0][k] = n2[k]; X[1][k] = v2[k]; X[2][k] = c2[k];
        Y[0][k] = n3[k]; Y[1][k] = v3[k]; Y[2][k] = c3[k];
    }
    for (int r = 0; r < 3; ++r) { normalize3(X[r]); normalize3(Y[r]); }
    double S[3][3];  // S = M^T with M = X^T Y, i.e. S[a][b] = sum_r Y[r][a] X[r][b]
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) S[i][j] = Y[0][i] * X[0][j] + Y[1][i] * X[1][j] + Y[2][i] * X[2][j];
    const double Sxx = S[0][0], Sxy = S[0][1], Sxz = S[0][2];
    const double Syx = S[1][0], Syy = S[1][1], Syz = S[1][2];
    const double Szx = S[2][0], Szy = S[2][1], Szz = S[2][2];
    double A[4][4] = {{Sxx + Syy + Szz, Syz - Szy, Szx - Sxz, Sxy - Syx},
                      {Syz - Szy, Sxx - Syy - Szz, Sxy + Syx, Szx + Sxz},
                      {Szx - Sxz, Sxy + Syx, -Sxx + Syy - Szz, Syz + Szy},
                      {Sxy - Syx, Szx + Sxz, Syz + Szy, -Sxx - Syy + Szz}};
    double V[4][4] = {{1, 0, 0, 0}, {0, 1, 0, 0}, {0, 0, 1, 0}, {0, 0, 0, 1}};
    // every loop below is unrolled, so A and V stay in registers (a run-time
    // index would place them in local memory)
    for (int sweep = 0; sweep < 50; ++sweep) {
        double off = 0.0, diag = 0.0;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            diag += A[i][i] * A[i][i];
#pragma unroll
            for (int j = i + 1; j < 4; ++j) off += A[i][j] * A[i][j];
        }
        if (off <= 1e-32 * (diag + 1e-300)) break;
#pragma unroll
        for (int pp = 0; pp < 3; ++pp)
#pragma unroll
            for (int q = pp + 1; q < 4; ++q) {
                const double apq = A[pp][q];
                if (fabs(apq) < 1e-300) continue;
                const double theta = (A[q][q] - A[pp][pp]) / (2.0 * apq);
                const double tt = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(tt * tt + 1.0), s = tt * c;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const double akp = A[k][pp], akq = A[k][q];
                    A[k][pp] = c * akp - s * akq;
                    A[k][q] = s * akp + c * akq;
                }
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const double apk = A[pp][k], aqk = A[q][k];
                    A[pp][k] = c * apk - s * aqk;
                    A[q][k] = s * apk + c * aqk;
                }
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const double vkp = V[k][pp], vkq = V[k][q];
                    V[k][pp] = c * vkp - s * vkq;
                    V[k][q] = s * vkp + c * vkq;
                }
            }
    }
    // the column of the largest eigenvalue (first index among equals)
    double q[4] = {V[0][0], V[1][0], V[2][0], V[3][0]};
    double bestVal = A[0][0];
#pragma unroll
    for (int i = 1; i < 4; ++i) {
        const bool take = A[i][i] > bestVal;
        bestVal = take ? A[i][i] : bestVal;
#pragma unroll
        for (int k = 0; k < 4; ++k) q[k] = take ? V[k][i] : q[k];
    }
    const double nq = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    return make_double4(q[0] / nq, q[1] / nq, q[2] / nq, q[3] / nq);
}


// The frame of conjugate node j in layer i depends only on a Y edge and the
// X edge j mod |EX| (higherOrderDeformationEnergy.cpp:95-134): the Y edge is
// i, or i - 1 for the degenerate-2d nodes |EX| <= j < 2|EX| of an unpruned
// graph.  The reference stores 3|EX| frames per layer; every one of them is
// a copy of frame (Y edge, X edge) of the |EX| x nY distinct ones, which is
// all that is computed here (quat_index maps a node to its frame).
__global__ void quaternion_kernel(QuatArgs a) {
    const long long total = (long long)a.nY * a.nEX;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i2 = (int)(idx / a.nEX), e3 = (int)(idx % a.nEX);
        double v2[3], n2[3], v3[3], n3[3];
        const int ya = a.EY[2 * i2], yb = a.EY[2 * i2 + 1];
        const int xa = a.EX[2 * e3], xb = a.EX[2 * e3 + 1];
        for (int k = 0; k < 3; ++k) {
            v2[k] = a.VY[3 * yb + k] - a.VY[3 * ya + k];
            n2[k] = a.NY[3 * ya + k];
            v3[k] = a.VX[3 * xb + k] - a.VX[3 * xa + k];
            n3[k] = (a.NX[3 * xa + k] + a.NX[3 * xb + k]) / 2;
        }
        a.out[idx] = frame_quaternion(v2, n2, v3, n3);
    }
}

__device__ __forceinline__ double so3_distance(const double4 a, const double4 b) {
    double ip = fabs(a.x * b.x + (a.y * b.y + a.z * b.z + a.w * b.w));
    if (ip > 1) ip = 1;
    if (isnan(ip)) return 0;
    return 2 * acos(ip);
}

__device__ __forceinline__ double robust_loss(const EnergyArgs& a, double x) {
    const double t = pow(x / a.rlC, a.rlPwr);
    const double am2 = fabs(a.rlAlpha - 2);
    return am2 / a.rlAlpha * (pow(t / am2 + 1, 0.5 * a.rlAlpha) - 1);
}

__device__ __forceinline__ double4 ldg_quat(const double4* q) {
    const double2 lo = __ldg(reinterpret_cast<const double2*>(q));
    const double2 hi = __ldg(reinterpret_cast<const double2*>(q) + 1);
    return make_double4(lo.x, lo.y, hi.x, hi.y);
}

// Frame of conjugate node j of layer i (see quaternion_kernel).
__device__ __forceinline__ long long quat_index(const EnergyArgs& a, int i, int j) {
    const int e3 = j % a.quatEX;
    const int i2 = (j >= a.quatEX && j < 2 * a.quatEX && !a.quatPrune) ? (i + a.nY - 1) % a.nY : i;
    return (long long)i2 * a.quatEX + e3;
}

// Work item: one block of template positions x a chunk of layers.  A thread
// keeps its position -- template edge, Y pattern, X columns, frame indices,
// the X half of the line integral -- and walks the chunk's layers, so per
// layer it reads only the layer's Y edge and the fd entry; the stores of a
// warp stay 32 consecutive entries of one layer.  Every value is computed
// with the same operations in the same order as per entry.
constexpr int kHoLayerChunk = 16;

__global__ void ho_energy_kernel(EnergyArgs a) {
    extern __shared__ unsigned int topSh[];  // [2][kTopBins] when a.hist0
    DigitRun r0, r1;
    top_digit_begin(a, topSh);
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    const double twoPi = 2 * 3.14159265358979323846;
    const bool needLi = (a.costMode == LENGTH || a.timeMode == LENGTH);
    // Without quaternions every SO(3) distance is 0: its robust loss is the
    // same number for every edge, computed once per thread by the same code.
    const double rl0 = robust_loss(a, 0.0);
    const int stride = (int)a.layerStride, inter = (int)a.interEntries, layers = a.nY + 1;
    const int posBlocks = (stride + (int)blockDim.x - 1) / (int)blockDim.x;
    const int chunks = (layers + kHoLayerChunk - 1) / kHoLayerChunk;
    const long long items = (long long)posBlocks * chunks;
    for (long long it = blockIdx.x; it < items; it += gridDim.x) {
        const int lc = (int)(it / posBlocks);
        const int pos = (int)(it - (long long)lc * posBlocks) * (int)blockDim.x + (int)threadIdx.x;
        if (pos >= stride) continue;
        const int l0 = lc * kHoLayerChunk, l1 = min(l0 + kHoLayerChunk, layers);
        const bool isInter = pos < inter;
        const int t = isInter ? __ldg(a.tedgeInter + pos) : __ldg(a.tedgeIntra + (pos - inter));
        if (t < 0) {
            for (int l = l0; l < l1; ++l) {
                const long long idx = (long long)l * stride + pos;
                a.out0[idx] = nan;
                if (a.out1) a.out1[idx] = nan;
            }
            continue;
        }
        const int pat = __ldg(a.eY + t);
        const int x0 = __ldg(a.eX + 3 * t), x1 = __ldg(a.eX + 3 * t + 1), x2 = __ldg(a.eX + 3 * t + 2);
        double dxx[3] = {0.0, 0.0, 0.0};
        if (needLi) {
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const double dx = __ldg(a.VX + 3 * x0 + j) - __ldg(a.VX + 3 * x1 + j);
                dxx[j] = dx * dx;
            }
        }
        int eSrc = 0, eTrgt = 0, eNext = 0;
        if (a.quat) {
            eSrc = __ldg(a.eSrc + t);
            eTrgt = __ldg(a.eTrgt + t);
            eNext = __ldg(a.eNext + t);
        }
        const double* fdRow = a.FD + (long long)x2 * a.nvy;
        for (int l = l0; l < l1; ++l) {
            const long long idx = (long long)l * stride + pos;
            if (isInter ? l < 1 : l >= a.nY) {  // no edge in this layer's slot
                a.out0[idx] = nan;
                if (a.out1) a.out1[idx] = nan;
                continue;
            }
            const int b = isInter ? l - 1 : l;
            const int s2 = __ldg(a.EY + 2 * b), m2 = __ldg(a.EY + 2 * b + 1);
            const int t2 = __ldg(a.EY + 2 * ((b + 1) % a.nY) + 1);
            int y0, y1, y2;
            switch (pat) {
                case 2: y0 = s2; y1 = s2; y2 = s2; break;
                case 3: y0 = s2; y1 = s2; y2 = m2; break;
                case 4: y0 = s2; y1 = m2; y2 = t2; break;
                default: y0 = s2; y1 = m2; y2 = m2; break;
            }
            double so3 = 0.0;
            if (a.quat) {
                const long long q0 = quat_index(a, b, eSrc);
                const long long q1 = quat_index(a, (b + eNext) % a.nY, eTrgt);
                so3 = so3_distance(ldg_quat(a.quat + q0), ldg_quat(a.quat + q1));
            }
            const double rl = a.quat ? robust_loss(a, so3) : rl0;
            const double fd = __ldg(fdRow + y2);
            double li = 0.0;
            if (needLi) {  // line_integral's sum, in its order
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    const double dy = __ldg(a.VY + 3 * y0 + j) - __ldg(a.VY + 3 * y1 + j);
                    li = li + dy * dy;
                    li = li + dxx[j];
                }
                li = sqrt(li);
            }
            const bool degenerate = (y2 == y1 || x2 == x1);
            const int cm = a.costMode, tm = a.timeMode;
            double c0 = 0, c1 = 0;
            if (cm == VANILLA && tm == VANILLA) {
                c0 = rl + fd;
            } else if (cm == VANILLA && tm == LENGTH) {
                c0 = rl + fd;
                c1 = li;
            } else if (cm == LENGTH && tm == VANILLA) {
                c0 = li;
            } else if (cm == VANILLA && tm == PENALISE_DEGENERATE) {
                c0 = rl + fd;
                c1 = degenerate ? 0.1 : 1;
            } else if (cm == PENALISE_DEGENERATE && tm == VANILLA) {
                c0 = degenerate ? 0.1 : 1;
            } else if (cm == FEATURE && tm == SO3_PLAIN) {
                c0 = fd;
                c1 = fmax(0.0, twoPi - so3);
            } else if (cm == FEATURE && tm == SO3_ROBUST) {
                c0 = fd;
                c1 = fmax(0.0, a.maxSO3 - rl);
            } else if (cm == SO3_ROBUST && tm == FEATURE) {
                c0 = rl;
                c1 = fmax(0.0, a.maxFd - fd);
            } else {  // SO3_PLAIN, FEATURE
                c0 = so3;
                c1 = fmax(0.0, a.maxFd - fd);
            }
            a.out0[idx] = c0;
            if (a.out1) a.out1[idx] = c1;
            if (a.hist0) {
                count_top_digit(topSh, r0, c0);
                if (a.hist1) count_top_digit(topSh + kTopBins, r1, c1);
            }
        }
    }
    top_digit_end(a, topSh, r0, r1);
}

// ---------------------------------------------------------------------------
// Median by radix selection over the valid entries of one column, decided on
// the device: the selection's state (MedianState) lives in device memory, so
// the host enqueues the whole chain -- digit passes, compaction of the last
// bucket, the in-bucket selection, the rescale -- and waits once.  Keys are
// the order-preserving 64-bit images of the doubles; digits from the most
// significant one: 12 bits (counted by the energy kernel while it wrote the
// column), 14, then 12 at a time, until the bucket holding the wanted rank
// has at most kMedianCompact members (or every bit is fixed).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double key_to_double(unsigned long long key) {
    const unsigned long long u = (key >> 63) ? (key & 0x7fffffffffffffffULL) : ~key;
    return __longlong_as_double((long long)u);
}

// Width of the digit counted after `shift` bits remain below the prefix.
__device__ __forceinline__ int median_digit_bits(int shift) {
    const int b = shift == 64 ? kTopDigitBits : shift == 64 - kTopDigitBits ? kMedianWideBits : kTopDigitBits;
    return b < shift ? b : shift;
}

__device__ __forceinline__ MedianState median_start(long long count) {
    MedianState m{};
    m.even = count % 2 == 0;
    m.rank = m.even ? (count - 2) / 2 : count / 2;
    m.bucket = count;
    m.shift = 64;
    m.bits = median_digit_bits(64);
    m.minAbove = ~0ull;
    return m;
}

__global__ void median_init_kernel(MedianState* st, long long count) { *st = median_start(count); }

// Histogram of the next digit of the keys that match the state's prefix.
// A grid of one wave (occupancy-sized) keeps the final flush of the block
// histograms short.  Nothing to do once the selection is done.
__global__ void median_hist_kernel(SelectArgs a, const MedianState* st) {
    extern __shared__ unsigned int sh[];
    __shared__ MedianState m;
    if (threadIdx.x == 0) m = *st;
    __syncthreads();
    if (m.done || m.bits < 1 || m.bits > kMedianWideBits || m.bits > m.shift) return;
    const int nb = 1 << m.bits;
    const int shift = m.shift - m.bits;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    // Each thread counts a run of equal digits in a register and adds the run
    // to the shared histogram when the digit changes: the most significant
    // digits of one column fall into a few bins, where per-entry atomics (or
    // warp matching) would serialise.
    unsigned runBin = 0xffffffffu, runCnt = 0;
    const unsigned long long prefix = m.prefix, mask = m.mask;
    for_stream_values<4>(a.col, a.layerStride, a.interEntries, a.nY, a.tedgeInter, a.tedgeIntra,
                         [&](long long, double x, bool valid, bool) {
                             if (!valid) return;
                             const unsigned long long k = order_key(x);
                             if ((k & mask) != prefix) return;
                             const unsigned bin = (unsigned)((k >> shift) & (unsigned long long)(nb - 1));
                             if (bin == runBin) {
                                 ++runCnt;
                             } else {
                                 if (runCnt) atomicAdd(&sh[runBin], runCnt);
                                 runBin = bin;
                                 runCnt = 1;
                             }
                         });
    if (runCnt) atomicAdd(&sh[runBin], runCnt);
    __syncthreads();
    for (int i = threadIdx.x; i < nb; i += blockDim.x)
        if (sh[i]) atomicAdd(a.hist + i, (unsigned long long)sh[i]);
}

// Block-wide search of a histogram of nb bins (1024 threads): the digit whose
// cumulative count first exceeds `rank`, and the count below it.  Returns
// false when the counts do not reach past the rank.
__device__ bool find_digit(const unsigned long long* hist, int nb, long long rank, int* digit, long long* below) {
    __shared__ long long part[1024];
    __shared__ int sDigit;
    __shared__ long long sBelow;
    const int per = (nb + 1023) / 1024;
    const int b0 = threadIdx.x * per, b1 = min(b0 + per, nb);
    long long mine = 0;
    for (int i = b0; i < b1; ++i) mine += (long long)hist[i];
    part[threadIdx.x] = mine;
    if (threadIdx.x == 0) sDigit = -1;
    __syncthreads();
    // inclusive scan of the parts (Hillis-Steele over 1024 entries)
    for (int o = 1; o < 1024; o <<= 1) {
        const long long x = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
        __syncthreads();
        part[threadIdx.x] += x;
        __syncthreads();
    }
    const long long before = threadIdx.x ? part[threadIdx.x - 1] : 0;
    if (before <= rank && rank < part[threadIdx.x]) {
        long long acc = before;
        for (int i = b0; i < b1; ++i) {
            const long long c = (long long)hist[i];
            if (acc + c > rank) {
                sDigit = i;
                sBelow = acc;
                break;
            }
            acc += c;
        }
    }
    __syncthreads();
    *digit = sDigit;
    *below = sBelow;
    return sDigit >= 0;
}

// The digit holding the wanted rank from the last pass's histogram: the
// prefix grows by it, the rank becomes the rank inside its bucket.  The
// histogram is cleared for the next pass.  One block of 1024 threads.
// init >= 0: the state starts here, for a column of `init` values (the first
// digit's histogram was counted before, by the energy kernel).
__global__ void median_scan_kernel(unsigned long long* hist, MedianState* st, long long init) {
    __shared__ MedianState m;
    if (threadIdx.x == 0) m = init >= 0 ? median_start(init) : *st;
    __syncthreads();
    if (m.done) return;
    if (m.bits < 1 || m.bits > kMedianWideBits || m.bits > m.shift) {
        if (threadIdx.x == 0) {
            st->err = 4;
            st->done = 1;
        }
        return;
    }
    const int nb = 1 << m.bits;
    int digit;
    long long below;
    const bool ok = find_digit(hist, nb, m.rank, &digit, &below);
    if (threadIdx.x == 0) {
        if (!ok) {
            m.err = 1;
            m.done = 1;
        } else {
            m.shift -= m.bits;
            m.rank -= below;
            m.bucket = (long long)hist[digit];
            m.prefix |= (unsigned long long)digit << m.shift;
            m.mask |= ((1ull << m.bits) - 1) << m.shift;
            if (m.shift == 0 || m.bucket <= kMedianCompact) m.done = 1;
            else m.bits = median_digit_bits(m.shift);
        }
        *st = m;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nb; i += blockDim.x) hist[i] = 0;
}

// Copies the last bucket's values (keys matching the prefix) to out[0..cap);
// nothing when every bit is fixed (the bucket's values are all equal).
// A selection that is not done after the passes enqueued (a column of few
// distinct values) is flagged (err 5) for the host, which runs the chain
// again with every pass.
__global__ void median_compact_kernel(SelectArgs a, MedianState* st, double* out, unsigned long long* count,
                                      long long cap) {
    __shared__ MedianState m;
    if (threadIdx.x == 0) m = *st;
    __syncthreads();
    if (!m.done && !m.err) {
        if (blockIdx.x == 0 && threadIdx.x == 0) st->err = 5;
        return;
    }
    if (m.shift == 0 || m.err) return;
    const unsigned long long prefix = m.prefix, mask = m.mask;
    for_stream_values<4>(a.col, a.layerStride, a.interEntries, a.nY, a.tedgeInter, a.tedgeIntra,
                         [&](long long, double x, bool valid, bool) {
                           if (!valid || (order_key(x) & mask) != prefix) return;
                           const unsigned long long at = atomicAdd(count, 1ull);
                           if ((long long)at < cap) out[at] = x;
                       });
}

// The order statistics inside the last bucket (one block of 1024 threads):
// xk of the rank, and for an even count the next one, either inside the
// bucket or -- when the rank is the bucket's largest -- the smallest key
// above it over the whole column (median_min_above_kernel, flagged here).
// Radix selection over the bucket's remaining bits, 11 at a time.
__global__ void median_select_kernel(MedianState* st, const double* band, const unsigned long long* count) {
    __shared__ MedianState m;
    __shared__ unsigned long long hist[1 << 11];
    __shared__ unsigned long long sMin;
    __shared__ long long sLess, sEq;
    if (threadIdx.x == 0) m = *st;
    __syncthreads();
    if (m.err) return;
    unsigned long long key;
    unsigned long long top;  // largest key the bucket can hold
    if (m.shift == 0) {
        key = m.prefix;  // every member equals it
        top = m.prefix;
    } else {
        const long long n = (long long)*count;
        if (n != m.bucket || n > kMedianCompact) {
            if (threadIdx.x == 0) {
                st->err = 2;
            }
            return;
        }
        unsigned long long prefix = m.prefix, mask = m.mask;
        long long rank = m.rank;
        int shift = m.shift;
        while (shift > 0) {
            const int b = shift < 11 ? shift : 11;
            shift -= b;
            const int nb = 1 << b;
            for (int i = threadIdx.x; i < nb; i += blockDim.x) hist[i] = 0;
            __syncthreads();
            // eight loads in flight per thread: one block reads the whole bucket
            for (long long i0 = threadIdx.x; i0 < n; i0 += 8LL * blockDim.x) {
                double x[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const long long i = i0 + (long long)u * blockDim.x;
                    x[u] = i < n ? __ldcg(band + i) : 0.0;
                }
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    if (i0 + (long long)u * blockDim.x >= n) break;
                    const unsigned long long k = order_key(x[u]);
                    if ((k & mask) == prefix) atomicAdd(&hist[(k >> shift) & (unsigned long long)(nb - 1)], 1ull);
                }
            }
            __syncthreads();
            int digit;
            long long below;
            if (!find_digit(hist, nb, rank, &digit, &below)) {
                if (threadIdx.x == 0) st->err = 3;
                return;
            }
            rank -= below;
            prefix |= (unsigned long long)digit << shift;
            mask |= ((unsigned long long)nb - 1) << shift;
            __syncthreads();
        }
        key = prefix;
        top = m.prefix | ~m.mask;
    }
    const double xk = key_to_double(key);
    double xk1 = 0;
    int needAbove = 0;
    if (m.even) {
        if (m.rank + 1 >= m.bucket) {
            needAbove = 1;  // the next key lies above the bucket
        } else if (m.shift == 0) {
            xk1 = xk;
        } else {
            // keys below and equal to xk's inside the bucket; the next order
            // statistic is xk again, or the smallest key above it
            if (threadIdx.x == 0) {
                sLess = 0;
                sEq = 0;
                sMin = ~0ull;
            }
            __syncthreads();
            const long long n = (long long)*count;
            long long less = 0, eq = 0;
            unsigned long long mn = ~0ull;
            for (long long i0 = threadIdx.x; i0 < n; i0 += 8LL * blockDim.x) {
                double x[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const long long i = i0 + (long long)u * blockDim.x;
                    x[u] = i < n ? __ldcg(band + i) : 0.0;
                }
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    if (i0 + (long long)u * blockDim.x >= n) break;
                    const unsigned long long k = order_key(x[u]);
                    if (k < key) ++less;
                    else if (k == key) ++eq;
                    else if (k < mn) mn = k;
                }
            }
            atomicAdd((unsigned long long*)&sLess, (unsigned long long)less);
            atomicAdd((unsigned long long*)&sEq, (unsigned long long)eq);
            atomicMin(&sMin, mn);
            __syncthreads();
            xk1 = m.rank + 1 < sLess + sEq ? xk : key_to_double(sMin);
        }
    }
    if (threadIdx.x == 0) {
        st->xk = xk;
        st->xk1 = xk1;
        st->needAbove = needAbove;
        st->bucketTop = top;
    }
}

// Smallest key strictly above the bucket over the whole column, when the
// selection flagged it.
__global__ void median_min_above_kernel(SelectArgs a, MedianState* st) {
    __shared__ MedianState m;
    if (threadIdx.x == 0) m = *st;
    __syncthreads();
    if (!m.needAbove || m.err) return;
    const unsigned long long above = m.bucketTop;
    unsigned long long best = ~0ull;
    for_stream_values<4>(a.col, a.layerStride, a.interEntries, a.nY, a.tedgeInter, a.tedgeIntra,
                         [&](long long, double x, bool valid, bool) {
                           if (!valid) return;
                           const unsigned long long k = order_key(x);
                           if (k > above && k < best) best = k;
                       });
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long x = __shfl_xor_sync(0xffffffffu, best, o);
        best = x < best ? x : best;
    }
    if ((threadIdx.x & 31) == 0 && best != ~0ull) atomicMin(&st->minAbove, best);
}

// median = xk (odd count) or (xk + xk1) / 2; factor = scaling / (2
// max(median, 0.001)), the host driver's double operations
// (cost_time_ratio_solver.cpp:709-721, utils.hpp:196-209).
__device__ __forceinline__ double median_factor(const MedianState& m, double scaling, double* median) {
    const double xk1 = m.needAbove ? key_to_double(m.minAbove) : m.xk1;
    *median = m.even ? __ddiv_rn(__dadd_rn(m.xk, xk1), 2.0) : m.xk;
    const double med = *median < 0.001 ? 0.001 : *median;
    return __ddiv_rn(scaling, __dmul_rn(2.0, med));
}

// x <- min(round(factor * x), clip) on the valid entries, factor from the
// selection's state: the float copy always, the double column in place only
// when writeF64 (the host first runs without it and keeps the float copy as
// the rescaled column when every value is exact); sets st->inexact when a
// value is not a float.
// The factor comes from the selection (the first pass, writeF64 == 0, also
// stores it and the median in the state) or, for the second pass, from the
// state; nothing is written when the selection failed.
__global__ void rescale_kernel(double* col, float* col32, long long layerStride, long long interEntries, int nY,
                               const int* tedgeInter, const int* tedgeIntra, MedianState* st, double scaling,
                               double clip, int writeF64) {
    __shared__ double sFactor;
    __shared__ int sErr;
    if (threadIdx.x == 0) {
        const MedianState m = *st;
        sErr = m.err;
        if (!m.err) {
            double median;
            sFactor = writeF64 ? m.factor : median_factor(m, scaling, &median);
            if (!writeF64 && blockIdx.x == 0) {
                st->median = median;
                st->factor = sFactor;
            }
        }
    }
    __syncthreads();
    if (sErr) return;
    const double factor = sFactor;
    int* inexact = &st->inexact;
    for_stream_values<4>(col, layerStride, interEntries, nY, tedgeInter, tedgeIntra,
                         [&](long long idx, double v, bool valid, bool inRange) {
                           if (!inRange) return;
                           if (!valid) {
                               if (col32) col32[idx] = __int_as_float(0x7fc00000);
                               return;
                           }
                           double x = round(__dmul_rn(factor, v));
                           if (x > clip) x = clip;
                           if (writeF64) col[idx] = x;
                           const float f = (float)x;
                           if (col32) col32[idx] = f;
                           if ((double)f != x) *inexact = 1;
                       });
}
// The double column from its exact float copy, on the valid entries.
__global__ void to_f64_kernel(const float* col32, double* col, long long layerStride, long long interEntries, int nY,
                              const int* tedgeInter, const int* tedgeIntra) {
    for_stream_layers(layerStride, interEntries, nY, tedgeInter, tedgeIntra,
                      [&](long long idx, int, long long, int t, bool inRange) {
                          if (inRange && t >= 0) col[idx] = (double)col32[idx];
                      });
}

__global__ void to_f32_kernel(const double* col, float* col32, long long total, long long layerStride,
                              long long interEntries, int nY, const int* tedgeInter, const int* tedgeIntra,
                              int* exact) {
    (void)total;
    for_stream_values<4>(col, layerStride, interEntries, nY, tedgeInter, tedgeIntra,
                         [&](long long idx, double x, bool valid, bool inRange) {
                           if (!inRange) return;
                           if (!valid) {
                               col32[idx] = __int_as_float(0x7fc00000);
                               return;
                           }
                           const float f = (float)x;
                           col32[idx] = f;
                           if ((double)f != x) *exact = 0;
                       });
}

__global__ void export_kernel(const double* col, double* out, int cols, int c, long long total,
                              long long layerStride, long long interEntries, int nY, long long eBlock,
                              const int* tedgeInter, const int* tedgeIntra) {
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long l = idx / layerStride;
        const long long pos = idx - l * layerStride;
        long long block;
        int t;
        if (pos < interEntries) {
            if (l < 1) continue;
            t = tedgeInter[pos];
            block = l - 1;
        } else {
            if (l >= nY) continue;
            t = tedgeIntra[pos - interEntries];
            block = l;
        }
        if (t < 0) continue;
        out[(block * eBlock + t) * cols + c] = col[idx];
    }
}

// Mean incoming cost of every node of layer 1, accumulated in float in
// in-edge order (cost_time_ratio_solver.cpp:656-675).
// CT: the fp64 column or its exact fp32 copy (the same values).
template <class CT>
__global__ void layer1_mean_kernel(const CT* cost, long long layerStride, long long interEntries, int n,
                                   int nslices, const int* spInter, const int* spIntra, const int* srcInter,
                                   const int* srcIntra, float* meanOut, int* countOut) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const int s = v >> 5, lane = v & 31;
    const CT* c1 = cost + layerStride;  // layer 1
    float mean = 0;
    int num = 0;
    for (int j = spInter[s]; j < spInter[s + 1]; ++j) {
        const long long e = (long long)j * 32 + lane;
        if (srcInter[e] < 0) continue;
        mean = (float)((double)mean + (double)c1[e]);
        ++num;
    }
    for (int j = spIntra[s]; j < spIntra[s + 1]; ++j) {
        const long long e = (long long)j * 32 + lane;
        if (srcIntra[e] < 0) continue;
        mean = (float)((double)mean + (double)c1[interEntries + e]);
        ++num;
    }
    meanOut[v] = mean / (float)num;
    countOut[v] = num;
    (void)nslices;
}

// ---------------------------------------------------------------------------
// Vertex normals on the device (utils::normals3d / normals2d,
// helper/utils.cpp:86-157).  Every value is computed with the operations, in
// the order, of the reference's host loops (this file is compiled without
// fused multiply-adds), so the results are the same bit for bit.
// ---------------------------------------------------------------------------

// 3D, step 1: every face's edge cross product (its unit normal times twice
// its area, libigl's area weighting) and each vertex's corner count.
__global__ void face_normals_kernel(const double* V, long long nv, const int* F, long long nf, double* fn, int* deg,
                                    int* bad) {
    for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < nf; f += (long long)gridDim.x * blockDim.x) {
        const int a = F[3 * f], b = F[3 * f + 1], c = F[3 * f + 2];
        if (a < 0 || b < 0 || c < 0 || a >= nv || b >= nv || c >= nv) {
            atomicExch(bad, 1);
            continue;
        }
        double u[3], w[3];
        for (int k = 0; k < 3; ++k) {
            u[k] = V[3 * b + k] - V[3 * a + k];
            w[k] = V[3 * c + k] - V[3 * a + k];
        }
        fn[3 * f] = u[1] * w[2] - u[2] * w[1];
        fn[3 * f + 1] = u[2] * w[0] - u[0] * w[2];
        fn[3 * f + 2] = u[0] * w[1] - u[1] * w[0];
        atomicAdd(deg + a, 1);
        atomicAdd(deg + b, 1);
        atomicAdd(deg + c, 1);
    }
}

// Exclusive prefix sum of n counts into off[0..n] by one CTA, tile by tile.
__global__ void exclusive_scan_kernel(const int* in, long long n, int* off) {
    __shared__ int warpSum[32];
    __shared__ int carry;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (long long base = 0; base < n; base += blockDim.x) {
        const long long i = base + threadIdx.x;
        const int x = i < n ? in[i] : 0;
        int incl = x;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) warpSum[w] = incl;
        __syncthreads();
        if (w == 0) {
            int ws = lane < nw ? warpSum[lane] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, ws, o);
                if (lane >= o) ws += y;
            }
            if (lane < nw) warpSum[lane] = ws;  // inclusive over warps
        }
        __syncthreads();
        const int before = (w > 0 ? warpSum[w - 1] : 0) + incl - x;
        if (i < n) off[i] = carry + before;
        __syncthreads();
        if (threadIdx.x == 0) carry += warpSum[nw - 1];
        __syncthreads();
    }
    if (threadIdx.x == 0) off[n] = carry;
}

// 3D, step 2: each vertex's incident faces (a face with a repeated vertex
// is listed once per corner, as the reference adds it once per corner).
// Faces with an index outside V were flagged by step 1 and are skipped, as
// they were not counted.
__global__ void face_lists_kernel(const int* F, long long nv, long long nf, const int* off, int* cursor, int* list) {
    for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < nf; f += (long long)gridDim.x * blockDim.x) {
        const int a = F[3 * f], b = F[3 * f + 1], c = F[3 * f + 2];
        if (a < 0 || b < 0 || c < 0 || a >= nv || b >= nv || c >= nv) continue;
        for (int k = 0; k < 3; ++k) {
            const int v = F[3 * f + k];
            list[off[v] + atomicAdd(cursor + v, 1)] = (int)f;
        }
    }
}

// 3D, step 3: per vertex, its faces in ascending order (the reference's
// accumulation order), their normals summed from 0, then unit length.
__global__ void vertex_normals_kernel(const double* fn, long long nv, const int* off, int* list, double* out) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nv; v += (long long)gridDim.x * blockDim.x) {
        const int lo = off[v], hi = off[v + 1];
        for (int j = lo + 1; j < hi; ++j) {  // insertion sort: vertex degrees are small
            const int f = list[j];
            int q = j - 1;
            while (q >= lo && list[q] > f) {
                list[q + 1] = list[q];
                --q;
            }
            list[q + 1] = f;
        }
        double x = 0.0, y = 0.0, z = 0.0;
        for (int j = lo; j < hi; ++j) {
            const long long f = list[j];
            x = x + fn[3 * f];
            y = y + fn[3 * f + 1];
            z = z + fn[3 * f + 2];
        }
        const double len = sqrt(x * x + y * y + z * z);
        if (len > 0) {
            x = x / len;
            y = y / len;
            z = z / len;
        }
        out[3 * v] = x;
        out[3 * v + 1] = y;
        out[3 * v + 2] = z;
    }
}

// 2D: the whole curve by one CTA.  `V` is scratch for the curve moved into
// the xy-plane, `en` and `el` for the edge normals and lengths.  *bad: 1 no
// coordinate plane, 2 an edge index outside V.
__global__ void curve_normals_kernel(const double* Vin, int nv, const int* E, double* V, double* en, double* el,
                                     double* out, int* bad) {
    __shared__ double sums[3];
    __shared__ int sZero, sBad;
    __shared__ double red[4][32];
    __shared__ double sMm;
    __shared__ float sMult, sMaxX;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (threadIdx.x < 3) {  // the column sums in row order, as the reference adds them
        double s = 0;
        for (int r = 0; r < nv; ++r) s += Vin[3 * r + threadIdx.x];
        sums[threadIdx.x] = s;
    }
    if (threadIdx.x == 0) sBad = 0;
    __syncthreads();
    if (threadIdx.x == 0) {
        int zero = -1;
        for (int i = 0; i < 3; ++i)
            if (fabs(sums[i]) < 1e-4) {
                zero = i;
                break;
            }
        sZero = zero;
        if (zero == -1) *bad = 1;
    }
    __syncthreads();
    const int zero = sZero;
    if (zero == -1) return;
    const int order[3] = {zero == 2 ? 0 : zero == 1 ? 0 : 1, zero == 2 ? 1 : 2, zero == 2 ? 2 : zero == 1 ? 1 : 0};
    for (int r = threadIdx.x; r < nv; r += blockDim.x)
        for (int k = 0; k < 3; ++k) V[3 * r + k] = Vin[3 * r + order[k]];
    __syncthreads();
    for (int i = threadIdx.x; i < nv; i += blockDim.x) {
        const int a = E[2 * i], b = E[2 * i + 1];
        if (a < 0 || b < 0 || a >= nv || b >= nv) {
            sBad = 2;
            continue;
        }
        const double ev0 = V[3 * a] - V[3 * b], ev1 = V[3 * a + 1] - V[3 * b + 1], ev2 = V[3 * a + 2] - V[3 * b + 2];
        el[i] = sqrt(ev0 * ev0 + ev1 * ev1 + ev2 * ev2);
        const double n0 = ev1, n1 = -ev0, n2 = ev2;  // rotation about z
        const double len = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
        en[3 * i] = len > 0 ? n0 / len : n0;
        en[3 * i + 1] = len > 0 ? n1 / len : n1;
        en[3 * i + 2] = len > 0 ? n2 / len : n2;
    }
    __syncthreads();
    if (sBad) {
        if (threadIdx.x == 0) *bad = sBad;
        return;
    }
    // extremes of x and y (exact in any order)
    double mx = -INFINITY, mn = INFINITY, my = -INFINITY, mny = INFINITY;
    for (int r = threadIdx.x; r < nv; r += blockDim.x) {
        mx = fmax(mx, V[3 * r]);
        mn = fmin(mn, V[3 * r]);
        my = fmax(my, V[3 * r + 1]);
        mny = fmin(mny, V[3 * r + 1]);
    }
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        my = fmax(my, __shfl_xor_sync(0xffffffffu, my, o));
        mny = fmin(mny, __shfl_xor_sync(0xffffffffu, mny, o));
    }
    if (lane == 0) {
        red[0][w] = mx;
        red[1][w] = mn;
        red[2][w] = my;
        red[3][w] = mny;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int q = 1; q < nw; ++q) {
            mx = fmax(mx, red[0][q]);
            mn = fmin(mn, red[1][q]);
            my = fmax(my, red[2][q]);
            mny = fmin(mny, red[3][q]);
        }
        const float maxX = (float)mx, minX = (float)mn, maxY = (float)my, minY = (float)mny;
        sMaxX = maxX;
        sMult = (float)(0.1 * (double)fminf(fabsf(maxX - minX), fabsf(maxY - minY)));
    }
    __syncthreads();
    // does the offset curve reach past maxX?  (utils.cpp:120-133, with the
    // reference's pairing of vertex r with edge r's normal)
    double mm = -INFINITY;
    const double mult = (double)sMult;
    for (int r = threadIdx.x; r < nv; r += blockDim.x) mm = fmax(mm, V[3 * r] + mult * en[3 * r]);
    for (int o = 16; o > 0; o >>= 1) mm = fmax(mm, __shfl_xor_sync(0xffffffffu, mm, o));
    if (lane == 0) red[0][w] = mm;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int q = 1; q < nw; ++q) mm = fmax(mm, red[0][q]);
        sMm = mm;
    }
    __syncthreads();
    // flipping every edge normal negates every sum below exactly
    const double sign = (float)sMm < sMaxX ? -1.0 : 1.0;
    for (int j = threadIdx.x; j < nv; j += blockDim.x) {
        const int ip = j == 0 ? nv - 1 : j - 1;
        double v[3];
        for (int k = 0; k < 3; ++k) v[k] = el[ip] * (sign * en[3 * ip + k]) + el[j] * (sign * en[3 * j + k]);
        const double len = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        for (int k = 0; k < 3; ++k) out[3 * j + k] = len > 0 ? v[k] / len : v[k];
    }
}

cudaError_t launch_normals_3d(const double* V, long long nv, const int* F, long long nf, double* fn, int* deg,
                              int* off, int* cursor, int* list, double* out, int* bad, cudaStream_t s) {
    const int threads = 256;
    const int fb = (int)std::min<long long>(std::max<long long>(1, (nf + threads - 1) / threads), 4096);
    const int vb = (int)std::min<long long>(std::max<long long>(1, (nv + threads - 1) / threads), 4096);
    note_launch();
    face_normals_kernel<<<fb, threads, 0, s>>>(V, nv, F, nf, fn, deg, bad);
    note_launch();
    exclusive_scan_kernel<<<1, 1024, 0, s>>>(deg, nv, off);
    note_launch();
    face_lists_kernel<<<fb, threads, 0, s>>>(F, nv, nf, off, cursor, list);
    note_launch();
    vertex_normals_kernel<<<vb, threads, 0, s>>>(fn, nv, off, list, out);
    return cudaGetLastError();
}

cudaError_t launch_normals_2d(const double* Vin, int nv, const int* E, double* V, double* en, double* el, double* out,
                              int* bad, cudaStream_t s) {
    note_launch();
    curve_normals_kernel<<<1, 256, 0, s>>>(Vin, nv, E, V, en, el, out, bad);
    return cudaGetLastError();
}

// Host wrappers -------------------------------------------------------------
// Persistent grid of a stream pass: as many CTAs as can be resident at once
// (one full wave; a partial second wave would double the pass).
// The grid is cached per (kernel, device, block, shared memory): the
// occupancy query is not free and every pass of every solve asks it.
// PGC_STREAM_GRID (measurement) caps it, so that the passes of many small
// graphs on concurrent streams can share the device.
static int stream_grid_cap() {
    static const int cap = [] {
        const char* v = std::getenv("PGC_STREAM_GRID");
        return v ? std::max(0, std::atoi(v)) : 0;
    }();
    return cap;
}
template <class K>
static int stream_grid_full(K kernel, int threads, size_t smem) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return 148;
    }
    static std::mutex mu;
    static std::map<std::tuple<const void*, int, int, size_t>, int> cache;
    const auto key = std::make_tuple((const void*)kernel, dev, threads, smem);
    {
        std::lock_guard<std::mutex> lk(mu);
        const auto it = cache.find(key);
        if (it != cache.end()) return it->second;
    }
    int grid = 148, per = 0;
    DeviceInfo info{};
    if (device_info(dev, &info) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem) != cudaSuccess || per < 1) {
        cudaGetLastError();
        return grid;
    }
    grid = info.sms * per;
    std::lock_guard<std::mutex> lk(mu);
    cache[key] = grid;
    return grid;
}

// `work` (>= 0 when many graphs' passes run side by side on concurrent
// streams): the stream entries the pass visits; a small column then gets
// one CTA per 128 entries a thread, fewer than a full wave, so that the
// passes share the device.  A lone graph's passes take a full wave.
template <class K>
static int stream_grid(K kernel, int threads, size_t smem, long long work = -1) {
    int g = stream_grid_full(kernel, threads, smem);
    if (work >= 0) {
        const long long want = std::max(1LL, work / ((long long)threads * 128));
        if (want < g) g = (int)want;
    }
    const int cap = stream_grid_cap();
    return cap > 0 && cap < g ? cap : g;
}

static int grid_for(long long total, int threads) {
    long long b = (total + threads - 1) / threads;
    if (b > 148LL * 32) b = 148LL * 32;
    if (b < 1) b = 1;
    return (int)b;
}

cudaError_t launch_plain_energy(const EnergyArgs& a, cudaStream_t s, bool shared) {
    const size_t smem = a.hist0 ? 2 * kTopBins * sizeof(unsigned) : 0;
    note_launch();
    plain_energy_kernel<<<stream_grid(plain_energy_kernel, 256, smem, shared ? a.total : -1), 256, smem, s>>>(a);
    return cudaGetLastError();
}
cudaError_t launch_ho_energy(const EnergyArgs& a, cudaStream_t s) {
    const size_t smem = a.hist0 ? 2 * kTopBins * sizeof(unsigned) : 0;
    note_launch();
    ho_energy_kernel<<<stream_grid(ho_energy_kernel, 256, smem), 256, smem, s>>>(a);
    return cudaGetLastError();
}
cudaError_t launch_quaternions(const QuatArgs& a, cudaStream_t s) {
    note_launch();
    quaternion_kernel<<<grid_for((long long)a.nY * a.nEX, 128), 128, 0, s>>>(a);
    return cudaGetLastError();
}
// The whole median-and-rescale chain of one column on stream s; the state
// holds the median, the factor and the error code when the stream reaches
// them.  `topHist`: the energy kernel's first-digit histogram of the column,
// or null (the first digit is counted here).  hist: 1 << kMedianWideBits
// zeroed counters; band: kMedianCompact doubles; count: one zeroed counter.
cudaError_t launch_median_rescale(const SelectArgs& a, unsigned long long* topHist, MedianState* st,
                                  unsigned long long* hist, double* band, unsigned long long* count, long long nValues,
                                  double scaling, float* col32, double clip, bool allPasses, bool shared,
                                  cudaStream_t s) {
    const size_t smem = sizeof(unsigned) << kMedianWideBits;
    {
        static std::mutex mu;
        static std::set<int> done;
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        std::lock_guard<std::mutex> lk(mu);
        if (!done.count(dev)) {
            // the 14-bit digit's shared histogram is above the default 48 KB
            e = cudaFuncSetAttribute(median_hist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            done.insert(dev);
        }
    }
    const int histGrid = stream_grid(median_hist_kernel, 512, smem, shared ? a.total : -1);
    const int grid = stream_grid(median_compact_kernel, 256, 0, shared ? a.total : -1);
    SelectArgs h = a;
    h.hist = hist;
    if (topHist) {
        note_launch();
        median_scan_kernel<<<1, 1024, 0, s>>>(topHist, st, nValues);
    } else {
        note_launch();
        median_init_kernel<<<1, 1, 0, s>>>(st, nValues);
        note_launch();
        median_hist_kernel<<<histGrid, 512, smem, s>>>(h, st);
        note_launch();
        median_scan_kernel<<<1, 1024, 0, s>>>(hist, st, -1);
    }
    // One more digit (14 bits) leaves a bucket of at most kMedianCompact
    // values on every column but those of few distinct values; for those the
    // compaction flags the state and the host runs the chain with all
    // passes: at most five more digits fix all 64 bits (12 + 14 + 12 + 12 +
    // 12 + 2), and the passes after the selection is done return at once.
    for (int pass = 0; pass < (allPasses ? 5 : 1); ++pass) {
        note_launch();
        median_hist_kernel<<<histGrid, 512, smem, s>>>(h, st);
        note_launch();
        median_scan_kernel<<<1, 1024, 0, s>>>(hist, st, -1);
    }
    note_launch();
    median_compact_kernel<<<grid, 256, 0, s>>>(a, st, band, count, kMedianCompact);
    note_launch();
    median_select_kernel<<<1, 1024, 0, s>>>(st, band, count);
    note_launch();
    median_min_above_kernel<<<grid, 256, 0, s>>>(a, st);
    note_launch();
    rescale_kernel<<<grid, 256, 0, s>>>(const_cast<double*>(a.col), col32, a.layerStride, a.interEntries, a.nY,
                                        a.tedgeInter, a.tedgeIntra, st, scaling, clip, 0);
    return cudaGetLastError();
}

// The double column rescaled in place with the factor of the state (when its
// float copy is not exact).
cudaError_t launch_rescale_f64(const SelectArgs& a, MedianState* st, double clip, cudaStream_t s) {
    note_launch();
    rescale_kernel<<<stream_grid(rescale_kernel, 256, 0), 256, 0, s>>>(const_cast<double*>(a.col), nullptr,
                                                                        a.layerStride, a.interEntries, a.nY,
                                                                        a.tedgeInter, a.tedgeIntra, st, 0.0, clip, 1);
    return cudaGetLastError();
}
cudaError_t launch_to_f64(const float* col32, double* col, long long layerStride, long long interEntries, int nY,
                          const int* ti, const int* tr, cudaStream_t s) {
    note_launch();
    to_f64_kernel<<<stream_grid(to_f64_kernel, 256, 0), 256, 0, s>>>(col32, col, layerStride, interEntries, nY, ti, tr);
    return cudaGetLastError();
}
cudaError_t launch_to_f32(const double* col, float* col32, long long total, long long layerStride,
                          long long interEntries, int nY, const int* ti, const int* tr, int* exact, cudaStream_t s) {
    note_launch();
    to_f32_kernel<<<stream_grid(to_f32_kernel, 256, 0), 256, 0, s>>>(col, col32, total, layerStride, interEntries, nY, ti, tr,
                                                       exact);
    return cudaGetLastError();
}
cudaError_t launch_export(const double* col, double* out, int cols, int c, long long total, long long layerStride,
                          long long interEntries, int nY, long long eBlock, const int* ti, const int* tr,
                          cudaStream_t s) {
    note_launch();
    export_kernel<<<grid_for(total, 256), 256, 0, s>>>(col, out, cols, c, total, layerStride, interEntries, nY,
                                                       eBlock, ti, tr);
    return cudaGetLastError();
}
// Fixed device scratch of the no-allocation cost export.  Some callers
// cannot let this library allocate device memory: a process whose HBM is
// already reserved by its own allocator (a PyTorch job's caching allocator, a
// serving engine that pre-reserves most of the GPU) would see cudaMalloc fail
// or force that allocator to give memory back, and cudaFree synchronizes the
// whole device, stalling the caller's other streams.  For them the export
// writes into this file-scope array instead: 2^21 doubles (16 MiB) that every
// GPU loading the library holds until the process exits.
static __device__ __align__(256) double g_noallocExport[kNoAllocExportValues];

// In host code g_noallocExport names a host-side stand-in, not device memory,
// so kernels are given the device address, taken here once per device with
// that device current (the caller sets it) and cached.  The first call on a
// device therefore does this set-up; it should come before any stream capture.
cudaError_t noalloc_export_scratch(int device, double** ptr) {
    static std::mutex mu;
    static std::map<int, double*> addr;
    std::lock_guard<std::mutex> lock(mu);
    const auto it = addr.find(device);
    if (it != addr.end()) {
        *ptr = it->second;
        return cudaSuccess;
    }
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noallocExport);
    if (e != cudaSuccess) return e;
    *ptr = static_cast<double*>(p);
    addr[device] = *ptr;
    return cudaSuccess;
}

cudaError_t launch_plain_energy_backward(const EnergyArgs& a, const long long* edges, int count, long long eBlock,
                                        double coef, double* grad, cudaStream_t s) {
    if (count <= 0) return cudaSuccess;
    note_launch();
    plain_energy_backward_kernel<<<(count + 127) / 128, 128, 0, s>>>(a, edges, count, eBlock, coef, grad);
    return cudaGetLastError();
}
cudaError_t launch_conj_energy_backward(const EnergyArgs& a, const long long* edges, int count, long long eBlock,
                                       double coef, double coefT, long long argmax, double* grad, cudaStream_t s) {
    if (count <= 0) return cudaSuccess;
    note_launch();
    conj_energy_backward_kernel<<<(count + 127) / 128, 128, 0, s>>>(a, edges, count, eBlock, coef, coefT, argmax,
                                                                      grad);
    return cudaGetLastError();
}
cudaError_t launch_import(const double* in, double* col, int cols, int c, long long total, long long layerStride,
                          long long interEntries, int nY, long long eBlock, const int* ti, const int* tr,
                          cudaStream_t s) {
    note_launch();
    import_kernel<<<grid_for(total, 256), 256, 0, s>>>(in, col, cols, c, total, layerStride, interEntries, nY, eBlock,
                                                       ti, tr);
    return cudaGetLastError();
}
cudaError_t launch_layer1_mean(const double* cost, long long layerStride, long long interEntries, int n, int nslices,
                               const int* spI, const int* spA, const int* srcI, const int* srcA, float* meanOut,
                               int* countOut, cudaStream_t s) {
    note_launch();
    layer1_mean_kernel<double><<<(n + 255) / 256, 256, 0, s>>>(cost, layerStride, interEntries, n, nslices, spI, spA,
                                                               srcI, srcA, meanOut, countOut);
    return cudaGetLastError();
}
cudaError_t launch_layer1_mean(const float* cost, long long layerStride, long long interEntries, int n, int nslices,
                               const int* spI, const int* spA, const int* srcI, const int* srcA, float* meanOut,
                               int* countOut, cudaStream_t s) {
    note_launch();
    layer1_mean_kernel<float><<<(n + 255) / 256, 256, 0, s>>>(cost, layerStride, interEntries, n, nslices, spI, spA,
                                                              srcI, srcA, meanOut, countOut);
    return cudaGetLastError();
}

}  // namespace pgc
