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

namespace pgc {

namespace {

struct EdgeOut {
    int src, trgt;
    int8_t next;
    int x0, x1, x2;
    int8_t y;
};

void emit(LayerTemplate& T, const EdgeOut& e) {
    T.eSrc.push_back(e.src);
    T.eTrgt.push_back(e.trgt);
    T.eNext.push_back(e.next);
    T.eX.push_back(e.x0);
    T.eX.push_back(e.x1);
    T.eX.push_back(e.x2);
    T.eY.push_back(e.y);
}

void build_plain(const int* EX, int64_t nEX, LayerTemplate& T) {
    for (int64_t j = 0; j < nEX; ++j) {
        const int a = EX[2 * j], b = EX[2 * j + 1];
        if (!T.prune) emit(T, {a, b, 0, a, b, 0, Y_SS});
        emit(T, {a, b, 1, a, b, 0, Y_SM});
    }
    for (int x = 0; x < T.nvx; ++x) emit(T, {x, x, 1, x, x, 0, Y_SM});
}

void build_conj(const int* EX, int64_t nEX, LayerTemplate& T) {
    std::vector<std::vector<int>> out((size_t)T.nvx);
    for (int64_t e = 0; e < nEX; ++e) out[(size_t)EX[2 * e]].push_back((int)e);
    const int off2d = (int)nEX;
    const int off3d = T.prune ? off2d : 2 * (int)nEX;
    if (!T.prune) {
        for (int j = 0; j < (int)nEX; ++j) {
            const int s3 = EX[2 * j], m3 = EX[2 * j + 1];
            for (int it : out[(size_t)m3]) {
                const int t3 = EX[2 * it + 1];
                if (t3 == s3) continue;
                emit(T, {off2d + j, off2d + it, 0, s3, m3, t3, Y_SSS});
                emit(T, {off2d + j, it, 0, s3, m3, t3, Y_SSM});
            }
        }
    }
    for (int j = 0; j < (int)nEX; ++j) {
        const int s3 = EX[2 * j], m3 = EX[2 * j + 1];
        for (int it : out[(size_t)m3]) {
            const int t3 = EX[2 * it + 1];
            if (t3 == s3) continue;
            emit(T, {j, it, 1, s3, m3, t3, Y_SMT});
            if (!T.prune) emit(T, {j, off2d + it, 1, s3, m3, t3, Y_SMM});
            emit(T, {off3d + j, it, 1, m3, m3, t3, Y_SMT});
        }
        emit(T, {j, off3d + j, 1, s3, m3, m3, Y_SMT});
        emit(T, {off3d + j, off3d + j, 1, m3, m3, m3, Y_SMT});
    }
}

void build_sell(LayerTemplate& T) {
    T.nslices = (T.n + 31) / 32;
    for (int p = 0; p < 2; ++p) {
        std::vector<std::vector<int>> lists((size_t)T.n);
        for (int64_t t = 0; t < T.eBlock; ++t) {
            const int part = T.eNext[(size_t)t] ? INTER : INTRA;
            if (part != p) continue;
            lists[(size_t)T.eTrgt[(size_t)t]].push_back((int)t);
        }
        std::vector<int>& sp = T.sp[p];
        sp.assign((size_t)T.nslices + 1, 0);
        for (int s = 0; s < T.nslices; ++s) {
            size_t w = 0;
            for (int i = 0; i < 32; ++i) {
                const int v = 32 * s + i;
                if (v < T.n) w = std::max(w, lists[(size_t)v].size());
            }
            sp[(size_t)s + 1] = sp[(size_t)s] + (int)w;
        }
        T.entries[p] = (int64_t)sp.back() * 32;
        T.src[p].assign((size_t)T.entries[p], -1);
        T.tedge[p].assign((size_t)T.entries[p], -1);
        for (int s = 0; s < T.nslices; ++s) {
            for (int i = 0; i < 32; ++i) {
                const int v = 32 * s + i;
                if (v >= T.n) continue;
                const auto& L = lists[(size_t)v];
                for (size_t j = 0; j < L.size(); ++j) {
                    const size_t at = ((size_t)sp[(size_t)s] + j) * 32 + (size_t)i;
                    T.src[p][at] = T.eSrc[(size_t)L[j]];
                    T.tedge[p][at] = L[j];
                    T.ePos[(size_t)L[j]] = (int)at | (p << 30);
                }
            }
        }
    }
    // The closing layer takes the INTER edges of block nY-1 whose global
    // source id is strictly greater than n (cost_time_ratio_solver.cpp:56);
    // with two layers that drops the edges leaving node 0 of layer 1.
    T.srcDummy = T.src[INTER];
    if (T.nY == 2)
        for (auto& s : T.srcDummy)
            if (s == 0) s = -1;
}

}  // namespace

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
    T.ePos.assign((size_t)T.eBlock, -1);
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

}  // namespace pgc
