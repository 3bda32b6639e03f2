// product_graph_generator_mex.cpp -- the reference's MATLAB entry point
// (mex/product_graph_generator_mex.cpp:29-151) over libpgc's C ABI:
//
//   [passes_layers_once, objective, matching] = product_graph_generator_mex( ...
//       VX, EX, VY, EY, feat_diff, use_conjugate_graph, use_regulariser, solver_id, ...
//       [prune_intralayer, [max_depth, [cost_id, time_id, [NX, NY, [rl_alpha, rl_c, rl_pwr]]]]])
//
// with 8, 9, 10, 12, 14 or 17 inputs.  Index matrices (EX, EY) are 1-based
// doubles as MATLAB passes them; the returned matching is 1-based.  Solver
// ids: 5 lawlercpu, 6 lawlergpu (ratio), 7 dijkstracpu, 8 dijkstragpu
// (minimum cost); any other id prints "solver not supported" and returns
// (0, 0, []), as the reference's dispatch does (-1, "export", included).
//
// Build (MATLAB R2018a or later):
//   mex -R2018a product_graph_generator_mex.cpp -I<repo>/include \
//       -L<repo>/product-graph-cycles_b200/lib -lpgc
#include <mex.h>

#include <cstdint>
#include <string>
#include <vector>

#include "pgc.h"

namespace {

// costTimeIdToName (mex.cpp:8-27), including its quirk: -1 gives "nomode"
// and still prints the error of the else-branch.
const char* cost_time_name(int id) {
    const char* name = "";
    if (id == -1) name = "nomode";
    if (id == 0)
        name = "vanilla";
    else if (id == 1)
        name = "feature";
    else if (id == 2)
        name = "lengthnormalisation";
    else if (id == 3)
        name = "plainso3";
    else if (id == 4)
        name = "robustso3";
    else if (id == 5)
        name = "tbd";
    else
        mexPrintf("[CPG-MEX] error: id not supported\n");
    return name;
}

// A MATLAB matrix (column-major doubles) as a row-major copy for the C ABI.
std::vector<double> row_major(const mxArray* a, int64_t& rows, int64_t& cols) {
    rows = (int64_t)mxGetM(a);
    cols = (int64_t)mxGetN(a);
    const double* p = mxGetPr(a);
    std::vector<double> out((size_t)(rows * cols));
    for (int64_t r = 0; r < rows; ++r)
        for (int64_t c = 0; c < cols; ++c) out[(size_t)(r * cols + c)] = p[c * rows + r];
    return out;
}

// A 1-based MATLAB index matrix as row-major 0-based int32 (the reference
// casts the doubles to int, then subtracts 1).
std::vector<int32_t> row_major_index(const mxArray* a, int64_t& rows, int64_t& cols) {
    const std::vector<double> d = row_major(a, rows, cols);
    std::vector<int32_t> out(d.size());
    for (size_t i = 0; i < d.size(); ++i) out[i] = (int32_t)d[i] - 1;
    return out;
}

double scalar(const mxArray* a) { return *mxGetPr(a); }

struct Handle {
    pgc_graph* g = nullptr;
    ~Handle() { pgc_destroy(g); }
};

void check(int rc) {
    if (rc != PGC_OK) mexErrMsgTxt(pgc_last_error());
}

}  // namespace

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    if (!(nrhs == 8 || nrhs == 9 || nrhs == 10 || nrhs == 12 || nrhs == 14 || nrhs == 17) || nlhs > 3) {
        mexErrMsgTxt(
            "Usage: [passes_layers_once, minimum_mean_mean, minimum_mean_matching] = "
            "product_graph_generator_mex(VX, EX, VY, EY, feat_diff, use_conjugate_graph, use_regulariser, "
            "mean_cycle_algo, prune_intralayer, maxDepth, ctCostName, ctTimeName, NX, NY, rl_alpha, rl_c, rl_gamma)");
        return;
    }
    int64_t rVX, cVX, rEX, cEX, rVY, cVY, rEY, cEY, rFD, cFD;
    const std::vector<double> VX = row_major(prhs[0], rVX, cVX);
    const std::vector<int32_t> EX = row_major_index(prhs[1], rEX, cEX);
    const std::vector<double> VY = row_major(prhs[2], rVY, cVY);
    const std::vector<int32_t> EY = row_major_index(prhs[3], rEY, cEY);
    const std::vector<double> FD = row_major(prhs[4], rFD, cFD);
    const bool conj = (int)scalar(prhs[5]) != 0;
    const bool reg = scalar(prhs[6]) != 0;
    const int solverId = (int)scalar(prhs[7]);
    bool prune = false;
    if (nrhs >= 9) {
        prune = scalar(prhs[8]) != 0;
        mexPrintf("pruneIntralayerEdges %d\n", prune ? 1 : 0);
    }
    if (cVX != 3 || cVY != 3 || cEX != 2 || cEY != 2 || rFD != rVX || cFD != rVY)
        mexErrMsgTxt("product_graph_generator_mex: VX, VY must be [n x 3], EX, EY [m x 2], feat_diff [|VX| x |VY|]");

    Handle h;
    check(pgc_create(VX.data(), rVX, EX.data(), rEX, VY.data(), rVY, EY.data(), rEY, FD.data(), conj ? 1 : 0,
                     reg ? 1 : 0, prune ? 1 : 0, &h.g));
    if (conj) {
        int64_t rNX = 0, cNX = 0, rNY = 0, cNY = 0;
        std::vector<double> NX, NY;
        if (nrhs >= 14) {
            NX = row_major(prhs[12], rNX, cNX);
            NY = row_major(prhs[13], rNY, cNY);
        }
        check(pgc_set_normals(h.g, NX.data(), rNX, cNX, NY.data(), rNY, cNY));
        if (nrhs >= 17) check(pgc_update_robust_loss_params(h.g, scalar(prhs[14]), scalar(prhs[15]), scalar(prhs[16])));
    }
    if (nrhs >= 10) check(pgc_set_max_depth(h.g, (int)scalar(prhs[9])));
    if (nrhs >= 12)
        check(pgc_set_cost_time_ratio_mode(h.g, cost_time_name((int)scalar(prhs[10])),
                                           cost_time_name((int)scalar(prhs[11]))));
    check(pgc_generate(h.g));

    int passes = 0;
    float objective = 0.0f;
    int64_t rows = 0, cols = 0;
    std::vector<int32_t> matching;
    const char* name = solverId == 5 ? "lawlercpu" : solverId == 6 ? "lawlergpu"
                       : solverId == 7 ? "dijkstracpu" : solverId == 8 ? "dijkstragpu"
                       : solverId == -1 ? "export" : "hartmannorlin";
    if (solverId > 4) {
        check(solverId > 6 ? pgc_solve_with_minimum_cost(h.g, name, -1)
                           : pgc_solve_with_cost_time_ratio(h.g, name, -1));
        check(pgc_result(h.g, &passes, &objective, &rows, &cols));
        matching.resize((size_t)(rows * cols));
        check(pgc_result_matching(h.g, matching.data()));
    } else {
        mexPrintf("solver not supported\n");
    }

    plhs[0] = mxCreateDoubleMatrix(1, 1, mxREAL);
    mxGetPr(plhs[0])[0] = passes ? 1.0 : 0.0;
    plhs[1] = mxCreateDoubleMatrix(1, 1, mxREAL);
    mxGetPr(plhs[1])[0] = (double)objective;
    plhs[2] = mxCreateDoubleMatrix((size_t)rows, (size_t)cols, mxREAL);
    double* m = mxGetPr(plhs[2]);
    for (int64_t r = 0; r < rows; ++r)
        for (int64_t c = 0; c < cols; ++c) m[c * rows + r] = (double)matching[(size_t)(r * cols + c)] + 1.0;
}
