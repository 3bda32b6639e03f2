// Test double of MATLAB's mex API: column-major double matrices, an error
// call that unwinds to the caller, and printed text kept in a buffer.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "mex.h"

struct FakeMxArray {
    size_t m, n;
    std::vector<double> data;
};

namespace {
std::string g_out, g_err;
struct MexError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
}  // namespace

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]);

extern "C" {
double* mxGetPr(const mxArray* a) { return const_cast<double*>(a->data.data()); }
size_t mxGetM(const mxArray* a) { return a->m; }
size_t mxGetN(const mxArray* a) { return a->n; }
mxArray* mxCreateDoubleMatrix(size_t m, size_t n, int) { return new FakeMxArray{m, n, std::vector<double>(m * n)}; }
void mexErrMsgTxt(const char* msg) { throw MexError(msg); }
int mexPrintf(const char* fmt, ...) {
    char buf[4096];
    va_list ap;
    va_start(ap, fmt);
    const int k = vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_out += buf;
    return k;
}

// helpers for the Python side of the tests
mxArray* fake_mx_new(size_t m, size_t n, const double* colMajor) {
    mxArray* a = mxCreateDoubleMatrix(m, n, mxREAL);
    if (colMajor) std::memcpy(a->data.data(), colMajor, m * n * sizeof(double));
    return a;
}
void fake_mx_free(mxArray* a) { delete a; }
const char* fake_mex_output() { return g_out.c_str(); }
const char* fake_mex_error() { return g_err.c_str(); }
int fake_mex_call(int nlhs, mxArray** plhs, int nrhs, mxArray** prhs) {
    g_out.clear();
    g_err.clear();
    try {
        mexFunction(nlhs, plhs, nrhs, const_cast<const mxArray**>(prhs));
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}
}
