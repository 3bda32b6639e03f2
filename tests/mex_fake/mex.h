/* A minimal stand-in for MATLAB's mex.h (the few calls the entry point
 * uses), so that tests can build and run it without MATLAB. */
#pragma once
#include <cstddef>

typedef struct FakeMxArray mxArray;
enum { mxREAL = 0 };

extern "C" {
double* mxGetPr(const mxArray* a);
size_t mxGetM(const mxArray* a);
size_t mxGetN(const mxArray* a);
mxArray* mxCreateDoubleMatrix(size_t m, size_t n, int complexity);
void mexErrMsgTxt(const char* msg);
int mexPrintf(const char* fmt, ...);
}
