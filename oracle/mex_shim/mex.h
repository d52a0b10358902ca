/*
 * Minimal host-side stand-in for the MATLAB/Octave MEX API.
 *
 * Test infrastructure only: it lets the reference's own MEX sources
 * (+CONSTITUTIVE_PROBLEM/mex/*.c, +ASSEMBLY/mex/*.c) compile unchanged with
 * gcc, so that their outputs can pin the oracle.  Only the handful of mx and mex
 * calls those files use are provided.  Arrays are dense, column-major, real.
 *
 * Errors raised through mexErrMsgTxt / mexErrMsgIdAndTxt unwind (longjmp) to
 * sgref_call(), which returns a non-zero status and keeps the message.
 */
#ifndef SG_MEX_SHIM_H
#define SG_MEX_SHIM_H

#include <stddef.h>
#include <stdint.h>
#include <stdbool.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef size_t mwSize;
typedef enum { mxREAL = 0 } mxComplexity;
typedef enum { mxDOUBLE_CLASS = 6, mxINT32_CLASS = 12, mxINT64_CLASS = 14 } mxClassID;

typedef struct mxArray_tag {
    mxClassID cls;
    size_t m, n;
    void *data;
    int owns;
} mxArray;

double *mxGetPr(const mxArray *a);
void *mxGetData(const mxArray *a);
size_t mxGetM(const mxArray *a);
size_t mxGetN(const mxArray *a);
bool mxIsInt64(const mxArray *a);
double mxGetScalar(const mxArray *a);
mxArray *mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity c);
void mexErrMsgTxt(const char *msg);
void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...);

/* Entry point defined by every MEX source. */
void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]);

#ifdef __cplusplus
}
#endif
#endif
