/*
 * Host-side MEX stand-in (test infrastructure for the oracle).
 *
 * sgref_call() wraps one mexFunction invocation: inputs are described by
 * plain pointers + class + shape, outputs are copied into caller buffers.
 * The wrapped sources are the reference's unchanged MEX files; nothing here
 * computes anything of the reference's algorithm.
 */
#include "mex.h"

#include <setjmp.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static jmp_buf g_err_jmp;
static char g_err_msg[512];

double *mxGetPr(const mxArray *a) { return (double *)a->data; }
void *mxGetData(const mxArray *a) { return a->data; }
size_t mxGetM(const mxArray *a) { return a->m; }
size_t mxGetN(const mxArray *a) { return a->n; }
bool mxIsInt64(const mxArray *a) { return a->cls == mxINT64_CLASS; }

double mxGetScalar(const mxArray *a)
{
    switch (a->cls) {
    case mxDOUBLE_CLASS: return ((const double *)a->data)[0];
    case mxINT32_CLASS: return (double)((const int32_t *)a->data)[0];
    case mxINT64_CLASS: return (double)((const int64_t *)a->data)[0];
    }
    return 0.0;
}

mxArray *mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity c)
{
    (void)c;
    mxArray *a = (mxArray *)calloc(1, sizeof(mxArray));
    a->cls = mxDOUBLE_CLASS;
    a->m = m;
    a->n = n;
    a->data = calloc(m * n ? m * n : 1, sizeof(double));
    a->owns = 1;
    return a;
}

void mexErrMsgTxt(const char *msg)
{
    snprintf(g_err_msg, sizeof g_err_msg, "%s", msg);
    longjmp(g_err_jmp, 1);
}

void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...)
{
    char body[400];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(body, sizeof body, fmt, ap);
    va_end(ap);
    snprintf(g_err_msg, sizeof g_err_msg, "%s: %s", id, body);
    longjmp(g_err_jmp, 1);
}

const char *sgref_last_error(void) { return g_err_msg; }

/*
 * Call the library's mexFunction.
 *   nrhs inputs: ptrs[i], cls[i] (mxClassID), m[i] x n[i]
 *   nlhs outputs: copied into outs[j] (doubles), capacity out_len[j] elements
 * Returns 0 on success, 1 if the MEX code raised an error, 2 on a size mismatch.
 */
int sgref_call(int nrhs, void *const *ptrs, const int *cls, const int64_t *m, const int64_t *n,
               int nlhs, double **outs, const int64_t *out_len)
{
    mxArray in[16];
    const mxArray *prhs[16];
    mxArray *plhs[8];
    int i, rc = 0;
    if (nrhs > 16 || nlhs > 8) return 2;
    for (i = 0; i < nrhs; i++) {
        in[i].cls = (mxClassID)cls[i];
        in[i].m = (size_t)m[i];
        in[i].n = (size_t)n[i];
        in[i].data = ptrs[i];
        in[i].owns = 0;
        prhs[i] = &in[i];
    }
    for (i = 0; i < 8; i++) plhs[i] = NULL;
    g_err_msg[0] = 0;
    if (setjmp(g_err_jmp) != 0) {
        rc = 1;
        goto cleanup;
    }
    mexFunction(nlhs, plhs, nrhs, prhs);
    for (i = 0; i < nlhs; i++) {
        if (!plhs[i]) continue;
        int64_t len = (int64_t)(plhs[i]->m * plhs[i]->n);
        if (len > out_len[i]) { rc = 2; goto cleanup; }
        memcpy(outs[i], plhs[i]->data, (size_t)len * sizeof(double));
    }
cleanup:
    for (i = 0; i < 8; i++) {
        if (plhs[i]) {
            if (plhs[i]->owns) free(plhs[i]->data);
            free(plhs[i]);
        }
    }
    return rc;
}
