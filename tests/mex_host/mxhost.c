/*
 * A small host for MEX gateways outside MATLAB: the mx* and mex* calls the
 * gateways under mex/ use, implemented in plain C so a test can build each
 * gateway into a shared library, hand it MATLAB-shaped arguments (structs of
 * double arrays, 1-based connectivity, char arrays) and read back what it
 * returns (dense and sparse doubles, structs).  Test infrastructure only: a
 * real build links the gateways against MATLAB's or Octave's mex library.
 *
 * Semantics kept from MATLAB's C API where the gateways rely on them:
 *  - double matrices are column-major, mxGetPr gives the data;
 *  - a sparse matrix has jc (n+1), ir and pr (nzmax), mwIndex = size_t;
 *  - mxGetField returns NULL for a missing field, mxSetField takes ownership;
 *  - mexErrMsgIdAndTxt does not return: it unwinds to mxhost_call, which
 *    reports the identifier and message to the caller.
 */
#include <setjmp.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mex.h"

enum { K_DOUBLE = 1, K_SPARSE = 2, K_STRUCT = 3, K_CHAR = 4 };

struct mxArray_tag {
    int kind;
    size_t m, n;
    double* pr;               /* double, sparse values */
    mwIndex *jc, *ir;         /* sparse */
    size_t nzmax;
    int nfields;              /* struct (1 x 1) */
    char** names;
    mxArray** values;
    char* str;                /* char */
};

static jmp_buf g_jmp;
static int g_in_call = 0;
static char g_err_id[256];
static char g_err_msg[1024];
static void (*g_atexit)(void) = NULL;

void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...) {
    va_list ap;
    snprintf(g_err_id, sizeof(g_err_id), "%s", id ? id : "");
    va_start(ap, fmt);
    vsnprintf(g_err_msg, sizeof(g_err_msg), fmt, ap);
    va_end(ap);
    if (g_in_call) longjmp(g_jmp, 1);
    fprintf(stderr, "mexErrMsgIdAndTxt outside a call: %s: %s\n", g_err_id, g_err_msg);
    abort();
}

int mexAtExit(void (*fn)(void)) {
    g_atexit = fn;
    return 0;
}

void mexLock(void) {}

void* mxMalloc(size_t n) { return malloc(n ? n : 1); }
void* mxCalloc(size_t n, size_t size) { return calloc(n ? n : 1, size ? size : 1); }
void mxFree(void* p) { free(p); }

static mxArray* alloc_array(int kind, size_t m, size_t n) {
    mxArray* a = (mxArray*)calloc(1, sizeof(mxArray));
    a->kind = kind;
    a->m = m;
    a->n = n;
    return a;
}

mxArray* mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity c) {
    mxArray* a = alloc_array(K_DOUBLE, m, n);
    (void)c;
    a->pr = (double*)calloc((m * n) > 0 ? m * n : 1, sizeof(double));
    return a;
}

mxArray* mxCreateDoubleScalar(double v) {
    mxArray* a = mxCreateDoubleMatrix(1, 1, mxREAL);
    a->pr[0] = v;
    return a;
}

mxArray* mxCreateSparse(mwSize m, mwSize n, mwSize nzmax, mxComplexity c) {
    mxArray* a = alloc_array(K_SPARSE, m, n);
    (void)c;
    if (nzmax < 1) nzmax = 1;
    a->nzmax = nzmax;
    a->pr = (double*)calloc(nzmax, sizeof(double));
    a->ir = (mwIndex*)calloc(nzmax, sizeof(mwIndex));
    a->jc = (mwIndex*)calloc(n + 1, sizeof(mwIndex));
    return a;
}

mxArray* mxCreateStructMatrix(mwSize m, mwSize n, int nfields, const char** names) {
    int k;
    mxArray* a = alloc_array(K_STRUCT, m, n);
    if (m * n != 1) {
        fprintf(stderr, "mxhost: only 1 x 1 structs\n");
        abort();
    }
    a->nfields = nfields;
    a->names = (char**)calloc(nfields ? nfields : 1, sizeof(char*));
    a->values = (mxArray**)calloc(nfields ? nfields : 1, sizeof(mxArray*));
    for (k = 0; k < nfields; ++k) {
        a->names[k] = (char*)malloc(strlen(names[k]) + 1);
        strcpy(a->names[k], names[k]);
    }
    return a;
}

mxArray* mxCreateString(const char* s) {
    mxArray* a = alloc_array(K_CHAR, 1, strlen(s));
    a->str = (char*)malloc(strlen(s) + 1);
    strcpy(a->str, s);
    return a;
}

void mxDestroyArray(mxArray* a) {
    int k;
    if (!a) return;
    free(a->pr);
    free(a->jc);
    free(a->ir);
    for (k = 0; k < a->nfields; ++k) {
        free(a->names[k]);
        mxDestroyArray(a->values[k]);
    }
    free(a->names);
    free(a->values);
    free(a->str);
    free(a);
}

static int field_index(const mxArray* s, const char* name) {
    int k;
    for (k = 0; k < s->nfields; ++k)
        if (!strcmp(s->names[k], name)) return k;
    return -1;
}

mxArray* mxGetField(const mxArray* s, mwIndex i, const char* name) {
    int k;
    if (!s || s->kind != K_STRUCT || i != 0) return NULL;
    k = field_index(s, name);
    return k < 0 ? NULL : s->values[k];
}

void mxSetField(mxArray* s, mwIndex i, const char* name, mxArray* v) {
    int k;
    if (!s || s->kind != K_STRUCT || i != 0) return;
    k = field_index(s, name);
    if (k < 0) return;
    mxDestroyArray(s->values[k]);
    s->values[k] = v;
}

int mxIsStruct(const mxArray* a) { return a && a->kind == K_STRUCT; }
int mxIsDouble(const mxArray* a) { return a && (a->kind == K_DOUBLE || a->kind == K_SPARSE); }
int mxIsChar(const mxArray* a) { return a && a->kind == K_CHAR; }
int mxIsSparse(const mxArray* a) { return a && a->kind == K_SPARSE; }
int mxIsEmpty(const mxArray* a) { return !a || a->m == 0 || a->n == 0; }
size_t mxGetM(const mxArray* a) { return a ? a->m : 0; }
size_t mxGetN(const mxArray* a) { return a ? a->n : 0; }
size_t mxGetNumberOfElements(const mxArray* a) { return a ? a->m * a->n : 0; }
double* mxGetPr(const mxArray* a) { return a ? a->pr : NULL; }
mwIndex* mxGetJc(const mxArray* a) { return a ? a->jc : NULL; }
mwIndex* mxGetIr(const mxArray* a) { return a ? a->ir : NULL; }
double mxGetScalar(const mxArray* a) { return a && a->pr ? a->pr[0] : 0.0; }

char* mxArrayToString(const mxArray* a) {
    char* s;
    if (!a || a->kind != K_CHAR) return NULL;
    s = (char*)mxMalloc(strlen(a->str) + 1);
    strcpy(s, a->str);
    return s;
}

/* ---- driver side (called from the test through ctypes) ---------------------------- */

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]);

/* Runs the gateway; returns 0, or 1 after mexErrMsgIdAndTxt (see mxhost_error). */
int mxhost_call(int nlhs, mxArray** plhs, int nrhs, const mxArray** prhs) {
    int k;
    for (k = 0; k < nlhs; ++k) plhs[k] = NULL;
    g_err_id[0] = g_err_msg[0] = 0;
    g_in_call = 1;
    if (setjmp(g_jmp)) {
        g_in_call = 0;
        return 1;
    }
    mexFunction(nlhs, plhs, nrhs, prhs);
    g_in_call = 0;
    return 0;
}

const char* mxhost_error_id(void) { return g_err_id; }
const char* mxhost_error_msg(void) { return g_err_msg; }

/* The gateway's mexAtExit function (frees its resident device state). */
void mxhost_unload(void) {
    if (g_atexit) g_atexit();
    g_atexit = NULL;
}

int mxhost_kind(const mxArray* a) { return a ? a->kind : 0; }
int mxhost_nfields(const mxArray* a) { return a ? a->nfields : 0; }
const char* mxhost_field_name(const mxArray* a, int k) { return a && k < a->nfields ? a->names[k] : NULL; }
mxArray* mxhost_field_value(const mxArray* a, int k) { return a && k < a->nfields ? a->values[k] : NULL; }
