/*
 * Compile-check stand-in for MATLAB's mex.h (declarations only, no
 * implementation).  It lets the gateways be syntax-checked where MATLAB and
 * Octave are not installed; real builds use the mex.h of MATLAB or Octave.
 */
#ifndef UA_STUB_MEX_H
#define UA_STUB_MEX_H
#include <stddef.h>
typedef struct mxArray_tag mxArray;
typedef size_t mwIndex;
typedef size_t mwSize;
typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;
void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...);
int mexAtExit(void (*fn)(void));
void mexLock(void);
mxArray* mxGetField(const mxArray* s, mwIndex i, const char* name);
void mxSetField(mxArray* s, mwIndex i, const char* name, mxArray* v);
int mxIsStruct(const mxArray* a);
int mxIsDouble(const mxArray* a);
int mxIsEmpty(const mxArray* a);
int mxIsChar(const mxArray* a);
char* mxArrayToString(const mxArray* a);
double mxGetScalar(const mxArray* a);
double* mxGetPr(const mxArray* a);
size_t mxGetM(const mxArray* a);
size_t mxGetN(const mxArray* a);
size_t mxGetNumberOfElements(const mxArray* a);
mwIndex* mxGetJc(const mxArray* a);
mwIndex* mxGetIr(const mxArray* a);
mxArray* mxCreateSparse(mwSize m, mwSize n, mwSize nzmax, mxComplexity c);
mxArray* mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity c);
mxArray* mxCreateDoubleScalar(double v);
mxArray* mxCreateStructMatrix(mwSize m, mwSize n, int nfields, const char** names);
mxArray* mxCreateString(const char* s);
void mxDestroyArray(mxArray* a);
int mxIsSparse(const mxArray* a);
void* mxMalloc(size_t n);
void* mxCalloc(size_t n, size_t size);
void mxFree(void* p);
#endif
