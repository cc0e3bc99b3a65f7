/*
 * Minimal stand-in for MATLAB's mex.h, written for the oracle so that the
 * unmodified ucodes/omc_matrad/omc_matrad.c compiles and runs as the D_ij
 * reference (test infrastructure only).  Implements exactly the mx and mex
 * calls that file makes, on a small in-memory mxArray: double, int32, char,
 * struct, cell and sparse arrays.  mexErrMsgIdAndTxt longjmps back to the
 * harness (MATLAB unwinds the same way); mexCallMATLAB implements "num2str"
 * and ignores the waitbar calls.
 */
#ifndef OMC_MEX_SHIM_H
#define OMC_MEX_SHIM_H
/* MATLAB's mex.h includes the C library headers before user code; the
   ucode relies on that when it redefines exit() right after the include. */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef size_t mwSize;
typedef size_t mwIndex;

typedef struct mxArray_tag mxArray;
struct mxArray_tag {
    int cls;                 /* 0 double, 1 int32, 2 char, 3 struct, 4 cell, 5 sparse */
    mwSize ndim;
    mwSize dims[4];
    double *pr;
    int32_t *i32;
    char *str;
    int nfields;
    const char **fnames;
    mxArray **fvals;
    mxArray **cells;
    mwIndex *ir, *jc;
    mwSize nzmax;
};

#define mxREAL 0

mxArray *mxGetField(const mxArray *a, mwIndex i, const char *name);
double *mxGetPr(const mxArray *a);
double mxGetScalar(const mxArray *a);
char *mxArrayToString(const mxArray *a);
int mxGetString(const mxArray *a, char *buf, mwSize buflen);
size_t mxGetNumberOfElements(const mxArray *a);
const mwSize *mxGetDimensions(const mxArray *a);
mwSize mxGetNumberOfDimensions(const mxArray *a);
mwIndex mxCalcSingleSubscript(const mxArray *a, mwSize nsubs, const mwIndex *subs);
mxArray *mxGetCell(const mxArray *a, mwIndex i);
int mxIsDouble(const mxArray *a);
int mxIsInt32(const mxArray *a);
int mxIsStruct(const mxArray *a);
int mxGetNumberOfFields(const mxArray *a);
mxArray *mxCreateSparse(mwSize m, mwSize n, mwSize nzmax, int flag);
mwIndex *mxGetIr(const mxArray *a);
mwIndex *mxGetJc(const mxArray *a);
void mxSetPr(mxArray *a, double *p);
void mxSetIr(mxArray *a, mwIndex *p);
void mxSetNzmax(mxArray *a, mwSize n);
void *mxRealloc(void *p, size_t n);
void *mxCalloc(size_t n, size_t sz);
void mxFree(void *p);
mxArray *mxCreateDoubleScalar(double v);
mxArray *mxCreateString(const char *s);
void mxDestroyArray(mxArray *a);
int mexPrintf(const char *fmt, ...);
void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...);
int mexCallMATLAB(int nlhs, mxArray *plhs[], int nrhs, mxArray *prhs[], const char *name);

#endif
