/* A minimal stand-in for MATLAB's mex.h (the documented C Matrix API names
 * and signatures the gateway uses), with a tiny in-memory implementation in
 * fake_mex.c, so that stokes-nnkifmm_b200/mex/nnk_mex.c compiles and runs on a
 * machine without MATLAB.  Test infrastructure only. */
#ifndef FAKE_MEX_H
#define FAKE_MEX_H
#include <stddef.h>
#include <stdint.h>

typedef size_t mwSize;
typedef size_t mwIndex;
typedef struct mxArray_tag mxArray;
typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;
typedef enum { mxUNKNOWN_CLASS = 0, mxCELL_CLASS, mxCHAR_CLASS, mxDOUBLE_CLASS, mxUINT64_CLASS } mxClassID;

void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...);
int mexAtExit(void (*fn)(void));
mxArray* mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity c);
mxArray* mxCreateDoubleScalar(double v);
mxArray* mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID cls, mxComplexity c);
mxArray* mxCreateSparse(mwSize m, mwSize n, mwSize nzmax, mxComplexity c);
mxArray* mxCreateCellMatrix(mwSize m, mwSize n);
void mxSetCell(mxArray* a, mwIndex i, mxArray* v);
void* mxGetData(const mxArray* a);
double* mxGetPr(const mxArray* a);
mwIndex* mxGetIr(const mxArray* a);
mwIndex* mxGetJc(const mxArray* a);
size_t mxGetM(const mxArray* a);
size_t mxGetN(const mxArray* a);
size_t mxGetNumberOfElements(const mxArray* a);
double mxGetScalar(const mxArray* a);
int mxIsDouble(const mxArray* a);
int mxIsUint64(const mxArray* a);
int mxIsComplex(const mxArray* a);
int mxIsSparse(const mxArray* a);
int mxIsChar(const mxArray* a);
int mxGetString(const mxArray* a, char* buf, mwSize len);
void* mxMalloc(size_t n);
void* mxCalloc(size_t n, size_t size);
void mxFree(void* p);
void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]);
#endif
