/*
 * mex.h -- minimal stand-in for MATLAB's MEX API, so that MEX sources build and run
 * without MATLAB.
 *
 * It covers the calls made by the Katsevich MEX entry points of CTRecon
 * (KatsevichFiltering_GPU.cu:939-978, KatsevichBkProj.cpp:314-352,
 * KatsevichBkProj_GPU.cu:332-429) and by this project's replacements of them:
 * numeric arrays (double/single, column-major), 1x1 structs with numbered fields,
 * mxGetPr / mxGetFieldByNumber / mxGetClassID, mxCalloc / mxFree, mexPrintf and
 * mexErrMsgTxt.
 *
 * mexErrMsgTxt never returns: it long-jumps back to mexshim_call(), which a harness
 * uses to invoke a mexFunction and which returns the message as an error, the way
 * MATLAB turns mexErrMsgTxt into a MATLAB error.
 *
 * The class-ID values are MATLAB's published enumeration (matrix.h), so a MEX source
 * that compares against mxDOUBLE_CLASS / mxSINGLE_CLASS behaves the same here.
 */
#ifndef CTRECON_MEX_SHIM_H
#define CTRECON_MEX_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef size_t mwSize;
typedef size_t mwIndex;
typedef long long mwSignedIndex;

typedef enum {
    mxUNKNOWN_CLASS = 0,
    mxCELL_CLASS = 1,
    mxSTRUCT_CLASS = 2,
    mxLOGICAL_CLASS = 3,
    mxCHAR_CLASS = 4,
    mxVOID_CLASS = 5,
    mxDOUBLE_CLASS = 6,
    mxSINGLE_CLASS = 7,
    mxINT8_CLASS = 8,
    mxUINT8_CLASS = 9,
    mxINT16_CLASS = 10,
    mxUINT16_CLASS = 11,
    mxINT32_CLASS = 12,
    mxUINT32_CLASS = 13,
    mxINT64_CLASS = 14,
    mxUINT64_CLASS = 15,
    mxFUNCTION_CLASS = 16
} mxClassID;

typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;

typedef struct mxArray_tag mxArray;

/* ---- creation / destruction ---- */
mxArray* mxCreateNumericArray(mwSize ndim, const mwSize* dims, mxClassID classid,
                              mxComplexity flag);
mxArray* mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID classid, mxComplexity flag);
mxArray* mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity flag);
mxArray* mxCreateDoubleScalar(double value);
mxArray* mxCreateStructMatrix(mwSize m, mwSize n, int nfields, const char** fieldnames);
void mxDestroyArray(mxArray* a);

/* ---- queries ---- */
mxClassID mxGetClassID(const mxArray* a);
int mxIsDouble(const mxArray* a);
int mxIsSingle(const mxArray* a);
int mxIsStruct(const mxArray* a);
mwSize mxGetNumberOfElements(const mxArray* a);
mwSize mxGetNumberOfDimensions(const mxArray* a);
const mwSize* mxGetDimensions(const mxArray* a);
size_t mxGetM(const mxArray* a);
size_t mxGetN(const mxArray* a);
double* mxGetPr(const mxArray* a);
void* mxGetData(const mxArray* a);
double mxGetScalar(const mxArray* a);
int mxGetNumberOfFields(const mxArray* a);
const char* mxGetFieldNameByNumber(const mxArray* a, int n);
mxArray* mxGetFieldByNumber(const mxArray* a, mwIndex index, int fieldnumber);
mxArray* mxGetField(const mxArray* a, mwIndex index, const char* fieldname);
void mxSetFieldByNumber(mxArray* a, mwIndex index, int fieldnumber, mxArray* value);

/* ---- memory ---- */
void* mxCalloc(mwSize n, mwSize size);
void* mxMalloc(mwSize n);
void mxFree(void* ptr);

/* ---- messages ---- */
int mexPrintf(const char* fmt, ...);
void mexErrMsgTxt(const char* msg)
#if defined(__GNUC__)
    __attribute__((noreturn))
#endif
    ;
void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...)
#if defined(__GNUC__)
    __attribute__((noreturn))
#endif
    ;
void mexWarnMsgTxt(const char* msg);

/* ---- the MEX entry point every MEX file defines ---- */
void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]);

/* ---- harness side (not part of MATLAB's API) ---- */
typedef void (*mexshim_entry)(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]);

/* Wrap caller-owned column-major numeric data without copying (the array does not
 * own `data`; mxDestroyArray leaves it alone). This is how a harness passes arrays
 * that a MEX function writes in place. */
mxArray* mexshim_wrap_numeric(mwSize ndim, const mwSize* dims, mxClassID classid,
                              void* data);

/* Call a mexFunction. Returns 0 on success; 1 if it raised mexErrMsgTxt, in which
 * case the message is copied into errbuf (NUL-terminated, truncated to errlen). */
int mexshim_call(mexshim_entry fn, int nlhs, mxArray* plhs[], int nrhs,
                 const mxArray* prhs[], char* errbuf, size_t errlen);

/* Route mexPrintf output: 1 = stdout (default), 0 = discard. */
void mexshim_set_print(int enabled);

#ifdef __cplusplus
}
#endif

#endif /* CTRECON_MEX_SHIM_H */
