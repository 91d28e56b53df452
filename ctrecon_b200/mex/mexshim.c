/*
 * mexshim.c -- implementation of the minimal MEX API declared in mex.h.
 *
 * Arrays are column-major with up to 8 dimensions; structs are m x n arrays of
 * numbered fields. mxCalloc/mxMalloc memory is plain heap memory (MATLAB frees it
 * when the MEX call returns; here the callers free it themselves, as the Katsevich
 * MEX sources do). mexErrMsgTxt long-jumps back into mexshim_call().
 */
#include "mex.h"

#include <setjmp.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define MEXSHIM_MAXDIM 8

struct mxArray_tag {
    mxClassID cls;
    mwSize ndim;
    mwSize dims[MEXSHIM_MAXDIM];
    void* data;
    int owns_data;
    int nfields;
    char** field_names;
    mxArray** fields; /* numel * nfields, row (element) major */
};

static __thread jmp_buf* g_jmp = NULL;
static __thread char g_errmsg[1024];
static int g_print = 1;

static size_t elem_size(mxClassID c) {
    switch (c) {
    case mxDOUBLE_CLASS: case mxINT64_CLASS: case mxUINT64_CLASS: return 8;
    case mxSINGLE_CLASS: case mxINT32_CLASS: case mxUINT32_CLASS: return 4;
    case mxINT16_CLASS: case mxUINT16_CLASS: case mxCHAR_CLASS: return 2;
    case mxINT8_CLASS: case mxUINT8_CLASS: case mxLOGICAL_CLASS: return 1;
    default: return 0;
    }
}

static mwSize numel_of(const mxArray* a) {
    mwSize n = 1;
    for (mwSize i = 0; i < a->ndim; ++i) n *= a->dims[i];
    return n;
}

static mxArray* new_header(mwSize ndim, const mwSize* dims, mxClassID cls) {
    mxArray* a = (mxArray*)calloc(1, sizeof(mxArray));
    if (!a) return NULL;
    if (ndim < 2) ndim = 2;
    if (ndim > MEXSHIM_MAXDIM) ndim = MEXSHIM_MAXDIM;
    a->cls = cls;
    a->ndim = ndim;
    for (mwSize i = 0; i < ndim; ++i) a->dims[i] = dims ? dims[i] : 1;
    /* MATLAB drops trailing singleton dimensions beyond the second */
    while (a->ndim > 2 && a->dims[a->ndim - 1] == 1) a->ndim--;
    return a;
}

mxArray* mxCreateNumericArray(mwSize ndim, const mwSize* dims, mxClassID classid,
                              mxComplexity flag) {
    (void)flag;
    mxArray* a = new_header(ndim, dims, classid);
    if (!a) return NULL;
    size_t bytes = (size_t)numel_of(a) * elem_size(classid);
    a->data = calloc(bytes ? bytes : 1, 1);
    a->owns_data = 1;
    return a;
}

mxArray* mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID classid, mxComplexity flag) {
    mwSize d[2] = {m, n};
    return mxCreateNumericArray(2, d, classid, flag);
}

mxArray* mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity flag) {
    return mxCreateNumericMatrix(m, n, mxDOUBLE_CLASS, flag);
}

mxArray* mxCreateDoubleScalar(double value) {
    mxArray* a = mxCreateDoubleMatrix(1, 1, mxREAL);
    if (a) ((double*)a->data)[0] = value;
    return a;
}

mxArray* mxCreateStructMatrix(mwSize m, mwSize n, int nfields, const char** fieldnames) {
    mwSize d[2] = {m, n};
    mxArray* a = new_header(2, d, mxSTRUCT_CLASS);
    if (!a) return NULL;
    a->nfields = nfields;
    a->field_names = (char**)calloc((size_t)(nfields > 0 ? nfields : 1), sizeof(char*));
    for (int i = 0; i < nfields; ++i) a->field_names[i] = strdup(fieldnames[i]);
    a->fields = (mxArray**)calloc((size_t)(numel_of(a) * (nfields > 0 ? nfields : 1)),
                                  sizeof(mxArray*));
    return a;
}

mxArray* mexshim_wrap_numeric(mwSize ndim, const mwSize* dims, mxClassID classid,
                              void* data) {
    mxArray* a = new_header(ndim, dims, classid);
    if (!a) return NULL;
    a->data = data;
    a->owns_data = 0;
    return a;
}

void mxDestroyArray(mxArray* a) {
    if (!a) return;
    if (a->cls == mxSTRUCT_CLASS) {
        mwSize n = numel_of(a) * (mwSize)a->nfields;
        for (mwSize i = 0; i < n; ++i) mxDestroyArray(a->fields[i]);
        for (int i = 0; i < a->nfields; ++i) free(a->field_names[i]);
        free(a->fields);
        free(a->field_names);
    }
    if (a->owns_data) free(a->data);
    free(a);
}

mxClassID mxGetClassID(const mxArray* a) { return a ? a->cls : mxUNKNOWN_CLASS; }
int mxIsDouble(const mxArray* a) { return a && a->cls == mxDOUBLE_CLASS; }
int mxIsSingle(const mxArray* a) { return a && a->cls == mxSINGLE_CLASS; }
int mxIsStruct(const mxArray* a) { return a && a->cls == mxSTRUCT_CLASS; }
mwSize mxGetNumberOfElements(const mxArray* a) { return a ? numel_of(a) : 0; }
mwSize mxGetNumberOfDimensions(const mxArray* a) { return a ? a->ndim : 0; }
const mwSize* mxGetDimensions(const mxArray* a) { return a ? a->dims : NULL; }
size_t mxGetM(const mxArray* a) { return a ? a->dims[0] : 0; }
size_t mxGetN(const mxArray* a) {
    if (!a) return 0;
    size_t n = 1;
    for (mwSize i = 1; i < a->ndim; ++i) n *= a->dims[i];
    return n;
}
double* mxGetPr(const mxArray* a) { return a ? (double*)a->data : NULL; }
void* mxGetData(const mxArray* a) { return a ? a->data : NULL; }

double mxGetScalar(const mxArray* a) {
    if (!a || !a->data || numel_of(a) == 0) return 0.0;
    switch (a->cls) {
    case mxDOUBLE_CLASS: return ((const double*)a->data)[0];
    case mxSINGLE_CLASS: return (double)((const float*)a->data)[0];
    case mxINT32_CLASS: return (double)((const int*)a->data)[0];
    case mxLOGICAL_CLASS: case mxUINT8_CLASS: return (double)((const unsigned char*)a->data)[0];
    default: return 0.0;
    }
}

int mxGetNumberOfFields(const mxArray* a) {
    return (a && a->cls == mxSTRUCT_CLASS) ? a->nfields : 0;
}

const char* mxGetFieldNameByNumber(const mxArray* a, int n) {
    if (!a || a->cls != mxSTRUCT_CLASS || n < 0 || n >= a->nfields) return NULL;
    return a->field_names[n];
}

mxArray* mxGetFieldByNumber(const mxArray* a, mwIndex index, int fieldnumber) {
    if (!a || a->cls != mxSTRUCT_CLASS) return NULL;
    if (fieldnumber < 0 || fieldnumber >= a->nfields || index >= numel_of(a)) return NULL;
    return a->fields[index * (mwSize)a->nfields + (mwSize)fieldnumber];
}

mxArray* mxGetField(const mxArray* a, mwIndex index, const char* fieldname) {
    if (!a || a->cls != mxSTRUCT_CLASS) return NULL;
    for (int i = 0; i < a->nfields; ++i)
        if (strcmp(a->field_names[i], fieldname) == 0)
            return mxGetFieldByNumber(a, index, i);
    return NULL;
}

void mxSetFieldByNumber(mxArray* a, mwIndex index, int fieldnumber, mxArray* value) {
    if (!a || a->cls != mxSTRUCT_CLASS) return;
    if (fieldnumber < 0 || fieldnumber >= a->nfields || index >= numel_of(a)) return;
    a->fields[index * (mwSize)a->nfields + (mwSize)fieldnumber] = value;
}

void* mxCalloc(mwSize n, mwSize size) { return calloc(n ? n : 1, size ? size : 1); }
void* mxMalloc(mwSize n) { return malloc(n ? n : 1); }
void mxFree(void* ptr) { free(ptr); }

void mexshim_set_print(int enabled) { g_print = enabled; }

int mexPrintf(const char* fmt, ...) {
    if (!g_print) return 0;
    va_list ap;
    va_start(ap, fmt);
    int r = vprintf(fmt, ap);
    va_end(ap);
    fflush(stdout);
    return r;
}

#if defined(__GNUC__)
__attribute__((noreturn))
#endif
static void raise_error(const char* msg) {
    snprintf(g_errmsg, sizeof g_errmsg, "%s", msg ? msg : "");
    if (g_jmp) longjmp(*g_jmp, 1);
    /* no harness frame: behave like an uncaught MATLAB error in a batch session */
    fprintf(stderr, "mexErrMsgTxt outside mexshim_call: %s\n", g_errmsg);
    abort();
}

void mexErrMsgTxt(const char* msg) { raise_error(msg); }

void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...) {
    (void)id;
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    raise_error(buf);
}

void mexWarnMsgTxt(const char* msg) {
    if (g_print) fprintf(stderr, "Warning: %s\n", msg);
}

int mexshim_call(mexshim_entry fn, int nlhs, mxArray* plhs[], int nrhs,
                 const mxArray* prhs[], char* errbuf, size_t errlen) {
    jmp_buf here;
    jmp_buf* saved = g_jmp;
    g_jmp = &here;
    if (setjmp(here) == 0) {
        fn(nlhs, plhs, nrhs, prhs);
        g_jmp = saved;
        if (errbuf && errlen) errbuf[0] = '\0';
        return 0;
    }
    g_jmp = saved;
    if (errbuf && errlen) snprintf(errbuf, errlen, "%s", g_errmsg);
    return 1;
}
