/*
 * mex.h — project-written stand-in for MATLAB's MEX/mx C API.
 *
 * TEST INFRASTRUCTURE ONLY. This header and mxshim.c let the reference's own
 * MEX sources (+MCmatlab/src/MCmatlab.c, +MCmatlab/src/finiteElementHeatPropagator.c)
 * and this project's MEX shims compile and run without MATLAB. An mxArray here is
 * either a dense numeric array (column-major, MATLAB layout) or a property bag
 * that stands for a MATLAB struct or object. Only the subset of the mx API that
 * those MEX files call is provided; signatures follow MATLAB's published API.
 */
#ifndef MCB_MXSHIM_MEX_H
#define MCB_MXSHIM_MEX_H

#include <stddef.h>
#include <stdbool.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <limits.h>
#include <float.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef size_t mwSize;
typedef size_t mwIndex;
typedef struct mxArray_tag mxArray;

typedef enum {
  mxUNKNOWN_CLASS = 0,
  mxCELL_CLASS,
  mxSTRUCT_CLASS,
  mxLOGICAL_CLASS,
  mxCHAR_CLASS,
  mxVOID_CLASS,
  mxDOUBLE_CLASS,
  mxSINGLE_CLASS,
  mxINT8_CLASS,
  mxUINT8_CLASS,
  mxINT16_CLASS,
  mxUINT16_CLASS,
  mxINT32_CLASS,
  mxUINT32_CLASS,
  mxINT64_CLASS,
  mxUINT64_CLASS
} mxClassID;

typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;

/* numeric arrays */
mxArray *mxCreateNumericArray(mwSize ndim, const mwSize *dims, mxClassID classid, mxComplexity flag);
mxArray *mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID classid, mxComplexity flag);
mxArray *mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity flag);
mxArray *mxCreateDoubleScalar(double value);
mxArray *mxCreateLogicalScalar(bool value);
void     mxDestroyArray(mxArray *pa);
mxArray *mxDuplicateArray(const mxArray *in);

double  *mxGetPr(const mxArray *pa);
void    *mxGetData(const mxArray *pa);
const mwSize *mxGetDimensions(const mxArray *pa);
mwSize   mxGetNumberOfDimensions(const mxArray *pa);
size_t   mxGetM(const mxArray *pa);
size_t   mxGetN(const mxArray *pa);
size_t   mxGetNumberOfElements(const mxArray *pa);
mxClassID mxGetClassID(const mxArray *pa);
bool     mxIsLogicalScalarTrue(const mxArray *pa);

/* structs and objects (property bags) */
mxArray *mxGetField(const mxArray *pa, mwIndex i, const char *fieldname);
void     mxSetField(mxArray *pa, mwIndex i, const char *fieldname, mxArray *value);
mxArray *mxGetProperty(const mxArray *pa, mwIndex i, const char *propname);
mxArray *mxGetPropertyShared(const mxArray *pa, mwIndex i, const char *propname);
void     mxSetProperty(mxArray *pa, mwIndex i, const char *propname, const mxArray *value);
void     mxSetPropertyShared(mxArray *pa, mwIndex i, const char *propname, const mxArray *value);

/* scalar predicates */
bool mxIsNaN(double x);
bool mxIsInf(double x);
bool mxIsFinite(double x);

/* memory and exit hooks */
void *mxMalloc(size_t n);
void *mxCalloc(size_t n, size_t size);
void  mxFree(void *ptr);
int   mexAtExit(void (*fn)(void));

/* MEX services */
int  mexPrintf(const char *fmt, ...);
int  mexEvalString(const char *cmd);
void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...);
void mexErrMsgTxt(const char *msg);

#ifdef __cplusplus
}
#endif

#endif
