/*
 * mxshim.c — project-written implementation of the MATLAB mx/MEX subset declared
 * in mex.h.
 *
 * TEST INFRASTRUCTURE ONLY: used to build and drive the reference MEX sources
 * (the oracle under oracle/_ref) and this project's MEX shims without MATLAB.
 * It is never linked into the product library.
 *
 * Semantics follow MATLAB's published mx API where the MEX files depend on them:
 *  - numeric arrays are column-major with at least two dimensions;
 *  - mxGetProperty/mxGetPropertyShared return the stored value (no copy is made;
 *    the reference never frees what they return);
 *  - mxSetProperty copies its argument, mxSetPropertyShared takes ownership;
 *  - mxIsLogicalScalarTrue is true only for a 1x1 logical array holding true;
 *  - mexErrMsgIdAndTxt does not return: it unwinds to mxshim_call with the message.
 */
#include "mex.h"
#include <math.h>
#include <setjmp.h>
#include <stdarg.h>

#define MXS_EXPORT __attribute__((visibility("default")))

struct mxArray_tag {
  int is_bag;          /* 1: struct/object property bag, 0: numeric array */
  mxClassID cls;
  mwSize ndim;
  mwSize dims[8];
  size_t numel;
  size_t elsize;
  void *data;
  int nfields;
  int cap;
  char **names;
  mxArray **values;
};

/* Harness controls (read by the per-library clock/omp wrappers in ref_hooks.c). */
MXS_EXPORT long long mxshim_fixed_us = -1; /* >= 0: clock reads return this many microseconds */
MXS_EXPORT int mxshim_nprocs = 0;          /* > 0: omp_get_num_procs() returns this value */
MXS_EXPORT int mxshim_quiet = 1;           /* suppress mexPrintf output */

static __thread jmp_buf *g_jmp = NULL;
static __thread char g_err[1024];

static size_t elsize_of(mxClassID c) {
  switch (c) {
    case mxDOUBLE_CLASS: case mxINT64_CLASS: case mxUINT64_CLASS: return 8;
    case mxSINGLE_CLASS: case mxINT32_CLASS: case mxUINT32_CLASS: return 4;
    case mxINT16_CLASS: case mxUINT16_CLASS: case mxCHAR_CLASS: return 2;
    case mxINT8_CLASS: case mxUINT8_CLASS: case mxLOGICAL_CLASS: return 1;
    default: return 0;
  }
}

static void fail(const char *id, const char *msg) {
  snprintf(g_err, sizeof g_err, "%s: %s", id ? id : "mxshim", msg);
  if (g_jmp) longjmp(*g_jmp, 1);
  fprintf(stderr, "mxshim fatal (no handler): %s\n", g_err);
  abort();
}

MXS_EXPORT mxArray *mxCreateNumericArray(mwSize ndim, const mwSize *dims, mxClassID classid, mxComplexity flag) {
  (void)flag;
  mxArray *a = (mxArray *)calloc(1, sizeof(mxArray));
  if (!a) fail("mxshim:nomem", "out of memory");
  a->cls = classid;
  a->elsize = elsize_of(classid);
  a->ndim = ndim < 2 ? 2 : ndim;
  if (a->ndim > 8) fail("mxshim:dims", "too many dimensions");
  a->numel = 1;
  for (mwSize i = 0; i < a->ndim; i++) {
    a->dims[i] = i < ndim ? dims[i] : 1;
    a->numel *= a->dims[i];
  }
  /* MATLAB drops trailing singleton dimensions beyond the second */
  while (a->ndim > 2 && a->dims[a->ndim - 1] == 1) a->ndim--;
  a->data = calloc(a->numel ? a->numel : 1, a->elsize ? a->elsize : 1);
  if (!a->data) fail("mxshim:nomem", "out of memory");
  return a;
}

MXS_EXPORT mxArray *mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID classid, mxComplexity flag) {
  mwSize d[2] = {m, n};
  return mxCreateNumericArray(2, d, classid, flag);
}

MXS_EXPORT mxArray *mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity flag) {
  return mxCreateNumericMatrix(m, n, mxDOUBLE_CLASS, flag);
}

MXS_EXPORT mxArray *mxCreateDoubleScalar(double value) {
  mxArray *a = mxCreateDoubleMatrix(1, 1, mxREAL);
  *(double *)a->data = value;
  return a;
}

MXS_EXPORT mxArray *mxCreateLogicalScalar(bool value) {
  mxArray *a = mxCreateNumericMatrix(1, 1, mxLOGICAL_CLASS, mxREAL);
  *(unsigned char *)a->data = value ? 1 : 0;
  return a;
}

MXS_EXPORT mxArray *mxshim_new_bag(void) {
  mxArray *a = (mxArray *)calloc(1, sizeof(mxArray));
  if (!a) fail("mxshim:nomem", "out of memory");
  a->is_bag = 1;
  a->cls = mxSTRUCT_CLASS;
  a->ndim = 2;
  a->dims[0] = a->dims[1] = 1;
  a->numel = 1;
  return a;
}

MXS_EXPORT void mxDestroyArray(mxArray *pa) {
  if (!pa) return;
  if (pa->is_bag) {
    for (int i = 0; i < pa->nfields; i++) {
      free(pa->names[i]);
      mxDestroyArray(pa->values[i]);
    }
    free(pa->names);
    free(pa->values);
  } else {
    free(pa->data);
  }
  free(pa);
}

MXS_EXPORT mxArray *mxDuplicateArray(const mxArray *in) {
  if (!in) return NULL;
  mxArray *a = (mxArray *)calloc(1, sizeof(mxArray));
  if (!a) fail("mxshim:nomem", "out of memory");
  *a = *in;
  if (in->is_bag) {
    a->names = (char **)calloc(in->cap ? in->cap : 1, sizeof(char *));
    a->values = (mxArray **)calloc(in->cap ? in->cap : 1, sizeof(mxArray *));
    for (int i = 0; i < in->nfields; i++) {
      a->names[i] = strdup(in->names[i]);
      a->values[i] = mxDuplicateArray(in->values[i]);
    }
  } else {
    size_t bytes = (in->numel ? in->numel : 1) * (in->elsize ? in->elsize : 1);
    a->data = malloc(bytes);
    if (!a->data) fail("mxshim:nomem", "out of memory");
    memcpy(a->data, in->data, bytes);
  }
  return a;
}

MXS_EXPORT double *mxGetPr(const mxArray *pa) { return (pa && !pa->is_bag) ? (double *)pa->data : NULL; }
MXS_EXPORT void *mxGetData(const mxArray *pa) { return (pa && !pa->is_bag) ? pa->data : NULL; }
MXS_EXPORT const mwSize *mxGetDimensions(const mxArray *pa) { return pa->dims; }
MXS_EXPORT mwSize mxGetNumberOfDimensions(const mxArray *pa) { return pa->ndim; }
MXS_EXPORT size_t mxGetM(const mxArray *pa) { return pa->dims[0]; }
MXS_EXPORT size_t mxGetN(const mxArray *pa) {
  size_t n = 1;
  for (mwSize i = 1; i < pa->ndim; i++) n *= pa->dims[i];
  return n;
}
MXS_EXPORT size_t mxGetNumberOfElements(const mxArray *pa) { return pa->is_bag ? 1 : pa->numel; }
MXS_EXPORT mxClassID mxGetClassID(const mxArray *pa) { return pa->cls; }

MXS_EXPORT bool mxIsLogicalScalarTrue(const mxArray *pa) {
  return pa && !pa->is_bag && pa->cls == mxLOGICAL_CLASS && pa->numel == 1 && *(unsigned char *)pa->data != 0;
}

static int find_field(const mxArray *pa, const char *name) {
  for (int i = 0; i < pa->nfields; i++)
    if (strcmp(pa->names[i], name) == 0) return i;
  return -1;
}

static mxArray *get_named(const mxArray *pa, const char *name, const char *what) {
  if (!pa || !pa->is_bag) {
    char msg[256];
    snprintf(msg, sizeof msg, "%s '%s' requested from a non-struct value", what, name);
    fail("mxshim:notstruct", msg);
  }
  int k = find_field(pa, name);
  if (k < 0) {
    char msg[256];
    snprintf(msg, sizeof msg, "no %s named '%s'", what, name);
    fail("mxshim:nofield", msg);
  }
  return pa->values[k];
}

static void set_named(mxArray *pa, const char *name, mxArray *value) {
  if (!pa || !pa->is_bag) fail("mxshim:notstruct", "set on a non-struct value");
  int k = find_field(pa, name);
  if (k >= 0) {
    if (pa->values[k] != value) mxDestroyArray(pa->values[k]);
    pa->values[k] = value;
    return;
  }
  if (pa->nfields == pa->cap) {
    int nc = pa->cap ? 2 * pa->cap : 16;
    char **nn = (char **)realloc(pa->names, nc * sizeof(char *));
    mxArray **nv = (mxArray **)realloc(pa->values, nc * sizeof(mxArray *));
    if (!nn || !nv) fail("mxshim:nomem", "out of memory");
    pa->names = nn;
    pa->values = nv;
    pa->cap = nc;
  }
  pa->names[pa->nfields] = strdup(name);
  pa->values[pa->nfields] = value;
  pa->nfields++;
}

MXS_EXPORT mxArray *mxGetField(const mxArray *pa, mwIndex i, const char *fieldname) {
  (void)i;
  return get_named(pa, fieldname, "field");
}
MXS_EXPORT void mxSetField(mxArray *pa, mwIndex i, const char *fieldname, mxArray *value) {
  (void)i;
  set_named(pa, fieldname, value);
}
/* As in MATLAB, a property that does not exist yields NULL. */
MXS_EXPORT mxArray *mxGetProperty(const mxArray *pa, mwIndex i, const char *propname) {
  (void)i;
  if (!pa || !pa->is_bag) return NULL;
  int k = find_field(pa, propname);
  return k < 0 ? NULL : pa->values[k];
}
MXS_EXPORT mxArray *mxGetPropertyShared(const mxArray *pa, mwIndex i, const char *propname) {
  return mxGetProperty(pa, i, propname);
}
MXS_EXPORT void mxSetProperty(mxArray *pa, mwIndex i, const char *propname, const mxArray *value) {
  (void)i;
  set_named(pa, propname, mxDuplicateArray(value));
}
MXS_EXPORT void mxSetPropertyShared(mxArray *pa, mwIndex i, const char *propname, const mxArray *value) {
  (void)i;
  set_named(pa, propname, (mxArray *)value);
}

MXS_EXPORT bool mxIsNaN(double x) { return isnan(x); }
MXS_EXPORT bool mxIsInf(double x) { return isinf(x); }
MXS_EXPORT bool mxIsFinite(double x) { return isfinite(x); }

MXS_EXPORT int mexPrintf(const char *fmt, ...) {
  if (mxshim_quiet) return 0;
  va_list ap;
  va_start(ap, fmt);
  int r = vprintf(fmt, ap);
  va_end(ap);
  return r;
}
MXS_EXPORT int mexEvalString(const char *cmd) { (void)cmd; return 0; }
MXS_EXPORT void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...) {
  char msg[768];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(msg, sizeof msg, fmt, ap);
  va_end(ap);
  fail(id, msg);
}
MXS_EXPORT void mexErrMsgTxt(const char *msg) { fail("MEX", msg); }

MXS_EXPORT int mxshim_interrupt = 0; /* what utIsInterruptPending reports (a test sets it) */
MXS_EXPORT bool utIsInterruptPending(void) { return __atomic_load_n(&mxshim_interrupt, __ATOMIC_ACQUIRE) != 0; }

MXS_EXPORT void *mxMalloc(size_t n) { return malloc(n ? n : 1); }
MXS_EXPORT void *mxCalloc(size_t n, size_t size) { return calloc(n ? n : 1, size ? size : 1); }
MXS_EXPORT void mxFree(void *ptr) { free(ptr); }
MXS_EXPORT int mexAtExit(void (*fn)(void)) {
  (void)fn;
  return 0;
}

/* ---- harness helpers (bag introspection, guarded calls) ---- */
MXS_EXPORT int mxshim_is_bag(const mxArray *pa) { return pa ? pa->is_bag : 0; }
MXS_EXPORT int mxshim_nfields(const mxArray *pa) { return (pa && pa->is_bag) ? pa->nfields : 0; }
MXS_EXPORT const char *mxshim_field_name(const mxArray *pa, int k) { return pa->names[k]; }
MXS_EXPORT mxArray *mxshim_field_value(const mxArray *pa, int k) { return pa->values[k]; }
MXS_EXPORT mxArray *mxshim_get(const mxArray *pa, const char *name) {
  if (!pa || !pa->is_bag) return NULL;
  int k = find_field(pa, name);
  return k < 0 ? NULL : pa->values[k];
}
MXS_EXPORT void mxshim_set(mxArray *pa, const char *name, mxArray *value) { set_named(pa, name, value); }
MXS_EXPORT size_t mxshim_elsize(const mxArray *pa) { return pa->elsize; }
MXS_EXPORT const char *mxshim_last_error(void) { return g_err; }

typedef void (*mex_fn)(int, mxArray **, int, const mxArray **);

/* Calls a mexFunction; returns 0 on success, 1 if it raised an error (message in mxshim_last_error). */
MXS_EXPORT int mxshim_call(mex_fn fn, int nlhs, mxArray **plhs, int nrhs, const mxArray **prhs) {
  jmp_buf here;
  jmp_buf *prev = g_jmp;
  g_err[0] = 0;
  if (setjmp(here)) {
    g_jmp = prev;
    return 1;
  }
  g_jmp = &here;
  fn(nlhs, plhs, nrhs, prhs);
  g_jmp = prev;
  return 0;
}
