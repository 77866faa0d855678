/*
 * getDownsampledParamVals_CUDA.c — MEX gateway for the sub-media binning on the device.
 *
 * Drop-in for the reference's MEX (+MCmatlab/src/getDownsampledParamVals.c:54 mexFunction),
 * called as
 *   [downsampledParamVals, binidx] = getDownsampledParamVals(paramVals, nSM)
 * from +MCmatlab/@model/private/getOpticalMediaProperties.m:151 and
 * getThermalMediaProperties.m:80. Same inputs (paramVals single [3, n]; nSM double scalar) and
 * outputs (single [3, nSM]; uint8 [1, n], 1-based), bit-identical to the reference build.
 * Building it under the reference's name (-output getDownsampledParamVals) into
 * +MCmatlab/@model/private/ replaces the CPU binning. Library errors become mexErrMsgIdAndTxt.
 *
 * Build in MATLAB (Linux):
 *   mex -I<repo>/include getDownsampledParamVals_CUDA.c -L<repo>/mcmatlab_b200 -lmcb200 -output getDownsampledParamVals
 */
#include "mex.h"

#include <stdint.h>

#include "mcb200.h"

static mcb_ctx *g_ctx = NULL;

static void cleanup(void) {
  if (g_ctx) mcb_ctx_destroy(g_ctx);
  g_ctx = NULL;
}

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
  (void)nlhs;
  if (nrhs < 2) mexErrMsgIdAndTxt("MCmatlab:CUDA", "usage: [downsampledParamVals, binidx] = f(paramVals, nSM)");
  if (mxGetClassID(prhs[0]) != mxSINGLE_CLASS || mxGetM(prhs[0]) != 3)
    mexErrMsgIdAndTxt("MCmatlab:CUDA", "paramVals must be a single [3, n] matrix");
  const int64_t n = (int64_t)mxGetN(prhs[0]);
  const int32_t nb = (int32_t)*mxGetPr(prhs[1]);
  plhs[0] = mxCreateNumericMatrix(3, nb > 0 ? nb : 0, mxSINGLE_CLASS, mxREAL);
  plhs[1] = mxCreateNumericMatrix(1, n, mxUINT8_CLASS, mxREAL);
  if (!g_ctx) {
    if (mcb_ctx_create(0, &g_ctx) != MCB_OK) mexErrMsgIdAndTxt("MCmatlab:CUDA", "no usable CUDA device");
    mexAtExit(cleanup);
  }
  const mcb_status st = mcb_downsample_params(g_ctx, (const float *)mxGetData(prhs[0]), n, nb,
                                             (float *)mxGetData(plhs[0]), (uint8_t *)mxGetData(plhs[1]));
  if (st != MCB_OK) mexErrMsgIdAndTxt("MCmatlab:CUDA", "%s", mcb_last_error(g_ctx));
}
