/*
 * finiteElementHeatPropagator_CUDA.c — MEX gateway for the B200 heat stepper.
 *
 * Drop-in for the reference's heat MEX (+MCmatlab/src/finiteElementHeatPropagator.c:688
 * mexFunction), called as
 *   [T, Omega, sensorTemps, maxMediaTemps] = finiteElementHeatPropagator_CUDA(T, Omega, heatSimParameters)
 * from +MCmatlab/@model/simulateHeatDistribution.m:259-264, :320-325, :381-386. Same inputs
 * (T single [nx ny nz]; Omega single [nx ny nz] or a NaN scalar for no damage; the
 * heatSimParameters struct) and outputs (T, Omega, sensorTemps double [nSensors, steps+1],
 * maxMediaTemps single [1, nM]). Library errors become mexErrMsgIdAndTxt.
 *
 * Build in MATLAB (Linux):
 *   mex -I<repo>/include finiteElementHeatPropagator_CUDA.c -L<repo>/mcmatlab_b200 -lmcb200
 */
#include "mex.h"

#include <math.h>
#include <stdint.h>
#include <string.h>

#include "mcb200.h"

static mcb_ctx *g_ctx = NULL;

static void cleanup(void) {
  if (g_ctx) mcb_ctx_destroy(g_ctx);
  g_ctx = NULL;
}

static const mxArray *field(const mxArray *s, const char *name) {
  const mxArray *f = mxGetField(s, 0, name);
  if (!f) mexErrMsgIdAndTxt("MCmatlab:CUDA", "heatSimParameters.%s is missing", name);
  return f;
}

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
  (void)nlhs;
  if (nrhs < 3) mexErrMsgIdAndTxt("MCmatlab:CUDA", "usage: [T,Omega,sensorTemps,maxMediaTemps] = f(T, Omega, params)");
  const mxArray *S = prhs[2];
  const size_t *dims = mxGetDimensions(prhs[0]);
  mcb_heat_params p;
  memset(&p, 0, sizeof p);
  p.nx = (int32_t)dims[0];
  p.ny = (int32_t)dims[1];
  p.nz = mxGetNumberOfDimensions(prhs[0]) > 2 ? (int32_t)dims[2] : 1;
  const mxArray *c = field(S, "dTdtperdeltaT");
  p.nM = (int32_t)mxGetM(c);
  p.dTdtperdeltaT = (const float *)mxGetData(c);
  p.M = (const uint8_t *)mxGetData(field(S, "M"));
  p.dTdt_abs = (const float *)mxGetData(field(S, "dTdt_abs"));
  p.A = mxGetPr(field(S, "A"));
  p.E = mxGetPr(field(S, "E"));
  p.lightsOn = mxIsLogicalScalarTrue(field(S, "lightsOn"));
  p.heatBoundaryType = (int32_t)*mxGetPr(field(S, "heatBoundaryType"));
  p.steps = (int64_t)*mxGetPr(field(S, "steps"));
  p.dt = *mxGetPr(field(S, "dt"));
  const mxArray *si = field(S, "tempSensorCornerIdxs");
  p.nSensors = (int32_t)mxGetM(si);
  p.tempSensorCornerIdxs = p.nSensors ? mxGetPr(si) : NULL;
  p.tempSensorInterpWeights = p.nSensors ? mxGetPr(field(S, "tempSensorInterpWeights")) : NULL;

  const size_t L = (size_t)p.nx * p.ny * p.nz;
  plhs[0] = mxCreateNumericArray(3, dims, mxSINGLE_CLASS, mxREAL);
  float *T = (float *)mxGetData(plhs[0]);
  memcpy(T, mxGetData(prhs[0]), sizeof(float) * L);
  const float *Om_in = (const float *)mxGetData(prhs[1]);
  const int damage = !mxIsNaN(Om_in[0]);
  plhs[1] = damage ? mxCreateNumericArray(3, dims, mxSINGLE_CLASS, mxREAL) : mxCreateNumericMatrix(1, 1, mxSINGLE_CLASS, mxREAL);
  float *Om = (float *)mxGetData(plhs[1]);
  if (damage) memcpy(Om, Om_in, sizeof(float) * L);
  else Om[0] = NAN;
  plhs[2] = p.nSensors ? mxCreateDoubleMatrix((size_t)p.nSensors, (size_t)p.steps + 1, mxREAL) : mxCreateDoubleMatrix(0, 0, mxREAL);
  plhs[3] = mxCreateNumericMatrix(1, (size_t)p.nM, mxSINGLE_CLASS, mxREAL);

  if (!g_ctx) {
    if (mcb_ctx_create(0, &g_ctx) != MCB_OK) mexErrMsgIdAndTxt("MCmatlab:CUDA", "no usable CUDA device");
    mexAtExit(cleanup);
  }
  const mcb_status st = mcb_heat_forward(g_ctx, &p, T, damage ? Om : NULL, p.nSensors ? mxGetPr(plhs[2]) : NULL,
                                         (float *)mxGetData(plhs[3]));
  if (st != MCB_OK) mexErrMsgIdAndTxt("MCmatlab:CUDA", "%s", mcb_last_error(g_ctx));
}
