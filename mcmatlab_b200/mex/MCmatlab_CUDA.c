/*
 * MCmatlab_CUDA.c — MEX gateway for the B200 transport library.
 *
 * Drop-in for the reference's MC MEX (+MCmatlab/src/MCmatlab.c:317 mexFunction, called as
 * model = MCmatlab_CUDA(model, simType) from +MCmatlab/@model/runMonteCarlo.m:99-104 and
 * :169-174). It reads the same model properties with the same meaning, fills an
 * mcb_mc_model, calls mcb_mc_run (include/mcb200.h) and writes the same output properties
 * as the reference (MCmatlab.c:461-493, :755-776). Library errors become
 * mexErrMsgIdAndTxt("MCmatlab:CUDA", ...).
 *
 * Build in MATLAB (Linux):
 *   mex -I<repo>/include MCmatlab_CUDA.c -L<repo>/mcmatlab_b200 -lmcb200 -lut
 * The RNG seed is the optional MC.seed property; without it the seed is taken from the
 * clock, as the reference seeds its generator (MCmatlab.c:241).
 *
 * Ctrl+C: the transport runs on a worker thread while the MATLAB thread polls
 * utIsInterruptPending (as MCmatlab.c:293-298, :690-693 do) and raises the library's cancel
 * flag; the run then stops and returns the results of the packets that ran, normalised over
 * them, as the reference does.
 */
#include "mex.h"

#include <math.h>
#include <pthread.h>
#include <stdbool.h>
#include <stdint.h>
#include <string.h>
#include <time.h>

#include "mcb200.h"

extern bool utIsInterruptPending(void); /* libut (MATLAB) */

struct run_job {
  mcb_ctx *ctx;
  const mcb_mc_model *m;
  mcb_mc_result *r;
  mcb_status st;
  int done;
};

static void *run_worker(void *arg) {
  struct run_job *j = (struct run_job *)arg;
  j->st = mcb_mc_run(j->ctx, j->m, j->r);
  __atomic_store_n(&j->done, 1, __ATOMIC_RELEASE);
  return NULL;
}

/* mcb_mc_run on a worker thread; this (MATLAB's) thread forwards Ctrl+C to the cancel flag. */
static mcb_status run_interruptible(mcb_ctx *ctx, const mcb_mc_model *m, mcb_mc_result *r) {
  volatile int *cancel = mcb_cancel_flag(ctx);
  struct run_job job = {ctx, m, r, MCB_OK, 0};
  pthread_t th;
  *cancel = 0;
  if (pthread_create(&th, NULL, run_worker, &job) != 0) return mcb_mc_run(ctx, m, r);
  const struct timespec tick = {0, 20000000}; /* 20 ms */
  while (!__atomic_load_n(&job.done, __ATOMIC_ACQUIRE)) {
    if (!*cancel && utIsInterruptPending()) *cancel = 1;
    nanosleep(&tick, NULL);
  }
  pthread_join(th, NULL);
  *cancel = 0;
  return job.st;
}

static mcb_ctx *g_ctx = NULL;
static int g_dev = -1;

static double num(const mxArray *a) { return *(const double *)mxGetData(a); }
static const mxArray *prop(const mxArray *o, const char *name) {
  const mxArray *p = mxGetPropertyShared(o, 0, name);
  if (!p) mexErrMsgIdAndTxt("MCmatlab:CUDA", "model property '%s' is missing", name);
  return p;
}
static double pnum(const mxArray *o, const char *name) { return num(prop(o, name)); }
static int pbool(const mxArray *o, const char *name) { return mxIsLogicalScalarTrue(prop(o, name)) ? 1 : 0; }

static mcb_distr distr(const mxArray *sid, const char *dname, const char *wname) {
  mcb_distr d;
  const mxArray *a = prop(sid, dname);
  d.values = (const double *)mxGetData(a);
  d.n = (int64_t)mxGetNumberOfElements(a);
  d.width = pnum(sid, wname);
  return d;
}

static void cleanup(void) {
  if (g_ctx) mcb_ctx_destroy(g_ctx);
  g_ctx = NULL;
}

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
  (void)nlhs;
  if (nrhs < 2) mexErrMsgIdAndTxt("MCmatlab:CUDA", "usage: model = MCmatlab_CUDA(model, simType)");
  const int simFluorescence = num(prhs[1]) == 2;
  const mxArray *MC = prop(prhs[0], simFluorescence ? "FMC" : "MC");
  const mxArray *G = prop(prhs[0], "G");
  const mxArray *LS = prop(MC, "LS");
  const mxArray *LC = prop(MC, "LC");
  const mxArray *DC = prop(MC, "depositionCriteria");
  const mxArray *mp = prop(MC, "mediaProperties");
  const mxArray *Marr = prop(MC, "M");

  mcb_mc_model m;
  memset(&m, 0, sizeof m);
  const size_t *dims = mxGetDimensions(Marr);
  m.nx = (int32_t)dims[0];
  m.ny = (int32_t)dims[1];
  m.nz = mxGetNumberOfDimensions(Marr) > 2 ? (int32_t)dims[2] : 1;
  m.dx = pnum(G, "dx");
  m.dy = pnum(G, "dy");
  m.dz = pnum(G, "dz");
  m.M = (const uint8_t *)mxGetData(Marr);
  const mxArray *mua = mxGetField(mp, 0, "mua");
  m.nM = (int32_t)mxGetM(mua);
  m.nL = (int32_t)mxGetN(mua);
  m.mua = (const double *)mxGetData(mua);
  m.mus = (const double *)mxGetData(mxGetField(mp, 0, "mus"));
  m.g = (const double *)mxGetData(mxGetField(mp, 0, "g"));
  m.n = (const double *)mxGetData(mxGetField(mp, 0, "n"));
  m.CDFidx = (const double *)mxGetData(mxGetField(mp, 0, "CDFidx"));
  const mxArray *cdfs = prop(MC, "CDFs");
  m.nCDFelems = (int64_t)mxGetNumberOfElements(cdfs);
  m.CDFs = m.nCDFelems ? (const double *)mxGetData(cdfs) : NULL;
  const mxArray *nrm = prop(MC, "interfaceNormals");
  m.interfaceNormals = mxIsNaN(*(const float *)mxGetData(nrm)) ? NULL : (const float *)mxGetData(nrm);
  const mxArray *sd = prop(MC, "sourceDistribution");
  m.sourceDistribution = mxIsNaN(*(const float *)mxGetData(sd)) ? NULL : (const float *)mxGetData(sd);
  m.spectrum = (const double *)mxGetData(prop(MC, "spectrum"));
  m.nPhotonsRequested = pnum(MC, "nPhotonsRequested");
  m.simulationTimeRequested = pnum(MC, "simulationTimeRequested");
  m.requestCollectedPhotons = pbool(MC, "requestCollectedPhotons");
  m.calcNFR = pbool(MC, "calcNFR");
  m.useLightCollector = pbool(MC, "useLightCollector");
  m.farFieldRes = (int32_t)pnum(MC, "farFieldRes");
  m.boundaryType = (int32_t)pnum(MC, "boundaryType");
  m.nExamplePaths = (int32_t)pnum(MC, "nExamplePaths");
  const mxArray *seed = mxGetPropertyShared(MC, 0, "seed");
  if (seed) {
    m.seed = (uint64_t)num(seed);
  } else {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    m.seed = (uint64_t)ts.tv_sec * 1000000u + (uint64_t)(ts.tv_nsec / 1000);
  }
  if (!m.sourceDistribution) {
    m.sourceType = (int32_t)pnum(LS, "sourceType");
    m.xFocus = pnum(LS, "xFocus");
    m.yFocus = pnum(LS, "yFocus");
    m.zFocus = pnum(LS, "zFocus");
    m.theta = pnum(LS, "theta");
    m.phi = pnum(LS, "phi");
    m.psi = pnum(LS, "psi");
    m.emitterLength = pnum(LS, "emitterLength");
    const mxArray *FP = prop(LS, "FPID"), *AI = prop(LS, "AID");
    m.FPID_radial = distr(FP, "radialDistr", "radialWidth");
    m.FPID_X = distr(FP, "XDistr", "XWidth");
    m.FPID_Y = distr(FP, "YDistr", "YWidth");
    m.AID_radial = distr(AI, "radialDistr", "radialWidth");
    m.AID_X = distr(AI, "XDistr", "XWidth");
    m.AID_Y = distr(AI, "YDistr", "YWidth");
    m.LC_tStart = pnum(LC, "tStart");
    m.LC_tEnd = pnum(LC, "tEnd");
    m.LC_nTimeBins = (int32_t)pnum(LC, "nTimeBins");
  }
  m.LC_x = pnum(LC, "x");
  m.LC_y = pnum(LC, "y");
  m.LC_z = pnum(LC, "z");
  m.LC_theta = pnum(LC, "theta");
  m.LC_phi = pnum(LC, "phi");
  m.LC_f = pnum(LC, "f");
  m.LC_diam = pnum(LC, "diam");
  m.LC_fieldSize = pnum(LC, "fieldSize");
  m.LC_NA = pnum(LC, "NA");
  m.LC_res = (int32_t)pnum(LC, "res");
  m.DC_minScatterings = pnum(DC, "minScatterings");
  m.DC_maxScatterings = pnum(DC, "maxScatterings");
  m.DC_minRefractions = pnum(DC, "minRefractions");
  m.DC_maxRefractions = pnum(DC, "maxRefractions");
  m.DC_minReflections = pnum(DC, "minReflections");
  m.DC_maxReflections = pnum(DC, "maxReflections");
  m.DC_minInterfaceTransitions = pnum(DC, "minInterfaceTransitions");
  m.DC_maxInterfaceTransitions = pnum(DC, "maxInterfaceTransitions");
  m.DC_minSubmediaIdx = pnum(DC, "minSubmediaIdx");
  m.DC_maxSubmediaIdx = pnum(DC, "maxSubmediaIdx");
  m.DC_onlyCollected = pbool(DC, "onlyCollected");
  m.DC_evaluateOnlyAtEndOfLife = pbool(DC, "evaluateOnlyAtEndOfLife");

  /* outputs, shaped as MCmatlab.c:461-493 allocates them */
  plhs[0] = mxDuplicateArray(prhs[0]);
  mxArray *MCout = mxGetPropertyShared(plhs[0], 0, simFluorescence ? "FMC" : "MC");
  mxArray *LCout = mxGetPropertyShared(MCout, 0, "LC");
  mcb_mc_result r;
  memset(&r, 0, sizeof r);
  const size_t nx = m.nx, ny = m.ny, nz = m.nz, nL = m.nL;
  if (m.calcNFR) {
    size_t d4[4] = {nx, ny, nz, nL};
    mxSetPropertyShared(MCout, 0, "NFR", mxCreateNumericArray(4, d4, mxSINGLE_CLASS, mxREAL));
    r.NFR = (float *)mxGetData(mxGetPropertyShared(MCout, 0, "NFR"));
  }
  const size_t nT = m.sourceDistribution ? 1 : (m.LC_nTimeBins ? (size_t)m.LC_nTimeBins + 2 : 1);
  if (m.useLightCollector) {
    size_t d4[4] = {(size_t)m.LC_res, (size_t)m.LC_res, nT, nL};
    mxSetPropertyShared(LCout, 0, "image", mxCreateNumericArray(4, d4, mxSINGLE_CLASS, mxREAL));
    r.image = (float *)mxGetData(mxGetPropertyShared(LCout, 0, "image"));
  }
  if (m.farFieldRes) {
    size_t d3[3] = {(size_t)m.farFieldRes, (size_t)m.farFieldRes, nL};
    mxSetPropertyShared(MCout, 0, "farField", mxCreateNumericArray(3, d3, mxSINGLE_CLASS, mxREAL));
    r.farField = (float *)mxGetData(mxGetPropertyShared(MCout, 0, "farField"));
  }
#define FACE(name, a, b, field)                                                    \
  do {                                                                             \
    size_t d3[3] = {(a), (b), nL};                                                 \
    mxSetPropertyShared(MCout, 0, name, mxCreateNumericArray(3, d3, mxSINGLE_CLASS, mxREAL)); \
    r.field = (float *)mxGetData(mxGetPropertyShared(MCout, 0, name));             \
  } while (0)
  if (m.boundaryType == 1) {
    FACE("NI_xpos", ny, nz, NI_xpos);
    FACE("NI_xneg", ny, nz, NI_xneg);
    FACE("NI_ypos", nx, nz, NI_ypos);
    FACE("NI_yneg", nx, nz, NI_yneg);
    FACE("NI_zpos", nx, ny, NI_zpos);
    FACE("NI_zneg", nx, ny, NI_zneg);
  } else if (m.boundaryType == 2) {
    FACE("NI_zneg", 5 * nx, 5 * ny, NI_zneg);
  } else if (m.boundaryType == 3) {
    FACE("NI_zpos", nx, ny, NI_zpos);
    FACE("NI_zneg", nx, ny, NI_zneg);
  }
#undef FACE
  double *paths = NULL;
  if (m.nExamplePaths > 0) {
    r.examplePathsCap = 2000 * (int64_t)m.nExamplePaths + 1000; /* INITIALPATHSSIZE per path, MCmatlab.c:162 */
    paths = (double *)mxMalloc(sizeof(double) * 4 * (size_t)r.examplePathsCap);
    r.examplePaths = paths;
  }

  const int dev = (int)pnum(MC, "GPUdevice");
  if (!g_ctx || g_dev != dev) {
    cleanup();
    if (mcb_ctx_create(dev, &g_ctx) != MCB_OK) mexErrMsgIdAndTxt("MCmatlab:CUDA", "no usable CUDA device %d", dev);
    g_dev = dev;
    mexAtExit(cleanup);
  }
  const mcb_status st = run_interruptible(g_ctx, &m, &r);
  if (st == MCB_ECANCELLED) mexPrintf("\nCtrl+C detected, stopping.");
  if (st != MCB_OK && st != MCB_ELAUNCH && st != MCB_ECANCELLED) {
    if (paths) mxFree(paths);
    mexErrMsgIdAndTxt("MCmatlab:CUDA", "%s", mcb_last_error(g_ctx));
  }
  if (st == MCB_ELAUNCH) mexPrintf("\nERROR: All photons launch outside simulation cuboid. Check your model definition.\n");

  mxArray *out = mxCreateDoubleMatrix(1, 1, mxREAL);
  *mxGetPr(out) = r.nPhotons;
  mxSetProperty(MCout, 0, "nPhotons", out);
  *mxGetPr(out) = r.nPhotonsCollected;
  mxSetProperty(MCout, 0, "nPhotonsCollected", out);
  *mxGetPr(out) = r.nThreads;
  mxSetProperty(MCout, 0, "nThreads", out);
  *mxGetPr(out) = r.simulationTime;
  mxSetProperty(MCout, 0, "simulationTime", out);
  mxDestroyArray(out);
  if (m.useLightCollector && (size_t)m.LC_res * m.LC_res * nT * nL == 1) {
    out = mxCreateNumericMatrix(1, 1, mxSINGLE_CLASS, mxREAL);
    *(float *)mxGetData(out) = r.image[0];
    mxSetProperty(LCout, 0, "image", out);
    mxDestroyArray(out);
  }
  if (m.nExamplePaths > 0) {
    mxArray *P = mxCreateNumericMatrix(4, (size_t)r.examplePathsN, mxDOUBLE_CLASS, mxREAL);
    if (r.examplePathsN) memcpy(mxGetPr(P), paths, sizeof(double) * 4 * (size_t)r.examplePathsN);
    mxSetPropertyShared(MCout, 0, "examplePaths", P);
    mxFree(paths);
  }
}
