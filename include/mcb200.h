/*
 * mcb200.h — C ABI of the B200 (sm_100a) implementation of MCmatlab's two hot paths.
 *
 * Plain C types only: host pointers, sizes and POD structs. Every entry point returns
 * an mcb_status; on failure mcb_last_error(ctx) holds a message. No entry point
 * prints, aborts or longjmps.
 *
 * Array layout follows MATLAB: column-major, x fastest. A grid array has
 * nx*ny*nz elements; a per-wavelength grid has nx*ny*nz*nL.
 *
 * Reference interfaces replaced (paths relative to the reference project):
 *   mcb_mc_run        <- mexFunction of +MCmatlab/src/MCmatlab.c:317-791
 *                        (called as MCmatlab(model,1) / MCmatlab_CUDA(model,1),
 *                         +MCmatlab/@model/runMonteCarlo.m:99-104, :169-174)
 *   mcb_heat_forward  <- mexFunction of +MCmatlab/src/finiteElementHeatPropagator.c:688-821
 *                        (called from +MCmatlab/@model/simulateHeatDistribution.m:259-264,
 *                         :320-325, :381-386)
 * The remaining entry points (batched MC, perturbation-MC gradients, the heat
 * adjoint, device-resident heat state) have no counterpart in the reference; each
 * says so below.
 */
#ifndef MCB200_H
#define MCB200_H

#include <stdint.h>
#include <stddef.h>

#if defined(__GNUC__)
#define MCB_API __attribute__((visibility("default")))
#else
#define MCB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  MCB_OK = 0,
  MCB_EINVAL = 1,     /* invalid argument or model */
  MCB_ENOMEM = 2,     /* device or host allocation failed */
  MCB_ECUDA = 3,      /* CUDA runtime error */
  MCB_ECANCELLED = 4, /* cancel flag was set during the run */
  MCB_ETIMEOUT = 5,   /* a bounded device-side wait gave up */
  MCB_ELAUNCH = 6     /* all packets launched outside the allowed region (MCmatlab.c:745) */
} mcb_status;

typedef struct mcb_ctx mcb_ctx;

/* One context per device and caller thread; it owns device buffers reused across calls. */
MCB_API mcb_status mcb_ctx_create(int device, mcb_ctx **out);
MCB_API mcb_status mcb_ctx_destroy(mcb_ctx *ctx);
MCB_API const char *mcb_last_error(const mcb_ctx *ctx);
/* Host-visible cancel flag polled by the transport kernel (stands in for utIsInterruptPending,
 * MCmatlab.c:293-298). Setting *flag != 0 makes the running mcb_mc_run return MCB_ECANCELLED;
 * its outputs then hold the results of the packets that ran, normalised over them, as the
 * reference returns them on Ctrl+C. The caller resets the flag. */
MCB_API volatile int *mcb_cancel_flag(mcb_ctx *ctx);

/* ------------------------------------------------------------------------------------------
 * Monte Carlo photon transport.
 * mcb_mc_model carries exactly the model properties MCmatlab.c's mexFunction reads, in their
 * MATLAB meaning (MCmatlab.c:317-616), plus a seed for the counter-based RNG.
 * ------------------------------------------------------------------------------------------ */
typedef struct mcb_distr {
  const double *values; /* custom distribution samples, or NULL */
  int64_t n;            /* number of samples; n == 1 means values[0] is a code: 0 top-hat, 1 Gaussian, 2 Lambertian */
  double width;         /* radialWidth / XWidth / YWidth */
} mcb_distr;

typedef struct mcb_mc_model {
  /* geometry (model.G and model.MC.M) */
  int32_t nx, ny, nz;
  double dx, dy, dz;
  const uint8_t *M;              /* [nx*ny*nz], 1-based sub-medium index (model.MC.M) */
  /* media (model.MC.mediaProperties), column-major [nM x nL] */
  int32_t nM, nL;
  const double *mua, *mus, *g, *n, *CDFidx; /* g NaN -> custom phase function CDFs[:, CDFidx] */
  const double *CDFs;            /* [201 x nCDF] or NULL */
  int64_t nCDFelems;             /* 201 * nCDF */
  const float *interfaceNormals; /* [2 x nx*ny*nz] (theta, phi) or NULL when matchedInterfaces */
  const float *sourceDistribution; /* [nx*ny*nz*nL] distributed source, or NULL */
  const double *spectrum;        /* [nL] power fraction per wavelength (model.MC.spectrum) */
  /* run control */
  double nPhotonsRequested;      /* NaN: timed run of simulationTimeRequested minutes */
  double simulationTimeRequested;
  int32_t requestCollectedPhotons;
  int32_t calcNFR;
  int32_t useLightCollector;
  int32_t farFieldRes;
  int32_t boundaryType;          /* 0 none escaping, 1 all faces, 2 top only, 3 top/bottom + cyclic x/y */
  int32_t nExamplePaths;
  uint64_t seed;                 /* Philox-4x32-10 key */
  /* light source (model.MC.LS) */
  int32_t sourceType;            /* 0..5, ignored when sourceDistribution != NULL */
  double xFocus, yFocus, zFocus, theta, phi, psi, emitterLength;
  mcb_distr FPID_radial, FPID_X, FPID_Y, AID_radial, AID_X, AID_Y;
  /* light collector (model.MC.LC) */
  double LC_x, LC_y, LC_z, LC_theta, LC_phi, LC_f, LC_diam, LC_fieldSize, LC_NA;
  double LC_tStart, LC_tEnd;
  int32_t LC_res, LC_nTimeBins;
  /* deposition criteria (model.MC.depositionCriteria); +inf allowed for the maxima */
  double DC_minScatterings, DC_maxScatterings, DC_minRefractions, DC_maxRefractions;
  double DC_minReflections, DC_maxReflections, DC_minInterfaceTransitions, DC_maxInterfaceTransitions;
  double DC_minSubmediaIdx, DC_maxSubmediaIdx; /* 1-based */
  int32_t DC_onlyCollected, DC_evaluateOnlyAtEndOfLife;
  /* Sharding (no counterpart in the reference): packet k of this run uses the random stream of
   * packet index packetOffset + k * packetStride (packetStride 0 means 1). Shards r = 0..W-1 of
   * one seed with offset r and stride W partition the packets of the unsharded run. Example paths
   * always replay packets 0, 1, 2, ... of the unsharded stream. */
  uint64_t packetOffset, packetStride;
} mcb_mc_model;

typedef struct mcb_mc_result {
  /* caller-owned output arrays (NULL = not wanted); sizes as the MEX allocates them (MCmatlab.c:461-493) */
  float *NFR;        /* [nx*ny*nz*nL] normalised fluence rate (when calcNFR) */
  float *image;      /* [res*res*(nTimeBins ? nTimeBins+2 : 1)*nL] (when useLightCollector) */
  float *farField;   /* [farFieldRes^2*nL] */
  float *NI_xpos, *NI_xneg, *NI_ypos, *NI_yneg; /* [ny*nz*nL], [nx*nz*nL] (boundaryType 1) */
  float *NI_zpos;    /* [nx*ny*nL] (boundaryType 1, 3) */
  float *NI_zneg;    /* [nx*ny*nL] (1, 3) or [5nx*5ny*nL] (2) */
  double *examplePaths;     /* [4 x examplePathsCap] x,y,z,weight columns, NaN-separated */
  int64_t examplePathsCap;  /* capacity in columns */
  /* results */
  int64_t examplePathsN;    /* columns written */
  double nPhotons, nPhotonsCollected, nThreads, simulationTime; /* simulationTime in minutes */
  /* kernel statistics (not in the reference) */
  uint64_t propagationSteps;   /* propagatePhoton-equivalent sub-steps executed */
  double kernelMs;             /* device time of the transport kernels */
  /* packets ended by the free-step limit (2e4 propagation sub-steps without a scattering event;
   * the reference has no such limit) and their remaining weight, summed over wavelengths, in
   * units of one launched packet's weight */
  double freeStepCuts, freeStepCutWeight;
  /* FP64 tallies before normalisation (no counterpart in the reference, whose MEX keeps them in
   * thread-local memory and returns only normalised single-precision outputs). NULL = not
   * wanted; else [mcb_mc_tally_count(model)] doubles, wavelength-major blocks of: the absorbed
   * weight per voxel (when calcNFR), the light-collector image, the far field, the escape-face
   * tallies, and last the launched and collected packet counts, 2 per wavelength. Tallies of runs
   * of one model on disjoint packet ranges (packetOffset) add up to the tallies of their union;
   * mcb_mc_normalize turns a sum into the outputs of that union. */
  double *tallies;
} mcb_mc_result;

/* Replaces MCmatlab.c mexFunction: runs all wavelengths, normalises and writes the outputs. */
MCB_API mcb_status mcb_mc_run(mcb_ctx *ctx, const mcb_mc_model *model, mcb_mc_result *result);

/* No counterpart in the reference: number of doubles mcb_mc_result.tallies receives for model
 * (0 for an invalid model). */
MCB_API int64_t mcb_mc_tally_count(const mcb_mc_model *model);

/* No counterpart in the reference: the normalisation of a run (normalizeDepositionAndResetO,
 * MCmatlablib.c:1186-1250, as mcb_mc_run applies it) applied to given FP64 tallies, e.g. the sum
 * of the tallies of several runs of model on disjoint packet ranges: writes the normalised
 * outputs, nPhotons and nPhotonsCollected of result (its tallies field is ignored). The merged
 * outputs equal those of one run over the union of the packets, up to FP64 summation order
 * (combineModels.m:59-101 merges normalised single-precision outputs instead). */
MCB_API mcb_status mcb_mc_normalize(mcb_ctx *ctx, const mcb_mc_model *model, const double *tallies,
                                    mcb_mc_result *result);

/* No counterpart in the reference, which sizes its launch with cudaOccupancyMaxPotentialBlockSize
 * (MCmatlab.c:641): the transport kernel's warp-grouping parameters. refillMin: a warp launches
 * new packets on its free lanes once at least this many lanes are free; scatterMin: packets whose
 * free path ran out wait until this many lanes of their warp are waiting before roulette and
 * scattering run (both 1..32). Results do not depend on them (each packet's random stream is
 * fixed); only the time does. */
typedef struct mcb_mc_launch {
  int32_t refillMin, scatterMin;
} mcb_mc_launch;

/* No counterpart in the reference: the launch-parameter class of a model (its voxel count in
 * powers of 4; +16 for gradient runs, +32 for batches). */
MCB_API int32_t mcb_mc_size_class(const mcb_mc_model *model, int32_t gradient, int32_t batched);

/* No counterpart in the reference: autotuner. Runs `model` with calibrationPackets packets for
 * every (refillMin, scatterMin) in {4, 8, 12, 16}^2 (twice each), keeps the fastest for the
 * model's size class in this context (later runs of that class use it), and, when the environment
 * variable MCB_TUNE_FILE names a file, records it there for this GPU model; contexts created later
 * read that file. Writes the choice to *chosen and, when table is not NULL, the 16 candidates as
 * rows {refillMin, scatterMin, best kernel ms} to table[48]. */
MCB_API mcb_status mcb_mc_autotune(mcb_ctx *ctx, const mcb_mc_model *model, double calibrationPackets, int32_t gradient,
                                   mcb_mc_launch *chosen, double *table);

/* No counterpart in the reference: runs n independent models (different grids, media,
 * wavelengths, photon counts) in one persistent launch. Each model's packets use the random
 * streams of its own seed, so results equal n calls of mcb_mc_run up to FP64 summation order.
 * Batched models need fixed launched-packet counts (no timed or collected-count runs). */
MCB_API mcb_status mcb_mc_run_batch(mcb_ctx *ctx, int32_t n, const mcb_mc_model *const *models,
                            mcb_mc_result *const *results);

/* No counterpart in the reference (which has no derivative code): perturbation Monte Carlo.
 * Each packet carries its path length L_m and scattering count k_m per medium, which gives the
 * derivatives of two objectives with respect to every medium's mua and mus in the same run:
 *   R_b  reflectance (escaping weight per unit area and incident power) on the z < 0 face in
 *        annuli of width radialBinWidth about (x, y) = (0, 0)       dW/dmua_m = -L_m W,
 *                                                                  dW/dmus_m = (k_m/mus_m - L_m) W
 *   F    mean normalised fluence rate over a target voxel box (absorbed weight / mua per
 *        sub-step, plus the sub-step's own dependence on mua_j)
 * Requirements: one wavelength, nM <= 10, a fixed packet count, default deposition criteria. */
typedef struct mcb_mc_objectives {
  int32_t nRadialBins;     /* 0..64 */
  double radialBinWidth;   /* [cm] */
  int32_t box[6];          /* [x0, x1) x [y0, y1) x [z0, z1), 0-based voxel ranges; x1 <= x0: no box */
} mcb_mc_objectives;

typedef struct mcb_mc_grad_result {
  double *R;        /* [nRadialBins] [1/cm^2] */
  double *dR_dmua;  /* [nRadialBins x nM] column-major (bin fastest) [1/cm] */
  double *dR_dmus;  /* [nRadialBins x nM] */
  double F;         /* box mean of the normalised fluence rate [1/cm^2] */
  double *dF_dmua;  /* [nM] */
  double *dF_dmus;  /* [nM] */
} mcb_mc_grad_result;

/* Forward transport (outputs as mcb_mc_run, result may hold NULL arrays) plus the objective
 * values and their per-medium derivatives. */
MCB_API mcb_status mcb_mc_grad(mcb_ctx *ctx, const mcb_mc_model *model, const mcb_mc_objectives *objectives,
                               mcb_mc_result *result, mcb_mc_grad_result *grad);

/* ------------------------------------------------------------------------------------------
 * Heat diffusion (Douglas-Gunn ADI) with Arrhenius damage.
 * mcb_heat_params carries the fields of heatSimParameters read by
 * finiteElementHeatPropagator.c:688-739.
 * ------------------------------------------------------------------------------------------ */
typedef struct mcb_heat_params {
  int32_t nx, ny, nz, nM;
  const uint8_t *M;             /* [nx*ny*nz] 0-based medium index (model.HS.M - 1) */
  const float *dTdtperdeltaT;   /* [nM x nM x 3] column-major: c(i,j,d) = TC_eff(i,j)/VHC_i/d_d^2 */
  const float *dTdt_abs;        /* [nx*ny*nz] heating rate while the light is on [K/s] */
  const double *A, *E;          /* [nM] Arrhenius frequency factor [1/s] and activation energy [J/mol] */
  int32_t lightsOn;
  int32_t heatBoundaryType;     /* 0 insulating, 1 constant-temperature (heat-sinked) faces */
  int64_t steps;                /* nt */
  double dt;
  int32_t nSensors;
  const double *tempSensorCornerIdxs;    /* [nSensors] 0-based linear corner index */
  const double *tempSensorInterpWeights; /* [nSensors x 3] column-major (wx, wy, wz) */
} mcb_heat_params;

/* Replaces finiteElementHeatPropagator.c mexFunction.
 *   T            in/out [nx*ny*nz]
 *   Omega        in/out [nx*ny*nz], or NULL for no damage (the MEX's NaN-scalar Omega)
 *   sensorTemps  out [nSensors x (steps+1)] (may be NULL when nSensors == 0)
 *   maxMediaTemps out [nM]: max over all voxels of medium m and all steps of T (-inf if none) */
MCB_API mcb_status mcb_heat_forward(mcb_ctx *ctx, const mcb_heat_params *p, float *T, float *Omega,
                            double *sensorTemps, float *maxMediaTemps);

/* No counterpart in the reference (whose MEX re-uploads every grid on each call,
 * finiteElementHeatPropagator.c:750, :811): a device-resident stepper state. The grids stay in
 * HBM between calls of mcb_heat_state_step, which runs p->steps steps with p's lightsOn, dt,
 * heatBoundaryType and sensors (p's grid and media must match the state's). */
typedef struct mcb_heat_state mcb_heat_state;
MCB_API mcb_status mcb_heat_state_create(mcb_ctx *ctx, const mcb_heat_params *p, const float *T, const float *Omega,
                                         mcb_heat_state **out);
MCB_API mcb_status mcb_heat_state_step(mcb_heat_state *state, const mcb_heat_params *p, double *sensorTemps,
                                       float *maxMediaTemps);
MCB_API mcb_status mcb_heat_state_read(mcb_heat_state *state, float *T, float *Omega);
MCB_API mcb_status mcb_heat_state_destroy(mcb_heat_state *state);

/* No counterpart in the reference (it has no derivative code): the reverse-time adjoint of the
 * heat stepper. Runs p->steps steps from T0 (no sensors, no damage state) and returns the
 * objective
 *   J = sum_v damageWeight_v * (Arrhenius damage gained by voxel v over the run)
 *     + sum_v peakWeight_v * max_{n = 1..steps} T_v^n
 * and its gradients with respect to the conduction table dTdtperdeltaT (c), the heat source
 * dTdt_abs (Q; zero when the light is off) and the initial temperature. States are checkpointed
 * every K = ceil(steps / nCheckpoints) steps (nCheckpoints <= 0: ceil(sqrt(steps))) and the K - 1
 * inner states of each segment are recomputed once during the reverse sweep; nCheckpoints =
 * steps stores every state (4 nx ny nz bytes each) and recomputes nothing. At most 32 media. */
typedef struct {
  const float *damageWeight; /* [nx*ny*nz] or NULL */
  const float *peakWeight;   /* [nx*ny*nz] or NULL */
} mcb_heat_objective;

typedef struct {
  double J, J_damage, J_peak;  /* out */
  double *dJ_dc;               /* out [nM x nM x 3], same layout as dTdtperdeltaT, or NULL */
  float *dJ_dQ;                /* out [nx*ny*nz] or NULL */
  float *dJ_dT0;               /* out [nx*ny*nz] or NULL */
  double forwardMs, adjointMs; /* out: device time of the checkpointed forward and of the reverse sweep */
} mcb_heat_grad;

MCB_API mcb_status mcb_heat_adjoint(mcb_ctx *ctx, const mcb_heat_params *p, const float *T0,
                                    const mcb_heat_objective *objective, int32_t nCheckpoints, mcb_heat_grad *grad);

/* No counterpart in the reference: mcb_heat_forward that allocates no memory, for callers that
 * cannot allocate at call time (a GPU whose HBM another allocator, e.g. MATLAB's gpuArray pool or
 * a PyTorch caching allocator, has already reserved; other streams' work that cudaFree's
 * device-wide synchronisation would stall). Same arguments, outputs and errors as
 * mcb_heat_forward. Its working set lives in one static 32 MiB device array of the library:
 * 26 bytes per voxel (18 without damage, 22 with damage but no light; the per-voxel grids are
 * stored with nx rounded up to a multiple of 16), about a 107^3 grid, or 66 bytes per voxel for
 * grids with an axis longer than 512; plus 8 per sensor and step (sensorTemps history) and
 * small per-medium tables. Larger problems return MCB_EINVAL naming the limit. The context comes from mcb_ctx_create, which does allocate: create it
 * at set-up. The first call on a device performs set-up (cudaGetSymbolAddress of the scratch).
 * The call is synchronous (it waits for ctx's stream and reads its events before returning), so
 * it must not be made while ctx's stream is being captured. There is one scratch per device:
 * calls that overlap in time on the same device race; serialise them. */
MCB_API mcb_status mcb_heat_forward_static(mcb_ctx *ctx, const mcb_heat_params *p, float *T, float *Omega,
                                           double *sensorTemps, float *maxMediaTemps);

/* Interface normals for mismatched refractive indices, on the device. No counterpart in the
 * reference's C code: its MATLAB host computes them before the MEX call
 * (getOpticalMediaProperties.m:222-244, imgradientxyz + smoothn). M1 [nx*ny*nz] holds 1-based
 * media; riClass [nM] the refractive-index class (0..nClass-1) of every medium (media with equal
 * refractive-index rows share a class). Per class, the 3D Sobel gradient of the class indicator
 * divided by the voxel size, smoothed when smoothingLengthScale > 0 with smoothness
 * s = max(1, round(smoothingLengthScale / max(dx, dy, dz))), is written into the class's voxels;
 * thetaPhi [2 x nx*ny*nz] (column-major, as the MC model's interfaceNormals) receives
 * theta = pi/2 - elevation and phi = azimuth. Smoothing needs every axis <= 1024 voxels. */
MCB_API mcb_status mcb_interface_normals(mcb_ctx *ctx, int32_t nx, int32_t ny, int32_t nz, const uint8_t *M1, int32_t nM,
                                         const int32_t *riClass, int32_t nClass, double dx, double dy, double dz,
                                         double smoothingLengthScale, float *thetaPhi);

/* Sub-media binning of a medium whose optical properties depend on fluence rate, temperature
 * or damage, on the device. Replaces the MEX getDownsampledParamVals (+MCmatlab/src/
 * getDownsampledParamVals.c:54-202, called from getOpticalMediaProperties.m:151): paramVals
 * [3 x n] (column-major: mua, mus, g of each of the medium's n voxels) are downsampled to nBins
 * representatives by greedy farthest-point selection in range-normalised coordinates;
 * downsampled [3 x nBins] receives them, binidx [n] each voxel's 1-based nearest representative.
 * Same arithmetic and index choices as the reference build, bit for bit. nBins in 1..255. */
MCB_API mcb_status mcb_downsample_params(mcb_ctx *ctx, const float *paramVals, int64_t n, int32_t nBins,
                                         float *downsampled, uint8_t *binidx);

/* No counterpart in the reference: measures the device's FP64 atomicAdd throughput to
 * scattered addresses of a buffer of `slots` doubles (the transport's roofline denominator:
 * one FP64 deposit per propagation sub-step). */
MCB_API mcb_status mcb_probe_atomics(mcb_ctx *ctx, int64_t slots, double *atomicsPerSecond);

/* No counterpart in the reference: device time in milliseconds (CUDA events on the context's
 * stream) of the transport kernel or stepping loop of the last call on this context. */
MCB_API double mcb_last_kernel_ms(const mcb_ctx *ctx);

#ifdef __cplusplus
}
#endif

#endif /* MCB200_H */
