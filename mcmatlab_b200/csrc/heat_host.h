// Host-side internals of the heat stepper shared by the forward entries (heat_adi.cu) and the
// adjoint (heat_adjoint.cu): the device-resident state and the stepping set-up.
#pragma once
#include <cuda.h>

#include <functional>

#include "heat_common.cuh"
#include "internal.h"

namespace mcb {
// Grid shape of the streamed stepper: every grid is stored with an x pitch px >= nx (a multiple
// of 16 that holds whole lane chunks of the X pass) so that every row starts on a TMA-aligned
// boundary.
struct StreamShape {
  int nx = 0, ny = 0, nz = 0, px = 0;
  long long Lp = 0;  // px * ny * nz
};
// TMA descriptors of the streamed stepper's tiles over this state's buffers.
struct StreamMaps {
  CUtensorMap xTh, xTr, xQr, xMh, xCr;  // X pass: T with y halo rows, T rows, Q rows, media with halo, codes
  CUtensorMap yA, yM;                   // Y pass: A and media, 16 columns x whole y lines
  CUtensorMap zA, zM, zT;               // Z pass: A, media and T, 16 columns x whole z lines
  CUtensorMap cyA, cyM, czA, czM, czT;  // column-layout Y/Z passes: 32 columns x whole lines
};
}  // namespace mcb

// Device-resident stepper state: grids stay in HBM across calls. A state is either streamed
// (heat_stream.cu: pitched grids, no stored factorisation) or factored (heat_adi.cu: dense grids
// with the line factorisation stored per voxel, used by the adjoint and for axes over 512).
struct mcb_heat_state {
  bool streamed = false;
  mcb::StreamShape shape;
  mcb::StreamMaps *maps = nullptr;
  uint8_t *code = nullptr;
  uint8_t *uniX = nullptr, *uniY = nullptr, *uniZ = nullptr;  // homogeneous-chunk tables (streamed)
  float *H = nullptr;
  float4 *Hd = nullptr;
  int codeHs = -1;
  bool qValid = false;
  int lastW = 0;
  mcb_ctx *ctx = nullptr;
  int nx = 0, ny = 0, nz = 0, nM = 0;
  long long L = 0;
  bool damage = false;
  int tw = 32;
  double base = 0.0;
  double factoredDt = -1.0;
  int factoredHs = -1;
  float *T = nullptr, *A = nullptr, *Q = nullptr, *ib = nullptr, *Om = nullptr, *dOm = nullptr, *stage = nullptr,
        *c = nullptr, *Sz = nullptr;
  float2 *fb = nullptr;
  uint8_t *nb = nullptr;
  uint8_t *M = nullptr;
  double *logA = nullptr, *E = nullptr;
  float2 *dmg = nullptr;
  unsigned int *maxEnc = nullptr;
  int *step = nullptr;
  double *sIdx = nullptr, *sW = nullptr, *sens = nullptr;
  long long sensCap = 0;
  int sCap = 0;
  void *block = nullptr;
};

namespace mcb {

// Launch configuration of one DG-ADI step on a state (three fused passes).
struct HeatStepper {
  HeatDev h;
  int gridX = 0, gridYZ = 0, tw = 32;
  size_t smemX = 0;
};

mcb_status heat_check_params(mcb_ctx *ctx, const mcb_heat_params *p);
// (Re)allocates the state's buffers for p's grid when needed and uploads T, Omega and p's tables.
mcb_status heat_state_init(mcb_ctx *ctx, mcb_heat_state *s, const mcb_heat_params *p, const float *T,
                           const float *Omega);
void heat_state_release(mcb_heat_state *s);
// Factors the line matrices if dt or the boundary type changed, sets the kernels' shared-memory
// limits, clears the per-call maxima, step counter and damage increments, and fills *out.
mcb_status heat_stepper(mcb_ctx *ctx, mcb_heat_state *s, const mcb_heat_params *p, HeatStepper *out);
// Enqueues one step.
void heat_step_launch(const HeatStepper &k, cudaStream_t st);
// Per medium {x0, E/R} with x0 = log A - E / (R T0), T0 = base temperature in kelvin.
void heat_damage_table(const mcb_heat_params *p, double base, float2 *out);

// Streamed stepper (heat_stream.cu).
struct StreamStepper;  // launch configuration of one streamed step (heat_stream.cu)
bool stream_supported(int nx, int ny, int nz);
// A streamed state for p's grid holding T (no damage), with p's source when the light is on
// (heat_adi.cu); release with heat_state_release.
mcb_status stream_state_create(mcb_ctx *ctx, mcb_heat_state *s, const mcb_heat_params *p, const float *T);
// Creates *out (the set-up of stream_step) for stepping s one step at a time (no sensors);
// release with stream_stepper_free.
mcb_status stream_stepper_new(mcb_ctx *ctx, mcb_heat_state *s, const mcb_heat_params *p, StreamStepper **out);
void stream_stepper_free(StreamStepper *k);
void stream_stepper_launch(const StreamStepper *k, cudaStream_t st);
StreamShape stream_shape(int nx, int ny, int nz);
int stream_warmup(const float *c, float hdt, int nM);
void stream_carve(const std::function<void *(size_t)> &take, mcb_heat_state *s, const mcb_heat_params *p, bool damage,
                  bool withQ);
mcb_status stream_maps(mcb_ctx *ctx, mcb_heat_state *s);
mcb_status stream_upload(mcb_ctx *ctx, mcb_heat_state *s, const mcb_heat_params *p, const float *T, const float *Omega);
mcb_status stream_upload_q(mcb_ctx *ctx, mcb_heat_state *s, const float *Q);
mcb_status stream_step(mcb_ctx *ctx, mcb_heat_state *s, const mcb_heat_params *p, double *sens, double *sensorTemps,
                       float *maxMediaTemps, bool graphs);
mcb_status stream_download(mcb_ctx *ctx, mcb_heat_state *s, float *T, float *Omega);
// T of a streamed state (pitched deviations) into a dense array of deviations, and back;
// asynchronous.
void stream_dense_copy(mcb_ctx *ctx, const mcb_heat_state *s, float *dense, cudaStream_t st);
void stream_dense_set(mcb_ctx *ctx, mcb_heat_state *s, const float *dense, cudaStream_t st);
// Index of voxel v (dense, column-major) in a streamed state's pitched grids.
long long stream_pitched_index(const mcb_heat_state *s, long long v);

}  // namespace mcb
