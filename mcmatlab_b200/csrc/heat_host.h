// Host-side internals of the heat stepper shared by the forward entries (heat_adi.cu) and the
// adjoint (heat_adjoint.cu): the device-resident state and the stepping set-up.
#pragma once
#include "heat_common.cuh"
#include "internal.h"

// Device-resident stepper state: grids stay in HBM across calls.
struct mcb_heat_state {
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

}  // namespace mcb
