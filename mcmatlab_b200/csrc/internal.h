// Shared host-side internals of libmcb200: the context, error reporting and a
// grow-only device buffer pool.
#pragma once
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <map>
#include <string>
#include <vector>

#include "../../include/mcb200.h"

struct DevBuf {
  void *ptr = nullptr;
  size_t bytes = 0;
};

struct mcb_heat_state;

struct mcb_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  volatile int *cancel_host = nullptr;  // pinned, mapped
  int *cancel_dev = nullptr;            // device alias of cancel_host
  std::string err;
  std::vector<DevBuf> pool;             // indexed slots, grow-only
  int num_sms = 0;
  mcb_heat_state *heat = nullptr;  // state reused by mcb_heat_forward
  double lastKernelMs = 0.0;        // device time of the last stepping / transport loop
  // transport launch parameters: tuned per size class (mcb_mc_autotune, or read from the tuning
  // file at context creation), and an override used while the autotuner calibrates
  std::string gpuName;
  std::map<int, mcb_mc_launch> tuned;
  mcb_mc_launch force{0, 0};
};

namespace mcb {

mcb_status set_error(mcb_ctx *ctx, mcb_status st, const char *fmt, ...);

// Returns a device buffer for `slot` of at least `bytes` (contents undefined).
mcb_status pool_get(mcb_ctx *ctx, int slot, size_t bytes, void **out);

// Reads the transport launch parameters tuned for this GPU from the file MCB_TUNE_FILE names.
void tune_file_load(mcb_ctx *ctx);

#define MCB_CUDA(ctx, call)                                                                      \
  do {                                                                                           \
    cudaError_t _e = (call);                                                                     \
    if (_e != cudaSuccess)                                                                       \
      return ::mcb::set_error((ctx), _e == cudaErrorMemoryAllocation ? MCB_ENOMEM : MCB_ECUDA,   \
                              "%s failed: %s (%s:%d)", #call, cudaGetErrorString(_e), __FILE__, \
                              __LINE__);                                                         \
  } while (0)

#define MCB_TRY(expr)                 \
  do {                                \
    mcb_status _s = (expr);           \
    if (_s != MCB_OK) return _s;      \
  } while (0)

// Buffer slots used by the pool.
enum PoolSlot {
  SLOT_MC_INST = 0,
  SLOT_MC_M,
  SLOT_MC_NRM_RAW,
  SLOT_MC_NRM,
  SLOT_MC_TABLES,
  SLOT_MC_S,
  SLOT_MC_ACC,
  SLOT_MC_OUT,
  SLOT_MC_CTR,
  SLOT_MC_PATHS,
  SLOT_HEAT_T = 20,
  SLOT_HEAT_A,
  SLOT_HEAT_M,
  SLOT_HEAT_Q,
  SLOT_HEAT_IB,
  SLOT_HEAT_OMEGA,
  SLOT_HEAT_MISC,
  SLOT_HEAT_SENS,
  SLOT_HEAT_ADJ,
  SLOT_PROBE,
  SLOT_NORMALS,
  SLOT_DOWNSAMPLE,
  SLOT_BATCH_BASE = 40
};

}  // namespace mcb
