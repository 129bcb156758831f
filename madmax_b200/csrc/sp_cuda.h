// sp_cuda.h -- CUDA-side internals shared by the .cu translation units:
// device state, the CUDA error check, device buffers and the cache of
// device-resident mesh plans.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "rve_device.cuh"
#include "sp_internal.h"

#define SP_CUDA_TRY(expr)                                                                   \
  do {                                                                                      \
    cudaError_t e_ = (expr);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      return sp_set_error(SP_ERR_CUDA, "%s failed: %s (%s:%d)", #expr, cudaGetErrorString(e_), \
                          __FILE__, __LINE__);                                              \
  } while (0)

#define SP_TRY(expr)        \
  do {                      \
    int rc_ = (expr);       \
    if (rc_) return rc_;    \
  } while (0)

namespace sp {

struct Device {
  int id = -1;
  int nsm = 0;
  cudaStream_t stream = nullptr; // library stream (non-blocking)
};

// Current device of the calling thread, initialised on first use.
// Returns SP_ERR_CUDA (no fallback) when no device is usable.
int device(Device **out);
cudaStream_t pick_stream(void *user_stream, Device *d);

// Device copy of a mesh plan (shared by every RVE of that size).
struct DevPlan {
  int n[3];
  MeshGeo geo;             // h and vol filled per RVE, not here
  int color_off[9];
  int *cols = nullptr;     // [ndof][SP_WP]
  int *nbr = nullptr;      // [nslice][27][32] node-sliced neighbour ids
  uint8_t *slot = nullptr; // [nelm][576]
  int *color_elems = nullptr;
  int boundary_nodes = 0;
  size_t bytes = 0;
  int refs = 0;
  int dev = -1;
};

// Build (or find) the plan for n[3] on the current device.
int plan_acquire(const int *n, DevPlan **out);
void plan_release(DevPlan *p);
// Host-side byte count of a plan's device arrays, without building it.
size_t plan_bytes(const int *n);

MeshGeo make_geo(const int *n, const double *len);

// device allocation helper that records the byte count
int dmalloc(void **p, size_t bytes, size_t *acct);

}  // namespace sp
