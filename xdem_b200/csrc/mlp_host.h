// mlp_host.h — the host object behind an xdem_mlp handle, shared by the
// training code (learn.cu) and the world code that harvests training pairs and
// runs the warm start (api.cu).
#pragma once
#include <cuda_runtime.h>

#include "mlp.cuh"

struct xdem_mlp_s {
  cudaStream_t stream = nullptr;
  float* theta = nullptr;         // FP32 master parameters (MlpLayout)
  float* adam_m = nullptr;        // Adam first moments
  float* adam_v = nullptr;        // Adam second moments
  __nv_bfloat16* wb = nullptr;    // BF16 weight copies (MlpBf16Layout)
  float* grad = nullptr;          // reduced gradient
  float* gpart = nullptr;         // per-block partial gradients
  float* lpart = nullptr;         // per-block partial losses
  int gpart_blocks = 0;
  int64_t adam_t = 0;             // Adam step count
  float scale[xdem::kMlpIn] = {0.25f, 0.25f, 1.0f, 1.0f, 0.5f, 0.5f, 1.0f};
  // training set: features [cap][7] (unscaled), target ratio (NaN: no root),
  // contact flag (0/1)
  float* x = nullptr;
  float* target = nullptr;
  float* contact = nullptr;
  int64_t size = 0, cap = 0;
  int32_t* perm = nullptr;        // sample order of an epoch
  int64_t perm_cap = 0;

  xdem::MlpDev dev() const {
    xdem::MlpDev d;
    d.wb = wb;
    d.theta = theta;
    for (int k = 0; k < xdem::kMlpIn; ++k) d.scale[k] = scale[k];
    return d;
  }
};

// grows the training set to hold `need` samples (keeps the current ones)
cudaError_t mlp_reserve(xdem_mlp_s* m, int64_t need);
