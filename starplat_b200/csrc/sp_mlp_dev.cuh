// The scheduler network evaluated inside a kernel, for decisions taken per iteration
// on the device (SSSP's bucket width per epoch, BC's direction per level).
//
// Network (as in sp_mlp.cu): x[SP_MLP_IN] -> tanh(W1 x + b1)[H] -> tanh(W2 h + b2)[H]
// -> w3 . h + b3. `model` packs the SP_MLP_PARAMS parameters, then the feature mean and
// scale (x' = (x - mean) * scale).
#pragma once
#include <cuda_runtime.h>

#include "../../include/starplat_b200.h"

namespace sp {

// The candidate whose score is lowest, among NC rows of raw inputs in shared memory
// (rows[c][i], written by the caller before the call, read only after the first
// barrier). NC x 32 threads of the CTA evaluate the hidden units (NC * 32 <= blockDim.x);
// every thread of the CTA must call it. Every CTA that evaluates the same rows runs the
// same instructions in the same order, so all return the same candidate: a decision
// taken this way needs no barrier between CTAs. Only candidates first .. NC-1 are
// eligible; ties go to the lower index. With dflt >= 0, the result is dflt unless the
// best score is lower than dflt's by more than margin.
template <int NC>
__device__ int mlp_argmin(const float* __restrict__ model, float (*rows)[SP_MLP_IN], int first = 0, int dflt = -1,
                          float margin = 0.0f) {
  constexpr int IN = SP_MLP_IN, H = SP_MLP_HIDDEN;
  constexpr int W1 = 0, B1 = W1 + H * IN, W2 = B1 + H, B2 = W2 + H * H, W3 = B2 + H, B3 = W3 + H;
  static_assert(B3 + 1 == SP_MLP_PARAMS, "parameter layout");
  __shared__ float s_h1[NC][H];
  __shared__ float s_y[NC];
  __shared__ int s_pick;
  const float* mean = model + SP_MLP_PARAMS;
  const float* scale = mean + IN;
  const int t = threadIdx.x;
  __syncthreads();  // the caller's rows are written
  if (t < NC * IN) {
    const int c = t / IN, i = t % IN;
    rows[c][i] = (rows[c][i] - mean[i]) * scale[i];
  }
  __syncthreads();
  const int c = t >> 5, j = t & 31;
  if (c < NC) {
    float z = model[B1 + j];
#pragma unroll
    for (int i = 0; i < IN; ++i) z = fmaf(model[W1 + j * IN + i], rows[c][i], z);
    s_h1[c][j] = tanhf(z);
  }
  __syncthreads();
  if (c < NC) {
    float z = model[B2 + j];
#pragma unroll 8
    for (int k = 0; k < H; ++k) z = fmaf(model[W2 + j * H + k], s_h1[c][k], z);
    float v = model[W3 + j] * tanhf(z);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (j == 0) s_y[c] = model[B3] + v;
  }
  __syncthreads();
  if (t == 0) {
    int best = first;
    for (int k = first + 1; k < NC; ++k)
      if (s_y[k] < s_y[best]) best = k;
    if (dflt >= first && dflt < NC && !(s_y[dflt] - s_y[best] > margin)) best = dflt;
    s_pick = best;
  }
  __syncthreads();
  return s_pick;
}

}  // namespace sp
