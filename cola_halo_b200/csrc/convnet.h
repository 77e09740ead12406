// Learned force correction: the 3-layer 3x3x3 conv net on the coarse mesh
// (convnet.cu, convnet_tc.cu).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "internal.h"

#define CNET_C 16                          // channels of every activation tensor
#define CNET_LAYER (27 * CNET_C * CNET_C + CNET_C)   // weights + bias of one layer
#define CNET_PARAMS (3 * CNET_LAYER)

struct CNet {
  int N;                       // coarse mesh cells per dimension
  int use_tc;                  // tcgen05 convolution when the mesh allows it
  long long step;              // Adam step count
  float in_scale[2];           // feature scales (delta, phi)
  float out_scale;             // force units per output unit
  float* params;               // float32 masters: per layer W[27][16][16], b[16]
  float* grads;
  float* m1;
  float* m2;
  int* trainable;              // 1 for live weights (masked channels stay 0)
  __nv_bfloat16* wb;           // bf16 weights used by the kernels, 3 x 27*16*16
  __nv_bfloat16* act[3];       // layer inputs: features, hidden 1, hidden 2 [v][16]
  float* out;                  // network output [v][16] (channels 0-2 used)
  float4* out4;                // its channels 0-3 packed [v]: what the interpolation reads
  float* g0;                   // gradient buffers [v][16]
  float* g1;
  __nv_bfloat16* gb;           // bf16 copy of the gradient fed to the data-gradient conv
  float* target;               // residual target [v][3] (in output units)
  float* mass;                 // deposited mass [v]
  double* loss;
  float* phi;                  // potential [v]
  float2* spec;                // half spectrum scratch
  MeshFFT fft;
};

cudaError_t cnet_alloc(CNet* n, int N, unsigned long long seed);
void cnet_free(CNet* n);
cudaError_t cnet_sync_bf16(CNet* n, cudaStream_t st);
cudaError_t cnet_features(CNet* n, const float* delta, cudaStream_t st);
// full: also write the [v][16] output that the loss and the host API read
// (the packed out4 is always written)
cudaError_t cnet_forward(CNet* n, cudaStream_t st, bool full = true);
cudaError_t cnet_loss_grad(CNet* n, double inv_msum, cudaStream_t st);
cudaError_t cnet_backward(CNet* n, cudaStream_t st);
cudaError_t cnet_adam(CNet* n, float lr, cudaStream_t st);
cudaError_t cnet_target(CNet* n, const float* const x[3], long long np, float boxsize,
                        const float* const f_fine[3], const float* const f_coarse[3],
                        cudaStream_t st);
cudaError_t cnet_apply(const CNet* n, const float* const x[3], long long np, float boxsize,
                       float* const f[3], cudaStream_t st);

// tcgen05 convolutions (convnet_tc.cu); cudaErrorNotSupported when the mesh
// is not a multiple of the 128-voxel tile.
cudaError_t conv_tc_forward(const __nv_bfloat16* in, int N, const __nv_bfloat16* w,
                            const float* bias, int act, float* out_f, __nv_bfloat16* out_b,
                            float4* out4, cudaStream_t st);
cudaError_t conv_tc_backward_data(const __nv_bfloat16* g, int N, const __nv_bfloat16* w,
                                  float* out_f, cudaStream_t st);
// Device error word of the tensor-core kernels (bounded waits that gave up).
unsigned conv_tc_error_word();
// Pipeline of the tensor-core convolutions: -1 by mesh size, 0 two stages,
// 1 one stage, 2 the line ring (128^3 only).  -1 returned on a bad value.
int conv_tc_set_variant(int v);
