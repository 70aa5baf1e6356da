// The learned proposal network (cnn.cu): geometry, parameter layout and the
// launchers the session and the C ABI use.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace gjxl_b200 {

constexpr int kCnnIn = 80;          // input tile side: 64 + 2 * 8 halo
constexpr int kCnnInChannels = 4;   // X, Y, B - Y (scaled), log2 distance
constexpr int kCnnC = 32;           // channels of every hidden layer
constexpr int kCnnStrategies = 27;  // AC strategy logits
constexpr int kCnnHead = 28;        // + the log field scale

// Parameter layout (FP32): conv weights [co][ky][kx][ci] then biases, per
// layer, then the head [k][c] and its biases.
constexpr int kCnnW1 = 0;
constexpr int kCnnB1 = kCnnW1 + kCnnC * 9 * kCnnInChannels;
constexpr int kCnnW2 = kCnnB1 + kCnnC;
constexpr int kCnnB2 = kCnnW2 + kCnnC * 9 * kCnnC;
constexpr int kCnnW3 = kCnnB2 + kCnnC;
constexpr int kCnnB3 = kCnnW3 + kCnnC * 9 * kCnnC;
constexpr int kCnnW4 = kCnnB3 + kCnnC;
constexpr int kCnnB4 = kCnnW4 + kCnnC * 9 * kCnnC;
constexpr int kCnnWh = kCnnB4 + kCnnC;
constexpr int kCnnBh = kCnnWh + kCnnHead * kCnnC;
constexpr int kCnnParams = kCnnBh + kCnnHead;

struct CnnActivations {
  __nv_bfloat16* act[5];  // input, conv1 .. conv4 outputs (NHWC, BF16)
  float* head;            // [n][64][28]
};

size_t CnnWorkspaceBytes(int tiles);
CnnActivations CnnLayout(void* workspace, int tiles);
int CnnGather(const float* opsin, size_t stride, size_t pitch, size_t pw, size_t ph,
              const int* tile_list, int n, float distance, __nv_bfloat16* out,
              cudaStream_t stream);
// tensor_cores: the convolutions as tcgen05 implicit GEMMs (inference);
// otherwise the SIMT kernels the training step's backward pass pairs with.
int CnnForward(const float* params, const CnnActivations& a, int n, cudaStream_t stream,
               bool tensor_cores = false, uint32_t* error = nullptr);
int CnnPropose(const float* head, int n, size_t blocks_x, size_t blocks_y, uint8_t* proposals,
               float* confidence, float* log_scale, cudaStream_t stream);
size_t CnnTrainScratchBytes(int tiles);
int CnnTrainStep(const float* params, const CnnActivations& a, int n, const uint8_t* labels,
                 const float* targets, const float* weights, float qf_weight, float* grads,
                 void* scratch, float* loss, cudaStream_t stream);
// Learned analysis mode.
int CnnTileMasks(const uint8_t* proposals, const float* mass, size_t blocks_x, size_t blocks_y,
                 float confidence, uint8_t* masks, cudaStream_t stream);
int CnnKeptTiles(const uint8_t* masks, size_t tiles, uint32_t* kept, uint32_t* counts,
                 cudaStream_t stream);
int CnnMaskCosts(float* costs, const uint8_t* masks, size_t blocks_x, size_t blocks_y,
                 cudaStream_t stream);
int CnnScaleField(float* field, const float* log_scale, size_t blocks, cudaStream_t stream);
int CnnAdamW(float* params, const float* grads, float* m, float* v, int step, float lr,
             float beta1, float beta2, float eps, float weight_decay, cudaStream_t stream);

}  // namespace gjxl_b200
