// Learned denoiser: a 5-level convolutional U-Net (widths 32-48-64-96-128,
// two 3x3 convolutions per level, 2x2 average pooling, nearest upsampling,
// concatenated skips, 1x1 output), about 1.01M parameters, computed with
// BF16 tensor-core convolutions and FP32 accumulation.
//
// Input per pixel (10 channels, padded to 16): log(1 + colour) RGB, albedo
// RGB, normal XYZ, log(1 + first-hit distance), where colour, albedo and
// depth are the accumulated averages and the normal the normalised sum, as
// RtDenoise prepares them. Output: log(1 + radiance) RGB. Trained with Adam
// on an L1 loss in that log space.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "rt_conv_tc.cuh"

namespace rt {

struct UnetLayer {
    int cin, cout;           // padded input channels, output channels
    size_t wOffset, bOffset; // into the flat parameter vector
};

class Unet {
public:
    explicit Unet(unsigned seed);
    ~Unet();
    Unet(const Unet&) = delete;
    Unet& operator=(const Unet&) = delete;

    size_t paramCount() const { return params_; }
    // Host copies of the FP32 master parameters, in the flat layout (per 3x3
    // layer: weights [tap][cin][cout] then bias [cout]; the 1x1 output layer:
    // weights [cin][3] then bias [3]).
    cudaError_t getParams(float* host) const;
    cudaError_t setParams(const float* host);
    // One forward and backward pass over host AOVs (n x h x w x 10) and
    // targets (n x h x w x 3, linear radiance). Writes the loss and, if
    // grads is not null, the FP32 gradient in the flat layout.
    cudaError_t lossAndGradient(const float* aovs, const float* targets, int n, int h, int w, float* loss,
                                float* grads, std::string& error);
    // Adam steps on random batches (with random flips) of a host data set.
    cudaError_t train(const float* aovs, const float* targets, int count, int h, int w, int steps, int batch,
                      float lr, unsigned seed, float* losses, std::string& error);
    // Inference from device AOV input (w x h x 10 FP32) to device linear
    // radiance (w x h x 3 FP32); any w, h (padded internally to 16).
    cudaError_t inferDevice(const float* aovs, int h, int w, float* radiance, cudaStream_t stream, std::string& error);
    // The same inference straight from a session's running sums (10 four-
    // byte fields per pixel: radiance, albedo and normal sums, coverage) and
    // first-hit distance sums after `samples` paths per pixel: the AOVs are
    // formed inside the input kernel with the expressions of RtxReadAovs, and
    // the output layer writes the cropped radiance directly.
    cudaError_t inferFromSums(const float* sums, const float* depthSums, unsigned samples, int h, int w,
                              float* radiance, cudaStream_t stream);
    // Checkpoint file: parameters, and the Adam state when optimizerState.
    cudaError_t save(const char* path, bool optimizerState, std::string& error) const;
    // After the work has finished: an error if a tensor-core convolution gave
    // up waiting (the flag is cleared).
    cudaError_t checkConvolutions(std::string& error);
    cudaError_t load(const char* path, std::string& error);

private:
    struct Activations;
    cudaError_t ensure(int n, int h, int w, bool training);
    // head (inference): the output head to fuse into the last convolution;
    // *headDone tells whether it was (else A.a[17] holds that layer's output).
    cudaError_t forward(cudaStream_t stream, bool training, bool outputLayer = true, const ConvHead* head = nullptr,
                        bool* headDone = nullptr);
    cudaError_t backward(cudaStream_t stream);
    cudaError_t syncWeights(cudaStream_t stream);

    std::vector<UnetLayer> layers_;
    size_t params_ = 0;
    float* master_ = nullptr;     // FP32 parameters
    float* grad_ = nullptr;       // FP32 gradients
    float* adamM_ = nullptr;
    float* adamV_ = nullptr;
    __nv_bfloat16* wbf_ = nullptr;   // BF16 3x3 weights [tap][cin][cout] per layer (same offsets)
    __nv_bfloat16* wT_ = nullptr;    // BF16 K-major weights [tap][cout][cin] for the forward convolutions
    int* convError_ = nullptr;       // set by a tensor-core convolution whose wait ran past its limit
    long long adamStep_ = 0;
    Activations* act_ = nullptr;
    int n_ = 0, h_ = 0, w_ = 0;
    bool training_ = false;
    cudaStream_t stream_ = nullptr;
};

}  // namespace rt
