// Launch interface of the render, query, sampler and denoise kernels.
#pragma once
#include <string>

#include "rt_integrator.cuh"

namespace rt {

// cuRAND's Sobol direction numbers (host copy), or null with a message.
const unsigned* hostSobolDirections(std::string& error);

struct RenderLaunch {
    SceneView scene;
    Camera cam;
    Settings set;
    int w, h;
    unsigned sample0;            // paths already accumulated per pixel
    const unsigned* passXor;     // [raysPerPixel][kSobolDims]
    const unsigned* seedHash;    // [kSobolDims]
    Accum* sums;                 // w*h running sums (read when sample0 > 0)
    float* depthSums;            // w*h running sums of first-hit distance (an added AOV)
    uchar4* pixels;              // w*h display image
    unsigned long long* counters;  // [0] primary, [1] secondary, [2] shadow rays
    int* errorFlag;              // set to 1 on traversal stack overflow
};

// Work buffers of the wavefront integrator, sized for `capacity` paths in flight.
struct WavefrontBuffers {
    int capacity = 0;
    float4* pathA = nullptr;     // origin.xyz, prevPdf
    float4* pathB = nullptr;     // dir.xyz, pixel index (bits)
    float4* pathC = nullptr;     // throughput.xyz, sample row r (bits)
    float4* radiance = nullptr;  // radiance.xyz, covered (bits)
    float4* albedo = nullptr;    // albedo.xyz
    float4* normal = nullptr;    // normal.xyz
    float4* hits = nullptr;      // per queue slot: distance, u, v, index (bits)
    int* queue[2] = {nullptr, nullptr};   // active path ids, ping-pong
    float4* shadowRay = nullptr;      // origin.xyz, limit
    float4* shadowDir = nullptr;      // dir.xyz, path id (bits)
    float4* shadowContrib = nullptr;  // contribution.xyz
    int* counts = nullptr;            // [0..1] queue sizes, [2] shadow queue size, [3..4] fetch counters
};

// Speed-only knobs of the persistent traversal kernels.
struct TraceTuning {
    int refill = 24;   // refill idle lanes when fewer lanes than this are busy
    int lanes = 2;     // waves in flight (1..kMaxLanes, see WaveOverlap)
    // Traversal stack entries a ray may use before the query stops with the
    // overflow error (1..kStackCapacity). Trees built here never need more
    // than kStackCapacity; a smaller limit forces the error path.
    int stackLimit = kStackCapacity;
};

// Lanes of waves: wave j runs on lane j % lanes, lane 0 on the caller's
// stream and buffers, lane k > 0 on streams[k - 1] with buffers[k - 1], so
// the kernels of one wave fill the SMs while those of another drain (every
// persistent traversal launch ends in a tail of a few slow warps, and shading
// is memory-bound where traversal is not). Only the accumulation is ordered
// across lanes (`accumulated`), which keeps each pixel's samples added in
// sample order.
constexpr int kMaxLanes = 4;
struct WaveOverlap {
    int lanes = 1;
    WavefrontBuffers* buffers[kMaxLanes - 1] = {};
    cudaStream_t streams[kMaxLanes - 1] = {};
    cudaEvent_t joins[kMaxLanes - 1] = {};
    cudaEvent_t fork = nullptr, accumulated = nullptr;
};

cudaError_t allocWavefront(WavefrontBuffers& b, int capacity);
void freeWavefront(WavefrontBuffers& b);

cudaError_t buildSobolTables(const unsigned* dirs, unsigned sample0, int rpp, unsigned seed, unsigned* passXor,
                             unsigned* seedHash, cudaStream_t stream);
// One kernel per path: returns the number of kernel launches in *launches.
cudaError_t launchMegakernel(const RenderLaunch& L, cudaStream_t stream, int* launches);
// Wavefront: generate -> (extend -> shade -> shadow)* per wave. Timing of the
// traversal kernels is accumulated into extendMs/shadowMs when timing != 0.
cudaError_t launchWavefront(const RenderLaunch& L, WavefrontBuffers& b, const TraceTuning& tuning, cudaStream_t stream,
                            int* launches, float* extendMs, float* shadowMs, bool timing,
                            float* primaryMs = nullptr, const WaveOverlap* overlap = nullptr);

// fetch: one device int of scratch (the work counter of the persistent kernel).
cudaError_t launchQueries(const uint4* wide, const float4* packed, const float4* queries /*2 per query*/, int count,
                          int any, float4* hits, int* fetch, int* errorFlag, int wideDepth, const TraceTuning& tuning,
                          cudaStream_t stream);
cudaError_t launchSobolSamples(const unsigned* dirs, const unsigned* pixel, const unsigned* sample, const unsigned* seed,
                               int count, int ndim, float* out, cudaStream_t stream);
// Denoise: prepare guides from the running sums, filter, tonemap into pixels.
// work holds 4 float4 regions of w*h: colour, albedo, normal, ping-pong; after
// the kAtrousPasses (odd) passes the filtered colour is in region 3.
constexpr int kAtrousPasses = 5;
cudaError_t launchDenoise(const Accum* sums, unsigned samples, int w, int h, float exposure, float4* work /*4*w*h*/,
                          uchar4* pixels, cudaStream_t stream);
// The last denoise's linear radiance (srcStride floats per pixel at src) as 3
// floats per pixel, uncovered pixels 0.
cudaError_t launchDenoisedRgb(const Accum* sums, const float* src, int srcStride, int count, float* out,
                              cudaStream_t stream);

// Denoiser input: per pixel colour = radiance / samples, albedo / samples,
// normalised normal sum (renderer.cu:422-428) and depth / samples (10 floats).
cudaError_t launchAovs(const Accum* sums, const float* depthSums, unsigned samples, int count, float* aov,
                       cudaStream_t stream);
// Tonemap linear radiance (3 floats per pixel) into the display image;
// uncovered pixels stay black (renderer.cu:429-435).
cudaError_t launchPresentRadiance(const Accum* sums, const float* radiance, int count, float exposure, uchar4* pixels,
                                  cudaStream_t stream);

}  // namespace rt
