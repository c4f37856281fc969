// Scene upload and preparation on the device (see rt_upload.cuh).
#include <algorithm>
#include <chrono>
#include <cstring>
#include <vector>

#include "rt_upload.cuh"

namespace rt {
namespace {

constexpr int kColourComponents = 6;  // color.xyz, specularColor.xyz
constexpr int kBlock = 256;

__device__ __forceinline__ float* component(SceneTri* t, int k) {
    return k < 3 ? &t->color.x + k : &t->specularColor.x + (k - 3);
}

__device__ __forceinline__ unsigned mixBits(unsigned k) {
    k ^= k >> 16; k *= 0x85ebca6bu;
    k ^= k >> 13; k *= 0xc2b2ae35u;
    return k ^ (k >> 16);
}

// Collects the distinct bit patterns of components that take the powf branch
// (!(c <= .04045f), NaN included) into an open-addressing set. Slots hold
// (1 << 32 | bits), 0 when empty. Stops with *overflow = 1 when `limit`
// distinct values are exceeded (the caller retries with a larger set).
__global__ void collectColoursKernel(const SceneTri* tris, long long components, unsigned long long* table,
                                     unsigned mask, unsigned* slotIndex, unsigned* distinct, unsigned limit,
                                     unsigned* values, int* overflow) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= components) return;
    const float c = *component(const_cast<SceneTri*>(tris) + i / kColourComponents, (int)(i % kColourComponents));
    if (c <= .04045f) return;
    const unsigned bits = __float_as_uint(c);
    const unsigned long long entry = (1ull << 32) | bits;
    unsigned slot = mixBits(bits) & mask;
    for (unsigned probe = 0; probe <= mask; probe++) {
        unsigned long long cur = *reinterpret_cast<volatile unsigned long long*>(&table[slot]);
        if (cur == entry) return;
        if (cur == 0ull) {
            unsigned long long prev = atomicCAS(&table[slot], 0ull, entry);
            if (prev == 0ull) {
                unsigned k = atomicAdd(distinct, 1u);
                if (k >= limit) { atomicExch(overflow, 1); return; }
                values[k] = bits;
                slotIndex[slot] = k;
                return;
            }
            if (prev == entry) return;
        }
        slot = (slot + 1u) & mask;
    }
    atomicExch(overflow, 1);
}

// Decodes every component in place: the division branch here, the powf
// branch through the host-decoded table.
__global__ void applyColoursKernel(SceneTri* tris, long long components, const unsigned long long* table,
                                   unsigned mask, const unsigned* slotIndex, const float* decoded, int* missing) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= components) return;
    float* p = component(tris + i / kColourComponents, (int)(i % kColourComponents));
    const float c = *p;
    if (c <= .04045f) { *p = c / 12.92f; return; }
    const unsigned bits = __float_as_uint(c);
    const unsigned long long entry = (1ull << 32) | bits;
    unsigned slot = mixBits(bits) & mask;
    for (unsigned probe = 0; probe <= mask; probe++) {
        unsigned long long cur = table[slot];
        if (cur == entry) { *p = decoded[slotIndex[slot]]; return; }
        if (cur == 0ull) break;
        slot = (slot + 1u) & mask;
    }
    atomicExch(missing, 1);
}

// Emitter count per block (emission > 0, the reference's test).
__global__ void emitterCountKernel(const SceneTri* tris, int n, unsigned* blockCounts) {
    __shared__ unsigned warpCounts[kBlock / 32];
    int i = blockIdx.x * kBlock + threadIdx.x;
    bool e = i < n && tris[i].emission > 0;
    unsigned m = __ballot_sync(0xFFFFFFFFu, e);
    if ((threadIdx.x & 31) == 0) warpCounts[threadIdx.x >> 5] = __popc(m);
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned s = 0;
        for (int w = 0; w < kBlock / 32; w++) s += warpCounts[w];
        blockCounts[blockIdx.x] = s;
    }
}

// Exclusive scan of the block counts in place (one block of 1024 threads).
__global__ void scanCountsKernel(unsigned* counts, int blocks, unsigned* total) {
    __shared__ unsigned sums[1024];
    const int per = (blocks + 1023) / 1024;
    const int begin = min(blocks, (int)threadIdx.x * per), end = min(blocks, begin + per);
    unsigned s = 0;
    for (int b = begin; b < end; b++) s += counts[b];
    sums[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned run = 0;
        for (int k = 0; k < 1024; k++) { unsigned v = sums[k]; sums[k] = run; run += v; }
        *total = run;
    }
    __syncthreads();
    unsigned run = sums[threadIdx.x];
    for (int b = begin; b < end; b++) { unsigned v = counts[b]; counts[b] = run; run += v; }
}

// Emitters in triangle order with their areas (renderer.cu:350-351).
__global__ void emitterScatterKernel(const SceneTri* tris, int n, const unsigned* blockOffsets, int* emitterTri,
                                     float* emitterArea) {
    __shared__ unsigned warpBase[kBlock / 32];
    const int i = blockIdx.x * kBlock + threadIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool e = i < n && tris[i].emission > 0;
    const unsigned m = __ballot_sync(0xFFFFFFFFu, e);
    if (lane == 0) warpBase[warp] = __popc(m);
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned run = 0;
        for (int w = 0; w < kBlock / 32; w++) { unsigned v = warpBase[w]; warpBase[w] = run; run += v; }
    }
    __syncthreads();
    if (e) {
        const unsigned pos = blockOffsets[blockIdx.x] + warpBase[warp] + __popc(m & ((1u << lane) - 1u));
        const SceneTri& t = tris[i];
        float3 an = cross(t.edge1, t.edge2);
        emitterTri[pos] = i;
        emitterArea[pos] = .5f * sqrtf(dot(an, an));
    }
}

// Cumulative areas in triangle order by one warp: every lane runs the same
// left-to-right chain of additions, so the sums round as the reference's.
__global__ void cumulativeAreaKernel(const int* emitterTri, const float* emitterArea, int count, Light* lights,
                                     float* totalArea) {
    const int lane = threadIdx.x;
    float carry = 0.0f;
    for (int base = 0; base < count; base += 32) {
        const int l = base + lane;
        const float a = l < count ? emitterArea[l] : 0.0f;
        const int m = min(32, count - base);
        float run = carry, mine = 0.0f;
        for (int k = 0; k < m; k++) {
            run = run + __shfl_sync(0xFFFFFFFFu, a, k);
            if (k == lane) mine = run;
        }
        if (l < count) lights[l] = Light{emitterTri[l], mine};
        carry = run;
    }
    if (lane == 0) *totalArea = carry;
}

inline int gridFor(long long n, int block) { return (int)((n + block - 1) / block); }

}  // namespace

cudaError_t uploadScene(const void* triangles, int count, cudaStream_t stream, SceneTri** dTrisOut, Light** dLightsOut,
                        UploadResult& R, std::string& error) {
    const auto t0 = std::chrono::steady_clock::now();
    *dTrisOut = nullptr;
    *dLightsOut = nullptr;
    R = UploadResult{};
    SceneTri* dTris = nullptr;
    Light* dLights = nullptr;
    unsigned long long* table = nullptr;
    unsigned *slotIndex = nullptr, *values = nullptr, *counters = nullptr, *blockCounts = nullptr;
    float *decoded = nullptr, *emitterArea = nullptr;
    int* emitterTri = nullptr;
    cudaError_t e = cudaSuccess;
    const long long components = (long long)count * kColourComponents;
    const int blocks = gridFor(count, kBlock);
    std::vector<unsigned> hostValues;
    std::vector<float> hostDecoded;
    unsigned hostCounters[4] = {0, 0, 0, 0};
    float area = 0.0f;
    unsigned cap = 1u << 12;  // set slots; grows until the distinct values fit in half
#define RT_TRY(x) do { if ((e = (x)) != cudaSuccess) goto done; } while (0)
    RT_TRY(rt::deviceAlloc(&dTris, sizeof(SceneTri) * (size_t)count));
    RT_TRY(cudaMemcpyAsync(dTris, triangles, sizeof(SceneTri) * (size_t)count, cudaMemcpyHostToDevice, stream));
    // counters: [0] distinct values, [1] overflow, [2] missing, [3] emitters
    RT_TRY(rt::deviceAlloc(&counters, 4 * sizeof(unsigned)));
    for (;;) {
        RT_TRY(rt::deviceAlloc(&table, sizeof(unsigned long long) * cap));
        RT_TRY(rt::deviceAlloc(&slotIndex, sizeof(unsigned) * cap));
        RT_TRY(rt::deviceAlloc(&values, sizeof(unsigned) * (cap / 2)));
        RT_TRY(cudaMemsetAsync(table, 0, sizeof(unsigned long long) * cap, stream));
        RT_TRY(cudaMemsetAsync(counters, 0, 4 * sizeof(unsigned), stream));
        collectColoursKernel<<<gridFor(components, kBlock), kBlock, 0, stream>>>(dTris, components, table, cap - 1,
                                                                                  slotIndex, &counters[0], cap / 2,
                                                                                  values, reinterpret_cast<int*>(&counters[1]));
        RT_TRY(cudaGetLastError());
        RT_TRY(cudaMemcpyAsync(hostCounters, counters, sizeof(hostCounters), cudaMemcpyDeviceToHost, stream));
        RT_TRY(cudaStreamSynchronize(stream));
        if (!hostCounters[1]) break;
        cudaFree(table); cudaFree(slotIndex); cudaFree(values);
        table = nullptr; slotIndex = nullptr; values = nullptr;
        if ((unsigned long long)cap * 4 > (1ull << 31)) { error = "too many distinct colour values"; e = cudaErrorInvalidValue; goto done; }
        cap *= 4;
    }
    R.distinctColours = (int)hostCounters[0];
    hostValues.resize(hostCounters[0]);
    hostDecoded.resize(hostCounters[0]);
    if (!hostValues.empty()) {
        RT_TRY(cudaMemcpy(hostValues.data(), values, sizeof(unsigned) * hostValues.size(), cudaMemcpyDeviceToHost));
        for (size_t k = 0; k < hostValues.size(); k++) {
            float c;
            std::memcpy(&c, &hostValues[k], sizeof(c));
            hostDecoded[k] = srgbToLinear(c);  // the reference's host expression (renderer.cu:84-85,347)
        }
        RT_TRY(rt::deviceAlloc(&decoded, sizeof(float) * hostDecoded.size()));
        RT_TRY(cudaMemcpyAsync(decoded, hostDecoded.data(), sizeof(float) * hostDecoded.size(), cudaMemcpyHostToDevice, stream));
    }
    applyColoursKernel<<<gridFor(components, kBlock), kBlock, 0, stream>>>(dTris, components, table, cap - 1, slotIndex,
                                                                            decoded, reinterpret_cast<int*>(&counters[2]));
    RT_TRY(cudaGetLastError());
    // Emitters.
    RT_TRY(rt::deviceAlloc(&blockCounts, sizeof(unsigned) * (size_t)blocks));
    emitterCountKernel<<<blocks, kBlock, 0, stream>>>(dTris, count, blockCounts);
    scanCountsKernel<<<1, 1024, 0, stream>>>(blockCounts, blocks, &counters[3]);
    RT_TRY(cudaGetLastError());
    RT_TRY(cudaMemcpyAsync(hostCounters, counters, sizeof(hostCounters), cudaMemcpyDeviceToHost, stream));
    RT_TRY(cudaStreamSynchronize(stream));
    if (hostCounters[2]) { error = "colour decode table is missing a value"; e = cudaErrorUnknown; goto done; }
    R.lightCount = (int)hostCounters[3];
    if (R.lightCount > 0) {
        RT_TRY(rt::deviceAlloc(&emitterTri, sizeof(int) * (size_t)R.lightCount));
        RT_TRY(rt::deviceAlloc(&emitterArea, sizeof(float) * (size_t)R.lightCount + sizeof(float)));
        RT_TRY(rt::deviceAlloc(&dLights, sizeof(Light) * (size_t)R.lightCount));
        emitterScatterKernel<<<blocks, kBlock, 0, stream>>>(dTris, count, blockCounts, emitterTri, emitterArea);
        cumulativeAreaKernel<<<1, 32, 0, stream>>>(emitterTri, emitterArea, R.lightCount, dLights,
                                                   emitterArea + R.lightCount);
        RT_TRY(cudaGetLastError());
        RT_TRY(cudaMemcpyAsync(&area, emitterArea + R.lightCount, sizeof(float), cudaMemcpyDeviceToHost, stream));
    }
    RT_TRY(cudaStreamSynchronize(stream));
    R.lightArea = area;
#undef RT_TRY
done:
    cudaFree(table); cudaFree(slotIndex); cudaFree(values); cudaFree(counters); cudaFree(blockCounts);
    cudaFree(decoded); cudaFree(emitterArea); cudaFree(emitterTri);
    if (e != cudaSuccess) {
        cudaFree(dTris);
        cudaFree(dLights);
        if (error.empty()) error = std::string("scene upload: ") + cudaGetErrorString(e);
        return e;
    }
    *dTrisOut = dTris;
    *dLightsOut = dLights;
    R.ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return cudaSuccess;
}

}  // namespace rt
