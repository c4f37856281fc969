// Render, query, sampler and denoise kernels for sm_100a.
//
// Two integrators produce bit-identical accumulations:
//  - wavefront (default): per wave of paths (one raysPerPixel row r over a
//    range of pixels) a generate kernel writes camera rays, then for every
//    bounce an extend kernel (closest hit) runs over the compacted queue of
//    live paths, a shade kernel applies the bounce and compacts survivors and
//    light-sample rays into queues with warp-aggregated atomics, and a shadow
//    kernel (any hit) resolves the light samples; an accumulate kernel adds
//    the wave's paths to the running sums in row order. Traversal kernels only
//    hold a ray and its stack, so they run at high occupancy on coherent work.
//  - one kernel per pixel (megakernel), the reference's launch shape with the
//    same traversal and shading code.
// Traversal stacks live in shared memory, one column per thread.
#include <vector>

#include "rt_render.cuh"
#include "rt_trace.cuh"

namespace rt {
namespace {

constexpr int kTileX = 16, kTileY = 8, kMegaBlock = kTileX * kTileY;
// Resident blocks per SM the traversal kernels are compiled for: 8 caps them
// at 64 registers (16-40 bytes of spills) for 32 resident warps. Measured on
// the 1M-triangle workload with waves of 2^24 paths: 6 blocks (77-79
// registers) 2,841 Mrays/s, 7 (72) 2,972, 8 (64) 3,003.
constexpr int kTraceMinBlocks = 8;

__global__ void sobolTablesKernel(const unsigned* dirs, unsigned sample0, int rpp, unsigned seed, unsigned* passXor,
                                  unsigned* seedHash) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int passEntries = rpp * kSobolDims;
    if (i < passEntries) {
        int r = i / kSobolDims, d = i % kSobolDims;
        passXor[i] = sobolXor(dirs, sample0 + (unsigned)r, (unsigned)d);
    } else if (i < passEntries + kSobolDims) {
        int d = i - passEntries;
        seedHash[d] = sobolHash(seed + (unsigned)d * 0x9e3779b9u);
    }
}

__device__ __forceinline__ void flushCounters(unsigned long long* counters, unsigned a, unsigned b, unsigned c) {
    unsigned sa = __reduce_add_sync(0xFFFFFFFFu, a), sb = __reduce_add_sync(0xFFFFFFFFu, b),
             sc = __reduce_add_sync(0xFFFFFFFFu, c);
    if ((threadIdx.x & 31) == 0) {
        if (sa) atomicAdd(&counters[0], (unsigned long long)sa);
        if (sb) atomicAdd(&counters[1], (unsigned long long)sb);
        if (sc) atomicAdd(&counters[2], (unsigned long long)sc);
    }
}

__global__ void __launch_bounds__(kMegaBlock) megakernel(RenderLaunch L) {
    extern __shared__ uint2 smemStack[];
    uint2* stack = smemStack + threadIdx.x;
    const int stride = kMegaBlock;
    int x = blockIdx.x * kTileX + (threadIdx.x % kTileX);
    int y = blockIdx.y * kTileY + (threadIdx.x / kTileX);
    unsigned nPrimary = 0, nSecondary = 0, nShadow = 0;
    int overflow = 0;
    if (x < L.w && y < L.h)
        renderPixel(L.scene, L.cam, L.set, x, y, L.w, L.h, L.sample0, L.passXor, L.seedHash, L.sums, L.depthSums,
                    L.pixels, stack, stride, &overflow, nPrimary, nSecondary, nShadow);
    flushCounters(L.counters, nPrimary, nSecondary, nShadow);
    if (overflow) atomicExch(L.errorFlag, 1);
}

// ---- wavefront stages ----
// A wave is the paths [start, start + n) of a pass, path k being sample row
// k / (w * h) of pixel k % (w * h); a wave may span several sample rows.
struct WaveArgs {
    RenderLaunch L;
    int start, n;
};
__device__ __forceinline__ int waveRow(const WaveArgs& A, int p) { return (A.start + p) / (A.L.w * A.L.h); }
__device__ __forceinline__ int wavePixel(const WaveArgs& A, int p) { return (A.start + p) % (A.L.w * A.L.h); }

__global__ void generateKernel(WaveArgs A, WavefrontBuffers B) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= A.n) return;
    int pix = wavePixel(A, p);
    int x = pix % A.L.w, y = pix / A.L.w;
    Sampler rng{A.L.passXor + waveRow(A, p) * kSobolDims, A.L.seedHash, (unsigned)pix, 0u};
    PathState st = startPath(A.L.cam, A.L.set, x, y, A.L.w, A.L.h, rng);
    B.pathA[p] = make_float4(st.origin.x, st.origin.y, st.origin.z, 0.0f);
    B.pathB[p] = make_float4(st.dir.x, st.dir.y, st.dir.z, 0.0f);
    B.pathC[p] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
    B.radiance[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    B.albedo[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    B.normal[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    B.queue[0][p] = p;
    if (p == 0) { B.counts[0] = A.n; B.counts[1] = 0; B.counts[2] = 0; }
}

// Closest hit for every queued path (persistent, dynamic fetch).
struct ExtendIO {
    const int* queue;
    const float4 *pathA, *pathB;
    float4* hits;
    __device__ void load(int k, float3& o, float3& d, float& limit, unsigned&) const {
        int p = queue[k];
        float4 a = pathA[p], b = pathB[p];
        o = v3(a.x, a.y, a.z); d = v3(b.x, b.y, b.z); limit = 1e30f;
    }
    __device__ void store(int k, const Hit& h) const {
        hits[queue[k]] = make_float4(h.distance, h.u, h.v, __int_as_float(h.index));
    }
};
__global__ void __launch_bounds__(kTraceBlock, kTraceMinBlocks) extendKernel(const uint4* wide, const float4* packed, WavefrontBuffers B,
                                                            int q, unsigned long long* counter, int* errorFlag,
                                                            int stackLimit, int refill) {
    ExtendIO io{B.queue[q], B.pathA, B.pathB, B.hits};
    persistentTrace<false>(io, B.counts[q], wide, packed, &B.counts[3], counter, errorFlag, stackLimit, refill);
}

// Appends to a queue with one atomic per warp.
__device__ __forceinline__ int warpAppend(int* counter, bool want) {
    unsigned mask = __ballot_sync(0xFFFFFFFFu, want);
    if (!mask) return -1;
    int lane = threadIdx.x & 31;
    int leader = __ffs(mask) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(counter, __popc(mask));
    base = __shfl_sync(0xFFFFFFFFu, base, leader);
    return want ? base + __popc(mask & ((1u << lane) - 1u)) : -1;
}

__global__ void shadeKernel(WaveArgs A, WavefrontBuffers B, int q, int bounce) {
    int count = B.counts[q];
    int nq = q ^ 1;
    int stride = gridDim.x * blockDim.x;
    int limit = ((count + 31) / 32) * 32;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < limit; k += stride) {
        bool valid = k < count;
        bool cont = false, shadow = false;
        int p = 0;
        ShadowRequest req;
        if (valid) {
            p = B.queue[q][k];
            float4 a = B.pathA[p], b = B.pathB[p], c = B.pathC[p], rad = B.radiance[p], hv = B.hits[p];
            PathState st;
            st.origin = v3(a.x, a.y, a.z); st.prevPdf = a.w;
            st.dir = v3(b.x, b.y, b.z);
            st.throughput = v3(c.x, c.y, c.z);
            st.radiance = v3(rad.x, rad.y, rad.z); st.covered = __float_as_uint(rad.w);
            float4 al = B.albedo[p], no = B.normal[p];
            st.albedo = v3(al.x, al.y, al.z); st.normal = v3(no.x, no.y, no.z);
            st.depth = al.w;
            Hit h{__float_as_int(hv.w), hv.x, hv.y, hv.z};
            Sampler rng{A.L.passXor + waveRow(A, p) * kSobolDims, A.L.seedHash, (unsigned)wavePixel(A, p),
                        4u + 8u * (unsigned)bounce};
            unsigned f = shadeBounce(A.L.scene, A.L.set, bounce, st, h, rng, req);
            cont = (f & kContinue) != 0;
            shadow = (f & kShadow) != 0;
            B.pathA[p] = make_float4(st.origin.x, st.origin.y, st.origin.z, st.prevPdf);
            B.pathB[p] = make_float4(st.dir.x, st.dir.y, st.dir.z, 0.0f);
            B.pathC[p] = make_float4(st.throughput.x, st.throughput.y, st.throughput.z, 0.0f);
            B.radiance[p] = make_float4(st.radiance.x, st.radiance.y, st.radiance.z, __uint_as_float(st.covered));
            if (bounce == 0) {
                B.albedo[p] = make_float4(st.albedo.x, st.albedo.y, st.albedo.z, st.depth);
                B.normal[p] = make_float4(st.normal.x, st.normal.y, st.normal.z, 0.0f);
            }
        }
        int slot = warpAppend(&B.counts[nq], cont);
        if (slot >= 0) B.queue[nq][slot] = p;
        int sslot = warpAppend(&B.counts[2], shadow);
        if (sslot >= 0) {
            B.shadowRay[sslot] = make_float4(req.origin.x, req.origin.y, req.origin.z, req.limit);
            B.shadowDir[sslot] = make_float4(req.dir.x, req.dir.y, req.dir.z, __int_as_float(p));
            B.shadowContrib[sslot] = make_float4(req.contribution.x, req.contribution.y, req.contribution.z, 0.0f);
        }
    }
}

// Light-sample visibility for every queued shadow ray (persistent, dynamic
// fetch); unoccluded samples add their contribution to the path's radiance.
struct ShadowIO {
    const float4 *ray, *dir, *contrib;
    float4* radiance;
    __device__ void load(int k, float3& o, float3& d, float& limit, unsigned&) const {
        float4 a = ray[k], b = dir[k];
        o = v3(a.x, a.y, a.z); d = v3(b.x, b.y, b.z); limit = a.w;
    }
    __device__ void store(int k, const Hit& h) const {
        if (h.index >= 0) return;
        int p = __float_as_int(dir[k].w);
        float4 c = contrib[k], rad = radiance[p];
        radiance[p] = make_float4(rad.x + c.x, rad.y + c.y, rad.z + c.z, rad.w);
    }
};
__global__ void __launch_bounds__(kTraceBlock, kTraceMinBlocks) shadowKernel(const uint4* wide, const float4* packed, WavefrontBuffers B,
                                                            unsigned long long* counter, int* errorFlag,
                                                            int stackLimit, int refill) {
    ShadowIO io{B.shadowRay, B.shadowDir, B.shadowContrib, B.radiance};
    persistentTrace<true>(io, B.counts[2], wide, packed, &B.counts[4], counter, errorFlag, stackLimit, refill);
}

__global__ void resetQueuesKernel(WavefrontBuffers B, int q) {
    if (threadIdx.x == 0) { B.counts[q ^ 1] = 0; B.counts[2] = 0; B.counts[3] = 0; B.counts[4] = 0; }
}

// Adds paths [first, first + count) of the wave (all of one sample row) to
// their pixels' sums; the rows of a wave are added by successive launches, so
// each pixel's samples are added in sample order.
__global__ void accumulateKernel(WaveArgs A, WavefrontBuffers B, int firstPath, int count) {
    int p = firstPath + blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= firstPath + count) return;
    size_t i = (size_t)wavePixel(A, p);
    const int row = waveRow(A, p);
    const bool first = row == 0 && A.L.sample0 == 0;
    Accum total = first ? Accum{v3(0, 0, 0), v3(0, 0, 0), v3(0, 0, 0), 0u} : A.L.sums[i];
    float depthTotal = first ? 0.0f : A.L.depthSums[i];
    float4 rad = B.radiance[p], al = B.albedo[p], no = B.normal[p];
    PathState st;
    st.radiance = v3(rad.x, rad.y, rad.z); st.covered = __float_as_uint(rad.w);
    st.albedo = v3(al.x, al.y, al.z); st.normal = v3(no.x, no.y, no.z);
    addPath(total, st);
    A.L.sums[i] = total;
    A.L.depthSums[i] = depthTotal + al.w;
    if (row == A.L.set.raysPerPixel - 1)
        A.L.pixels[i] = displayPixel(total, A.L.sample0 + (unsigned)A.L.set.raysPerPixel, A.L.set.exposure);
}

// ---- per-ray queries, sampler values ----
struct QueryIO {
    const float4* q;
    float4* out;
    __device__ void load(int k, float3& o, float3& d, float& limit, unsigned&) const {
        float4 a = q[2 * k], b = q[2 * k + 1];
        o = v3(a.x, a.y, a.z); d = v3(a.w, b.x, b.y); limit = b.z;
    }
    __device__ void store(int k, const Hit& h) const {
        out[k] = make_float4(__int_as_float(h.index), h.distance, h.u, h.v);
    }
};
template <bool ANY>
__global__ void __launch_bounds__(kTraceBlock) queryKernel(const uint4* wide, const float4* packed, const float4* q,
                                                           int count, float4* out, int* fetch, int* errorFlag,
                                                           int stackLimit, int refill) {
    QueryIO io{q, out};
    persistentTrace<ANY>(io, count, wide, packed, fetch, nullptr, errorFlag, stackLimit, refill);
}

__global__ void sobolSamplesKernel(const unsigned* dirs, const unsigned* pixel, const unsigned* sample,
                                   const unsigned* seed, int count, int ndim, float* out) {
    long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (long long)count * ndim) return;
    int i = (int)(k / ndim), d = (int)(k % ndim);
    out[k] = sobolDirect(dirs, pixel[i], sample[i], seed[i], (unsigned)d);
}

// ---- denoise: guides, edge-avoiding a-trous wavelet filter, present ----
__global__ void denoisePrepareKernel(const Accum* sums, unsigned samples, int count, float4* color, float4* albedo,
                                     float4* normal) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    Accum s = sums[i];
    float inv = 1.0f / (float)samples;
    float3 c = scale(s.radiance, inv), a = scale(s.albedo, inv), n = normalize(s.normal);
    color[i] = make_float4(c.x, c.y, c.z, s.covered ? 1.0f : 0.0f);
    albedo[i] = make_float4(a.x, a.y, a.z, 0.0f);
    normal[i] = make_float4(n.x, n.y, n.z, 0.0f);
}
__global__ void atrousKernel(const float4* in, const float4* albedo, const float4* normal, float4* out, int w, int h,
                             int step, float colorPhi) {
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const float kernel[3] = {3.0f / 8.0f, 1.0f / 4.0f, 1.0f / 16.0f};
    int i = y * w + x;
    float4 c0 = in[i], a0 = albedo[i], n0 = normal[i];
    if (c0.w == 0.0f) { out[i] = c0; return; }
    float3 sum = v3(0, 0, 0);
    float wsum = 0.0f;
    for (int dy = -2; dy <= 2; dy++)
        for (int dx = -2; dx <= 2; dx++) {
            int xx = x + dx * step, yy = y + dy * step;
            if (xx < 0 || yy < 0 || xx >= w || yy >= h) continue;
            int j = yy * w + xx;
            float4 c = in[j];
            if (c.w == 0.0f) continue;
            float4 a = albedo[j], n = normal[j];
            float3 dc = v3(c.x - c0.x, c.y - c0.y, c.z - c0.z);
            float3 da = v3(a.x - a0.x, a.y - a0.y, a.z - a0.z);
            float wc = expf(-dot(dc, dc) / colorPhi);
            float wa = expf(-dot(da, da) / 0.02f);
            float wn = powf(fmaxf(0.0f, n.x * n0.x + n.y * n0.y + n.z * n0.z), 64.0f);
            float wk = kernel[abs(dx)] * kernel[abs(dy)] * wc * wa * wn;
            sum = add(sum, scale(v3(c.x, c.y, c.z), wk));
            wsum += wk;
        }
    float3 r = wsum > 0 ? scale(sum, 1.0f / wsum) : v3(c0.x, c0.y, c0.z);
    out[i] = make_float4(r.x, r.y, r.z, c0.w);
}
__global__ void denoisePresentKernel(const Accum* sums, const float4* color, int count, float exposure, uchar4* pixels) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    float4 c4 = color[i];
    float3 c = sums[i].covered ? v3(c4.x, c4.y, c4.z) : v3(0, 0, 0);
    pixels[i] = make_uchar4(tonemap(c.x, exposure), tonemap(c.y, exposure), tonemap(c.z, exposure), 255);
}

__global__ void aovKernel(const Accum* sums, const float* depthSums, unsigned samples, int count, float* aov) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    Accum s = sums[i];
    float inv = 1.0f / (float)samples;
    float3 c = scale(s.radiance, inv), a = scale(s.albedo, inv), n = normalize(s.normal);
    float* o = aov + (size_t)i * 10;
    o[0] = c.x; o[1] = c.y; o[2] = c.z;
    o[3] = a.x; o[4] = a.y; o[5] = a.z;
    o[6] = n.x; o[7] = n.y; o[8] = n.z;
    o[9] = depthSums[i] * inv;
}
__global__ void presentRadianceKernel(const Accum* sums, const float* radiance, int count, float exposure,
                                      uchar4* pixels) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float* r = radiance + (size_t)i * 3;
    float3 c = sums[i].covered ? v3(r[0], r[1], r[2]) : v3(0, 0, 0);
    pixels[i] = make_uchar4(tonemap(c.x, exposure), tonemap(c.y, exposure), tonemap(c.z, exposure), 255);
}

inline int blocks(long long n, int b) { return (int)((n + b - 1) / b); }

int smCount() {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    return sms;
}
int persistentBlocks(int blockSize) {
    int perSm = 2048 / blockSize;
    return smCount() * (perSm > 0 ? perSm : 1);
}
// Resident blocks of a traversal kernel, for a grid of exactly one wave.
template <class K>
int traceBlocks(K kernel, size_t smem) {
    int perSm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kernel, kTraceBlock, smem) != cudaSuccess || perSm <= 0)
        perSm = 1;
    return smCount() * perSm;
}
constexpr size_t kTraceSmem = traceSharedBytes(kTraceBlock);

}  // namespace

cudaError_t allocWavefront(WavefrontBuffers& b, int capacity) {
    freeWavefront(b);
    size_t n = (size_t)capacity;
    cudaError_t e;
#define RT_ALLOC(p, count) if ((e = rt::deviceAlloc(reinterpret_cast<void**>(&(p)), sizeof(*(p)) * (count))) != cudaSuccess) { freeWavefront(b); return e; }
    RT_ALLOC(b.pathA, n); RT_ALLOC(b.pathB, n); RT_ALLOC(b.pathC, n);
    RT_ALLOC(b.radiance, n); RT_ALLOC(b.albedo, n); RT_ALLOC(b.normal, n); RT_ALLOC(b.hits, n);
    RT_ALLOC(b.queue[0], n); RT_ALLOC(b.queue[1], n);
    RT_ALLOC(b.shadowRay, n); RT_ALLOC(b.shadowDir, n); RT_ALLOC(b.shadowContrib, n);
    RT_ALLOC(b.counts, 8);
#undef RT_ALLOC
    b.capacity = capacity;
    return cudaSuccess;
}
void freeWavefront(WavefrontBuffers& b) {
    void* owned[] = {b.pathA, b.pathB, b.pathC, b.radiance, b.albedo, b.normal, b.hits, b.queue[0], b.queue[1],
                     b.shadowRay, b.shadowDir, b.shadowContrib, b.counts};
    for (void* p : owned)
        if (p) cudaFree(p);
    b = WavefrontBuffers{};
}

cudaError_t buildSobolTables(const unsigned* dirs, unsigned sample0, int rpp, unsigned seed, unsigned* passXor,
                             unsigned* seedHash, cudaStream_t stream) {
    int total = (rpp + 1) * kSobolDims;
    sobolTablesKernel<<<blocks(total, 256), 256, 0, stream>>>(dirs, sample0, rpp, seed, passXor, seedHash);
    return cudaGetLastError();
}

cudaError_t launchMegakernel(const RenderLaunch& L, cudaStream_t stream, int* launches) {
    size_t smem = sizeof(uint2) * kStackCapacity * kMegaBlock;
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(megakernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        configured = true;
    }
    dim3 grid((L.w + kTileX - 1) / kTileX, (L.h + kTileY - 1) / kTileY);
    megakernel<<<grid, kMegaBlock, smem, stream>>>(L);
    if (launches) *launches = 1;
    return cudaGetLastError();
}

cudaError_t launchWavefront(const RenderLaunch& L, WavefrontBuffers& B, const TraceTuning& tuning, cudaStream_t stream,
                            int* launches, float* extendMs, float* shadowMs, bool timing, float* primaryMs,
                            const WaveOverlap* overlap) {
    static int extendBlocks = 0, shadowBlocks = 0;
    if (!extendBlocks) {
        extendBlocks = traceBlocks(extendKernel, kTraceSmem);
        shadowBlocks = traceBlocks(shadowKernel, kTraceSmem);
    }
    const size_t smem = kTraceSmem;
    const int stackLimit = tuning.stackLimit;
    const int refill = tuning.refill;
    int shadeBlocks = persistentBlocks(256);
    int pixels = L.w * L.h;
    int n = 0;
    static thread_local std::vector<cudaEvent_t> pool;
    struct Mark { cudaEvent_t a, b; int kind; };  // 0 primary closest-hit, 1 secondary, 2 shadow
    std::vector<Mark> marks;
    auto event = [&](size_t k) -> cudaEvent_t {
        while (pool.size() <= k) { cudaEvent_t e; cudaEventCreate(&e); pool.push_back(e); }
        return pool[k];
    };
    size_t ev = 0;
    int nLanes = overlap ? std::max(1, std::min(overlap->lanes, kMaxLanes)) : 1;
    for (int k = 1; k < nLanes; k++)
        if (!overlap->buffers[k - 1] || !overlap->streams[k - 1] || overlap->buffers[k - 1]->capacity != B.capacity)
            nLanes = 1;
    const bool two = nLanes > 1;
    WavefrontBuffers* lanes[kMaxLanes] = {&B};
    cudaStream_t laneStream[kMaxLanes] = {stream};
    for (int k = 1; k < nLanes; k++) {
        lanes[k] = overlap->buffers[k - 1];
        laneStream[k] = overlap->streams[k - 1];
    }
    if (two) {
        cudaEventRecord(overlap->fork, stream);  // the other lanes start after the work queued so far
        for (int k = 1; k < nLanes; k++) cudaStreamWaitEvent(laneStream[k], overlap->fork, 0);
    }
    int wave = 0;
    const int total = pixels * L.set.raysPerPixel;  // paths of the pass (at most 4096^2 * 16 < 2^31)
    {
        for (int start = 0; start < total; start += B.capacity, wave++) {
            WavefrontBuffers& W = *lanes[wave % nLanes];
            cudaStream_t ws = laneStream[wave % nLanes];
            WaveArgs A{L, start, total - start < B.capacity ? total - start : B.capacity};
            generateKernel<<<blocks(A.n, 256), 256, 0, ws>>>(A, W);
            n++;
            int q = 0;
            for (int bounce = 0; bounce < L.set.maxBounces; bounce++) {
                resetQueuesKernel<<<1, 32, 0, ws>>>(W, q);
                Mark m{nullptr, nullptr, bounce == 0 ? 0 : 1};
                if (timing) { m.a = event(ev++); m.b = event(ev++); cudaEventRecord(m.a, ws); }
                extendKernel<<<extendBlocks, kTraceBlock, smem, ws>>>(L.scene.wide, L.scene.packed, W, q,
                                                                      &L.counters[bounce == 0 ? 0 : 1], L.errorFlag,
                                                                      stackLimit, refill);
                if (timing) { cudaEventRecord(m.b, ws); marks.push_back(m); }
                shadeKernel<<<shadeBlocks, 256, 0, ws>>>(A, W, q, bounce);
                Mark s{nullptr, nullptr, 2};
                if (timing) { s.a = event(ev++); s.b = event(ev++); cudaEventRecord(s.a, ws); }
                shadowKernel<<<shadowBlocks, kTraceBlock, smem, ws>>>(L.scene.wide, L.scene.packed, W, &L.counters[2],
                                                                      L.errorFlag, stackLimit, refill);
                if (timing) { cudaEventRecord(s.b, ws); marks.push_back(s); }
                n += 4;
                q ^= 1;
            }
            // Samples of a pixel are added in sample order: after the
            // previous wave's accumulation, whichever lane ran it.
            // Within the wave, one launch per sample row it covers.
            if (two && wave > 0) cudaStreamWaitEvent(ws, overlap->accumulated, 0);
            for (int first = 0; first < A.n;) {
                const int rowEnd = ((A.start + first) / pixels + 1) * pixels - A.start;
                const int count = (rowEnd < A.n ? rowEnd : A.n) - first;
                accumulateKernel<<<blocks(count, 256), 256, 0, ws>>>(A, W, first, count);
                first += count;
                n++;
            }
            if (two) cudaEventRecord(overlap->accumulated, ws);
        }
    }
    for (int k = 1; k < nLanes; k++) {
        cudaEventRecord(overlap->joins[k - 1], laneStream[k]);
        cudaStreamWaitEvent(stream, overlap->joins[k - 1], 0);
    }
    cudaError_t e = cudaGetLastError();
    if (launches) *launches = n;
    if (timing && e == cudaSuccess) {
        e = cudaStreamSynchronize(stream);
        float kindMs[3] = {0, 0, 0};
        for (const Mark& m : marks) {
            float ms = 0;
            cudaEventElapsedTime(&ms, m.a, m.b);
            kindMs[m.kind] += ms;
        }
        if (extendMs) *extendMs = kindMs[0] + kindMs[1];
        if (shadowMs) *shadowMs = kindMs[2];
        if (primaryMs) *primaryMs = kindMs[0];
    }
    return e;
}

cudaError_t launchQueries(const uint4* wide, const float4* packed, const float4* queries, int count, int any,
                          float4* hits, int* fetch, int* errorFlag, int wideDepth, const TraceTuning& tuning,
                          cudaStream_t stream) {
    (void)wideDepth;
    const int stackLimit = tuning.stackLimit;
    const int refill = tuning.refill;
    cudaError_t e = cudaMemsetAsync(fetch, 0, sizeof(int), stream);
    if (e != cudaSuccess) return e;
    if (any) {
        static int blocks = traceBlocks(queryKernel<true>, kTraceSmem);
        queryKernel<true><<<blocks, kTraceBlock, kTraceSmem, stream>>>(wide, packed, queries, count, hits, fetch, errorFlag,
                                                                      stackLimit, refill);
    } else {
        static int blocks = traceBlocks(queryKernel<false>, kTraceSmem);
        queryKernel<false><<<blocks, kTraceBlock, kTraceSmem, stream>>>(wide, packed, queries, count, hits, fetch, errorFlag,
                                                                       stackLimit, refill);
    }
    return cudaGetLastError();
}

cudaError_t launchSobolSamples(const unsigned* dirs, const unsigned* pixel, const unsigned* sample, const unsigned* seed,
                               int count, int ndim, float* out, cudaStream_t stream) {
    long long total = (long long)count * ndim;
    sobolSamplesKernel<<<blocks(total, 256), 256, 0, stream>>>(dirs, pixel, sample, seed, count, ndim, out);
    return cudaGetLastError();
}

// Denoised linear radiance as 3 floats per pixel (uncovered pixels 0, as the
// display shows them): src holds srcStride floats per pixel.
__global__ void denoisedRgbKernel(const Accum* sums, const float* src, int srcStride, int count, float* out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float* r = src + (size_t)i * srcStride;
    const bool covered = sums[i].covered != 0u;
    out[3 * (size_t)i] = covered ? r[0] : 0.0f;
    out[3 * (size_t)i + 1] = covered ? r[1] : 0.0f;
    out[3 * (size_t)i + 2] = covered ? r[2] : 0.0f;
}

cudaError_t launchDenoisedRgb(const Accum* sums, const float* src, int srcStride, int count, float* out,
                              cudaStream_t stream) {
    denoisedRgbKernel<<<blocks(count, 256), 256, 0, stream>>>(sums, src, srcStride, count, out);
    return cudaGetLastError();
}

cudaError_t launchDenoise(const Accum* sums, unsigned samples, int w, int h, float exposure, float4* work,
                          uchar4* pixels, cudaStream_t stream) {
    int count = w * h;
    float4 *color = work, *albedo = work + count, *normal = work + 2 * (size_t)count, *tmp = work + 3 * (size_t)count;
    denoisePrepareKernel<<<blocks(count, 256), 256, 0, stream>>>(sums, samples, count, color, albedo, normal);
    dim3 block(16, 16), grid((w + 15) / 16, (h + 15) / 16);
    float4 *src = color, *dst = tmp;
    float phi = 0.5f;
    for (int it = 0; it < kAtrousPasses; it++) {
        atrousKernel<<<grid, block, 0, stream>>>(src, albedo, normal, dst, w, h, 1 << it, phi);
        float4* t = src; src = dst; dst = t;
        phi *= 0.5f;
    }
    denoisePresentKernel<<<blocks(count, 256), 256, 0, stream>>>(sums, src, count, exposure, pixels);
    return cudaGetLastError();
}

cudaError_t launchAovs(const Accum* sums, const float* depthSums, unsigned samples, int count, float* aov,
                       cudaStream_t stream) {
    aovKernel<<<blocks(count, 256), 256, 0, stream>>>(sums, depthSums, samples, count, aov);
    return cudaGetLastError();
}
cudaError_t launchPresentRadiance(const Accum* sums, const float* radiance, int count, float exposure, uchar4* pixels,
                                  cudaStream_t stream) {
    presentRadianceKernel<<<blocks(count, 256), 256, 0, stream>>>(sums, radiance, count, exposure, pixels);
    return cudaGetLastError();
}

}  // namespace rt
