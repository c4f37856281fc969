// Batched multi-scene rendering (the RtxBatch* entry points): many views of
// many scenes traced in shared waves, one traversal launch per stage for the
// rays of every scene, frames replayed from a CUDA graph, and an autotuner
// for the launch shape and the BVH width.
//
// Scenes are built one by one with the single-scene builder, then copied
// into arenas: shading triangles, wide nodes, packed triangles and emitters
// of all scenes one after another. The copy rebases the indices inside it (a
// node's childBase and triBase by the scene's node and packed-triangle
// offsets, a packed triangle's original index and an emitter's triangle by
// its triangle offset), so a traversal that starts at
// the scene's root node meets only that scene's nodes and triangles, and hit
// indices address the shared shading arena. The offsets keep the order of
// indices within a scene, so the reference's tie-break (smaller index at equal
// distance, renderer.cu:153) picks the same triangle as in the scene alone.
//
// Views are concatenated into one pixel range; a wave is a range of that
// global pixel index, so one wave holds paths of many views. A path carries
// its view; the view gives the camera, the scene and the pixel's index within
// the view, which is the Sobol pixel index (renderer.cu:198). Frames read the
// accumulated sample count from device memory, so one captured graph serves
// every frame with the same settings.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cuda_ray_tracer.h"
#include "rt_build.cuh"
#include "rt_render.cuh"
#include "rt_trace.cuh"
#include "rt_upload.cuh"

namespace rt {
namespace {

struct BatchView { Camera cam; int w, h, scene; unsigned pixelStart; };
struct BatchScene { SceneView view; unsigned root; };

struct BatchFrame {
    const BatchView* views;
    int viewCount;
    const BatchScene* scenes;
    Settings set;
    const unsigned* passXor;   // [raysPerPixel][kSobolDims]
    const unsigned* seedHash;  // [kSobolDims]
    const unsigned* sample;    // paths per pixel accumulated before this frame (device)
    Accum* sums;
    float* depthSums;
    uchar4* pixels;
    unsigned long long* counters;  // [0] primary, [1] secondary, [2] shadow rays
    int* errorFlag;
};
// A wave is the paths [start, start + n) of a frame, path k being sample
// row k / pixels of global pixel k % pixels; a wave may span several rows.
struct BatchWave {
    BatchFrame F;
    unsigned long long start;  // first path
    unsigned pixels;           // pixels of all views
    int n;                     // paths in the wave
};
__device__ __forceinline__ int batchRow(const BatchWave& A, int p) { return (int)((A.start + (unsigned)p) / A.pixels); }
__device__ __forceinline__ unsigned batchPixel(const BatchWave& A, int p) {
    return (unsigned)((A.start + (unsigned)p) % A.pixels);
}

// View holding global pixel g: the last view whose first pixel is <= g.
__device__ __forceinline__ int findView(const BatchView* views, int count, unsigned g) {
    int lo = 0, hi = count - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (views[mid].pixelStart <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__global__ void batchSobolKernel(const unsigned* dirs, const unsigned* sample, int rpp, unsigned seed,
                                 unsigned* passXor, unsigned* seedHash) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned sample0 = *sample;
    int passEntries = rpp * kSobolDims;
    if (i < passEntries) {
        int r = i / kSobolDims, d = i % kSobolDims;
        passXor[i] = sobolXor(dirs, sample0 + (unsigned)r, (unsigned)d);
    } else if (i < passEntries + kSobolDims) {
        int d = i - passEntries;
        seedHash[d] = sobolHash(seed + (unsigned)d * 0x9e3779b9u);
    }
}

__global__ void batchGenerateKernel(BatchWave A, WavefrontBuffers B) {
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= A.n) return;
    const unsigned g = batchPixel(A, p);
    const int v = findView(A.F.views, A.F.viewCount, g);
    const BatchView& V = A.F.views[v];
    const unsigned local = g - V.pixelStart;
    const int x = (int)(local % (unsigned)V.w), y = (int)(local / (unsigned)V.w);
    Sampler rng{A.F.passXor + batchRow(A, p) * kSobolDims, A.F.seedHash, local, 0u};
    PathState st = startPath(V.cam, A.F.set, x, y, V.w, V.h, rng);
    B.pathA[p] = make_float4(st.origin.x, st.origin.y, st.origin.z, 0.0f);
    B.pathB[p] = make_float4(st.dir.x, st.dir.y, st.dir.z, __int_as_float(v));
    B.pathC[p] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
    B.radiance[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    B.albedo[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    B.normal[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    B.queue[0][p] = p;
    if (p == 0) { B.counts[0] = A.n; B.counts[1] = 0; B.counts[2] = 0; }
}

// Closest hit for every queued path; each ray starts at its scene's root.
struct BatchExtendIO {
    const int* queue;
    const float4 *pathA, *pathB;
    float4* hits;
    const BatchView* views;
    const BatchScene* scenes;
    __device__ void load(int k, float3& o, float3& d, float& limit, unsigned& root) const {
        int p = queue[k];
        float4 a = pathA[p], b = pathB[p];
        o = v3(a.x, a.y, a.z); d = v3(b.x, b.y, b.z); limit = 1e30f;
        root = scenes[views[__float_as_int(b.w)].scene].root;
    }
    __device__ void store(int k, const Hit& h) const {
        hits[queue[k]] = make_float4(h.distance, h.u, h.v, __int_as_float(h.index));
    }
};
// Traversal kernels are compiled for 1,024 resident threads per SM (64
// registers), as the single-scene ones.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, 1024 / BLOCK) batchExtendKernel(const uint4* wide, const float4* packed,
                                                           WavefrontBuffers B, int q, const BatchView* views,
                                                           const BatchScene* scenes, unsigned long long* counter,
                                                           int* errorFlag, int refill) {
    BatchExtendIO io{B.queue[q], B.pathA, B.pathB, B.hits, views, scenes};
    persistentTrace<false>(io, B.counts[q], wide, packed, &B.counts[3], counter, errorFlag, kStackCapacity, refill);
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

__global__ void batchShadeKernel(BatchWave A, WavefrontBuffers B, int q, int bounce) {
    int count = B.counts[q];
    int nq = q ^ 1;
    int stride = gridDim.x * blockDim.x;
    int limit = ((count + 31) / 32) * 32;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < limit; k += stride) {
        bool valid = k < count;
        bool cont = false, shadow = false;
        int p = 0;
        unsigned root = 0;
        ShadowRequest req;
        if (valid) {
            p = B.queue[q][k];
            float4 a = B.pathA[p], b = B.pathB[p], c = B.pathC[p], rad = B.radiance[p], hv = B.hits[p];
            const int v = __float_as_int(b.w);
            const BatchView& V = A.F.views[v];
            const BatchScene& S = A.F.scenes[V.scene];
            root = S.root;
            PathState st;
            st.origin = v3(a.x, a.y, a.z); st.prevPdf = a.w;
            st.dir = v3(b.x, b.y, b.z);
            st.throughput = v3(c.x, c.y, c.z);
            st.radiance = v3(rad.x, rad.y, rad.z); st.covered = __float_as_uint(rad.w);
            float4 al = B.albedo[p], no = B.normal[p];
            st.albedo = v3(al.x, al.y, al.z); st.normal = v3(no.x, no.y, no.z);
            st.depth = al.w;
            Hit h{__float_as_int(hv.w), hv.x, hv.y, hv.z};
            const unsigned local = batchPixel(A, p) - V.pixelStart;
            Sampler rng{A.F.passXor + batchRow(A, p) * kSobolDims, A.F.seedHash, local, 4u + 8u * (unsigned)bounce};
            unsigned f = shadeBounce(S.view, A.F.set, bounce, st, h, rng, req);
            cont = (f & kContinue) != 0;
            shadow = (f & kShadow) != 0;
            B.pathA[p] = make_float4(st.origin.x, st.origin.y, st.origin.z, st.prevPdf);
            B.pathB[p] = make_float4(st.dir.x, st.dir.y, st.dir.z, __int_as_float(v));
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
            B.shadowContrib[sslot] =
                make_float4(req.contribution.x, req.contribution.y, req.contribution.z, __uint_as_float(root));
        }
    }
}

// Light-sample visibility; the root node travels in the contribution's w.
struct BatchShadowIO {
    const float4 *ray, *dir, *contrib;
    float4* radiance;
    __device__ void load(int k, float3& o, float3& d, float& limit, unsigned& root) const {
        float4 a = ray[k], b = dir[k];
        o = v3(a.x, a.y, a.z); d = v3(b.x, b.y, b.z); limit = a.w;
        root = __float_as_uint(contrib[k].w);
    }
    __device__ void store(int k, const Hit& h) const {
        if (h.index >= 0) return;
        int p = __float_as_int(dir[k].w);
        float4 c = contrib[k], rad = radiance[p];
        radiance[p] = make_float4(rad.x + c.x, rad.y + c.y, rad.z + c.z, rad.w);
    }
};
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, 1024 / BLOCK) batchShadowKernel(const uint4* wide, const float4* packed,
                                                           WavefrontBuffers B, unsigned long long* counter,
                                                           int* errorFlag, int refill) {
    BatchShadowIO io{B.shadowRay, B.shadowDir, B.shadowContrib, B.radiance};
    persistentTrace<true>(io, B.counts[2], wide, packed, &B.counts[4], counter, errorFlag, kStackCapacity, refill);
}

__global__ void batchResetQueuesKernel(WavefrontBuffers B, int q) {
    if (threadIdx.x == 0) { B.counts[q ^ 1] = 0; B.counts[2] = 0; B.counts[3] = 0; B.counts[4] = 0; }
}

// Adds paths [firstPath, firstPath + count) of the wave (all of one sample
// row) to their pixels; the rows of a wave are added by successive launches.
__global__ void batchAccumulateKernel(BatchWave A, WavefrontBuffers B, int firstPath, int count) {
    int p = firstPath + blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= firstPath + count) return;
    const size_t i = batchPixel(A, p);
    const int row = batchRow(A, p);
    const unsigned sample0 = *A.F.sample;
    const bool first = row == 0 && sample0 == 0;
    Accum total = first ? Accum{v3(0, 0, 0), v3(0, 0, 0), v3(0, 0, 0), 0u} : A.F.sums[i];
    float depthTotal = first ? 0.0f : A.F.depthSums[i];
    float4 rad = B.radiance[p], al = B.albedo[p], no = B.normal[p];
    PathState st;
    st.radiance = v3(rad.x, rad.y, rad.z); st.covered = __float_as_uint(rad.w);
    st.albedo = v3(al.x, al.y, al.z); st.normal = v3(no.x, no.y, no.z);
    addPath(total, st);
    A.F.sums[i] = total;
    A.F.depthSums[i] = depthTotal + al.w;
    if (row == A.F.set.raysPerPixel - 1)
        A.F.pixels[i] = displayPixel(total, sample0 + (unsigned)A.F.set.raysPerPixel, A.F.set.exposure);
}

__global__ void batchAdvanceKernel(unsigned* sample, int rpp) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *sample += (unsigned)rpp;
}

// ---- one persistent launch per frame (RTX_BATCH_PERSISTENT) ----
// Resident blocks pull tiles of 16 x 8 pixels from one queue over every
// view of every scene (tiles[v] .. tiles[v + 1] - 1 are view v's, in rows;
// tiles[viewCount + 1] is the queue's cursor) and trace each pixel's paths
// with the reference's launch shape (renderPixel, one thread per pixel, the
// whole traversal stack in shared memory), starting at the view's scene's
// root in the arena.
constexpr int kBatchTileX = 16, kBatchTileY = 8, kBatchMegaBlock = kBatchTileX * kBatchTileY;
__global__ void __launch_bounds__(kBatchMegaBlock) batchMegaKernel(BatchFrame F, unsigned* tiles) {
    extern __shared__ uint2 smemStack[];
    __shared__ unsigned tile;
    uint2* stack = smemStack + threadIdx.x;
    const unsigned total = tiles[F.viewCount];
    const unsigned sample0 = *F.sample;
    unsigned nPrimary = 0, nSecondary = 0, nShadow = 0;
    int overflow = 0;
    for (;;) {
        if (threadIdx.x == 0) tile = atomicAdd(&tiles[F.viewCount + 1], 1u);
        __syncthreads();
        const unsigned t = tile;
        __syncthreads();
        if (t >= total) break;
        int lo = 0, hi = F.viewCount - 1;  // the view v with tiles[v] <= t < tiles[v + 1]
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (tiles[mid] <= t) lo = mid; else hi = mid - 1;
        }
        const BatchView V = F.views[lo];
        const BatchScene& S = F.scenes[V.scene];
        const unsigned local = t - tiles[lo], tilesX = (unsigned)(V.w + kBatchTileX - 1) / kBatchTileX;
        const int x = (int)(local % tilesX) * kBatchTileX + (int)threadIdx.x % kBatchTileX;
        const int y = (int)(local / tilesX) * kBatchTileY + (int)threadIdx.x / kBatchTileX;
        if (x < V.w && y < V.h) {
            SceneView sv = S.view;
            sv.root = S.root;
            renderPixel(sv, V.cam, F.set, x, y, V.w, V.h, sample0, F.passXor, F.seedHash, F.sums + V.pixelStart,
                        F.depthSums + V.pixelStart, F.pixels + V.pixelStart, stack, kBatchMegaBlock, &overflow,
                        nPrimary, nSecondary, nShadow);
        }
    }
    const unsigned sa = __reduce_add_sync(0xFFFFFFFFu, nPrimary), sb = __reduce_add_sync(0xFFFFFFFFu, nSecondary),
                   sc = __reduce_add_sync(0xFFFFFFFFu, nShadow);
    if ((threadIdx.x & 31) == 0) {
        if (sa) atomicAdd(&F.counters[0], (unsigned long long)sa);
        if (sb) atomicAdd(&F.counters[1], (unsigned long long)sb);
        if (sc) atomicAdd(&F.counters[2], (unsigned long long)sc);
    }
    if (overflow) atomicExch(F.errorFlag, 1);
}

// Arena copies: indices of scene k move by its node / triangle offsets.
__global__ void rebaseNodesKernel(uint4* nodes, int count, unsigned nodeBase, unsigned triBase) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    uint4 w1 = nodes[(size_t)i * 5 + 1];
    w1.x += nodeBase;
    w1.y += triBase;
    nodes[(size_t)i * 5 + 1] = w1;
}
__global__ void rebasePackedKernel(float4* packed, int count, unsigned triBase) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    float4 c = packed[(size_t)i * 3 + 2];
    c.z = __uint_as_float(__float_as_uint(c.z) + triBase);
    packed[(size_t)i * 3 + 2] = c;
}

inline int blocksFor(long long n, int b) { return (int)((n + b - 1) / b); }

int deviceSms() {
    int device = 0, sms = 0;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    return sms > 0 ? sms : 1;
}

template <int BLOCK>
struct TraceLaunch {
    static int extendBlocks, shadowBlocks;
    static void configure() {
        if (extendBlocks) return;
        const size_t smem = traceSharedBytes(BLOCK);
        // Blocks of 256 threads take more than the 48 KB of dynamic shared
        // memory a kernel gets without opting in.
        cudaFuncSetAttribute(batchExtendKernel<BLOCK>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(batchShadowKernel<BLOCK>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        int perSm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, batchExtendKernel<BLOCK>, BLOCK, smem) != cudaSuccess ||
            perSm <= 0)
            perSm = 1;
        extendBlocks = deviceSms() * perSm;
        perSm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, batchShadowKernel<BLOCK>, BLOCK, smem) != cudaSuccess ||
            perSm <= 0)
            perSm = 1;
        shadowBlocks = deviceSms() * perSm;
    }
};
template <int BLOCK> int TraceLaunch<BLOCK>::extendBlocks = 0;
template <int BLOCK> int TraceLaunch<BLOCK>::shadowBlocks = 0;

template <int BLOCK>
void launchTraversal(bool shadow, const uint4* wide, const float4* packed, const WavefrontBuffers& B, int q,
                     const BatchView* views, const BatchScene* scenes, unsigned long long* counter, int* errorFlag,
                     int refill, cudaStream_t stream) {
    TraceLaunch<BLOCK>::configure();
    const size_t smem = traceSharedBytes(BLOCK);
    if (shadow)
        batchShadowKernel<BLOCK><<<TraceLaunch<BLOCK>::shadowBlocks, BLOCK, smem, stream>>>(wide, packed, B, counter,
                                                                                            errorFlag, refill);
    else
        batchExtendKernel<BLOCK><<<TraceLaunch<BLOCK>::extendBlocks, BLOCK, smem, stream>>>(
            wide, packed, B, q, views, scenes, counter, errorFlag, refill);
}

}  // namespace
}  // namespace rt

using namespace rt;

namespace {

struct BatchSceneData {
    std::vector<Light> lights;  // triangle indices local to the scene
    float lightArea = 0.0f;
    SceneTri* dTris = nullptr;  // the scene's own copy (source of the arena)
    int count = 0;
    BuiltBvh bvh;
    BuildResult build;
    int builtWidth = 0, builtPieces = 0, builtLeaf = 0;
    unsigned triBase = 0, nodeBase = 0, lightBase = 0, packedBase = 0;
};
struct BatchViewData {
    Camera cam;
    int w, h, scene;
    unsigned pixelStart;
};

struct Batch {
    std::string error;
    int device = -1;
    cudaStream_t stream = nullptr;
    cudaEvent_t start = nullptr, stop = nullptr;
    std::vector<BatchSceneData> scenes;
    std::vector<BatchViewData> views;
    // Arenas of all scenes and the tables the kernels read.
    SceneTri* aTris = nullptr;
    uint4* aWide = nullptr;
    float4* aPacked = nullptr;
    Light* aLights = nullptr;
    BatchScene* dScenes = nullptr;
    BatchView* dViews = nullptr;
    bool arenaReady = false, viewsReady = false;
    // Accumulation of all views, concatenated.
    Accum* dSum = nullptr;
    float* dDepth = nullptr;
    uchar4* dPixels = nullptr;
    size_t pixels = 0;
    // Sampler tables and the device sample count.
    unsigned *dDirs = nullptr, *dPassXor = nullptr, *dSeedHash = nullptr, *dSample = nullptr;
    unsigned samples = 0;
    unsigned long long* dCounters = nullptr;
    int* dError = nullptr;
    WavefrontBuffers wave;
    // Lanes of waves beyond the first (wave j on lane j % lanes; WaveOverlap).
    WavefrontBuffers laneWaves[kMaxLanes - 1];
    cudaStream_t laneStreams[kMaxLanes - 1] = {};
    cudaEvent_t laneJoins[kMaxLanes - 1] = {};
    cudaEvent_t fork = nullptr, accumulated = nullptr;
    int lanesReady = 1;
    // Tuning.
    int block = 128, capacity = 0, refill = 24, width = 8, useGraph = 1, pieces = 3, leaf = 2, lanes = 2;
    int persistent = 0;             // RTX_BATCH_PERSISTENT: one persistent launch per frame
    unsigned* dTiles = nullptr;     // [views + 2]: tile prefix per view, then the frame's tile cursor
    int environmentMode = 0;
    float3 environment = make_float3(0.0f, 0.0f, 0.0f);
    // Frame state.
    RenderSettings last{};
    bool haveLast = false;
    cudaGraphExec_t exec = nullptr;
    bool graphValid = false;
    int frameLaunches = 0;
    RtxBatchStats stats{};
};

bool failB(Batch* b, cudaError_t e, const char* what = nullptr) {
    b->error = what ? std::string(what) + (e != cudaSuccess ? std::string(": ") + cudaGetErrorString(e) : "")
                    : std::string(cudaGetErrorString(e));
    return false;
}

void dropGraph(Batch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
    b->graphValid = false;
}

void freeArena(Batch* b) {
    void* owned[] = {b->aTris, b->aWide, b->aPacked, b->aLights, b->dScenes};
    for (void* p : owned)
        if (p) cudaFree(p);
    b->aTris = nullptr; b->aWide = nullptr; b->aPacked = nullptr; b->aLights = nullptr; b->dScenes = nullptr;
    b->arenaReady = false;
    dropGraph(b);
}

void freeViews(Batch* b) {
    void* owned[] = {b->dViews, b->dSum, b->dDepth, b->dPixels, b->dTiles};
    for (void* p : owned)
        if (p) cudaFree(p);
    b->dViews = nullptr; b->dSum = nullptr; b->dDepth = nullptr; b->dPixels = nullptr; b->dTiles = nullptr;
    b->viewsReady = false;
    dropGraph(b);
}

void resetSamples(Batch* b) {
    b->samples = 0;
    if (b->dSample) cudaMemsetAsync(b->dSample, 0, sizeof(unsigned), b->stream);
}

bool ensureBase(Batch* b) {
    if (b->stream) return true;
    cudaError_t e;
    if ((e = cudaGetDevice(&b->device)) != cudaSuccess) return failB(b, e);
    std::string why;
    const unsigned* dirs = hostSobolDirections(why);
    if (!dirs) { b->error = why; return false; }
    if ((e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) != cudaSuccess) return failB(b, e);
    if ((e = cudaEventCreate(&b->start)) != cudaSuccess) return failB(b, e);
    if ((e = cudaEventCreate(&b->stop)) != cudaSuccess) return failB(b, e);
    if ((e = rt::deviceAlloc(&b->dDirs, sizeof(unsigned) * kSobolDims * 32)) != cudaSuccess) return failB(b, e);
    // Copies and fills on b->stream: a non-blocking stream is not ordered
    // after the legacy default stream.
    if ((e = cudaMemcpyAsync(b->dDirs, dirs, sizeof(unsigned) * kSobolDims * 32, cudaMemcpyHostToDevice, b->stream)) !=
        cudaSuccess)
        return failB(b, e);
    if ((e = rt::deviceAlloc(&b->dPassXor, sizeof(unsigned) * 16 * kSobolDims)) != cudaSuccess) return failB(b, e);
    if ((e = rt::deviceAlloc(&b->dSeedHash, sizeof(unsigned) * kSobolDims)) != cudaSuccess) return failB(b, e);
    if ((e = rt::deviceAlloc(&b->dSample, sizeof(unsigned))) != cudaSuccess) return failB(b, e);
    if ((e = cudaMemsetAsync(b->dSample, 0, sizeof(unsigned), b->stream)) != cudaSuccess) return failB(b, e);
    if ((e = rt::deviceAlloc(&b->dCounters, 4 * sizeof(unsigned long long))) != cudaSuccess) return failB(b, e);
    if ((e = rt::deviceAlloc(&b->dError, 2 * sizeof(int))) != cudaSuccess) return failB(b, e);
    return true;
}

// Traversal tree of a scene at the batch's BVH width and pieces per triangle
// (only the wide nodes and packed triangles are kept).
bool buildScene(Batch* b, BatchSceneData& S) {
    if (S.builtWidth == b->width && S.builtPieces == b->pieces && S.builtLeaf == b->leaf) return true;
    freeBvh(S.bvh);
    const char* why = nullptr;
    cudaError_t e = buildBvh(S.dTris, S.count, b->stream, S.bvh, S.build, &why, 3, b->width, b->pieces, b->leaf);
    if (e != cudaSuccess) { S.builtWidth = 0; return failB(b, e, why); }
    void* unused[] = {S.bvh.binNodes, S.bvh.order, S.bvh.primLo, S.bvh.primHi};
    for (void* q : unused) cudaFree(q);
    S.bvh.binNodes = nullptr; S.bvh.order = nullptr; S.bvh.primLo = nullptr; S.bvh.primHi = nullptr;
    S.builtWidth = b->width;
    S.builtPieces = b->pieces;
    S.builtLeaf = b->leaf;
    return true;
}

// Builds (at the current width) and copies every scene into the arenas.
bool ensureArena(Batch* b) {
    if (b->arenaReady) return true;
    freeArena(b);
    size_t tris = 0, nodes = 0, lights = 0, packedCount = 0;
    for (BatchSceneData& S : b->scenes) {
        if (!buildScene(b, S)) return false;
        S.triBase = (unsigned)tris;
        S.nodeBase = (unsigned)nodes;
        S.lightBase = (unsigned)lights;
        S.packedBase = (unsigned)packedCount;
        tris += (size_t)S.count;
        nodes += (size_t)S.build.wideNodes;
        lights += S.lights.size();
        packedCount += (size_t)S.build.packedTriangles;
    }
    if (tris > 0x7FFFFFFFull || nodes > 0x7FFFFFFFull || packedCount > 0x7FFFFFFFull) {
        b->error = "batch too large for 31-bit indices";
        return false;
    }
    cudaError_t e;
    if ((e = rt::deviceAlloc(&b->aTris, sizeof(SceneTri) * tris)) != cudaSuccess) return failB(b, e, "arena");
    if ((e = rt::deviceAlloc(&b->aWide, sizeof(uint4) * 5 * nodes)) != cudaSuccess) return failB(b, e, "arena");
    if ((e = rt::deviceAlloc(&b->aPacked, sizeof(float4) * 3 * packedCount)) != cudaSuccess) return failB(b, e, "arena");
    if ((e = rt::deviceAlloc(&b->aLights, sizeof(Light) * std::max<size_t>(lights, 1))) != cudaSuccess) return failB(b, e, "arena");
    if ((e = rt::deviceAlloc(&b->dScenes, sizeof(BatchScene) * b->scenes.size())) != cudaSuccess) return failB(b, e, "arena");
    std::vector<BatchScene> table;
    std::vector<Light> allLights;
    allLights.reserve(lights);
    for (BatchSceneData& S : b->scenes) {
        const size_t n = (size_t)S.count, w = (size_t)S.build.wideNodes, np = (size_t)S.build.packedTriangles;
        if ((e = cudaMemcpyAsync(b->aTris + S.triBase, S.dTris, sizeof(SceneTri) * n, cudaMemcpyDeviceToDevice,
                                 b->stream)) != cudaSuccess) return failB(b, e);
        if ((e = cudaMemcpyAsync(b->aWide + (size_t)S.nodeBase * 5, S.bvh.wideNodes, sizeof(uint4) * 5 * w,
                                 cudaMemcpyDeviceToDevice, b->stream)) != cudaSuccess) return failB(b, e);
        if ((e = cudaMemcpyAsync(b->aPacked + (size_t)S.packedBase * 3, S.bvh.packedTris, sizeof(float4) * 3 * np,
                                 cudaMemcpyDeviceToDevice, b->stream)) != cudaSuccess) return failB(b, e);
        rebaseNodesKernel<<<blocksFor((long long)w, 256), 256, 0, b->stream>>>(b->aWide + (size_t)S.nodeBase * 5, (int)w,
                                                                              S.nodeBase, S.packedBase);
        rebasePackedKernel<<<blocksFor((long long)np, 256), 256, 0, b->stream>>>(b->aPacked + (size_t)S.packedBase * 3,
                                                                                (int)np, S.triBase);
        if ((e = cudaGetLastError()) != cudaSuccess) return failB(b, e);
        for (const Light& L : S.lights) allLights.push_back(Light{L.triangle + (int)S.triBase, L.cumulativeArea});
        SceneView view{b->aTris, b->aWide, b->aPacked, b->aLights + S.lightBase, (int)S.lights.size(), S.lightArea,
                       S.build.wideDepth, b->environmentMode, b->environment};
        table.push_back(BatchScene{view, S.nodeBase});
    }
    if (!allLights.empty() &&
        (e = cudaMemcpyAsync(b->aLights, allLights.data(), sizeof(Light) * allLights.size(), cudaMemcpyHostToDevice,
                             b->stream)) != cudaSuccess) return failB(b, e);
    if ((e = cudaMemcpyAsync(b->dScenes, table.data(), sizeof(BatchScene) * table.size(), cudaMemcpyHostToDevice,
                             b->stream)) != cudaSuccess) return failB(b, e);
    if ((e = cudaStreamSynchronize(b->stream)) != cudaSuccess) return failB(b, e);
    b->arenaReady = true;
    resetSamples(b);
    return true;
}

bool ensureViews(Batch* b) {
    if (b->viewsReady) return true;
    freeViews(b);
    std::vector<BatchView> table;
    std::vector<unsigned> tiles(1, 0u);
    size_t pixels = 0;
    for (BatchViewData& V : b->views) {
        V.pixelStart = (unsigned)pixels;
        table.push_back(BatchView{V.cam, V.w, V.h, V.scene, V.pixelStart});
        pixels += (size_t)V.w * V.h;
        tiles.push_back(tiles.back() + (unsigned)(((V.w + kBatchTileX - 1) / kBatchTileX) *
                                                  ((V.h + kBatchTileY - 1) / kBatchTileY)));
    }
    tiles.push_back(0u);  // the cursor
    if (pixels > 0x7FFFFFFFull) { b->error = "batch has more than 2^31 pixels"; return false; }
    cudaError_t e;
    if ((e = rt::deviceAlloc(&b->dViews, sizeof(BatchView) * table.size())) != cudaSuccess) return failB(b, e);
    if ((e = rt::deviceAlloc(&b->dSum, sizeof(Accum) * pixels)) != cudaSuccess) return failB(b, e, "accumulation");
    if ((e = rt::deviceAlloc(&b->dDepth, sizeof(float) * pixels)) != cudaSuccess) return failB(b, e, "accumulation");
    if ((e = rt::deviceAlloc(&b->dPixels, sizeof(uchar4) * pixels)) != cudaSuccess) return failB(b, e, "accumulation");
    if ((e = rt::deviceAlloc(&b->dTiles, sizeof(unsigned) * tiles.size())) != cudaSuccess) return failB(b, e);
    if ((e = cudaMemcpyAsync(b->dTiles, tiles.data(), sizeof(unsigned) * tiles.size(), cudaMemcpyHostToDevice,
                             b->stream)) != cudaSuccess)
        return failB(b, e);
    if ((e = cudaMemcpyAsync(b->dViews, table.data(), sizeof(BatchView) * table.size(), cudaMemcpyHostToDevice,
                             b->stream)) != cudaSuccess)
        return failB(b, e);
    b->pixels = pixels;
    b->viewsReady = true;
    resetSamples(b);
    return true;
}

// Paths per wave: RTX_BATCH_CAPACITY (default 2^24), at most the paths of a
// frame of raysPerPixel rows.
int waveCapacity(const Batch* b, int raysPerPixel) {
    const long long want = b->capacity > 0 ? b->capacity : (1ll << 24);
    return (int)std::min<long long>(want, (long long)b->pixels * raysPerPixel);
}

void freeLanes(Batch* b) {
    for (int k = 0; k < kMaxLanes - 1; k++) {
        freeWavefront(b->laneWaves[k]);
        if (b->laneStreams[k]) cudaStreamDestroy(b->laneStreams[k]);
        if (b->laneJoins[k]) cudaEventDestroy(b->laneJoins[k]);
        b->laneStreams[k] = nullptr;
        b->laneJoins[k] = nullptr;
    }
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->accumulated) cudaEventDestroy(b->accumulated);
    b->fork = b->accumulated = nullptr;
    b->lanesReady = 1;
}

bool ensureWave(Batch* b, int raysPerPixel) {
    const int cap = waveCapacity(b, raysPerPixel);
    cudaError_t e;
    if (b->wave.capacity != cap) {
        dropGraph(b);
        if ((e = allocWavefront(b->wave, cap)) != cudaSuccess) return failB(b, e, "wavefront buffers");
    }
    if (b->lanes < b->lanesReady) { dropGraph(b); freeLanes(b); }
    if (b->lanes < 2) return true;
    if (!b->fork && ((e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming)) != cudaSuccess ||
                     (e = cudaEventCreateWithFlags(&b->accumulated, cudaEventDisableTiming)) != cudaSuccess)) {
        freeLanes(b);
        return failB(b, e, "wave lane events");
    }
    for (int k = 0; k < b->lanes - 1; k++) {
        if (b->laneWaves[k].capacity != cap) {
            dropGraph(b);
            if ((e = allocWavefront(b->laneWaves[k], cap)) != cudaSuccess) { freeLanes(b); return failB(b, e, "wavefront buffers"); }
        }
        if ((!b->laneStreams[k] && (e = cudaStreamCreateWithFlags(&b->laneStreams[k], cudaStreamNonBlocking)) != cudaSuccess) ||
            (!b->laneJoins[k] && (e = cudaEventCreateWithFlags(&b->laneJoins[k], cudaEventDisableTiming)) != cudaSuccess)) {
            freeLanes(b);
            return failB(b, e, "wave lanes");
        }
    }
    if (b->lanesReady != b->lanes) dropGraph(b);
    b->lanesReady = b->lanes;
    return true;
}

// The kernels of one frame on b->stream and the lane streams forked from it
// (captured or launched).
cudaError_t enqueueFrame(Batch* b, const Settings& set, int* launches) {
    cudaStream_t main = b->stream;
    int n = 0;
    const int nLanes = b->lanesReady;
    WavefrontBuffers* laneWave[kMaxLanes] = {&b->wave};
    cudaStream_t laneStream[kMaxLanes] = {main};
    for (int k = 1; k < nLanes; k++) {
        laneWave[k] = &b->laneWaves[k - 1];
        laneStream[k] = b->laneStreams[k - 1];
    }
    cudaStream_t s = main;
    cudaError_t e;
    if ((e = cudaMemsetAsync(b->dCounters, 0, 4 * sizeof(unsigned long long), s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(b->dError, 0, sizeof(int), s)) != cudaSuccess) return e;
    const int tables = (set.raysPerPixel + 1) * kSobolDims;
    batchSobolKernel<<<blocksFor(tables, 256), 256, 0, s>>>(b->dDirs, b->dSample, set.raysPerPixel, set.seed, b->dPassXor,
                                                          b->dSeedHash);
    n++;
    BatchFrame F{b->dViews, (int)b->views.size(), b->dScenes, set, b->dPassXor, b->dSeedHash, b->dSample,
                 b->dSum, b->dDepth, b->dPixels, b->dCounters, b->dError};
    if (b->persistent) {
        // One launch traces the frame; the cursor restarts every frame.
        const size_t smem = sizeof(uint2) * kStackCapacity * kBatchMegaBlock;
        static bool configured = false;
        if (!configured) {
            if ((e = cudaFuncSetAttribute(batchMegaKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) !=
                cudaSuccess)
                return e;
            configured = true;
        }
        int perSm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, batchMegaKernel, kBatchMegaBlock, smem) != cudaSuccess ||
            perSm < 1)
            perSm = 1;
        if ((e = cudaMemsetAsync(b->dTiles + b->views.size() + 1, 0, sizeof(unsigned), s)) != cudaSuccess) return e;
        batchMegaKernel<<<deviceSms() * perSm, kBatchMegaBlock, smem, s>>>(F, b->dTiles);
        batchAdvanceKernel<<<1, 32, 0, s>>>(b->dSample, set.raysPerPixel);
        n += 2;
        if (launches) *launches = n;
        return cudaGetLastError();
    }
    const int cap = b->wave.capacity;
    const int shadeBlocks = deviceSms() * (2048 / 256);
    if (nLanes > 1) {
        if ((e = cudaEventRecord(b->fork, main)) != cudaSuccess) return e;
        for (int k = 1; k < nLanes; k++)
            if ((e = cudaStreamWaitEvent(laneStream[k], b->fork, 0)) != cudaSuccess) return e;
    }
    int wave = 0;
    const unsigned long long total = (unsigned long long)b->pixels * (unsigned long long)set.raysPerPixel;
    {
        for (unsigned long long start = 0; start < total; start += (unsigned long long)cap, wave++) {
            s = laneStream[wave % nLanes];
            WavefrontBuffers& W = *laneWave[wave % nLanes];
            BatchWave A{F, start, (unsigned)b->pixels, (int)std::min<unsigned long long>((unsigned long long)cap, total - start)};
            batchGenerateKernel<<<blocksFor(A.n, 256), 256, 0, s>>>(A, W);
            n++;
            int q = 0;
            for (int bounce = 0; bounce < set.maxBounces; bounce++) {
                batchResetQueuesKernel<<<1, 32, 0, s>>>(W, q);
                unsigned long long* rays = &b->dCounters[bounce == 0 ? 0 : 1];
                switch (b->block) {
                    case 64: launchTraversal<64>(false, b->aWide, b->aPacked, W, q, b->dViews, b->dScenes, rays, b->dError, b->refill, s); break;
                    case 256: launchTraversal<256>(false, b->aWide, b->aPacked, W, q, b->dViews, b->dScenes, rays, b->dError, b->refill, s); break;
                    default: launchTraversal<128>(false, b->aWide, b->aPacked, W, q, b->dViews, b->dScenes, rays, b->dError, b->refill, s); break;
                }
                batchShadeKernel<<<shadeBlocks, 256, 0, s>>>(A, W, q, bounce);
                unsigned long long* shadowRays = &b->dCounters[2];
                switch (b->block) {
                    case 64: launchTraversal<64>(true, b->aWide, b->aPacked, W, q, b->dViews, b->dScenes, shadowRays, b->dError, b->refill, s); break;
                    case 256: launchTraversal<256>(true, b->aWide, b->aPacked, W, q, b->dViews, b->dScenes, shadowRays, b->dError, b->refill, s); break;
                    default: launchTraversal<128>(true, b->aWide, b->aPacked, W, q, b->dViews, b->dScenes, shadowRays, b->dError, b->refill, s); break;
                }
                n += 4;
                q ^= 1;
            }
            // Samples of a pixel are added in sample order, whichever lane
            // ran the previous wave.
            if (nLanes > 1 && wave > 0 && (e = cudaStreamWaitEvent(s, b->accumulated, 0)) != cudaSuccess) return e;
            for (int first = 0; first < A.n;) {
                const long long rowEnd = (long long)((A.start + (unsigned)first) / b->pixels + 1) * (long long)b->pixels -
                                         (long long)A.start;
                const int count = (int)std::min<long long>(rowEnd, A.n) - first;
                batchAccumulateKernel<<<blocksFor(count, 256), 256, 0, s>>>(A, W, first, count);
                first += count;
                n++;
            }
            if (nLanes > 1 && (e = cudaEventRecord(b->accumulated, s)) != cudaSuccess) return e;
        }
    }
    for (int k = 1; k < nLanes; k++) {
        if ((e = cudaEventRecord(b->laneJoins[k - 1], laneStream[k])) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(main, b->laneJoins[k - 1], 0)) != cudaSuccess) return e;
    }
    s = main;
    batchAdvanceKernel<<<1, 32, 0, s>>>(b->dSample, set.raysPerPixel);
    n++;
    if (launches) *launches = n;
    return cudaGetLastError();
}

bool validBatchSettings(const RenderSettings* st) {
    return st->raysPerPixel >= 1 && st->raysPerPixel <= 16 && st->maxBounces >= 1 && st->maxBounces <= 32 &&
           st->exposure > 0 && st->aperture >= 0 && st->focusDistance > 0 && st->skyStrength >= 0;
}

bool renderFrame(Batch* b, const RenderSettings* settings, float* ms) {
    if (b->scenes.empty() || b->views.empty()) { b->error = "RtxBatchRender: add a scene and a view first"; return false; }
    if (!validBatchSettings(settings)) { b->error = "RtxBatchRender: invalid settings"; return false; }
    if (cudaSetDevice(b->device) != cudaSuccess) { b->error = "RtxBatchRender: could not make the batch's device current"; return false; }
    if (!ensureArena(b) || !ensureViews(b) || !ensureWave(b, settings->raysPerPixel)) return false;
    if (!b->haveLast || std::memcmp(settings, &b->last, sizeof(RenderSettings))) {
        resetSamples(b);
        dropGraph(b);
        b->last = *settings;
        b->haveLast = true;
    }
    Settings set;
    std::memcpy(&set, settings, sizeof(set));
    cudaError_t e;
    int launches = 0;
    if (b->useGraph && !b->graphValid) {
        cudaGraph_t graph = nullptr;
        if ((e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) return failB(b, e, "graph capture");
        cudaError_t enq = enqueueFrame(b, set, &launches);
        e = cudaStreamEndCapture(b->stream, &graph);
        if (enq != cudaSuccess) { if (graph) cudaGraphDestroy(graph); return failB(b, enq, "graph capture"); }
        if (e != cudaSuccess) return failB(b, e, "graph capture");
        e = cudaGraphInstantiate(&b->exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) { b->exec = nullptr; return failB(b, e, "graph instantiation"); }
        b->graphValid = true;
        b->frameLaunches = launches;
    }
    if ((e = cudaEventRecord(b->start, b->stream)) != cudaSuccess) return failB(b, e);
    if (b->useGraph) {
        e = cudaGraphLaunch(b->exec, b->stream);
    } else {
        e = enqueueFrame(b, set, &launches);
        b->frameLaunches = launches;
    }
    if (e != cudaSuccess) return failB(b, e, "frame launch");
    if ((e = cudaEventRecord(b->stop, b->stream)) != cudaSuccess) return failB(b, e);
    if ((e = cudaEventSynchronize(b->stop)) != cudaSuccess) return failB(b, e, "frame");
    float elapsed = 0;
    if ((e = cudaEventElapsedTime(&elapsed, b->start, b->stop)) != cudaSuccess) return failB(b, e);
    unsigned long long counters[4];
    int overflow = 0;
    if ((e = cudaMemcpy(counters, b->dCounters, sizeof(counters), cudaMemcpyDeviceToHost)) != cudaSuccess) return failB(b, e);
    if ((e = cudaMemcpy(&overflow, b->dError, sizeof(int), cudaMemcpyDeviceToHost)) != cudaSuccess) return failB(b, e);
    if (overflow) { b->error = "BVH traversal stack overflow"; return false; }
    b->samples += (unsigned)settings->raysPerPixel;
    RtxBatchStats& st = b->stats;
    st.primaryRays = counters[0];
    st.secondaryRays = counters[1];
    st.shadowRays = counters[2];
    st.paths = (unsigned long long)b->pixels * (unsigned long long)settings->raysPerPixel;
    st.frameMs = elapsed;
    st.kernelLaunches = b->frameLaunches;
    st.graph = b->useGraph;
    if (ms) *ms = elapsed;
    b->error.clear();
    return true;
}

}  // namespace

void* RtxBatchCreate(void) { return new Batch(); }

void RtxBatchDestroy(void* p) {
    Batch* b = static_cast<Batch*>(p);
    if (!b) return;
    if (b->device >= 0) (void)cudaSetDevice(b->device);  // freeing goes on regardless
    freeArena(b);
    freeViews(b);
    freeWavefront(b->wave);
    freeLanes(b);
    for (BatchSceneData& S : b->scenes) {
        freeBvh(S.bvh);
        if (S.dTris) cudaFree(S.dTris);
    }
    void* owned[] = {b->dDirs, b->dPassXor, b->dSeedHash, b->dSample, b->dCounters, b->dError};
    for (void* q : owned)
        if (q) cudaFree(q);
    if (b->start) cudaEventDestroy(b->start);
    if (b->stop) cudaEventDestroy(b->stop);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

const char* RtxBatchLastError(void* p) { return p ? static_cast<Batch*>(p)->error.c_str() : "null batch"; }

int RtxBatchAddScene(void* p, const Triangle* triangles, int count) {
    Batch* b = static_cast<Batch*>(p);
    if (!b) return -1;
    if (!triangles || count <= 0) { b->error = "RtxBatchAddScene: need triangles and count > 0"; return -1; }
    if (!ensureBase(b)) return -1;
    if (cudaSetDevice(b->device) != cudaSuccess) { b->error = "RtxBatchAddScene: could not make the batch's device current"; return -1; }
    // Prepared on the device like RtInitialize's scenes (rt_upload.cuh); the
    // emitters come back to the host for the arena's emitter list.
    BatchSceneData S;
    S.count = count;
    Light* dLights = nullptr;
    UploadResult up;
    std::string why;
    cudaError_t e = uploadScene(triangles, count, b->stream, &S.dTris, &dLights, up, why);
    if (e != cudaSuccess) { b->error = why; return -1; }
    S.lightArea = up.lightArea;
    S.lights.resize((size_t)up.lightCount);
    if (up.lightCount &&
        (e = cudaMemcpy(S.lights.data(), dLights, sizeof(Light) * S.lights.size(), cudaMemcpyDeviceToHost)) != cudaSuccess) {
        cudaFree(dLights);
        cudaFree(S.dTris);
        failB(b, e, "scene");
        return -1;
    }
    cudaFree(dLights);
    if (!buildScene(b, S)) { freeBvh(S.bvh); cudaFree(S.dTris); return -1; }
    b->scenes.push_back(S);
    b->stats.buildMs += S.build.buildMs + S.build.collapseMs;
    b->stats.triangles += count;
    b->stats.scenes = (int)b->scenes.size();
    freeArena(b);
    return (int)b->scenes.size() - 1;
}

int RtxBatchAddView(void* p, int scene, const CameraData* camera, int width, int height) {
    Batch* b = static_cast<Batch*>(p);
    if (!b) return -1;
    if (!camera || scene < 0 || scene >= (int)b->scenes.size() || width < 1 || height < 1 || width > 4096 ||
        height > 4096) {
        b->error = "RtxBatchAddView: need a scene id, a camera and 1 <= width, height <= 4096";
        return -1;
    }
    BatchViewData V;
    std::memcpy(&V.cam, camera, sizeof(Camera));
    V.w = width; V.h = height; V.scene = scene; V.pixelStart = 0;
    b->views.push_back(V);
    b->stats.pixels += (long long)width * height;
    b->stats.views = (int)b->views.size();
    freeViews(b);
    return (int)b->views.size() - 1;
}

int RtxBatchSetEnvironment(void* p, int mode, float r, float g, float bl) {
    Batch* b = static_cast<Batch*>(p);
    if (!b) return 0;
    if ((mode != 0 && mode != 1) || !(r >= 0) || !(g >= 0) || !(bl >= 0)) {
        b->error = "RtxBatchSetEnvironment: mode 0 or 1 and non-negative radiance";
        return 0;
    }
    float3 c = mode ? make_float3(r, g, bl) : make_float3(0.0f, 0.0f, 0.0f);
    if (mode != b->environmentMode || std::memcmp(&c, &b->environment, sizeof(c))) {
        b->environmentMode = mode;
        b->environment = c;
        freeArena(b);  // the scene table carries the environment
    }
    return 1;
}

int RtxBatchRender(void* p, const RenderSettings* settings, float* milliseconds) {
    Batch* b = static_cast<Batch*>(p);
    if (!b || !settings) return 0;
    return renderFrame(b, settings, milliseconds) ? 1 : 0;
}

void RtxBatchReset(void* p) {
    Batch* b = static_cast<Batch*>(p);
    if (b && b->stream) resetSamples(b);
}

unsigned RtxBatchSampleCount(void* p) { return p ? static_cast<Batch*>(p)->samples : 0u; }

int RtxBatchReadImage(void* p, int view, unsigned char* output, int outputBytes) {
    Batch* b = static_cast<Batch*>(p);
    if (!b) return 0;
    if (view < 0 || view >= (int)b->views.size() || !output || !b->viewsReady || !b->samples) {
        b->error = "RtxBatchReadImage: render first and pass a view id";
        return 0;
    }
    const BatchViewData& V = b->views[view];
    const size_t bytes = (size_t)V.w * V.h * 4;
    if (outputBytes < 0 || (size_t)outputBytes < bytes) { b->error = "RtxBatchReadImage: buffer too small"; return 0; }
    cudaError_t e = cudaMemcpy(output, b->dPixels + V.pixelStart, bytes, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? 1 : (failB(b, e), 0);
}

int RtxBatchReadAccumulation(void* p, int view, PixelSum* sums, int count) {
    Batch* b = static_cast<Batch*>(p);
    if (!b) return 0;
    if (view < 0 || view >= (int)b->views.size() || !sums || !b->viewsReady || !b->samples) {
        b->error = "RtxBatchReadAccumulation: render first and pass a view id";
        return 0;
    }
    const BatchViewData& V = b->views[view];
    const size_t n = (size_t)V.w * V.h;
    if (count < 0 || (size_t)count < n) { b->error = "RtxBatchReadAccumulation: buffer too small"; return 0; }
    cudaError_t e = cudaMemcpy(sums, b->dSum + V.pixelStart, n * sizeof(Accum), cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? 1 : (failB(b, e), 0);
}

int RtxBatchSetTuning(void* p, int key, int value) {
    Batch* b = static_cast<Batch*>(p);
    if (!b) return 0;
    switch (key) {
        case RTX_BATCH_BLOCK:
            if (value != 64 && value != 128 && value != 256) break;
            if (value != b->block) { b->block = value; dropGraph(b); }
            return 1;
        case RTX_BATCH_CAPACITY:
            if (value < 1024) break;
            b->capacity = value;
            return 1;
        case RTX_BATCH_REFILL:
            if (value < 1 || value > 32) break;
            if (value != b->refill) { b->refill = value; dropGraph(b); }
            return 1;
        case RTX_BATCH_GRAPH:
            if (value != 0 && value != 1) break;
            b->useGraph = value;
            if (!value) dropGraph(b);
            return 1;
        case RTX_BATCH_WIDTH:
            if (value != 4 && value != 8) break;
            if (value != b->width) { b->width = value; freeArena(b); }
            return 1;
        case RTX_BATCH_PIECES:
            if (value < 1 || value > 8) break;
            if (value != b->pieces) { b->pieces = value; freeArena(b); }
            return 1;
        case RTX_BATCH_LEAF:
            if (value < 1 || value > 8) break;
            if (value != b->leaf) { b->leaf = value; freeArena(b); }
            return 1;
        case RTX_BATCH_LANES:
            if (value < 1 || value > kMaxLanes) break;
            if (value != b->lanes) { b->lanes = value; dropGraph(b); }
            return 1;
        case RTX_BATCH_PERSISTENT:
            if (value != 0 && value != 1) break;
            if (value != b->persistent) { b->persistent = value; dropGraph(b); }
            return 1;
        default:
            break;
    }
    b->error = "RtxBatchSetTuning: unknown key or value out of range";
    return 0;
}

int RtxBatchAutotune(void* p, const RenderSettings* settings, RtxBatchTune* results, int maxResults, int* count) {
    Batch* b = static_cast<Batch*>(p);
    if (!b) return 0;
    if (!settings || !validBatchSettings(settings) || maxResults < 0 || (maxResults > 0 && !results)) {
        b->error = "RtxBatchAutotune: invalid settings or result buffer";
        return 0;
    }
    RenderSettings probe = *settings;
    probe.raysPerPixel = 1;
    std::vector<RtxBatchTune> tried;
    // Frame time of the current tuning: best of two frames after a warm-up.
    auto measure = [&](float& best) -> bool {
        best = 1e30f;
        for (int i = 0; i < 3; i++) {
            float ms = 0;
            if (!renderFrame(b, &probe, &ms)) return false;
            if (i > 0) best = std::min(best, ms);
        }
        tried.push_back(RtxBatchTune{b->block, waveCapacity(b, probe.raysPerPixel), b->refill, b->width, best, b->pieces,
                                     b->lanes});
        return true;
    };
    auto trial = [&](int key, int value, float& ms) -> bool {
        return RtxBatchSetTuning(b, key, value) && measure(ms);
    };
    // Coordinate search: pieces per triangle, BVH width, block size, queue
    // capacity, refill, lanes of waves.
    float bestMs = 0;
    if (!measure(bestMs)) return 0;
    struct Axis { int key; std::vector<int> values; int* current; };
    std::vector<int> caps;
    for (long long c : {262144ll, 1048576ll, 4194304ll, 16777216ll})
        if (c < (long long)b->pixels || caps.empty()) caps.push_back((int)std::min<long long>(c, (long long)b->pixels));
    if ((long long)b->pixels <= 16777216ll && caps.back() != (int)b->pixels) caps.push_back((int)b->pixels);
    Axis axes[] = {{RTX_BATCH_PIECES, {3, 1, 2}, &b->pieces},
                   {RTX_BATCH_WIDTH, {8, 4}, &b->width},
                   {RTX_BATCH_BLOCK, {64, 128, 256}, &b->block},
                   {RTX_BATCH_CAPACITY, caps, &b->capacity},
                   {RTX_BATCH_REFILL, {8, 16, 24, 32}, &b->refill},
                   {RTX_BATCH_LANES, {4, 2, 1}, &b->lanes}};
    if (b->capacity <= 0) b->capacity = waveCapacity(b, probe.raysPerPixel);
    for (Axis& a : axes) {
        int bestValue = *a.current;
        for (int v : a.values) {
            if (v == bestValue) continue;
            float ms = 0;
            if (!trial(a.key, v, ms)) return 0;
            if (ms < bestMs) { bestMs = ms; bestValue = v; }
        }
        if (!RtxBatchSetTuning(b, a.key, bestValue)) return 0;
    }
    if (!ensureArena(b)) return 0;
    resetSamples(b);
    b->haveLast = false;
    dropGraph(b);
    const int n = (int)std::min<size_t>(tried.size(), (size_t)maxResults);
    for (int i = 0; i < n; i++) results[i] = tried[i];
    if (count) *count = (int)tried.size();
    return 1;
}

int RtxBatchStatsGet(void* p, RtxBatchStats* stats) {
    Batch* b = static_cast<Batch*>(p);
    if (!b || !stats) return 0;
    b->stats.block = b->block;
    b->stats.capacity = b->viewsReady ? waveCapacity(b, b->haveLast ? b->last.raysPerPixel : 1) : b->capacity;
    b->stats.refill = b->refill;
    b->stats.width = b->width;
    b->stats.pieces = b->pieces;
    b->stats.lanes = b->lanes;
    *stats = b->stats;
    return 1;
}
