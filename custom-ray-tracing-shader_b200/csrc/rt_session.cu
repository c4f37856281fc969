// The C ABI (include/cuda_ray_tracer.h): session lifecycle, validation,
// progressive accumulation and the additive query entry points.
//
// Behaviour follows the reference's session layer (Native/renderer.cu:309-458):
//  - RtInitialize copies the triangles, converts colours from sRGB on the host
//    and builds the emitter CDF in triangle order (renderer.cu:344-353; the
//    host conversion keeps the reference's exact powf results), uploads the
//    scene and builds the BVH on the GPU;
//  - RtRender validates (renderer.cu:377-382), resets the accumulation when
//    the backend or the bytes of camera/settings change (renderer.cu:388-389),
//    renders raysPerPixel paths per pixel, reports compute time and copies the
//    RGBA8 image out; samples += raysPerPixel (renderer.cu:417);
//  - backends 0/1 run the same integrator and traversal code compiled for the
//    host, on one thread or all OpenMP threads; backend 3 (Embree) is not
//    part of this build and is rejected with a message;
//  - RtDenoise never changes the accumulation, the sample count or the version.
#include <omp.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <curand.h>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/cuda_ray_tracer.h"
#include "rt_render.cuh"
#include "rt_conv_tc.cuh"
#include "rt_unet.cuh"
#include "rt_upload.cuh"

using namespace rt;

static_assert(sizeof(Triangle) == 116 && sizeof(CameraData) == 64 && sizeof(RenderSettings) == 28, "ABI sizes");
static_assert(sizeof(PixelSum) == 40 && sizeof(BvhNode) == 32, "record sizes");
static_assert(sizeof(RtxQuery) == 28 && sizeof(RtxHit) == 16, "query sizes");

// Pieces per triangle of the traversal tree (RTX_TUNE_PIECES; 1: traverse the
// collapse of the reference's tree).
constexpr int kDefaultPieces = 3;
// Leaf size of the traversal tree over pieces (RTX_TUNE_LEAF; the reference's
// tree keeps its own rule of 4). Measured on the 1M-triangle room at most 3
// pieces: leaves of 1, 2, 3, 4, 6, 8 gave 2,108, 2,114, 2,094, 2,078, 2,031,
// 1,987 Mrays/s.
constexpr int kDefaultTraversalLeaf = 2;

// A denoising network with its last error message (RtxUnet* entry points).
struct UnetHandle {
    rt::Unet net;
    std::string error;
    explicit UnetHandle(unsigned seed) : net(seed) {}
};

namespace rt {
// Countdown of RtxDebugFailAllocation: when it reaches the call that brings
// it from 1 to 0, that allocation fails without calling cudaMalloc.
static std::atomic<long long> g_failAllocationIn{0};
cudaError_t deviceAllocBytes(void** p, size_t bytes) {
    long long n = g_failAllocationIn.load();
    while (n > 0 && !g_failAllocationIn.compare_exchange_weak(n, n - 1)) {
    }
    if (n == 1) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    return cudaMalloc(p, bytes);
}

// The sampler's direction numbers: cuRAND's JOEKUO6 table, fetched at run
// time like the reference (sampling.cuh:10), 260 dimensions x 32 words.
const unsigned* hostSobolDirections(std::string& error) {
    static curandDirectionVectors32_t* table = nullptr;
    static curandStatus_t status = curandGetDirectionVectors32(&table, CURAND_DIRECTION_VECTORS_32_JOEKUO6);
    if (status != CURAND_STATUS_SUCCESS || !table) { error = "Could not load cuRAND Sobol direction vectors"; return nullptr; }
    return &table[0][0];
}
}  // namespace rt

namespace {

struct Session {
    std::string hostError;
    cudaError_t error = cudaSuccess;
    bool ready = false;
    int width = 0, height = 0, device = 0;
    int lastBackend = -1, cpuThreads = 0;
    unsigned samples = 0, accumulationVersion = 0;
    CameraData lastCamera{};
    RenderSettings lastSettings{};
    // Scene size and emitters (prepared on the device at RtInitialize); host
    // copies of the prepared triangles and emitters for the CPU backends,
    // fetched on their first use.
    int triCount = 0, lightCount = 0;
    float lightArea = 0;
    std::vector<SceneTri> tris;
    std::vector<Light> lights;
    bool hostSceneReady = false;
    UploadResult upload;
    // Device scene.
    cudaStream_t stream = nullptr;
    cudaEvent_t start = nullptr, stop = nullptr;
    SceneTri* dTris = nullptr;
    Light* dLights = nullptr;
    unsigned* dDirs = nullptr;
    unsigned* dPassXor = nullptr;
    unsigned* dSeedHash = nullptr;
    Accum* dSum = nullptr;
    float* dDepth = nullptr;      // running sums of first-hit distance (added AOV)
    uchar4* dPixels = nullptr;
    unsigned long long* dCounters = nullptr;
    int* dError = nullptr;
    float4* dDenoise = nullptr;
    BuiltBvh bvh;          // the reference's binary tree (RtBvhInfo, RtxExportBvh) and its wide collapse
    BuildResult build;
    BuiltBvh pieceBvh;     // traversal tree over triangle pieces (when pieces > 1)
    BuildResult pieceBuild;
    bool referenceTreeReady = false;  // bvh/build hold the reference's tree
    int pieces = kDefaultPieces;
    int traversalLeaf = kDefaultTraversalLeaf;
    WavefrontBuffers wave;
    WavefrontBuffers laneWaves[kMaxLanes - 1];  // buffers of lanes 1.. (tuning.lanes > 1)
    WaveOverlap overlap;
    // Host mirrors for the CPU backends (filled on first use).
    std::vector<Accum> hostSum;
    std::vector<float> hostDepth;
    std::vector<uint4> hostWide;
    std::vector<float4> hostPacked;
    bool hostBvhReady = false;
    // Statistics and tuning.
    RtxRenderStats stats{};
    double sahCost = -1.0;
    int integrator = 0, pathsInFlight = 0;
    TraceTuning tuning;
    int environmentMode = 0;
    float3 environment = make_float3(0.0f, 0.0f, 0.0f);
    UnetHandle* denoiser = nullptr;  // learned denoiser used by RtDenoise (not owned)
    // Where the last RtDenoise left its linear radiance inside dDenoise (float
    // offset and floats per pixel), valid until the accumulation changes.
    bool denoisedValid = false;
    size_t denoisedOffset = 0;
    int denoisedStride = 0;
};

bool fail(Session* s, cudaError_t e, const char* what = nullptr) {
    s->error = e;
    if (what) s->hostError = what;
    return false;
}

// Makes the session's device current; false (with the error recorded) when
// the runtime refuses.
bool useDevice(Session* s) {
    cudaError_t e = cudaSetDevice(s->device);
    if (e != cudaSuccess) return fail(s, e, "could not make the session's device current");
    return true;
}

// The tree that traversal uses: over triangle pieces when built, else the
// collapse of the reference's tree.
// The reference's tree, built on first use when the session traces a tree
// over triangle pieces (RtInitialize builds only the traced tree).
bool ensureReferenceTree(Session* s) {
    if (s->referenceTreeReady) return true;
    if (!s->ready) return false;
    if (!useDevice(s)) return false;
    const char* why = nullptr;
    cudaError_t e = buildBvh(s->dTris, s->triCount, s->stream, s->bvh, s->build, &why);
    if (e != cudaSuccess) return fail(s, e, why);
    s->referenceTreeReady = true;
    return true;
}

const uint4* travWide(const Session* s) { return s->pieceBvh.wideNodes ? s->pieceBvh.wideNodes : s->bvh.wideNodes; }
const float4* travPacked(const Session* s) { return s->pieceBvh.wideNodes ? s->pieceBvh.packedTris : s->bvh.packedTris; }
const BuildResult& travBuild(const Session* s) { return s->pieceBvh.wideNodes ? s->pieceBuild : s->build; }

void releaseOverlap(Session* s) {
    WaveOverlap& o = s->overlap;
    for (int k = 0; k < kMaxLanes - 1; k++) {
        freeWavefront(s->laneWaves[k]);
        if (o.streams[k]) cudaStreamDestroy(o.streams[k]);
        if (o.joins[k]) cudaEventDestroy(o.joins[k]);
    }
    if (o.fork) cudaEventDestroy(o.fork);
    if (o.accumulated) cudaEventDestroy(o.accumulated);
    o = WaveOverlap{};
}

void releaseScene(Session* s) {
    freeBvh(s->bvh);
    freeBvh(s->pieceBvh);
    s->pieceBuild = BuildResult{};
    freeWavefront(s->wave);
    releaseOverlap(s);
    void* owned[] = {s->dTris, s->dLights, s->dDirs, s->dPassXor, s->dSeedHash, s->dSum, s->dDepth, s->dPixels,
                     s->dCounters, s->dError, s->dDenoise};
    for (void* p : owned)
        if (p) cudaFree(p);
    s->dTris = nullptr; s->dLights = nullptr; s->dDirs = nullptr; s->dPassXor = nullptr; s->dSeedHash = nullptr;
    s->dSum = nullptr; s->dDepth = nullptr; s->dPixels = nullptr; s->dCounters = nullptr; s->dError = nullptr;
    s->dDenoise = nullptr;
    if (s->start) cudaEventDestroy(s->start);
    if (s->stop) cudaEventDestroy(s->stop);
    s->start = s->stop = nullptr;
    if (s->stream) cudaStreamDestroy(s->stream);
    s->stream = nullptr;
    s->tris.clear(); s->lights.clear(); s->hostSum.clear(); s->hostDepth.clear(); s->hostWide.clear();
    s->hostPacked.clear();
    s->tris.shrink_to_fit(); s->hostWide.shrink_to_fit(); s->hostPacked.shrink_to_fit();
    s->hostBvhReady = false;
    s->hostSceneReady = false;
    s->triCount = 0;
    s->lightCount = 0;
    s->upload = UploadResult{};
    s->ready = false;
    s->width = s->height = 0;
    s->samples = 0;
    s->lightArea = 0;
    s->lastBackend = -1;
    s->build = BuildResult{};
    s->referenceTreeReady = false;
    s->sahCost = -1.0;
    s->stats = RtxRenderStats{};
    s->denoisedValid = false;
}

bool validSettings(const RenderSettings* st) {
    return st->raysPerPixel >= 1 && st->raysPerPixel <= 16 && st->maxBounces >= 1 && st->maxBounces <= 32 &&
           st->exposure > 0 && st->aperture >= 0 && st->focusDistance > 0 && st->skyStrength >= 0;
}

SceneView deviceView(Session* s) {
    return SceneView{s->dTris, travWide(s), travPacked(s), s->dLights, s->lightCount, s->lightArea,
                     travBuild(s).wideDepth, s->environmentMode, s->environment, s->tuning.stackLimit};
}

// Paths per wave: RTX_TUNE_PATHS_IN_FLIGHT (default kDefaultPathsInFlight),
// at most the paths of a pass of raysPerPixel rows. Large waves make few,
// long traversal launches, so the drain at the end of each launch weighs
// little: on the 1920x1080, 16-path workload waves of one row (2.07M paths)
// gave 2,567 Mrays/s, of 2^24 paths 2,960 (168 B of path state per path and
// lane: 2.8 GB per lane).
constexpr int kDefaultPathsInFlight = 1 << 24;
// Buffers only grow while they fit the limit (the setting, or 16 rows of the
// image), so passes of different sizes do not reallocate them; a wave is at
// most the buffers' capacity.
bool ensureWave(Session* s, int raysPerPixel) {
    const long long pixels = (long long)s->width * s->height;
    const long long setting = s->pathsInFlight > 0 ? s->pathsInFlight : kDefaultPathsInFlight;
    const int need = (int)std::min<long long>(setting, pixels * raysPerPixel);
    const int limit = (int)std::min<long long>(setting, pixels * 16);
    const int cap = (s->wave.capacity >= need && s->wave.capacity <= limit) ? s->wave.capacity : need;
    cudaError_t e;
    if (s->wave.capacity != cap && (e = allocWavefront(s->wave, cap)) != cudaSuccess)
        return fail(s, e, "could not allocate wavefront buffers");
    const int lanes = s->tuning.lanes;
    WaveOverlap& o = s->overlap;
    if (lanes < o.lanes) releaseOverlap(s);  // fewer lanes: drop the extra ones
    if (lanes < 2) return true;
    if (!o.fork && ((e = cudaEventCreateWithFlags(&o.fork, cudaEventDisableTiming)) != cudaSuccess ||
                    (e = cudaEventCreateWithFlags(&o.accumulated, cudaEventDisableTiming)) != cudaSuccess)) {
        releaseOverlap(s);
        return fail(s, e, "could not create the wave lane events");
    }
    for (int k = 0; k < lanes - 1; k++) {
        if ((s->laneWaves[k].capacity != cap && (e = allocWavefront(s->laneWaves[k], cap)) != cudaSuccess) ||
            (!o.streams[k] && (e = cudaStreamCreateWithFlags(&o.streams[k], cudaStreamNonBlocking)) != cudaSuccess) ||
            (!o.joins[k] && (e = cudaEventCreateWithFlags(&o.joins[k], cudaEventDisableTiming)) != cudaSuccess)) {
            releaseOverlap(s);
            return fail(s, e, "could not allocate a wave lane");
        }
        o.buffers[k] = &s->laneWaves[k];
    }
    o.lanes = lanes;
    return true;
}

// Common render path of RtRender / RtxRenderDevice for backend 2.
bool renderDevice(Session* s, const CameraData* camera, const RenderSettings* settings, float* computeMs, bool timing) {
    Camera cam; Settings set;
    std::memcpy(&cam, camera, sizeof(cam));
    std::memcpy(&set, settings, sizeof(set));
    cudaError_t e;
    // Path buffers are (re)allocated before the timed span; the span covers
    // all of the pass's device work: sampler tables, counter resets, the
    // integrator's kernels.
    if (s->integrator != 1 && !ensureWave(s, set.raysPerPixel)) return false;
    if ((e = cudaEventRecord(s->start, s->stream)) != cudaSuccess) return fail(s, e);
    if ((e = buildSobolTables(s->dDirs, s->samples, set.raysPerPixel, set.seed, s->dPassXor, s->dSeedHash, s->stream)) != cudaSuccess) return fail(s, e);
    if ((e = cudaMemsetAsync(s->dCounters, 0, 4 * sizeof(unsigned long long), s->stream)) != cudaSuccess) return fail(s, e);
    if ((e = cudaMemsetAsync(s->dError, 0, sizeof(int), s->stream)) != cudaSuccess) return fail(s, e);
    RenderLaunch L{deviceView(s), cam, set, s->width, s->height, s->samples, s->dPassXor, s->dSeedHash,
                   s->dSum, s->dDepth, s->dPixels, s->dCounters, s->dError};
    int launches = 0;
    float extendMs = 0, shadowMs = 0, primaryMs = 0;
    if (s->integrator == 1) {
        e = launchMegakernel(L, s->stream, &launches);
    } else {
        e = launchWavefront(L, s->wave, s->tuning, s->stream, &launches, &extendMs, &shadowMs, timing, &primaryMs,
                            s->tuning.lanes > 1 ? &s->overlap : nullptr);
    }
    if (e != cudaSuccess) return fail(s, e);
    if ((e = cudaEventRecord(s->stop, s->stream)) != cudaSuccess) return fail(s, e);
    if ((e = cudaEventSynchronize(s->stop)) != cudaSuccess) return fail(s, e);
    if ((e = cudaEventElapsedTime(computeMs, s->start, s->stop)) != cudaSuccess) return fail(s, e);
    unsigned long long counters[4];
    int overflow = 0;
    if ((e = cudaMemcpy(counters, s->dCounters, sizeof(counters), cudaMemcpyDeviceToHost)) != cudaSuccess) return fail(s, e);
    if ((e = cudaMemcpy(&overflow, s->dError, sizeof(int), cudaMemcpyDeviceToHost)) != cudaSuccess) return fail(s, e);
    if (overflow) return fail(s, cudaErrorUnknown, "BVH traversal stack overflow");
    s->stats.primaryRays = counters[0];
    s->stats.secondaryRays = counters[1];
    s->stats.shadowRays = counters[2];
    s->stats.paths = (unsigned long long)s->width * s->height * set.raysPerPixel;
    s->stats.renderMs = *computeMs;
    s->stats.extendMs = extendMs;
    s->stats.shadowMs = shadowMs;
    s->stats.primaryMs = primaryMs;
    s->stats.kernelLaunches = launches + 1;  // + the sampler-table kernel
    return true;
}

// Host copies of the prepared triangles and emitters (CPU backends).
bool ensureHostScene(Session* s) {
    if (s->hostSceneReady) return true;
    s->tris.resize((size_t)s->triCount);
    s->lights.resize((size_t)s->lightCount);
    cudaError_t e = cudaMemcpy(s->tris.data(), s->dTris, sizeof(SceneTri) * s->tris.size(), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && s->lightCount)
        e = cudaMemcpy(s->lights.data(), s->dLights, sizeof(Light) * s->lights.size(), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return fail(s, e);
    s->hostSceneReady = true;
    return true;
}

bool ensureHostBvh(Session* s) {
    if (!ensureHostScene(s)) return false;
    if (s->hostBvhReady) return true;
    s->hostWide.resize((size_t)travBuild(s).wideNodes * 5);
    s->hostPacked.resize((size_t)travBuild(s).packedTriangles * 3);
    cudaError_t e = cudaMemcpy(s->hostWide.data(), travWide(s), s->hostWide.size() * sizeof(uint4), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
        e = cudaMemcpy(s->hostPacked.data(), travPacked(s), s->hostPacked.size() * sizeof(float4), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return fail(s, e);
    s->hostBvhReady = true;
    return true;
}

// Backends 0 and 1: the integrator compiled for the host (renderer.cu:405-415).
bool renderHost(Session* s, const CameraData* camera, const RenderSettings* settings, unsigned char* output, int backend,
                float* computeMs) {
    if (!ensureHostBvh(s)) return false;
    std::string err;
    const unsigned* dirs = hostSobolDirections(err);
    if (!dirs) { s->hostError = err; return false; }
    Camera cam; Settings set;
    std::memcpy(&cam, camera, sizeof(cam));
    std::memcpy(&set, settings, sizeof(set));
    std::vector<unsigned> passXor((size_t)set.raysPerPixel * kSobolDims), seedHash(kSobolDims);
    for (int r = 0; r < set.raysPerPixel; r++)
        for (int d = 0; d < kSobolDims; d++) passXor[(size_t)r * kSobolDims + d] = sobolXor(dirs, s->samples + (unsigned)r, (unsigned)d);
    for (int d = 0; d < kSobolDims; d++) seedHash[d] = sobolHash(set.seed + (unsigned)d * 0x9e3779b9u);
    if (s->hostSum.size() != (size_t)s->width * s->height) s->hostSum.assign((size_t)s->width * s->height, Accum{});
    if (s->hostDepth.size() != (size_t)s->width * s->height) s->hostDepth.assign((size_t)s->width * s->height, 0.0f);
    float* depthSums = s->hostDepth.data();
    SceneView sc{s->tris.data(), s->hostWide.data(), s->hostPacked.data(), s->lights.data(), (int)s->lights.size(),
                 s->lightArea, travBuild(s).wideDepth, s->environmentMode, s->environment, s->tuning.stackLimit};
    const int w = s->width, h = s->height;
    const unsigned sample0 = s->samples;
    Accum* sums = s->hostSum.data();
    uchar4* pixels = reinterpret_cast<uchar4*>(output);
    unsigned long long nPrimary = 0, nSecondary = 0, nShadow = 0;
    int overflow = 0, threads = 1;
    auto begin = std::chrono::steady_clock::now();
#pragma omp parallel num_threads(backend == 1 ? omp_get_max_threads() : 1) reduction(+ : nPrimary, nSecondary, nShadow) reduction(| : overflow)
    {
#pragma omp single
        threads = omp_get_num_threads();
        uint2 stack[kStackCapacity];
        unsigned p = 0, q = 0, sh = 0;
#pragma omp for schedule(dynamic, 1)
        for (int y = 0; y < h; y++)
            for (int x = 0; x < w; x++)
                renderPixel(sc, cam, set, x, y, w, h, sample0, passXor.data(), seedHash.data(), sums, depthSums, pixels,
                            stack, 1, &overflow, p, q, sh);
        nPrimary += p; nSecondary += q; nShadow += sh;
    }
    *computeMs = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - begin).count();
    if (overflow) { s->hostError = "BVH traversal stack overflow"; return false; }
    s->cpuThreads = threads;
    s->stats = RtxRenderStats{};
    s->stats.primaryRays = nPrimary; s->stats.secondaryRays = nSecondary; s->stats.shadowRays = nShadow;
    s->stats.paths = (unsigned long long)w * h * set.raysPerPixel;
    s->stats.renderMs = *computeMs;
    return true;
}

// Shared front half of RtRender and RtxRenderDevice (renderer.cu:376-390).
bool beginRender(Session* s, const CameraData* camera, const RenderSettings* settings, int backend) {
    s->denoisedValid = false;
    if (s->ready && s->device >= 0 && !useDevice(s)) return false;
    if (backend == 3) {
        s->hostError = "Embree backend (3) is not available in this build";
        s->error = cudaErrorInvalidValue;
        return false;
    }
    s->hostError.clear();
    if (s->lastBackend != backend || std::memcmp(camera, &s->lastCamera, sizeof(CameraData)) ||
        std::memcmp(settings, &s->lastSettings, sizeof(RenderSettings))) {
        s->samples = 0;
        s->accumulationVersion++;
    }
    s->lastBackend = backend;
    s->lastCamera = *camera;
    s->lastSettings = *settings;
    s->cpuThreads = 0;
    return true;
}

}  // namespace

extern "C" {

void* RtCreate(void) { return new Session(); }

void RtReset(void* p) {
    Session* s = static_cast<Session*>(p);
    if (s) { s->samples = 0; s->accumulationVersion++; s->denoisedValid = false; }
}
unsigned RtAccumulationVersion(void* p) { return p ? static_cast<Session*>(p)->accumulationVersion : 0u; }
unsigned RtSampleCount(void* p) { return p ? static_cast<Session*>(p)->samples : 0u; }
float RtEmbreeBuildMilliseconds(void*) { return 0.0f; }
int RtCpuThreadCount(void* p) { return p ? static_cast<Session*>(p)->cpuThreads : 0; }
void RtBvhInfo(void* p, int* nodes, int* depth, float* buildMs) {
    Session* s = static_cast<Session*>(p);
    if (s && s->ready && !ensureReferenceTree(s)) s = nullptr;  // zeros, and RtLastError says why
    if (nodes) *nodes = s ? s->build.binaryNodes : 0;
    if (depth) *depth = s ? s->build.binaryDepth : 0;
    if (buildMs) *buildMs = s ? s->build.buildMs : 0.0f;
}
const char* RtLastError(void* p) {
    Session* s = static_cast<Session*>(p);
    if (s && !s->hostError.empty()) return s->hostError.c_str();
    return cudaGetErrorString(s ? s->error : cudaErrorInvalidValue);
}
void RtShutdown(void* p) {
    Session* s = static_cast<Session*>(p);
    if (!s) return;
    // Releasing on another device than the scene's would free nothing; the
    // attempt goes on regardless so the session is left empty.
    if (s->device >= 0 && s->stream) (void)useDevice(s);
    releaseScene(s);
    s->hostError.clear();
}
void RtDestroy(void* p) {
    Session* s = static_cast<Session*>(p);
    if (s) { RtShutdown(s); delete s; }
}

int RtInitialize(void* p, const Triangle* triangles, int count, int width, int height) {
    Session* s = static_cast<Session*>(p);
    if (!s) return 0;
    RtShutdown(s);
    if (!triangles || count <= 0 || width <= 0 || height <= 0 || width > 4096 || height > 4096) {
        s->hostError = "RtInitialize: need triangles, count > 0 and 1 <= width, height <= 4096";
        s->error = cudaErrorInvalidValue;
        return 0;
    }
    cudaError_t e = cudaGetDevice(&s->device);
    if (e != cudaSuccess) { fail(s, e); return 0; }
    std::string err;
    const unsigned* dirs = hostSobolDirections(err);
    if (!dirs) { s->hostError = err; return 0; }
#define RT_CHECK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { fail(s, e_); releaseScene(s); return 0; } } while (0)
    RT_CHECK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    RT_CHECK(cudaEventCreate(&s->start));
    RT_CHECK(cudaEventCreate(&s->stop));
    // The triangles go to the device as they are; sRGB decode and the
    // emitter list are computed there with the reference's results
    // (renderer.cu:344-353; rt_upload.cuh).
    e = uploadScene(triangles, count, s->stream, &s->dTris, &s->dLights, s->upload, err);
    if (e != cudaSuccess) {
        fail(s, e);
        releaseScene(s);
        s->hostError = err;
        return 0;
    }
    s->triCount = count;
    s->lightCount = s->upload.lightCount;
    s->lightArea = s->upload.lightArea;
    RT_CHECK(rt::deviceAlloc(&s->dDirs, sizeof(unsigned) * kSobolDims * 32));
    RT_CHECK(cudaMemcpyAsync(s->dDirs, dirs, sizeof(unsigned) * kSobolDims * 32, cudaMemcpyHostToDevice, s->stream));
    RT_CHECK(rt::deviceAlloc(&s->dPassXor, sizeof(unsigned) * 16 * kSobolDims));
    RT_CHECK(rt::deviceAlloc(&s->dSeedHash, sizeof(unsigned) * kSobolDims));
    RT_CHECK(rt::deviceAlloc(&s->dSum, sizeof(Accum) * (size_t)width * height));
    RT_CHECK(rt::deviceAlloc(&s->dDepth, sizeof(float) * (size_t)width * height));
    RT_CHECK(rt::deviceAlloc(&s->dPixels, sizeof(uchar4) * (size_t)width * height));
    RT_CHECK(rt::deviceAlloc(&s->dCounters, 4 * sizeof(unsigned long long)));
    RT_CHECK(rt::deviceAlloc(&s->dError, 2 * sizeof(int)));
    const char* why = nullptr;
    // The tree that is traced is built here: over triangle pieces when some
    // triangle is split, else the reference's own tree. The reference's tree
    // (RtBvhInfo, RtxExportBvh, RtxBvhStatsGet) is then built on its first
    // use (ensureReferenceTree), so RtInitialize pays for the traced tree
    // only.
    int pieceTotal = count;
    s->referenceTreeReady = false;
    e = cudaSuccess;
    if (s->pieces > 1) e = pieceMap(s->dTris, count, s->pieces, s->stream, nullptr, &pieceTotal);
    if (e == cudaSuccess && pieceTotal > count) {
        e = buildBvh(s->dTris, count, s->stream, s->pieceBvh, s->pieceBuild, &why, 3, 8, s->pieces, s->traversalLeaf);
        if (e == cudaSuccess) {
            void* unused[] = {s->pieceBvh.binNodes, s->pieceBvh.order, s->pieceBvh.primLo, s->pieceBvh.primHi};
            for (void* q : unused) cudaFree(q);
            s->pieceBvh.binNodes = nullptr; s->pieceBvh.order = nullptr;
            s->pieceBvh.primLo = nullptr; s->pieceBvh.primHi = nullptr;
        }
    } else if (e == cudaSuccess) {
        e = buildBvh(s->dTris, count, s->stream, s->bvh, s->build, &why);
        s->referenceTreeReady = e == cudaSuccess;
    }
    if (e != cudaSuccess) {
        fail(s, e, why);
        std::string keep = s->hostError;
        releaseScene(s);
        s->hostError = keep;
        return 0;
    }
#undef RT_CHECK
    s->width = width;
    s->height = height;
    s->ready = true;
    return 1;
}

int RtRender(void* p, const CameraData* camera, const RenderSettings* settings, unsigned char* output, int outputBytes,
             int backend, float* computeMs) {
    Session* s = static_cast<Session*>(p);
    if (!s) return 0;
    if (!camera || !settings || !output || !computeMs || !s->ready || backend < 0 || backend > 3 || outputBytes < 0 ||
        (size_t)outputBytes < (size_t)s->width * s->height * 4 || !validSettings(settings)) {
        s->error = cudaErrorInvalidValue;
        s->hostError = !s->ready ? "RtRender: session is not initialised"
                                 : "RtRender: invalid camera, settings, backend or output buffer";
        return 0;
    }
    if (!beginRender(s, camera, settings, backend)) return 0;
    if (backend == 2) {
        if (!renderDevice(s, camera, settings, computeMs, false)) return 0;
        cudaError_t e = cudaMemcpy(output, s->dPixels, (size_t)s->width * s->height * 4, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) { fail(s, e); return 0; }
    } else {
        if (!renderHost(s, camera, settings, output, backend, computeMs)) return 0;
    }
    s->samples += (unsigned)settings->raysPerPixel;
    s->error = cudaSuccess;
    return 1;
}

int RtDenoise(void* p, unsigned char* output, int outputBytes, float* milliseconds) {
    Session* s = static_cast<Session*>(p);
    if (!s) return 0;
    if (!s->ready || !s->samples || !output || !milliseconds || outputBytes < 0 ||
        (size_t)outputBytes < (size_t)s->width * s->height * 4) {
        s->error = cudaErrorInvalidValue;
        s->hostError = !s->ready ? "RtDenoise: session is not initialised"
                     : !s->samples ? "RtDenoise: render at least one pass before denoising"
                                   : "RtDenoise: invalid output buffer";
        return 0;
    }
    if (!useDevice(s)) return 0;
    auto begin = std::chrono::steady_clock::now();
    s->hostError.clear();
    size_t count = (size_t)s->width * s->height;
    cudaError_t e;
    if (!s->dDenoise && (e = rt::deviceAlloc(&s->dDenoise, sizeof(float4) * 4 * count)) != cudaSuccess) { fail(s, e); return 0; }
    if (s->lastBackend != 2) {
        if ((e = cudaMemcpyAsync(s->dSum, s->hostSum.data(), count * sizeof(Accum), cudaMemcpyHostToDevice, s->stream)) != cudaSuccess) { fail(s, e); return 0; }
    }
    if (s->lastBackend != 2 && s->hostDepth.size() == count) {
        if ((e = cudaMemcpyAsync(s->dDepth, s->hostDepth.data(), count * sizeof(float), cudaMemcpyHostToDevice, s->stream)) != cudaSuccess) { fail(s, e); return 0; }
    }
    if ((e = cudaEventRecord(s->start, s->stream)) != cudaSuccess) { fail(s, e); return 0; }
    if (s->denoiser) {
        // Learned denoiser: running sums -> U-Net (AOVs formed in its input
        // kernel, as RtxReadAovs forms them) -> display, on the session stream.
        float* radiance = reinterpret_cast<float*>(s->dDenoise) + 10 * count;
        if ((e = s->denoiser->net.inferFromSums(reinterpret_cast<const float*>(s->dSum), s->dDepth, s->samples,
                                                s->height, s->width, radiance, s->stream)) != cudaSuccess) { fail(s, e); return 0; }
        if ((e = launchPresentRadiance(s->dSum, radiance, (int)count, s->lastSettings.exposure, s->dPixels, s->stream)) != cudaSuccess) { fail(s, e); return 0; }
        s->denoisedOffset = 10 * count;
        s->denoisedStride = 3;
    } else {
        if ((e = launchDenoise(s->dSum, s->samples, s->width, s->height, s->lastSettings.exposure, s->dDenoise, s->dPixels, s->stream)) != cudaSuccess) { fail(s, e); return 0; }
        s->denoisedOffset = 4 * 3 * count;  // region 3 of the filter's work buffer
        s->denoisedStride = 4;
    }
    if ((e = cudaEventRecord(s->stop, s->stream)) != cudaSuccess) { fail(s, e); return 0; }
    if ((e = cudaStreamSynchronize(s->stream)) != cudaSuccess) { fail(s, e); return 0; }
    if ((e = cudaEventElapsedTime(&s->stats.denoiseMs, s->start, s->stop)) != cudaSuccess) { fail(s, e); return 0; }
    if (s->denoiser) {
        std::string why;
        if ((e = s->denoiser->net.checkConvolutions(why)) != cudaSuccess) { fail(s, e, why.c_str()); return 0; }
    }
    if ((e = cudaMemcpy(output, s->dPixels, count * 4, cudaMemcpyDeviceToHost)) != cudaSuccess) { fail(s, e); return 0; }
    *milliseconds = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - begin).count();
    if (!(*milliseconds > 0)) *milliseconds = 1e-6f;
    s->denoisedValid = true;
    s->error = cudaSuccess;
    return 1;
}

// ---- additive entry points ----

int RtxQueryRays(void* p, const RtxQuery* queries, int count, int any, RtxHit* hits) {
    Session* s = static_cast<Session*>(p);
    if (!s) return 0;
    if (!s->ready || !queries || !hits || count < 0) { s->error = cudaErrorInvalidValue; s->hostError = "RtxQueryRays: invalid arguments"; return 0; }
    if (count == 0) return 1;
    if (!useDevice(s)) return 0;
    std::vector<float4> packed((size_t)count * 2);
    for (int i = 0; i < count; i++) {
        const RtxQuery& q = queries[i];
        packed[2 * (size_t)i] = make_float4(q.origin.x, q.origin.y, q.origin.z, q.direction.x);
        packed[2 * (size_t)i + 1] = make_float4(q.direction.y, q.direction.z, q.limit, 0.0f);
    }
    float4 *dq = nullptr, *dh = nullptr;
    std::vector<float4> out((size_t)count);
    int overflow = 0;
    cudaError_t e = rt::deviceAlloc(&dq, sizeof(float4) * packed.size());
    if (e == cudaSuccess) e = rt::deviceAlloc(&dh, sizeof(float4) * (size_t)count);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dq, packed.data(), sizeof(float4) * packed.size(), cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->dError, 0, sizeof(int), s->stream);
    if (e == cudaSuccess) e = launchQueries(travWide(s), travPacked(s), dq, count, any, dh, s->dError + 1, s->dError,
                                            travBuild(s).wideDepth, s->tuning, s->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out.data(), dh, sizeof(float4) * (size_t)count, cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&overflow, s->dError, sizeof(int), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    cudaFree(dq); cudaFree(dh);
    if (e != cudaSuccess) { fail(s, e); return 0; }
    if (overflow) { s->hostError = "BVH traversal stack overflow"; return 0; }
    for (int i = 0; i < count; i++) {
        int index;
        std::memcpy(&index, &out[i].x, 4);
        hits[i] = RtxHit{index, out[i].y, out[i].z, out[i].w};
    }
    return 1;
}

int RtxSobolSamples(const unsigned* pixel, const unsigned* sample, const unsigned* seed, int count, int ndim, float* out) {
    if (!pixel || !sample || !seed || !out || count < 0 || ndim < 0 || ndim > kSobolDims) return 0;
    if (count == 0 || ndim == 0) return 1;
    std::string err;
    const unsigned* dirs = hostSobolDirections(err);
    if (!dirs) return 0;
    unsigned *dd = nullptr, *dp = nullptr, *ds = nullptr, *dseed = nullptr;
    float* dout = nullptr;
    size_t n = (size_t)count;
    cudaError_t e = rt::deviceAlloc(&dd, sizeof(unsigned) * kSobolDims * 32);
    if (e == cudaSuccess) e = rt::deviceAlloc(&dp, sizeof(unsigned) * n);
    if (e == cudaSuccess) e = rt::deviceAlloc(&ds, sizeof(unsigned) * n);
    if (e == cudaSuccess) e = rt::deviceAlloc(&dseed, sizeof(unsigned) * n);
    if (e == cudaSuccess) e = rt::deviceAlloc(&dout, sizeof(float) * n * ndim);
    if (e == cudaSuccess) e = cudaMemcpy(dd, dirs, sizeof(unsigned) * kSobolDims * 32, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dp, pixel, sizeof(unsigned) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(ds, sample, sizeof(unsigned) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dseed, seed, sizeof(unsigned) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = launchSobolSamples(dd, dp, ds, dseed, count, ndim, dout, 0);
    if (e == cudaSuccess) e = cudaMemcpy(out, dout, sizeof(float) * n * ndim, cudaMemcpyDeviceToHost);
    cudaFree(dd); cudaFree(dp); cudaFree(ds); cudaFree(dseed); cudaFree(dout);
    return e == cudaSuccess ? 1 : 0;
}

int RtxExportBvh(void* p, BvhNode* nodes, int nodeCapacity, int* order, int orderCapacity) {
    Session* s = static_cast<Session*>(p);
    if (!s) return 0;
    if (s->ready && !ensureReferenceTree(s)) return 0;
    if (!s->ready || (nodes && nodeCapacity < s->build.binaryNodes) || (order && orderCapacity < s->triCount)) {
        s->error = cudaErrorInvalidValue; s->hostError = "RtxExportBvh: not initialised or buffers too small"; return 0;
    }
    if (!useDevice(s)) return 0;
    cudaError_t e = cudaSuccess;
    if (nodes) e = cudaMemcpy(nodes, s->bvh.binNodes, sizeof(BvhNode) * (size_t)s->build.binaryNodes, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && order) e = cudaMemcpy(order, s->bvh.order, sizeof(int) * (size_t)s->triCount, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) { fail(s, e); return 0; }
    return 1;
}

int RtxBvhStatsGet(void* p, RtxBvhStats* out) {
    Session* s = static_cast<Session*>(p);
    if (!s || !out) return 0;
    if (!s->ready) { s->hostError = "RtxBvhStatsGet: session is not initialised"; return 0; }
    if (!ensureReferenceTree(s)) return 0;
    if (s->sahCost < 0) {
        std::vector<BvhNode> nodes((size_t)s->build.binaryNodes);
        if (!useDevice(s)) return 0;
        cudaError_t e = cudaMemcpy(nodes.data(), s->bvh.binNodes, sizeof(BvhNode) * nodes.size(), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) { fail(s, e); return 0; }
        auto area = [](const BvhNode& n) {
            double x = std::max(0.0, (double)n.high.x - n.low.x), y = std::max(0.0, (double)n.high.y - n.low.y),
                   z = std::max(0.0, (double)n.high.z - n.low.z);
            return x * y + x * z + y * z;
        };
        double root = area(nodes[0]), total = 0;
        for (const BvhNode& n : nodes) total += n.count > 0 ? area(n) * n.count : area(n);
        s->sahCost = root > 0 ? total / root : 0.0;
    }
    out->binaryNodes = s->build.binaryNodes;
    out->binaryDepth = s->build.binaryDepth;
    out->wideNodes = travBuild(s).wideNodes;
    out->wideDepth = travBuild(s).wideDepth;
    out->buildMs = s->build.buildMs;
    out->collapseMs = s->build.collapseMs;
    out->sahCost = s->sahCost;
    out->uploadMs = s->upload.ms;
    out->distinctColours = s->upload.distinctColours;
    out->lightCount = s->lightCount;
    out->lightArea = s->lightArea;
    out->pieces = s->pieceBvh.wideNodes ? s->pieces : 1;
    out->pieceBuildMs = s->pieceBvh.wideNodes ? s->pieceBuild.buildMs + s->pieceBuild.collapseMs : 0.0f;
    return 1;
}

int RtxReadAccumulation(void* p, PixelSum* out, int count) {
    Session* s = static_cast<Session*>(p);
    if (!s) return 0;
    size_t need = (size_t)s->width * s->height;
    if (!s->ready || !out || count < 0 || (size_t)count < need) {
        s->error = cudaErrorInvalidValue; s->hostError = "RtxReadAccumulation: not initialised or buffer too small"; return 0;
    }
    if (s->lastBackend == 0 || s->lastBackend == 1) {
        if (s->hostSum.size() != need) return 0;
        std::memcpy(out, s->hostSum.data(), need * sizeof(PixelSum));
        return 1;
    }
    if (!useDevice(s)) return 0;
    cudaError_t e = cudaMemcpy(out, s->dSum, need * sizeof(PixelSum), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) { fail(s, e); return 0; }
    return 1;
}

int RtxRenderStatsGet(void* p, RtxRenderStats* out) {
    Session* s = static_cast<Session*>(p);
    if (!s || !out) return 0;
    *out = s->stats;
    return 1;
}

int RtxRenderDevice(void* p, const CameraData* camera, const RenderSettings* settings, float* computeMs) {
    Session* s = static_cast<Session*>(p);
    if (!s) return 0;
    if (!camera || !settings || !computeMs || !s->ready || !validSettings(settings)) {
        s->error = cudaErrorInvalidValue;
        s->hostError = "RtxRenderDevice: invalid arguments or session not initialised";
        return 0;
    }
    if (!beginRender(s, camera, settings, 2)) return 0;
    if (!renderDevice(s, camera, settings, computeMs, true)) return 0;
    s->samples += (unsigned)settings->raysPerPixel;
    s->error = cudaSuccess;
    return 1;
}

int RtxSetIntegrator(void* p, int mode) {
    Session* s = static_cast<Session*>(p);
    if (!s || mode < 0 || mode > 1) return 0;
    s->integrator = mode;
    return 1;
}

// ---- learned denoiser ----

void* RtxUnetCreate(unsigned seed) {
    UnetHandle* h = new UnetHandle(seed);
    if (cudaGetLastError() != cudaSuccess) { delete h; return nullptr; }
    return h;
}
void RtxUnetDestroy(void* p) { delete static_cast<UnetHandle*>(p); }
long long RtxUnetParamCount(void* p) { return p ? (long long)static_cast<UnetHandle*>(p)->net.paramCount() : 0; }
const char* RtxUnetLastError(void* p) { return p ? static_cast<UnetHandle*>(p)->error.c_str() : "null network"; }
static int unetResult(UnetHandle* h, cudaError_t e, const std::string& why) {
    if (e == cudaSuccess) { h->error.clear(); return 1; }
    h->error = why.empty() ? cudaGetErrorString(e) : why;
    return 0;
}
int RtxUnetGetParams(void* p, float* out) {
    UnetHandle* h = static_cast<UnetHandle*>(p);
    if (!h || !out) return 0;
    return unetResult(h, h->net.getParams(out), "");
}
int RtxUnetSetParams(void* p, const float* in) {
    UnetHandle* h = static_cast<UnetHandle*>(p);
    if (!h || !in) return 0;
    return unetResult(h, h->net.setParams(in), "");
}
int RtxUnetLossGrad(void* p, const float* aovs, const float* targets, int n, int h, int w, float* loss, float* grads) {
    UnetHandle* u = static_cast<UnetHandle*>(p);
    if (!u || !aovs || !targets || !loss || n < 1 || h < 16 || w < 16) return 0;
    std::string why;
    return unetResult(u, u->net.lossAndGradient(aovs, targets, n, h, w, loss, grads, why), why);
}
int RtxUnetTrain(void* p, const float* aovs, const float* targets, int count, int h, int w, int steps, int batch,
                 float lr, unsigned seed, float* losses) {
    UnetHandle* u = static_cast<UnetHandle*>(p);
    if (!u || !aovs || !targets || count < 1 || steps < 0 || batch < 1 || !(lr > 0)) return 0;
    std::string why;
    return unetResult(u, u->net.train(aovs, targets, count, h, w, steps, batch, lr, seed, losses, why), why);
}
int RtxUnetInfer(void* p, const float* aovs, int h, int w, float* radiance) {
    UnetHandle* u = static_cast<UnetHandle*>(p);
    if (!u || !aovs || !radiance || h < 1 || w < 1) return 0;
    float *dIn = nullptr, *dOut = nullptr;
    size_t px = (size_t)w * h;
    std::string why;
    cudaError_t e = rt::deviceAlloc(&dIn, sizeof(float) * px * 10);
    if (e == cudaSuccess) e = rt::deviceAlloc(&dOut, sizeof(float) * px * 3);
    if (e == cudaSuccess) e = cudaMemcpy(dIn, aovs, sizeof(float) * px * 10, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = u->net.inferDevice(dIn, h, w, dOut, 0, why);
    if (e == cudaSuccess) e = cudaMemcpy(radiance, dOut, sizeof(float) * px * 3, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = u->net.checkConvolutions(why);
    cudaFree(dIn); cudaFree(dOut);
    return unetResult(u, e, why);
}
int RtxUnetSave(void* p, const char* path, int optimizerState) {
    UnetHandle* u = static_cast<UnetHandle*>(p);
    if (!u || !path) return 0;
    std::string why;
    return unetResult(u, u->net.save(path, optimizerState != 0, why), why);
}
int RtxUnetLoad(void* p, const char* path) {
    UnetHandle* u = static_cast<UnetHandle*>(p);
    if (!u || !path) return 0;
    std::string why;
    return unetResult(u, u->net.load(path, why), why);
}
int RtxSetDenoiser(void* p, void* net) {
    Session* s = static_cast<Session*>(p);
    if (!s) return 0;
    s->denoiser = static_cast<UnetHandle*>(net);
    return 1;
}
int RtxReadAovs(void* p, float* out, int count) {
    Session* s = static_cast<Session*>(p);
    if (!s) return 0;
    size_t need = (size_t)s->width * s->height;
    if (!s->ready || !s->samples || !out || count < 0 || (size_t)count < need) {
        s->error = cudaErrorInvalidValue;
        s->hostError = "RtxReadAovs: render first, and pass room for width*height pixels";
        return 0;
    }
    if (!useDevice(s)) return 0;
    cudaError_t e;
    if (!s->dDenoise && (e = rt::deviceAlloc(&s->dDenoise, sizeof(float4) * 4 * need)) != cudaSuccess) { fail(s, e); return 0; }
    if (s->lastBackend != 2) {
        if ((e = cudaMemcpyAsync(s->dSum, s->hostSum.data(), need * sizeof(Accum), cudaMemcpyHostToDevice, s->stream)) != cudaSuccess) { fail(s, e); return 0; }
        if (s->hostDepth.size() == need &&
            (e = cudaMemcpyAsync(s->dDepth, s->hostDepth.data(), need * sizeof(float), cudaMemcpyHostToDevice, s->stream)) != cudaSuccess) { fail(s, e); return 0; }
    }
    float* aov = reinterpret_cast<float*>(s->dDenoise);
    if ((e = launchAovs(s->dSum, s->dDepth, s->samples, (int)need, aov, s->stream)) != cudaSuccess) { fail(s, e); return 0; }
    if ((e = cudaStreamSynchronize(s->stream)) != cudaSuccess) { fail(s, e); return 0; }
    if ((e = cudaMemcpy(out, aov, need * 10 * sizeof(float), cudaMemcpyDeviceToHost)) != cudaSuccess) { fail(s, e); return 0; }
    return 1;
}

int RtxReadDenoised(void* p, float* rgb, int count) {
    Session* s = static_cast<Session*>(p);
    if (!s) return 0;
    const size_t need = (size_t)s->width * s->height;
    if (!s->ready || !s->denoisedValid || !rgb || count < 0 || (size_t)count < need) {
        s->error = cudaErrorInvalidValue;
        s->hostError = "RtxReadDenoised: call RtDenoise after the last render, and pass room for width*height pixels";
        return 0;
    }
    if (!useDevice(s)) return 0;
    float* base = reinterpret_cast<float*>(s->dDenoise);
    // Staged in floats [0, 3 * count), free once the denoise is done and below
    // both result locations (10 * count for the network, 12 * count for the
    // filter), so the result stays readable.
    float* out = base;
    cudaError_t e;
    if ((e = launchDenoisedRgb(s->dSum, base + s->denoisedOffset, s->denoisedStride, (int)need, out, s->stream)) != cudaSuccess) { fail(s, e); return 0; }
    if ((e = cudaMemcpyAsync(rgb, out, need * 3 * sizeof(float), cudaMemcpyDeviceToHost, s->stream)) != cudaSuccess) { fail(s, e); return 0; }
    if ((e = cudaStreamSynchronize(s->stream)) != cudaSuccess) { fail(s, e); return 0; }
    return 1;
}

int RtxSetEnvironment(void* p, int mode, float r, float g, float b) {
    Session* s = static_cast<Session*>(p);
    if (!s) return 0;
    if (mode < 0 || mode > 1 || !(r >= 0) || !(g >= 0) || !(b >= 0)) {
        s->error = cudaErrorInvalidValue;
        s->hostError = "RtxSetEnvironment: mode 0 or 1 and non-negative radiance";
        return 0;
    }
    float3 c = mode == 1 ? make_float3(r, g, b) : make_float3(0.0f, 0.0f, 0.0f);
    if (mode != s->environmentMode || std::memcmp(&c, &s->environment, sizeof(c))) {
        s->environmentMode = mode;
        s->environment = c;
        RtReset(s);  // a different light field: restart the accumulation
    }
    return 1;
}

int RtxSetConvPath(int mode) {
    if (mode < 0 || mode > 2) return 0;
    rt::setConvPath(mode == 1 ? 1 : 0);
    rt::setConvPipeReference(mode == 2);
    return 1;
}

int RtxDebugConvWaitProbe(void) { return rt::convPipeWaitProbe(); }

int RtxConvLaunchCounts(long long* pipelined, long long* singleRole) {
    rt::convLaunchCounts(pipelined, singleRole);
    return 1;
}

int RtxDebugFailAllocation(int n) {
    if (n < 0) return 0;
    rt::g_failAllocationIn.store(n);
    return 1;
}

int RtxSetTuning(void* p, int key, int value) {
    Session* s = static_cast<Session*>(p);
    if (!s) return 0;
    switch (key) {
        case RTX_TUNE_PATHS_IN_FLIGHT:
            if (value < 1024) return 0;
            s->pathsInFlight = value;
            return 1;
        case RTX_TUNE_POSTPONE:  // no effect on this traversal schedule; accepted for compatibility
            return value == 0 || value == 1;
        case RTX_TUNE_REFILL:
            if (value < 1 || value > 32) return 0;
            s->tuning.refill = value;
            return 1;
        case RTX_TUNE_PIECES:
            if (value < 1 || value > 8) return 0;
            s->pieces = value;  // used by the next RtInitialize
            return 1;
        case RTX_TUNE_LEAF:
            if (value < 1 || value > 8) return 0;
            s->traversalLeaf = value;  // used by the next RtInitialize
            return 1;
        case RTX_TUNE_LANES:
            if (value < 1 || value > kMaxLanes) return 0;
            s->tuning.lanes = value;
            return 1;
        case RTX_TUNE_STACK_LIMIT:
            if (value < 1 || value > kStackCapacity) return 0;
            s->tuning.stackLimit = value;
            return 1;
        default:
            return 0;
    }
}

}  // extern "C"

// ---- ray queries without device allocation ----
//
// RtxQueryRaysStatic serves callers that must not allocate device memory
// during the call: code that runs while another thread captures CUDA work
// into a graph, or latency-critical loops where cudaMalloc/cudaFree would
// serialise with the whole device, or hosts whose device memory is owned by
// a pool the library must not touch. It stages rays and hits in one
// file-scope device array instead of cudaMalloc'd buffers.
namespace {

constexpr int kStaticQueryRays = 16384;  // largest count one call accepts
constexpr size_t kStaticPacked = 0;                                    // 2 float4 per ray, kernel layout
constexpr size_t kStaticHits = 2 * (size_t)kStaticQueryRays;           // 1 float4 per ray, RtxHit layout
constexpr size_t kStaticRaw = 3 * (size_t)kStaticQueryRays;            // caller's 28-byte RtxQuery records
constexpr size_t kStaticCounters = kStaticRaw + (7 * (size_t)kStaticQueryRays + 3) / 4;  // work counter, error flag
constexpr size_t kStaticFloat4s = kStaticCounters + 1;                 // 1,245,200 bytes in total
constexpr int kStaticMaxDevices = 64;

// One copy per GPU that loads the library, held until the process exits.
// Every call on a device shares it: calls whose GPU work overlaps race.
static __device__ __align__(256) float4 g_staticQueryScratch[kStaticFloat4s];

std::mutex g_staticScratchLock;
float4* g_staticScratchAddress[kStaticMaxDevices] = {};

// Device address of g_staticQueryScratch on the current device, looked up
// once per device (the host-side symbol is not a device address). The cached
// address is valid while the device's primary context lives; a
// cudaDeviceReset makes it stale.
float4* staticQueryScratch(int device, std::string& error) {
    if (device < 0 || device >= kStaticMaxDevices) { error = "RtxQueryRaysStatic: device index out of range"; return nullptr; }
    std::lock_guard<std::mutex> guard(g_staticScratchLock);
    if (!g_staticScratchAddress[device]) {
        void* address = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&address, g_staticQueryScratch);
        if (e != cudaSuccess || !address) {
            error = std::string("RtxQueryRaysStatic: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e);
            return nullptr;
        }
        g_staticScratchAddress[device] = static_cast<float4*>(address);
    }
    return g_staticScratchAddress[device];
}

// 28-byte RtxQuery records -> the query kernel's two-float4 layout.
__global__ void packStaticQueriesKernel(const float* raw, float4* packed, int count) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float* q = raw + 7 * (size_t)i;
    packed[2 * (size_t)i] = make_float4(q[0], q[1], q[2], q[3]);
    packed[2 * (size_t)i + 1] = make_float4(q[4], q[5], q[6], 0.0f);
}

}  // namespace

extern "C" int RtxQueryRaysStatic(void* p, const RtxQuery* queries, int count, int any, RtxHit* hits) {
    Session* s = static_cast<Session*>(p);
    if (!s) return 0;
    if (!s->ready || !queries || !hits || count < 0) {
        s->error = cudaErrorInvalidValue;
        s->hostError = "RtxQueryRaysStatic: invalid arguments or session not initialised";
        return 0;
    }
    if (count > kStaticQueryRays) {
        s->error = cudaErrorInvalidValue;
        s->hostError = "RtxQueryRaysStatic: count exceeds the static scratch capacity of 16384 rays per call";
        return 0;
    }
    if (count == 0) return 1;
    if (!useDevice(s)) return 0;
    cudaError_t e;
    std::string why;
    float4* scratch = staticQueryScratch(s->device, why);
    if (!scratch) { s->hostError = why; return 0; }
    float4* packed = scratch + kStaticPacked;
    float4* deviceHits = scratch + kStaticHits;
    float* raw = reinterpret_cast<float*>(scratch + kStaticRaw);
    int* counters = reinterpret_cast<int*>(scratch + kStaticCounters);  // [0] work counter, [1] error flag
    int overflow = 0;
    e = cudaMemcpyAsync(raw, queries, sizeof(RtxQuery) * (size_t)count, cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) {
        packStaticQueriesKernel<<<(count + 255) / 256, 256, 0, s->stream>>>(raw, packed, count);
        e = cudaGetLastError();
    }
    // The array keeps the previous call's contents: clear the counters.
    if (e == cudaSuccess) e = cudaMemsetAsync(counters, 0, 2 * sizeof(int), s->stream);
    if (e == cudaSuccess)
        e = launchQueries(travWide(s), travPacked(s), packed, count, any, deviceHits, counters, counters + 1,
                          travBuild(s).wideDepth, s->tuning, s->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(hits, deviceHits, sizeof(RtxHit) * (size_t)count, cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&overflow, counters + 1, sizeof(int), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) { fail(s, e); return 0; }
    if (overflow) { s->hostError = "BVH traversal stack overflow"; return 0; }
    return 1;
}
