/*
 * C ABI of libCudaRayTracer.so: a drop-in for the reference renderer's native
 * library (Ekansh-K/custom-ray-tracing-shader, Native/renderer.cu), rebuilt for
 * NVIDIA B200 (sm_100a).
 *
 * The thirteen Rt* entry points keep the reference's names, argument meaning,
 * return convention (1 = success, 0 = failure, message in RtLastError) and
 * struct layouts, so the Unity P/Invoke bindings
 * (UnityRayTracer/Assets/RayTracing/RayTraceSession.cs:36-63) and the ctypes
 * bindings (Tools/native_api.py:28-43) load it unchanged.
 *
 * The Rtx* entry points are additive: they have no counterpart in the
 * reference's exported ABI. Each one names the reference test harness whose
 * job it takes over (per-ray queries, sampler values, the built BVH, the raw
 * accumulation buffer, ray counters).
 *
 * All entry points use plain C types and pointers. A session is not
 * thread-safe; use one session per thread (the reference's rule).
 */
#ifndef CUDA_RAY_TRACER_H
#define CUDA_RAY_TRACER_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- records (layouts fixed by Native/renderer.cu:11-30,46 and Native/bvh.cuh:7) ---- */

typedef struct RtVector { float x, y, z; } RtVector;

/* Scene primitive, 116 bytes (Native/renderer.cu:11-18). Colours are sRGB
 * encoded; the library converts them to linear at RtInitialize
 * (Native/renderer.cu:347). */
typedef struct Triangle {
    RtVector origin, edge1, edge2, color;
    float emission;
    int oneSided;
    RtVector normal0, normal1, normal2;
    int mesh;
    RtVector specularColor;
    float smoothness, specularProbability;
} Triangle;

/* Camera, 64 bytes (Native/renderer.cu:21-24). */
typedef struct CameraData {
    RtVector origin, right, up, forward;
    float tanHalfFov, aspect, orthographicSize;
    int orthographic;
} CameraData;

/* Per-call settings, 28 bytes (Native/renderer.cu:25-30). */
typedef struct RenderSettings {
    int maxBounces;
    float exposure, aperture, focusDistance, skyStrength;
    unsigned seed;
    int raysPerPixel;
} RenderSettings;

/* Progressive accumulation record, 40 bytes per pixel, row-major with row 0 at
 * the bottom of the image (Native/renderer.cu:46, :291). */
typedef struct PixelSum {
    RtVector radiance, albedo, normal;
    unsigned covered;
} PixelSum;

/* Binary BVH node in the reference layout, 32 bytes (Native/bvh.cuh:7). A
 * leaf has count > 0 and covers order[first .. first+count); an interior node
 * has count == 0 and children first, first+1. */
typedef struct BvhNode {
    RtVector low;
    int first;
    RtVector high;
    int count;
} BvhNode;

/* Ray query and its result (Tools/verify_bvh.cu:8 and Native/renderer.cu:43). */
typedef struct RtxQuery { RtVector origin, direction; float limit; } RtxQuery;
typedef struct RtxHit { int index; float distance, u, v; } RtxHit;

/* Counters and timings of the last successful RtRender / RtxRenderDevice. */
typedef struct RtxRenderStats {
    unsigned long long primaryRays;   /* closest-hit queries at bounce 0 */
    unsigned long long secondaryRays; /* closest-hit queries at bounces >= 1 */
    unsigned long long shadowRays;    /* any-hit queries for light sampling */
    unsigned long long paths;         /* width * height * raysPerPixel */
    float renderMs;                   /* device time of the render kernels (CUDA events) */
    float extendMs;                   /* part of renderMs spent in closest-hit traversal kernels */
    float shadowMs;                   /* part of renderMs spent in any-hit traversal kernels */
    int kernelLaunches;               /* kernels launched by the render */
    float primaryMs;                  /* part of extendMs spent on bounce 0 (wavefront integrator) */
    float denoiseMs;                  /* device time of the last RtDenoise's kernels (AOVs, network or
                                         filter, display), without its read-back */
} RtxRenderStats;

/* Summary of the acceleration structure built at RtInitialize. */
typedef struct RtxBvhStats {
    int binaryNodes;        /* reference-layout nodes (same count as Native/bvh.cuh) */
    int binaryDepth;        /* deepest binary node (the reference's maxDepth) */
    int wideNodes;          /* 8-wide compressed nodes used for traversal */
    int wideDepth;          /* deepest wide node of the traversal tree */
    float buildMs;          /* device time of the binned-SAH build (CUDA events) */
    float collapseMs;       /* device time of the wide collapse and triangle packing */
    double sahCost;         /* SAH cost of the binary tree, normalised by the root area */
    float uploadMs;         /* wall time of the upload with sRGB decode and emitter list on the device */
    int distinctColours;    /* colour values decoded through the host's powf (the rest on the device) */
    int lightCount;         /* emitting triangles */
    float lightArea;        /* their total area */
    int pieces;             /* pieces per triangle of the traversal tree (1: the reference's tree) */
    float pieceBuildMs;     /* device time of the traversal tree's build and collapse (0 with 1 piece) */
} RtxBvhStats;

/* ---- the reference's thirteen exports ---- */

/* Native/renderer.cu:309. Returns a new, empty session. */
void* RtCreate(void);
/* Native/renderer.cu:332. Frees the session and everything it owns. */
void RtDestroy(void* session);
/* Native/renderer.cu:319. Frees scene and image buffers; the session stays usable. */
void RtShutdown(void* session);
/* Native/renderer.cu:340. Copies the triangles, builds the BVH on the GPU and
 * allocates a width x height image. 1 <= width, height <= 4096, count > 0. */
int RtInitialize(void* session, const Triangle* triangles, int count, int width, int height);
/* Native/renderer.cu:374. Adds settings->raysPerPixel paths per pixel to the
 * accumulation and writes the tonemapped RGBA8 image (width*height*4 bytes,
 * bottom row first) to output. backend: 0 CPU one thread, 1 CPU all threads,
 * 2 CUDA, 3 Embree (not available in this build: returns 0). computeMs
 * receives the render time (CUDA events for backend 2). */
int RtRender(void* session, const CameraData* camera, const RenderSettings* settings,
             unsigned char* output, int outputBytes, int backend, float* computeMs);
/* Native/renderer.cu:436. Filters the current accumulation into output without
 * changing it, the sample count or the accumulation version. */
int RtDenoise(void* session, unsigned char* output, int outputBytes, float* milliseconds);
/* Native/renderer.cu:310. Clears the accumulation and bumps its version. */
void RtReset(void* session);
/* Native/renderer.cu:311. */
unsigned RtAccumulationVersion(void* session);
/* Native/renderer.cu:312. Paths accumulated per pixel since the last reset. */
unsigned RtSampleCount(void* session);
/* Native/renderer.cu:313. Always 0: this build has no Embree backend. */
float RtEmbreeBuildMilliseconds(void* session);
/* Native/renderer.cu:314. 0 after a CUDA render, else the CPU thread count. */
int RtCpuThreadCount(void* session);
/* Native/renderer.cu:315. Binary node count, depth and BVH build time in ms. */
void RtBvhInfo(void* session, int* nodes, int* depth, float* buildMs);
/* Native/renderer.cu:318. Message for the last failure on this session. */
const char* RtLastError(void* session);

/* ---- additive entry points (no counterpart in the reference's exported ABI) ---- */

/* Per-ray BVH queries on the GPU for a host array of rays, closest hit
 * (any = 0) or any hit (any != 0), against the session's scene. Takes over the
 * job of the reference's differential checker kernel (Tools/verify_bvh.cu:26-34). */
int RtxQueryRays(void* session, const RtxQuery* queries, int count, int any, RtxHit* hits);
/* Sampler values on the GPU: out[i*ndim + d] = sample d of the path
 * (pixel[i], sample[i], seed[i]); ndim <= 260. Takes over the job of the
 * reference's sampler check kernel (Tools/verify_sampling.cu:8-13). */
int RtxSobolSamples(const unsigned* pixel, const unsigned* sample, const unsigned* seed, int count, int ndim, float* out);
/* Copies the GPU-built binary BVH in the reference layout (node count from
 * RtBvhInfo) and its primitive order (one int per triangle). The BVH checker
 * reads the same arrays from the reference session (Tools/verify_bvh.cu:42-66). */
int RtxExportBvh(void* session, BvhNode* nodes, int nodeCapacity, int* order, int orderCapacity);
/* BVH summary (node counts, depths, build times, SAH cost). */
int RtxBvhStatsGet(void* session, RtxBvhStats* stats);
/* Copies the raw accumulation (width*height PixelSum records) of the last
 * backend used. The reference keeps it private (Native/renderer.cu:55,61). */
int RtxReadAccumulation(void* session, PixelSum* out, int count);
/* Counters and device timings of the last render. */
int RtxRenderStatsGet(void* session, RtxRenderStats* stats);
/* RtRender on the CUDA backend without the image copy to the host: the
 * accumulation and the device-side RGBA8 image are updated in HBM. Same
 * validation, auto-reset and sample-count rules as RtRender. */
int RtxRenderDevice(void* session, const CameraData* camera, const RenderSettings* settings, float* computeMs);
/* Selects the CUDA integrator: 0 = wavefront (queues per bounce, default),
 * 1 = one-kernel path tracer. Both give bit-identical accumulations. */
int RtxSetIntegrator(void* session, int mode);
/* Tunables of the wavefront integrator, one key at a time. Results do not
 * depend on them, only speed does (except RTX_TUNE_STACK_LIMIT below its
 * default, which makes traversal fail). Returns 0 for an unknown key or a
 * value out of range.
 *   RTX_TUNE_PATHS_IN_FLIGHT  paths per wave (>= 1024; default 16,777,216,
 *                             at most width * height * raysPerPixel); a wave
 *                             may span several of a pass's raysPerPixel rows.
 *                             Path state takes 168 bytes per path and lane
 *                             (2.8 GB per lane at the default)
 *   RTX_TUNE_POSTPONE         0 or 1; no effect on the current traversal
 *                             schedule (accepted for compatibility)
 *   RTX_TUNE_REFILL           refill a warp's idle lanes when fewer than this
 *                             many lanes are busy (1..32, default 24)
 *   RTX_TUNE_PIECES           most pieces per triangle of the traversal tree
 *                             (1..8, default 3; applies from the next
 *                             RtInitialize): triangles whose box holds much
 *                             empty space (box half area at least 12 times the
 *                             triangle's area) are cut into slabs along the
 *                             longest axis of their box, and the traversal tree
 *                             is built over the pieces' padded boxes, which
 *                             overlap less than the whole triangles' boxes; with
 *                             no such triangle, traversal uses the reference's
 *                             tree. The reference's tree is always built for
 *                             RtBvhInfo and RtxExportBvh; hits do not depend on
 *                             the tree
 *   RTX_TUNE_LEAF             leaf size of that traversal tree (1..8, default 2;
 *                             the reference tree keeps 4; applies from the next
 *                             RtInitialize)
 *   RTX_TUNE_LANES            waves in flight (1..4, default 2): wave j runs
 *                             on lane j % lanes, each lane a stream with its
 *                             own path buffers, so the end of one wave's
 *                             kernels overlaps another's; samples are still
 *                             added to each pixel in sample order
 *   RTX_TUNE_STACK_LIMIT      traversal stack entries a ray may use (1..48,
 *                             default 48, which every tree built here fits):
 *                             a query that needs more stops, and RtRender,
 *                             RtxRenderDevice and RtxQueryRays return 0 with
 *                             "BVH traversal stack overflow" (the accumulation
 *                             of that pass is not valid; RtReset before the
 *                             next one). For testing the failure path.
 */
#define RTX_TUNE_PATHS_IN_FLIGHT 1
#define RTX_TUNE_POSTPONE 2
#define RTX_TUNE_REFILL 3
#define RTX_TUNE_PIECES 4
#define RTX_TUNE_LEAF 5
#define RTX_TUNE_LANES 6
#define RTX_TUNE_STACK_LIMIT 7
int RtxSetTuning(void* session, int key, int value);

/* Which tensor-core convolution kernel the learned denoiser runs, no
 * counterpart in the reference: 0 (default) the warp-specialised TMA-fed
 * kernel wherever its shared memory allows (inference then also runs the
 * decoders' concatenated layers as two passes and fuses the output head
 * into the last layer; input rows are staged as swizzled slabs of 16-64
 * channels, and unsplit 32-channel layers issue one MMA per input row and
 * column tap over the three kernel rows' weights side by side), 1 the
 * single-role kernel for every layer, one pass each, 2 as 0 with every
 * layer's MMAs issued tap by tap per output tile over rows staged as planes
 * of 8 channels. Process-wide; 0 and 2 give identical results, 1 agrees with
 * them to BF16 rounding. */
int RtxSetConvPath(int mode);
/* Convolutions launched so far in this process by the warp-specialised
 * kernel and by the single-role kernel (either pointer may be null); no
 * counterpart in the reference. */
int RtxConvLaunchCounts(long long* pipelined, long long* singleRole);
/* Failure path of the warp-specialised convolution, no counterpart in the
 * reference: one launch whose wait on a barrier that nothing completes runs
 * out (2 ms limit) must report it through its error flag and free its
 * tensor memory without a CUDA error, and a normal launch after it must give
 * the right output. Returns 1 when both hold. Runs on the current device. */
int RtxDebugConvWaitProbe(void);

/* Failure injection on the host, no counterpart in the reference: the n-th
 * next device allocation made by the renderer (sessions, scene upload, BVH
 * build, wave buffers, batches) fails with cudaErrorMemoryAllocation without
 * calling cudaMalloc, as if the device were out of memory; n = 0 disarms it.
 * Process-wide; for testing the error paths (each must return 0, report the
 * error through RtLastError and leave the session usable). Returns 0 for
 * n < 0. */
int RtxDebugFailAllocation(int n);
/* Light arriving from outside the scene on rays that leave it after the first
 * bounce (primary misses stay black, as in the reference). mode 0: the
 * reference's sky gradient times settings->skyStrength (Native/renderer.cu:
 * 193-196, the default); mode 1: constant radiance (r, g, b), skyStrength
 * ignored. A change resets the accumulation. No counterpart in the
 * reference's exported ABI. */
int RtxSetEnvironment(void* session, int mode, float r, float g, float b);
/* Learned denoiser (no counterpart in the reference: it replaces the OptiX
 * denoiser of Native/denoiser.cuh). A 5-level convolutional U-Net (widths
 * 32-48-64-96-128, about 1.01M parameters) on BF16 tensor cores with FP32
 * accumulation. Input per pixel: the 10 floats RtxReadAovs returns; output:
 * linear radiance RGB. Returns 1 on success, 0 on failure (RtxUnetLastError).
 *   RtxUnetCreate     new network, He-normal initialisation from seed
 *   RtxUnetGetParams / RtxUnetSetParams  FP32 parameters, RtxUnetParamCount floats
 *   RtxUnetLossGrad   one forward/backward over n crops (h, w multiples of 16):
 *                     L1 loss on log(1 + radiance) and its gradient
 *   RtxUnetTrain      Adam steps over random batches (with flips) of a data set
 *   RtxUnetInfer      host-to-host inference for any h, w
 *   RtxUnetSave / RtxUnetLoad  checkpoint: parameters, and the Adam state
 *                     when optimizerState is non-zero
 *   RtxSetDenoiser    RtDenoise runs this network (NULL: guided filter) */
void* RtxUnetCreate(unsigned seed);
void RtxUnetDestroy(void* net);
long long RtxUnetParamCount(void* net);
const char* RtxUnetLastError(void* net);
int RtxUnetGetParams(void* net, float* params);
int RtxUnetSetParams(void* net, const float* params);
int RtxUnetLossGrad(void* net, const float* aovs, const float* targets, int n, int h, int w, float* loss, float* grads);
int RtxUnetTrain(void* net, const float* aovs, const float* targets, int count, int h, int w, int steps, int batch,
                 float learningRate, unsigned seed, float* losses);
int RtxUnetInfer(void* net, const float* aovs, int h, int w, float* radiance);
int RtxUnetSave(void* net, const char* path, int optimizerState);
int RtxUnetLoad(void* net, const char* path);
int RtxSetDenoiser(void* session, void* net);
/* Denoiser inputs of the current accumulation, 10 floats per pixel: colour
 * (radiance / samples), albedo / samples, normalised normal sum, first-hit
 * distance / samples (the distance is an added AOV). */
int RtxReadAovs(void* session, float* aovs, int count);
/* The linear radiance of the last RtDenoise (learned network or filter), 3
 * floats per pixel in the accumulation's order, uncovered pixels 0: what
 * RtDenoise tonemaps into its RGBA8 image, before quantisation, so quality
 * can be measured on float values. Fails unless RtDenoise succeeded after
 * the last render or reset. count >= width * height. No counterpart in the
 * reference (its OptiX pass returns only the RGBA8 image). */
int RtxReadDenoised(void* session, float* rgb, int count);
/* ---- Batched multi-scene rendering (no counterpart in the reference) ----
 * Many views of many scenes of uneven size, rendered together: every frame
 * traces the paths of all views in shared waves, so each traversal launch
 * serves rays of every scene (the scenes' BVHs live in one node array, each
 * ray starting at its scene's root), and the frame's kernel sequence is
 * replayed from a CUDA graph. A view rendered in a batch accumulates exactly
 * what RtRender (backend 2) accumulates for the same scene, camera and
 * settings: the same Sobol pixel index (y * width + x of the view), sample
 * numbers and seed.
 *   RtxBatchAddScene   copies and prepares triangles like RtInitialize and
 *                      builds its BVH; returns the scene id (>= 0) or -1
 *   RtxBatchAddView    a camera on a scene with its own resolution (1..4096)
 *                      and accumulation; returns the view id or -1
 *   RtxBatchRender     one frame: raysPerPixel paths for every pixel of every
 *                      view; the accumulation restarts when the settings
 *                      bytes change or a view or scene is added
 *   RtxBatchReadImage / RtxBatchReadAccumulation  one view's RGBA8 image /
 *                      PixelSum records (bottom-up rows like RtRender)
 *   RtxBatchSetTuning  RTX_BATCH_* keys below
 *   RtxBatchAutotune   times candidate pieces per triangle, BVH widths, block
 *                      sizes, queue capacities, refill thresholds and lanes
 *                      of waves on this batch (frames of
 *                      one path per pixel), keeps the fastest and writes
 *                      the candidates to results (up to maxResults)
 * Returns 1 on success and 0 on failure (RtxBatchLastError) unless noted. */
#define RTX_BATCH_BLOCK 1     /* threads per block of the traversal kernels: 64, 128 or 256 */
#define RTX_BATCH_CAPACITY 2  /* paths per wave (>= 1024, default 16,777,216); a wave may span sample rows */
#define RTX_BATCH_REFILL 3    /* refill threshold of the persistent traversal (1..32) */
#define RTX_BATCH_GRAPH 4     /* 1: replay frames from a CUDA graph (default), 0: launch kernels */
#define RTX_BATCH_WIDTH 5     /* BVH node width: 4 or 8 (default 8); rebuilds every scene */
#define RTX_BATCH_PIECES 6    /* most pieces per triangle of the traversal trees (1..8, default 3; see RTX_TUNE_PIECES) */
#define RTX_BATCH_LEAF 7      /* leaf size of the traversal trees (1..8, default 2) */
#define RTX_BATCH_LANES 8     /* waves in flight (1..4, default 2; see RTX_TUNE_LANES) */
#define RTX_BATCH_PERSISTENT 9 /* 1: one persistent launch per frame pulling 16x8 tiles of every view from one
                                  queue, a thread per pixel tracing its whole paths; 0 (default): waves */
typedef struct RtxBatchTune {
    int block, capacity, refill, width;
    float frameMs;  /* device time of one frame of one path per pixel */
    int pieces;     /* pieces per triangle of the traversal trees */
    int lanes;      /* waves in flight */
} RtxBatchTune;
typedef struct RtxBatchStats {
    unsigned long long primaryRays, secondaryRays, shadowRays, paths;  /* of the last frame */
    float frameMs;                 /* device time of the last frame (CUDA events) */
    float buildMs;                 /* total BVH build time of all scenes */
    long long triangles, pixels;   /* over all scenes / views */
    int scenes, views;
    int kernelLaunches;            /* kernels in one frame (graph nodes when replayed) */
    int graph;                     /* 1 if the last frame was a graph launch */
    int block, capacity, refill, width;  /* tuning in use */
    int pieces, lanes;
} RtxBatchStats;
void* RtxBatchCreate(void);
void RtxBatchDestroy(void* batch);
const char* RtxBatchLastError(void* batch);
int RtxBatchAddScene(void* batch, const Triangle* triangles, int count);
int RtxBatchAddView(void* batch, int scene, const CameraData* camera, int width, int height);
int RtxBatchSetEnvironment(void* batch, int mode, float r, float g, float b);
int RtxBatchRender(void* batch, const RenderSettings* settings, float* milliseconds);
void RtxBatchReset(void* batch);
unsigned RtxBatchSampleCount(void* batch);
int RtxBatchReadImage(void* batch, int view, unsigned char* output, int outputBytes);
int RtxBatchReadAccumulation(void* batch, int view, PixelSum* sums, int count);
int RtxBatchSetTuning(void* batch, int key, int value);
int RtxBatchAutotune(void* batch, const RenderSettings* settings, RtxBatchTune* results, int maxResults, int* count);
int RtxBatchStatsGet(void* batch, RtxBatchStats* stats);

/* RtxQueryRays without any device allocation; no counterpart in the reference.
 * For callers that must not allocate device memory during the call (work
 * running beside a CUDA graph capture, latency-critical loops where
 * cudaMalloc/cudaFree would synchronise the device, hosts whose device memory
 * belongs to a pool). Rays and hits are staged in a file-scope device array
 * of 1,245,200 bytes (about 1.19 MiB) that every GPU loading the library
 * keeps until the process exits; count may be at most 16384 per call (larger
 * counts return 0 with a message). The first call on each device looks up
 * that array's device address, so make it before any stream capture; the
 * address is cached per device and stays valid while the device's primary
 * context lives (after cudaDeviceReset the cached address is stale, so do
 * not call this entry point again in that process). All calls on a device
 * share the array: calls whose GPU work overlaps race and must be serialised
 * by the caller. Results equal RtxQueryRays. */
int RtxQueryRaysStatic(void* session, const RtxQuery* queries, int count, int any, RtxHit* hits);

#ifdef __cplusplus
}
#endif
#endif /* CUDA_RAY_TRACER_H */
