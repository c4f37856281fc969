// Reference harness: the reference renderer's own code, compiled from its
// source file where it lies (Native/renderer.cu, which pulls in
// Native/bvh.cuh and Native/sampling.cuh), with a few extern "C" wrappers so
// tests can call its host-side functions directly.
//
// Test infrastructure only. This file is the checker, never the product: it
// is built into oracle/_ref/libref.so by oracle/Makefile, and only tests/,
// the smoke check and the CPU-baseline leg of bench.py load it. Its purpose is
// to pin the CPU restatement in oracle/oracle.cpp against the reference itself
// and to time the reference's own CPU backend.
//
// Why wrappers: RtInitialize (Native/renderer.cu:340) uploads to the GPU, so
// on a machine without a GPU it fails. The wrappers repeat its host steps
// (Native/renderer.cu:344-357: copy, sRGB->linear, emitter CDF, BvhBuilder)
// by calling the reference's own helpers, then drive collision()
// (renderer.cu:136), pixel() (renderer.cu:289) and PathSampler
// (sampling.cuh:17) the same way Tools/verify_bvh.cu does.
//
// The reference's exported Rt* functions are compiled in unchanged as well;
// on a machine with a GPU, RtRender backend 2 runs the reference's own CUDA
// renderer (renderKernel, renderer.cu:303) built for sm_100a.
#include "renderer.cu"

namespace {
struct RefScene {
    std::vector<Triangle> triangles;
    std::vector<Emitter> lights;
    std::vector<BvhNode> nodes;
    std::vector<int> order;
    float lightArea = 0, buildMs = 0;
    int depth = 0;
    Scene view() const {
        return Scene{triangles.data(), nodes.data(), order.data(), lights.data(), (int)triangles.size(),
                     (int)lights.size(), lightArea, sobolDirections()};
    }
};
}  // namespace

// Ray query record (origin, direction, limit), as in Tools/verify_bvh.cu:8.
struct RefQuery { float3 origin, direction; float limit; };
static_assert(sizeof(RefQuery) == 28 && sizeof(Hit) == 16 && sizeof(PixelSum) == 40 && sizeof(BvhNode) == 32);

extern "C" {

// Host steps of RtInitialize (renderer.cu:344-357) on a private scene object.
void* refh_scene_create(const Triangle* triangles, int count) {
    if (!triangles || count <= 0) return nullptr;
    auto* s = new RefScene();
    s->triangles.assign(triangles, triangles + count);
    for (int i = 0; i < count; i++) {
        Triangle& t = s->triangles[i];
        t.color = toLinear(t.color);
        t.specularColor = toLinear(t.specularColor);
        if (t.emission > 0) {
            float3 areaNormal = cross(t.edge1, t.edge2);
            s->lightArea += .5f * sqrtf(dot(areaNormal, areaNormal));
            s->lights.push_back({i, s->lightArea});
        }
    }
    auto start = std::chrono::steady_clock::now();
    BvhBuilder bvh(s->triangles);
    s->nodes = std::move(bvh.nodes);
    s->order = std::move(bvh.order);
    s->depth = bvh.maxDepth;
    s->buildMs = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - start).count();
    return s;
}
void refh_scene_destroy(void* scene) { delete static_cast<RefScene*>(scene); }
int refh_scene_node_count(void* scene) { return (int)static_cast<RefScene*>(scene)->nodes.size(); }
int refh_scene_depth(void* scene) { return static_cast<RefScene*>(scene)->depth; }
float refh_scene_build_ms(void* scene) { return static_cast<RefScene*>(scene)->buildMs; }
int refh_scene_light_count(void* scene) { return (int)static_cast<RefScene*>(scene)->lights.size(); }
float refh_scene_light_area(void* scene) { return static_cast<RefScene*>(scene)->lightArea; }
void refh_scene_nodes(void* scene, BvhNode* out) {
    auto* s = static_cast<RefScene*>(scene);
    std::memcpy(out, s->nodes.data(), s->nodes.size() * sizeof(BvhNode));
}
void refh_scene_order(void* scene, int* out) {
    auto* s = static_cast<RefScene*>(scene);
    std::memcpy(out, s->order.data(), s->order.size() * sizeof(int));
}
void refh_scene_lights(void* scene, Emitter* out) {
    auto* s = static_cast<RefScene*>(scene);
    std::memcpy(out, s->lights.data(), s->lights.size() * sizeof(Emitter));
}
void refh_scene_triangles(void* scene, Triangle* out) {
    auto* s = static_cast<RefScene*>(scene);
    std::memcpy(out, s->triangles.data(), s->triangles.size() * sizeof(Triangle));
}

// Sobol values: out[i*ndim+d] = PathSampler{pixel[i], sample[i], seed[i]}.get(d).
int refh_sobol(const unsigned* pixel, const unsigned* sample, const unsigned* seed, int count, int ndim, float* out) {
    if (ndim > SobolDimensions) return 0;
    const unsigned* directions = sobolDirections();
    for (int i = 0; i < count; i++) {
        PathSampler s{directions, pixel[i], sample[i], seed[i]};
        for (int d = 0; d < ndim; d++) out[(size_t)i * ndim + d] = s.get((unsigned)d);
    }
    return 1;
}

// The reference's BVH traversal (collision, renderer.cu:136) for a batch of rays.
void refh_query(void* scene, const RefQuery* queries, int count, int any, Hit* out, int threads) {
    Scene view = static_cast<RefScene*>(scene)->view();
    #pragma omp parallel for schedule(dynamic, 256) num_threads(threads > 0 ? threads : 1)
    for (int i = 0; i < count; i++)
        out[i] = collision(queries[i].origin, queries[i].direction, view, queries[i].limit, any != 0);
}

// The reference's CPU backend loop (renderer.cu:405-414) over rows [y0, y1):
// pixel() per pixel with the session's accumulated sample count.
void refh_render(void* scene, const CameraData* camera, const RenderSettings* settings, int w, int h,
                 unsigned sample, PixelSum* sum, unsigned char* rgba, int y0, int y1, int threads) {
    Scene view = static_cast<RefScene*>(scene)->view();
    CameraData cam = *camera;
    RenderSettings set = *settings;
    #pragma omp parallel for schedule(dynamic, 1) num_threads(threads > 0 ? threads : 1)
    for (int y = y0; y < y1; y++)
        for (int x = 0; x < w; x++)
            pixel(x, y, cam, view, set, sum, reinterpret_cast<uchar4*>(rgba), w, h, sample);
}

int refh_max_threads() { return omp_get_max_threads(); }

// Copies the raw accumulation of a session created with the reference's own
// RtCreate/RtInitialize after a backend-2 render (the reference keeps it
// private, Native/renderer.cu:61). Needs a GPU.
int refh_session_sums(void* session, PixelSum* out, int count) {
    auto* s = static_cast<Session*>(session);
    if (!s || !s->ready || count < s->width * s->height) return 0;
    if (s->lastBackend != 2) {
        std::memcpy(out, s->sum.data(), sizeof(PixelSum) * (size_t)s->width * s->height);
        return 1;
    }
    return cudaMemcpy(out, s->deviceSum, sizeof(PixelSum) * (size_t)s->width * s->height, cudaMemcpyDeviceToHost) == cudaSuccess;
}

}  // extern "C"
