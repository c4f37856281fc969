// Host build of the library's portable code paths, for CPU-only checks.
//
// Test infrastructure: the wide-BVH collapse (rt_collapse.cuh), the traversal
// (rt_bvh.cuh) and the integrator (rt_integrator.cuh) are written for host and
// device; this file compiles them for the host so tests can compare them with
// the oracle without a GPU. The binary tree fed to the collapse comes from the
// caller (the oracle's builder, which equals the reference's); the GPU builder
// itself is checked by the GPU tests.
#include <vector>

#include "../../custom-ray-tracing-shader_b200/csrc/rt_collapse.cuh"
#include "../../custom-ray-tracing-shader_b200/csrc/rt_integrator.cuh"

using namespace rt;

extern "C" {

// Padded primitive boxes with the builder's expressions (Native/bvh.cuh:38-48).
static void primBoxes(const SceneTri* tris, int n, std::vector<float4>& lo, std::vector<float4>& hi) {
    lo.resize(n); hi.resize(n);
    for (int i = 0; i < n; i++) {
        const SceneTri& t = tris[i];
        float3 o = t.origin;
        float3 b = v3(o.x + t.edge1.x, o.y + t.edge1.y, o.z + t.edge1.z);
        float3 c = v3(o.x + t.edge2.x, o.y + t.edge2.y, o.z + t.edge2.z);
        float l[3], h[3];
        for (int a = 0; a < 3; a++) {
            float oa = comp(o, a), ba = comp(b, a), ca = comp(c, a);
            l[a] = fminf(fminf(fminf(FLT_MAX, oa), ba), ca);
            h[a] = fmaxf(fmaxf(fmaxf(-FLT_MAX, oa), ba), ca);
            float pad = 1e-5f + 1e-6f * fmaxf(fabsf(l[a]), fabsf(h[a]));
            l[a] -= pad; h[a] += pad;
        }
        lo[i] = make_float4(l[0], l[1], l[2], 0.0f);
        hi[i] = make_float4(h[0], h[1], h[2], 0.0f);
    }
}

// Collapses a reference-layout binary BVH. result: [0] wide nodes, [1] depth,
// [2] error code, [3] packed triangle count.
int hc_collapse(const BinNode* bn, const int* order, const SceneTri* tris, int n, uint4* wideOut, int wideCapacity,
                float4* packedOut, int* result, int group, int width) {
    std::vector<float4> plo, phi;
    primBoxes(tris, n, plo, phi);
    int jobCapacity = 2 * n + 8;
    std::vector<Job> jobs{Job{0, 0, 0, 0, 0}}, next((size_t)jobCapacity);
    int counters[4] = {1, 0, 0, 0};
    int depth = 0;
    while (!jobs.empty()) {
        depth++;
        counters[2] = 0;
        for (const Job& j : jobs)
            collapseJob(j, bn, order, plo.data(), phi.data(), tris, next.data(), reinterpret_cast<WideNode*>(wideOut),
                        packedOut, counters, wideCapacity, jobCapacity, n, group, width);
        if (counters[3]) break;
        jobs.assign(next.begin(), next.begin() + counters[2]);
    }
    result[0] = counters[0];
    result[1] = depth;
    result[2] = counters[3];
    result[3] = counters[1];
    return counters[3] == 0;
}

// Ray queries (28-byte origin/direction/limit records) against a wide BVH.
// stats: [0] node visits, [1] triangle tests, [2] stack overflows.
// stats: [0] node visits, [1] triangle tests, [2] queries that overflowed a
// stack of stackLimit entries (0: the library's default, kStackCapacity).
void hc_query(const uint4* wide, const float4* packed, const float* queries, int count, int any, Hit* out,
              unsigned long long* stats, unsigned* perRay, int stackLimit) {
    uint2 stack[kStackCapacity];
    const int limit = stackLimit > 0 && stackLimit < kStackCapacity ? stackLimit : kStackCapacity;
    for (int i = 0; i < count; i++) {
        const float* q = queries + 7 * (size_t)i;
        int overflow = 0;
        TraversalCounters tc{0, 0};
        float3 o = v3(q[0], q[1], q[2]), d = v3(q[3], q[4], q[5]);
        out[i] = any ? traverse<true>(wide, packed, o, d, q[6], stack, 1, &overflow, &tc, limit)
                     : traverse<false>(wide, packed, o, d, q[6], stack, 1, &overflow, &tc, limit);
        stats[0] += tc.nodes; stats[1] += tc.tris; stats[2] += (unsigned)overflow;
        if (perRay) { perRay[2 * (size_t)i] = tc.nodes; perRay[2 * (size_t)i + 1] = tc.tris; }
    }
}

// One render pass with the library's integrator on the host. tris are the
// linearised scene triangles; dirs the 260x32 Sobol direction numbers.
int hc_render(const SceneTri* tris, const Light* lights, int lightCount, float lightArea, const uint4* wide,
              const float4* packed, const unsigned* dirs, const Camera* cam, const Settings* set, int w, int h,
              unsigned sample0, Accum* sums, uchar4* pixels, unsigned long long* counts) {
    std::vector<unsigned> passXor((size_t)set->raysPerPixel * kSobolDims), seedHash(kSobolDims);
    for (int r = 0; r < set->raysPerPixel; r++)
        for (int d = 0; d < kSobolDims; d++) passXor[(size_t)r * kSobolDims + d] = sobolXor(dirs, sample0 + (unsigned)r, (unsigned)d);
    for (int d = 0; d < kSobolDims; d++) seedHash[d] = sobolHash(set->seed + (unsigned)d * 0x9e3779b9u);
    SceneView sc{tris, wide, packed, lights, lightCount, lightArea, 0, 0, make_float3(0.0f, 0.0f, 0.0f)};
    uint2 stack[kStackCapacity];
    int overflow = 0;
    unsigned p = 0, q = 0, s = 0;
    static std::vector<float> depth;
    if (sample0 == 0 || depth.size() != (size_t)w * h) depth.assign((size_t)w * h, 0.0f);
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++)
            renderPixel(sc, *cam, *set, x, y, w, h, sample0, passXor.data(), seedHash.data(), sums, depth.data(),
                        pixels, stack, 1, &overflow, p, q, s);
    counts[0] = p; counts[1] = q; counts[2] = s;
    return overflow == 0;
}

}  // extern "C"
