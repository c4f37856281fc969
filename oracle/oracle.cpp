// CPU restatement of the reference renderer's hot path.
//
// TEST INFRASTRUCTURE, NOT PRODUCT CODE. Only tests/, the smoke check and the
// CPU-baseline leg of bench.py load this library, always as the checker. The
// product library (libCudaRayTracer.so) never links or calls it.
//
// It restates, in this project's own code, the arithmetic of
//   Native/sampling.cuh:17-36   scrambled Sobol sampler (PathSampler)
//   Native/bvh.cuh:11-106       binned-SAH BVH builder (BvhBuilder)
//   Native/renderer.cu:74-96    vector helpers, sRGB, display tonemap
//   Native/renderer.cu:99-178   Moller-Trumbore, slab test, BVH traversal
//   Native/renderer.cu:180-302  BRDF, sky, path integrator, pixel accumulation
//   Native/renderer.cu:344-353  scene preparation in RtInitialize
// Every floating-point expression keeps the reference's operand order, so the
// results are bit-identical to the reference's host build (pinned by
// tests/test_oracle_pin.py against oracle/_ref/libref.so and by the committed
// fixtures in tests/golden/). Compile without FMA contraction
// (-ffp-contract=off), as the reference is built with --fmad=false.
//
// The Sobol direction numbers come from the same cuRAND call the reference
// makes (curandGetDirectionVectors32, JOEKUO6 table), at run time.
#include <curand.h>
#include <omp.h>

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

namespace {

struct V3 { float x, y, z; };
inline V3 mk(float x, float y, float z) { return V3{x, y, z}; }
inline float& at(V3& v, int a) { return (&v.x)[a]; }
inline float at(const V3& v, int a) { return (&v.x)[a]; }

// ABI records, field for field as in Native/renderer.cu:11-30,46 and bvh.cuh:7.
struct Tri {
    V3 origin, edge1, edge2, color;
    float emission; int oneSided;
    V3 normal0, normal1, normal2;
    int mesh;
    V3 specularColor;
    float smoothness, specularProbability;
};
struct Camera { V3 origin, right, up, forward; float tanHalfFov, aspect, orthographicSize; int orthographic; };
struct Settings { int maxBounces; float exposure, aperture, focusDistance, skyStrength; unsigned seed; int raysPerPixel; };
struct Node { V3 low; int first; V3 high; int count; };
struct Sum { V3 radiance, albedo, normal; unsigned covered; };
struct HitRec { int index; float distance, u, v; };
struct Query { V3 origin, direction; float limit; };
struct Light { int triangle; float cumulativeArea; };
static_assert(sizeof(Tri) == 116 && sizeof(Camera) == 64 && sizeof(Settings) == 28, "ABI sizes");
static_assert(sizeof(Node) == 32 && sizeof(Sum) == 40 && sizeof(HitRec) == 16 && sizeof(Query) == 28, "record sizes");

constexpr float kPi = 3.14159265358979323846f;
constexpr int kMaxDepth = 32;      // bvh.cuh:9
constexpr int kBins = 12;          // bvh.cuh:29
constexpr int kSobolDims = 4 + 8 * 32;  // sampling.cuh:6

// ---- vector helpers (renderer.cu:76-96) ----
inline V3 add(V3 a, V3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 sub(V3 a, V3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 scale(V3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
inline V3 mul(V3 a, V3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
inline V3 normalize(V3 a) { return scale(a, 1.0f / sqrtf(fmaxf(dot(a, a), 1e-20f))); }
inline V3 mirror(V3 d, V3 n) { return sub(d, scale(n, 2.0f * dot(d, n))); }
inline float srgbToLinear(float c) { return c <= .04045f ? c / 12.92f : powf((c + .055f) / 1.055f, 2.4f); }
inline unsigned char tonemap(float c, float exposure) {
    c = 1.0f - expf(-fmaxf(c, 0.0f) * exposure);
    c = c <= .0031308f ? 12.92f * c : 1.055f * powf(c, 1.0f / 2.4f) - .055f;
    return (unsigned char)(255.0f * fminf(c, 1.0f) + .5f);
}
inline V3 orient(V3 axis, float cosine, float angle) {
    V3 tangent = normalize(cross(fabsf(axis.y) < .999f ? mk(0, 1, 0) : mk(1, 0, 0), axis));
    float sine = sqrtf(fmaxf(0.0f, 1.0f - cosine * cosine));
    return normalize(add(scale(axis, cosine), add(scale(tangent, sine * cosf(angle)), scale(cross(axis, tangent), sine * sinf(angle)))));
}
inline float power2(float a, float b) { return a * a / fmaxf(a * a + b * b, 1e-30f); }

// ---- Sobol sampler (sampling.cuh:17-36) ----
const unsigned* directionTable() {
    static const unsigned* table = [] {
        curandDirectionVectors32_t* vectors = nullptr;
        if (curandGetDirectionVectors32(&vectors, CURAND_DIRECTION_VECTORS_32_JOEKUO6) != CURAND_STATUS_SUCCESS)
            return (const unsigned*)nullptr;
        return (const unsigned*)&vectors[0][0];
    }();
    return table;
}
inline unsigned mix(unsigned v) {
    v ^= v >> 16; v *= 0x7feb352du;
    v ^= v >> 15; v *= 0x846ca68bu;
    return v ^ (v >> 16);
}
struct Sampler {
    const unsigned* dirs;
    unsigned pixel, sample, seed, base;
    float operator()(unsigned dim) const {
        dim += base;
        unsigned value = mix(pixel ^ mix(seed + dim * 0x9e3779b9u));
        unsigned gray = sample ^ (sample >> 1);
        for (unsigned bit = 0; gray; gray >>= 1, bit++)
            if (gray & 1) value ^= dirs[dim * 32 + bit];
        return (value >> 8) * (1.0f / 16777216.0f);
    }
};

// ---- binned SAH builder (bvh.cuh:11-106) ----
struct Box {
    V3 low = mk(FLT_MAX, FLT_MAX, FLT_MAX), high = mk(-FLT_MAX, -FLT_MAX, -FLT_MAX);
    void include(V3 a, V3 b) {
        for (int k = 0; k < 3; k++) { at(low, k) = fminf(at(low, k), at(a, k)); at(high, k) = fmaxf(at(high, k), at(b, k)); }
    }
    void include(const Box& o) { include(o.low, o.high); }
    float halfArea() const {
        float x = fmaxf(0.0f, high.x - low.x), y = fmaxf(0.0f, high.y - low.y), z = fmaxf(0.0f, high.z - low.z);
        return x * y + x * z + y * z;
    }
};
struct Prim { Box box; V3 centroid; };
inline int binOf(float c, float lo, float s) { return std::min(kBins - 1, std::max(0, (int)((c - lo) * s))); }

struct Builder {
    std::vector<Prim> prims;
    std::vector<int> order;
    std::vector<Node> nodes;
    int maxDepth = 0;

    explicit Builder(const std::vector<Tri>& tris) {
        size_t n = tris.size();
        prims.resize(n); order.resize(n);
        std::iota(order.begin(), order.end(), 0);
        for (size_t i = 0; i < n; i++) {
            const Tri& t = tris[i];
            V3 b = mk(t.origin.x + t.edge1.x, t.origin.y + t.edge1.y, t.origin.z + t.edge1.z);
            V3 c = mk(t.origin.x + t.edge2.x, t.origin.y + t.edge2.y, t.origin.z + t.edge2.z);
            Prim& p = prims[i];
            p.box.include(t.origin, t.origin); p.box.include(b, b); p.box.include(c, c);
            for (int k = 0; k < 3; k++) {
                at(p.centroid, k) = (at(t.origin, k) + at(b, k) + at(c, k)) / 3.0f;
                float pad = 1e-5f + 1e-6f * fmaxf(fabsf(at(p.box.low, k)), fabsf(at(p.box.high, k)));
                at(p.box.low, k) -= pad; at(p.box.high, k) += pad;
            }
        }
        nodes.reserve(n * 2); nodes.resize(1);
        // Depth-first, left before right: the same node numbering as the
        // reference's recursion (children appended in pairs when a node splits).
        struct Task { int node, first, count, depth; };
        std::vector<Task> stack{{0, 0, (int)n, 0}};
        while (!stack.empty()) {
            Task t = stack.back(); stack.pop_back();
            int left = splitNode(t.node, t.first, t.count, t.depth);
            if (left < 0) continue;
            int child = nodes[t.node].first;
            stack.push_back({child + 1, t.first + left, t.count - left, t.depth + 1});
            stack.push_back({child, t.first, left, t.depth + 1});
        }
    }
    // Returns the left child's primitive count, or -1 when the node stays a leaf.
    int splitNode(int index, int first, int count, int depth) {
        maxDepth = std::max(maxDepth, depth);
        Box box, cent;
        for (int i = first; i < first + count; i++) { const Prim& p = prims[order[i]]; box.include(p.box); cent.include(p.centroid, p.centroid); }
        nodes[index] = Node{box.low, first, box.high, count};
        if (count <= 4 || depth == kMaxDepth) return -1;
        int bestAxis = -1, bestBin = -1;
        float bestCost = box.halfArea() * count;
        for (int axis = 0; axis < 3; axis++) {
            float extent = at(cent.high, axis) - at(cent.low, axis);
            if (extent <= 1e-12f) continue;
            float s = kBins / extent, lo = at(cent.low, axis);
            Box binBox[kBins]; int binCount[kBins] = {};
            for (int i = first; i < first + count; i++) {
                const Prim& p = prims[order[i]];
                int b = binOf(at(p.centroid, axis), lo, s);
                binCount[b]++; binBox[b].include(p.box);
            }
            Box suffixBox[kBins], acc; int suffixCount[kBins], accCount = 0;
            for (int b = kBins - 1; b >= 0; b--) {
                if (binCount[b]) acc.include(binBox[b]);
                accCount += binCount[b]; suffixBox[b] = acc; suffixCount[b] = accCount;
            }
            Box prefix; int prefixCount = 0;
            for (int b = 0; b < kBins - 1; b++) {
                if (binCount[b]) prefix.include(binBox[b]);
                prefixCount += binCount[b];
                if (!prefixCount || !suffixCount[b + 1]) continue;
                float cost = box.halfArea() + prefix.halfArea() * prefixCount + suffixBox[b + 1].halfArea() * suffixCount[b + 1];
                if (cost < bestCost) { bestCost = cost; bestAxis = axis; bestBin = b; }
            }
        }
        if (bestAxis < 0) return -1;
        float lo = at(cent.low, bestAxis);
        float s = kBins / (at(cent.high, bestAxis) - lo);
        auto mid = std::partition(order.begin() + first, order.begin() + first + count,
                                  [&](int i) { return binOf(at(prims[i].centroid, bestAxis), lo, s) <= bestBin; });
        int left = (int)(mid - (order.begin() + first));
        if (left == 0 || left == count) return -1;
        int child = (int)nodes.size();
        nodes.resize(nodes.size() + 2);
        nodes[index].first = child; nodes[index].count = 0;
        return left;
    }
};

// ---- prepared scene (renderer.cu:344-353) ----
struct Stats {  // traversal work, for the algorithmic-bytes model
    long long queries = 0, interior = 0, pops = 0, tris = 0;
};
struct OScene {
    std::vector<Tri> tris;
    std::vector<Light> lights;
    std::vector<Node> nodes;
    std::vector<int> order;
    float lightArea = 0;
    int depth = 0;
    const unsigned* dirs = nullptr;
};

// ---- ray queries (renderer.cu:99-178) ----
inline float triangleHit(V3 o, V3 d, const Tri& t, float& u, float& v) {
    V3 p = cross(d, t.edge2);
    float det = dot(t.edge1, p);
    if (fabsf(det) < 1e-7f || (t.oneSided && det < 0)) return -1;
    float inv = 1.0f / det;
    V3 s = sub(o, t.origin);
    u = dot(s, p) * inv;
    if (u < 0 || u > 1) return -1;
    V3 q = cross(s, t.edge1);
    v = dot(d, q) * inv;
    if (v < 0 || u + v > 1) return -1;
    float dist = dot(t.edge2, q) * inv;
    return dist > 1e-4f ? dist : -1;
}
inline float slabEntry(V3 o, V3 inv, const Node& n, float limit) {
    float tn = 0, tf = limit;
    for (int k = 0; k < 3; k++) {
        float ok = at(o, k), ik = at(inv, k), lo = at(n.low, k), hi = at(n.high, k);
        if (ik == 0) { if (ok < lo || ok > hi) return FLT_MAX; continue; }
        float a = (lo - ok) * ik, b = (hi - ok) * ik;
        if (a > b) std::swap(a, b);
        if (a > tn) tn = a;
        if (b < tf) tf = b;
        if (tn > tf) return FLT_MAX;
    }
    return tn;
}
HitRec closest(const OScene& sc, V3 o, V3 d, float limit, bool any, Stats* st) {
    HitRec hit{-1, limit, 0, 0};
    if (st) st->queries++;
    V3 inv = mk(fabsf(d.x) < FLT_MIN ? 0 : 1.0f / d.x, fabsf(d.y) < FLT_MIN ? 0 : 1.0f / d.y, fabsf(d.z) < FLT_MIN ? 0 : 1.0f / d.z);
    if (slabEntry(o, inv, sc.nodes[0], limit) == FLT_MAX) return hit;
    int stack[kMaxDepth], top = 0, cur = 0;
    for (;;) {
        const Node& n = sc.nodes[cur];
        if (n.count > 0) {
            for (int j = n.first; j < n.first + n.count; j++) {
                int i = sc.order[j];
                float u, v, t = triangleHit(o, d, sc.tris[i], u, v);
                if (st) st->tris++;
                if (t > 0 && (t < hit.distance || (t == hit.distance && i < hit.index))) {
                    hit = HitRec{i, t, u, v};
                    if (any) return hit;
                }
            }
        } else {
            if (st) st->interior++;
            int a = n.first, b = a + 1;
            float ta = slabEntry(o, inv, sc.nodes[a], hit.distance), tb = slabEntry(o, inv, sc.nodes[b], hit.distance);
            if (tb < ta) { std::swap(a, b); std::swap(ta, tb); }
            if (ta != FLT_MAX) {
                if (tb != FLT_MAX) stack[top++] = b;
                cur = a;
                continue;
            }
        }
        bool more = false;
        while (top > 0) {
            cur = stack[--top];
            if (st) st->pops++;
            if (slabEntry(o, inv, sc.nodes[cur], hit.distance) != FLT_MAX) { more = true; break; }
        }
        if (!more) break;
    }
    return hit;
}
// Plain triangle loop (Tools/verify_bvh.cu:9-19): the independent check.
HitRec bruteForce(const OScene& sc, V3 o, V3 d, float limit, bool any) {
    HitRec hit{-1, limit, 0, 0};
    for (int i = 0; i < (int)sc.tris.size(); i++) {
        float u, v, t = triangleHit(o, d, sc.tris[i], u, v);
        if (t > 0 && t < hit.distance) { hit = HitRec{i, t, u, v}; if (any) return hit; }
    }
    return hit;
}

// ---- integrator (renderer.cu:180-302) ----
inline float phongExponent(const Tri& t) { float r = fmaxf(1.0f - t.smoothness, .015f); return fmaxf(0.0f, 2.0f / (r * r) - 2.0f); }
inline V3 bsdf(const Tri& t, V3 n, V3 refl, V3 dir, float& pdf) {
    float cosine = fmaxf(0.0f, dot(n, dir)), p = t.specularProbability;
    pdf = (1.0f - p) * cosine / kPi;
    V3 value = scale(t.color, (1.0f - p) / kPi);
    if (p > 0 && t.smoothness < .999f) {
        float e = phongExponent(t), lobe = powf(fmaxf(0.0f, dot(refl, dir)), e);
        pdf += p * (e + 1.0f) * lobe / (2.0f * kPi);
        value = add(value, scale(t.specularColor, p * (e + 2.0f) * lobe / (2.0f * kPi)));
    }
    return value;
}
inline V3 sky(V3 d, float strength) {
    float t = fminf(1.0f, fmaxf(0.0f, d.y));
    return scale(add(scale(mk(.65f, .72f, .82f), 1.0f - t), scale(mk(.15f, .32f, .65f), t)), strength);
}
struct RayCounts { long long primary = 0, secondary = 0, shadow = 0; Stats closestWork, shadowWork; };

Sum tracePath(const OScene& sc, const Camera& cam, const Settings& set, int x, int y, int w, int h, unsigned sample, RayCounts* rc) {
    Sampler rng{sc.dirs, (unsigned)(y * w + x), sample, set.seed, 0};
    float px = 2.0f * ((float)x + rng(0)) / (float)w - 1.0f, py = 2.0f * ((float)y + rng(1)) / (float)h - 1.0f;
    V3 o = cam.origin;
    V3 d = normalize(add(cam.forward, add(scale(cam.right, px * cam.aspect * cam.tanHalfFov), scale(cam.up, py * cam.tanHalfFov))));
    if (cam.orthographic) {
        o = add(o, add(scale(cam.right, px * cam.aspect * cam.orthographicSize), scale(cam.up, py * cam.orthographicSize)));
        d = cam.forward;
    } else if (set.aperture > 0) {
        float angle = 2.0f * kPi * rng(2), radius = .5f * set.aperture * sqrtf(rng(3));
        V3 lens = add(scale(cam.right, radius * cosf(angle)), scale(cam.up, radius * sinf(angle)));
        V3 focus = add(o, scale(d, set.focusDistance / dot(d, cam.forward)));
        o = add(o, lens); d = normalize(sub(focus, o));
    }
    Sum out{};
    V3 thr = mk(1, 1, 1);
    float prevPdf = 0;
    for (int bounce = 0; bounce < set.maxBounces; bounce++) {
        rng.base = 4 + 8 * bounce;
        if (rc) (bounce == 0 ? rc->primary : rc->secondary)++;
        HitRec hit = closest(sc, o, d, 1e30f, false, rc ? &rc->closestWork : nullptr);
        if (hit.index < 0) {
            if (bounce > 0) out.radiance = add(out.radiance, mul(thr, sky(d, set.skyStrength)));
            break;
        }
        const Tri& t = sc.tris[hit.index];
        V3 g = normalize(cross(t.edge1, t.edge2));
        if (dot(g, d) > 0) g = scale(g, -1.0f);
        if (bounce == 0) {
            out.covered = 1;
            out.albedo = t.emission > 0 ? mk(1, 1, 1) : add(scale(t.color, 1.0f - t.specularProbability), scale(t.specularColor, t.specularProbability));
            out.normal = g;
        }
        if (t.emission > 0) {
            float lightPdf = sc.lightArea > 0 ? hit.distance * hit.distance / (sc.lightArea * fmaxf(1e-6f, -dot(g, d))) : 0;
            float wgt = prevPdf > 0 ? power2(prevPdf, lightPdf) : 1.0f;
            out.radiance = add(out.radiance, scale(mul(thr, t.color), t.emission * wgt));
            break;
        }
        V3 n = normalize(add(scale(t.normal0, 1.0f - hit.u - hit.v), add(scale(t.normal1, hit.u), scale(t.normal2, hit.v))));
        if (dot(n, g) < 0) n = scale(n, -1.0f);
        if (dot(n, d) >= 0) n = g;
        if (bounce == 0) out.normal = n;
        V3 p = add(o, scale(d, hit.distance));
        V3 refl = mirror(d, n);
        o = add(p, scale(g, .0005f));
        if (!sc.lights.empty()) {
            int count = (int)sc.lights.size();
            float pick = rng(0) * sc.lightArea;
            int l = 0;
            while (l < count - 1 && pick >= sc.lights[l].cumulativeArea) l++;
            const Tri& L = sc.tris[sc.lights[l].triangle];
            float root = sqrtf(rng(1)), v = rng(2);
            V3 target = add(L.origin, add(scale(L.edge1, root * (1.0f - v)), scale(L.edge2, root * v)));
            V3 off = sub(target, o);
            float dist2 = dot(off, off), dist = sqrtf(dist2);
            V3 wi = scale(off, 1.0f / dist), ln = normalize(cross(L.edge1, L.edge2));
            float lightCos = -dot(ln, wi);
            if (!L.oneSided) lightCos = fabsf(lightCos);
            float surfCos = fmaxf(0.0f, dot(n, wi));
            if (lightCos > 0 && surfCos > 0 && dot(g, wi) > 0) {
                if (rc) rc->shadow++;
                if (closest(sc, o, wi, dist - .001f, true, rc ? &rc->shadowWork : nullptr).index < 0) {
                    float pdf, lightPdf = dist2 / (sc.lightArea * lightCos);
                    V3 f = bsdf(t, n, refl, wi, pdf);
                    float wgt = bounce + 1 == set.maxBounces ? 1.0f : power2(lightPdf, pdf);
                    out.radiance = add(out.radiance, scale(mul(mul(thr, f), L.color), L.emission * surfCos * wgt / lightPdf));
                }
            }
        }
        if (bounce + 1 == set.maxBounces) break;
        bool spec = rng(3) < t.specularProbability;
        if (spec && t.smoothness >= .999f) {
            d = refl; thr = mul(thr, t.specularColor); prevPdf = 0;
        } else {
            float cosine = spec ? powf(rng(4), 1.0f / (phongExponent(t) + 1.0f)) : sqrtf(rng(4));
            d = orient(spec ? refl : n, cosine, 2.0f * kPi * rng(5));
            if (dot(g, d) <= 0 || dot(n, d) <= 0) break;
            float pdf;
            V3 f = bsdf(t, n, refl, d, pdf);
            if (pdf < 1e-12f) break;
            thr = mul(thr, scale(f, dot(n, d) / pdf)); prevPdf = pdf;
        }
        if (bounce >= 3) {
            float survive = fminf(.95f, fmaxf(thr.x, fmaxf(thr.y, thr.z)));
            if (rng(6) >= survive) break;
            thr = scale(thr, 1.0f / survive);
        }
    }
    return out;
}
void shadePixel(const OScene& sc, const Camera& cam, const Settings& set, int x, int y, int w, int h, unsigned sample,
                Sum* sums, unsigned char* rgba, RayCounts* rc) {
    size_t i = (size_t)y * w + x;
    Sum total = sample ? sums[i] : Sum{};
    for (int r = 0; r < set.raysPerPixel; r++) {
        Sum s = tracePath(sc, cam, set, x, y, w, h, sample + (unsigned)r, rc);
        total.radiance = add(total.radiance, s.radiance);
        total.albedo = add(total.albedo, s.albedo);
        total.normal = add(total.normal, s.normal);
        total.covered += s.covered;
    }
    sums[i] = total;
    V3 avg = scale(total.radiance, 1.0f / (float)(sample + (unsigned)set.raysPerPixel));
    if (rgba) {
        rgba[i * 4 + 0] = tonemap(avg.x, set.exposure);
        rgba[i * 4 + 1] = tonemap(avg.y, set.exposure);
        rgba[i * 4 + 2] = tonemap(avg.z, set.exposure);
        rgba[i * 4 + 3] = 255;
    }
}

}  // namespace

extern "C" {

// ---- sampler ----
int orc_sobol(const unsigned* pixel, const unsigned* sample, const unsigned* seed, int count, int ndim, float* out) {
    const unsigned* dirs = directionTable();
    if (!dirs || ndim > kSobolDims) return 0;
    for (int i = 0; i < count; i++) {
        Sampler s{dirs, pixel[i], sample[i], seed[i], 0};
        for (int d = 0; d < ndim; d++) out[(size_t)i * ndim + d] = s((unsigned)d);
    }
    return 1;
}
int orc_sobol_directions(unsigned* out) {
    const unsigned* dirs = directionTable();
    if (!dirs) return 0;
    std::memcpy(out, dirs, sizeof(unsigned) * kSobolDims * 32);
    return 1;
}

// ---- scene ----
void* orc_scene_create(const void* triangles, int count) {
    if (!triangles || count <= 0) return nullptr;
    auto* sc = new OScene();
    const Tri* in = static_cast<const Tri*>(triangles);
    sc->tris.assign(in, in + count);
    for (int i = 0; i < count; i++) {
        Tri& t = sc->tris[i];
        t.color = mk(srgbToLinear(t.color.x), srgbToLinear(t.color.y), srgbToLinear(t.color.z));
        t.specularColor = mk(srgbToLinear(t.specularColor.x), srgbToLinear(t.specularColor.y), srgbToLinear(t.specularColor.z));
        if (t.emission > 0) {
            V3 an = cross(t.edge1, t.edge2);
            sc->lightArea += .5f * sqrtf(dot(an, an));
            sc->lights.push_back(Light{i, sc->lightArea});
        }
    }
    Builder b(sc->tris);
    sc->nodes = std::move(b.nodes);
    sc->order = std::move(b.order);
    sc->depth = b.maxDepth;
    sc->dirs = directionTable();
    return sc;
}
void orc_scene_destroy(void* s) { delete static_cast<OScene*>(s); }
int orc_scene_node_count(void* s) { return (int)static_cast<OScene*>(s)->nodes.size(); }
int orc_scene_depth(void* s) { return static_cast<OScene*>(s)->depth; }
int orc_scene_light_count(void* s) { return (int)static_cast<OScene*>(s)->lights.size(); }
float orc_scene_light_area(void* s) { return static_cast<OScene*>(s)->lightArea; }
void orc_scene_nodes(void* s, void* out) { auto* sc = static_cast<OScene*>(s); std::memcpy(out, sc->nodes.data(), sc->nodes.size() * sizeof(Node)); }
void orc_scene_order(void* s, int* out) { auto* sc = static_cast<OScene*>(s); std::memcpy(out, sc->order.data(), sc->order.size() * sizeof(int)); }
void orc_scene_lights(void* s, void* out) { auto* sc = static_cast<OScene*>(s); std::memcpy(out, sc->lights.data(), sc->lights.size() * sizeof(Light)); }
void orc_scene_triangles(void* s, void* out) { auto* sc = static_cast<OScene*>(s); std::memcpy(out, sc->tris.data(), sc->tris.size() * sizeof(Tri)); }

// SAH cost of a binary tree in the reference layout, normalised by the root:
// sum over interior nodes of A(n)/A(root) + sum over leaves of A(n)*count/A(root)
// (C_trav = C_isect = 1, consistent with the split cost at bvh.cuh:89).
double orc_sah_cost(const void* nodes, int count) {
    const Node* n = static_cast<const Node*>(nodes);
    auto area = [](const Node& x) {
        double a = std::max(0.0, (double)x.high.x - x.low.x), b = std::max(0.0, (double)x.high.y - x.low.y),
               c = std::max(0.0, (double)x.high.z - x.low.z);
        return a * b + a * c + b * c;
    };
    double root = area(n[0]), total = 0;
    if (root <= 0) return 0;
    for (int i = 0; i < count; i++) total += n[i].count > 0 ? area(n[i]) * n[i].count : area(n[i]);
    return total / root;
}

// ---- ray queries ----
// stats (nullable): [queries, interior visits, stack pops, triangle tests]
void orc_query(void* s, const void* queries, int count, int any, void* out, int brute, long long* stats, int threads) {
    const OScene& sc = *static_cast<OScene*>(s);
    const Query* q = static_cast<const Query*>(queries);
    HitRec* hits = static_cast<HitRec*>(out);
    std::atomic<long long> a0{0}, a1{0}, a2{0}, a3{0};
    #pragma omp parallel num_threads(threads > 0 ? threads : 1)
    {
        Stats st;
        #pragma omp for schedule(dynamic, 256)
        for (int i = 0; i < count; i++)
            hits[i] = brute ? bruteForce(sc, q[i].origin, q[i].direction, q[i].limit, any != 0)
                            : closest(sc, q[i].origin, q[i].direction, q[i].limit, any != 0, &st);
        a0 += st.queries; a1 += st.interior; a2 += st.pops; a3 += st.tris;
    }
    if (stats) { stats[0] = a0; stats[1] = a1; stats[2] = a2; stats[3] = a3; }
}

// ---- rendering ----
// One progressive pass over rows [y0, y1), like the reference's CPU backend
// (renderer.cu:405-414). counts (nullable, 11 entries): primary, secondary,
// shadow rays; then closest-ray [queries, interior, pops, tris] and
// shadow-ray [queries, interior, pops, tris].
void orc_render(void* s, const void* camera, const void* settings, int w, int h, unsigned sample, void* sums,
                unsigned char* rgba, int y0, int y1, int threads, long long* counts) {
    const OScene& sc = *static_cast<OScene*>(s);
    const Camera& cam = *static_cast<const Camera*>(camera);
    const Settings& set = *static_cast<const Settings*>(settings);
    Sum* sum = static_cast<Sum*>(sums);
    std::atomic<long long> c[11];
    for (auto& x : c) x = 0;
    #pragma omp parallel num_threads(threads > 0 ? threads : 1)
    {
        RayCounts rc;
        #pragma omp for schedule(dynamic, 1)
        for (int y = y0; y < y1; y++)
            for (int x = 0; x < w; x++) shadePixel(sc, cam, set, x, y, w, h, sample, sum, rgba, counts ? &rc : nullptr);
        if (counts) {
            c[0] += rc.primary; c[1] += rc.secondary; c[2] += rc.shadow;
            c[3] += rc.closestWork.queries; c[4] += rc.closestWork.interior; c[5] += rc.closestWork.pops; c[6] += rc.closestWork.tris;
            c[7] += rc.shadowWork.queries; c[8] += rc.shadowWork.interior; c[9] += rc.shadowWork.pops; c[10] += rc.shadowWork.tris;
        }
    }
    if (counts) for (int i = 0; i < 11; i++) counts[i] = c[i];
}

// Sampled pixels: render only the listed pixel indices (for bounded CPU timing
// on large frames). sums/rgba are full-frame buffers. counts (nullable) as in
// orc_render.
void orc_render_pixels(void* s, const void* camera, const void* settings, int w, int h, unsigned sample, void* sums,
                       unsigned char* rgba, const int* pixels, int npix, int threads, long long* counts) {
    const OScene& sc = *static_cast<OScene*>(s);
    const Camera& cam = *static_cast<const Camera*>(camera);
    const Settings& set = *static_cast<const Settings*>(settings);
    Sum* sum = static_cast<Sum*>(sums);
    std::atomic<long long> c[11];
    for (auto& x : c) x = 0;
    #pragma omp parallel num_threads(threads > 0 ? threads : 1)
    {
        RayCounts rc;
        #pragma omp for schedule(dynamic, 64)
        for (int k = 0; k < npix; k++)
            shadePixel(sc, cam, set, pixels[k] % w, pixels[k] / w, w, h, sample, sum, rgba, counts ? &rc : nullptr);
        if (counts) {
            c[0] += rc.primary; c[1] += rc.secondary; c[2] += rc.shadow;
            c[3] += rc.closestWork.queries; c[4] += rc.closestWork.interior; c[5] += rc.closestWork.pops; c[6] += rc.closestWork.tris;
            c[7] += rc.shadowWork.queries; c[8] += rc.shadowWork.interior; c[9] += rc.shadowWork.pops; c[10] += rc.shadowWork.tris;
        }
    }
    if (counts) for (int i = 0; i < 11; i++) counts[i] = c[i];
}

// Tonemap used for display (renderer.cu:86-90), exposed for tests.
unsigned char orc_tonemap(float c, float exposure) { return tonemap(c, exposure); }

int orc_max_threads() { return omp_get_max_threads(); }

}  // extern "C"
