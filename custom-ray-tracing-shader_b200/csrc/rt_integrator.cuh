// Path integrator (host and device), split into stages so the same code runs
// as one kernel per path or as wavefront stages over ray queues.
//
// The arithmetic is the reference's trace()/pixel() (Native/renderer.cu:
// 180-302) with the same operation order: camera ray (:198-210), per-bounce
// closest hit, sky on misses after the first bounce (:218-221), emission with
// power-heuristic MIS (:232-237), shading-normal rules (:238-241), next-event
// estimation on the emitter CDF (:247-267), diffuse/Phong/mirror sampling
// (:268-280), Russian roulette from bounce 3 (:281-285), first-hit AOVs
// (:226-231, :241) and in-order per-pixel accumulation (:289-301).
//
// The Sobol sampler (Native/sampling.cuh:17-36) is evaluated through two
// small tables built once per render pass: passXor[r][dim], the XOR of the
// direction numbers selected by the Gray code of sample (sample0 + r), and
// seedHash[dim] = hash(seed + dim * 0x9e3779b9). A value is then
// hash(pixel ^ seedHash[dim]) ^ passXor[r][dim], bit-identical to the
// reference's loop because XOR is associative and commutative.
#pragma once
#include "rt_build.cuh"

namespace rt {

constexpr int kSobolDims = 4 + 8 * 32;  // sampling.cuh:6

struct Light { int triangle; float cumulativeArea; };

struct Camera { float3 origin, right, up, forward; float tanHalfFov, aspect, orthographicSize; int orthographic; };
struct Settings { int maxBounces; float exposure, aperture, focusDistance, skyStrength; unsigned seed; int raysPerPixel; };
struct Accum { float3 radiance, albedo, normal; unsigned covered; };
static_assert(sizeof(Camera) == 64 && sizeof(Settings) == 28 && sizeof(Accum) == 40, "ABI layouts");

RT_HD unsigned sobolHash(unsigned v) {  // sampling.cuh:21-25
    v ^= v >> 16; v *= 0x7feb352du;
    v ^= v >> 15; v *= 0x846ca68bu;
    return v ^ (v >> 16);
}
// The reference's per-call form (sampling.cuh:26-35), used for sampler checks
// and to build the pass tables.
RT_HD unsigned sobolXor(const unsigned* dirs, unsigned sample, unsigned dim) {
    unsigned value = 0, gray = sample ^ (sample >> 1);
    for (unsigned bit = 0; gray; gray >>= 1, bit++)
        if (gray & 1u) value ^= dirs[dim * 32 + bit];
    return value;
}
RT_HD float sobolDirect(const unsigned* dirs, unsigned pixel, unsigned sample, unsigned seed, unsigned dim) {
    unsigned value = sobolHash(pixel ^ sobolHash(seed + dim * 0x9e3779b9u)) ^ sobolXor(dirs, sample, dim);
    return (value >> 8) * (1.0f / 16777216.0f);
}

struct Sampler {
    const unsigned* passXor;   // this path's row of the pass table (kSobolDims entries)
    const unsigned* seedHash;  // kSobolDims entries
    unsigned pixel, base;
    RT_HD float operator()(unsigned dim) const {
        unsigned d = dim + base;
#ifdef __CUDA_ARCH__
        unsigned value = sobolHash(pixel ^ __ldg(seedHash + d)) ^ __ldg(passXor + d);
#else
        unsigned value = sobolHash(pixel ^ seedHash[d]) ^ passXor[d];
#endif
        return (value >> 8) * (1.0f / 16777216.0f);
    }
};

struct SceneView {
    const SceneTri* tris;    // by original index, colours already linear
    const uint4* wide;       // WideNode records
    const float4* packed;    // triangles in wide-leaf order
    const Light* lights;
    int lightCount;
    float lightArea;
    int wideDepth;           // levels of the wide BVH (bounds the traversal stack)
    int environmentMode;     // 0: the reference's sky gradient x skyStrength; 1: constant radiance
    float3 environment;      // the constant radiance of mode 1
    int stackLimit = kStackCapacity;  // traversal stack entries before the overflow error
    unsigned root = 0;                // root node of the scene's wide tree (its first node in a batch arena)
};

// ---- BRDF and sky (renderer.cu:181-196) ----
RT_HD float phongExponent(const SceneTri& t) {
    float rough = fmaxf(1.0f - t.smoothness, .015f);
    return fmaxf(0.0f, 2.0f / (rough * rough) - 2.0f);
}
RT_HD float3 evaluateBsdf(const SceneTri& t, float3 n, float3 refl, float3 dir, float& pdf) {
    float cosine = fmaxf(0.0f, dot(n, dir)), p = t.specularProbability;
    pdf = (1.0f - p) * cosine / kPi;
    float3 value = scale(t.color, (1.0f - p) / kPi);
    if (p > 0 && t.smoothness < .999f) {
        float e = phongExponent(t), lobe = powf(fmaxf(0.0f, dot(refl, dir)), e);
        pdf += p * (e + 1.0f) * lobe / (2.0f * kPi);
        value = add(value, scale(t.specularColor, p * (e + 2.0f) * lobe / (2.0f * kPi)));
    }
    return value;
}
RT_HD float3 skyRadiance(float3 d, float strength) {
    float t = fminf(1.0f, fmaxf(0.0f, d.y));
    return scale(add(scale(v3(.65f, .72f, .82f), 1.0f - t), scale(v3(.15f, .32f, .65f), t)), strength);
}
// Radiance of rays that leave the scene after the first bounce
// (renderer.cu:218-221). Mode 0 is the reference's sky; mode 1, a constant
// environment, is an addition that leaves mode 0's results untouched.
RT_HD float3 environmentRadiance(const SceneView& sc, float3 d, float skyStrength) {
    return sc.environmentMode == 1 ? sc.environment : skyRadiance(d, skyStrength);
}
RT_HD float3 orientAround(float3 axis, float cosine, float angle) {
    float3 tangent = normalize(cross(fabsf(axis.y) < .999f ? v3(0, 1, 0) : v3(1, 0, 0), axis));
    float sine = sqrtf(fmaxf(0.0f, 1.0f - cosine * cosine));
    return normalize(add(scale(axis, cosine), add(scale(tangent, sine * cosf(angle)), scale(cross(axis, tangent), sine * sinf(angle)))));
}
RT_HD float powerHeuristic(float a, float b) { return a * a / fmaxf(a * a + b * b, 1e-30f); }

// State of one path between bounces.
struct PathState {
    float3 origin, dir, throughput;
    float prevPdf;
    float3 radiance, albedo, normal;
    unsigned covered;
    float depth;  // distance to the first hit (0 on a primary miss); an added AOV
};

// Camera ray and initial state (renderer.cu:198-214). rng.base must be 0.
RT_HD PathState startPath(const Camera& cam, const Settings& set, int x, int y, int w, int h, const Sampler& rng) {
    PathState s;
    float px = 2.0f * ((float)x + rng(0)) / (float)w - 1.0f, py = 2.0f * ((float)y + rng(1)) / (float)h - 1.0f;
    float3 o = cam.origin;
    float3 d = normalize(add(cam.forward, add(scale(cam.right, px * cam.aspect * cam.tanHalfFov), scale(cam.up, py * cam.tanHalfFov))));
    if (cam.orthographic) {
        o = add(o, add(scale(cam.right, px * cam.aspect * cam.orthographicSize), scale(cam.up, py * cam.orthographicSize)));
        d = cam.forward;
    } else if (set.aperture > 0) {
        float angle = 2.0f * kPi * rng(2), radius = .5f * set.aperture * sqrtf(rng(3));
        float3 lens = add(scale(cam.right, radius * cosf(angle)), scale(cam.up, radius * sinf(angle)));
        float3 focus = add(o, scale(d, set.focusDistance / dot(d, cam.forward)));
        o = add(o, lens);
        d = normalize(sub(focus, o));
    }
    s.origin = o; s.dir = d;
    s.throughput = v3(1, 1, 1);
    s.prevPdf = 0;
    s.radiance = v3(0, 0, 0); s.albedo = v3(0, 0, 0); s.normal = v3(0, 0, 0);
    s.covered = 0;
    s.depth = 0.0f;
    return s;
}

constexpr unsigned kContinue = 1u, kShadow = 2u;

struct ShadowRequest { float3 origin, dir; float limit; float3 contribution; };

// Everything the reference does after the closest-hit query of one bounce
// (renderer.cu:218-285). Returns kContinue when the path goes on (state holds
// the next ray) and kShadow when a light-sample ray must be tested; if that
// ray is unoccluded, the caller adds req.contribution to the radiance before
// anything of the next bounce is added. rng.base must be 4 + 8 * bounce.
RT_HD unsigned shadeBounce(const SceneView& sc, const Settings& set, int bounce, PathState& st, const Hit& hit,
                           const Sampler& rng, ShadowRequest& req) {
    if (hit.index < 0) {
        if (bounce > 0) st.radiance = add(st.radiance, mul(st.throughput, environmentRadiance(sc, st.dir, set.skyStrength)));
        return 0;
    }
    const SceneTri& t = sc.tris[hit.index];
    float3 g = normalize(cross(t.edge1, t.edge2));
    if (dot(g, st.dir) > 0) g = scale(g, -1.0f);
    if (bounce == 0) {
        st.covered = 1;
        st.depth = hit.distance;
        st.albedo = t.emission > 0 ? v3(1, 1, 1)
                                   : add(scale(t.color, 1.0f - t.specularProbability), scale(t.specularColor, t.specularProbability));
        st.normal = g;
    }
    if (t.emission > 0) {
        float lightPdf = sc.lightArea > 0 ? hit.distance * hit.distance / (sc.lightArea * fmaxf(1e-6f, -dot(g, st.dir))) : 0.0f;
        float w = st.prevPdf > 0 ? powerHeuristic(st.prevPdf, lightPdf) : 1.0f;
        st.radiance = add(st.radiance, scale(mul(st.throughput, t.color), t.emission * w));
        return 0;
    }
    float3 n = normalize(add(scale(t.normal0, 1.0f - hit.u - hit.v), add(scale(t.normal1, hit.u), scale(t.normal2, hit.v))));
    if (dot(n, g) < 0) n = scale(n, -1.0f);
    if (dot(n, st.dir) >= 0) n = g;
    if (bounce == 0) st.normal = n;
    float3 p = add(st.origin, scale(st.dir, hit.distance));
    float3 refl = mirror(st.dir, n);
    st.origin = add(p, scale(g, .0005f));
    unsigned flags = 0;
    if (sc.lightCount > 0) {
        // The reference scans the cumulative areas (renderer.cu:250) for the
        // first light with pick < cumulativeArea, else the last light. The
        // test is monotone in l (cumulative areas never decrease; once one is
        // NaN all later ones are), so a binary search picks the same light.
        float pick = rng(0) * sc.lightArea;
        int l = 0, hi = sc.lightCount - 1;
        while (l < hi) {
            int mid = (l + hi) >> 1;
            if (pick >= sc.lights[mid].cumulativeArea) l = mid + 1;
            else hi = mid;
        }
        const SceneTri& L = sc.tris[sc.lights[l].triangle];
        float root = sqrtf(rng(1)), v = rng(2);
        float3 target = add(L.origin, add(scale(L.edge1, root * (1.0f - v)), scale(L.edge2, root * v)));
        float3 off = sub(target, st.origin);
        float dist2 = dot(off, off), dist = sqrtf(dist2);
        float3 wi = scale(off, 1.0f / dist), ln = normalize(cross(L.edge1, L.edge2));
        float lightCos = -dot(ln, wi);
        if (!L.oneSided) lightCos = fabsf(lightCos);
        float surfCos = fmaxf(0.0f, dot(n, wi));
        if (lightCos > 0 && surfCos > 0 && dot(g, wi) > 0) {
            float pdf, lightPdf = dist2 / (sc.lightArea * lightCos);
            float3 f = evaluateBsdf(t, n, refl, wi, pdf);
            float w = bounce + 1 == set.maxBounces ? 1.0f : powerHeuristic(lightPdf, pdf);
            req.origin = st.origin; req.dir = wi; req.limit = dist - .001f;
            req.contribution = scale(mul(mul(st.throughput, f), L.color), L.emission * surfCos * w / lightPdf);
            flags |= kShadow;
        }
    }
    if (bounce + 1 == set.maxBounces) return flags;
    bool spec = rng(3) < t.specularProbability;
    if (spec && t.smoothness >= .999f) {
        st.dir = refl;
        st.throughput = mul(st.throughput, t.specularColor);
        st.prevPdf = 0;
    } else {
        float cosine = spec ? powf(rng(4), 1.0f / (phongExponent(t) + 1.0f)) : sqrtf(rng(4));
        st.dir = orientAround(spec ? refl : n, cosine, 2.0f * kPi * rng(5));
        if (dot(g, st.dir) <= 0 || dot(n, st.dir) <= 0) return flags;
        float pdf;
        float3 f = evaluateBsdf(t, n, refl, st.dir, pdf);
        if (pdf < 1e-12f) return flags;
        st.throughput = mul(st.throughput, scale(f, dot(n, st.dir) / pdf));
        st.prevPdf = pdf;
    }
    if (bounce >= 3) {
        float survive = fminf(.95f, fmaxf(st.throughput.x, fmaxf(st.throughput.y, st.throughput.z)));
        if (rng(6) >= survive) return flags;
        st.throughput = scale(st.throughput, 1.0f / survive);
    }
    return flags | kContinue;
}

// Adds one finished path to a pixel's running total (renderer.cu:295-297).
RT_HD void addPath(Accum& total, const PathState& s) {
    total.radiance = add(total.radiance, s.radiance);
    total.albedo = add(total.albedo, s.albedo);
    total.normal = add(total.normal, s.normal);
    total.covered += s.covered;
}
RT_HD uchar4 displayPixel(const Accum& total, unsigned samples, float exposure) {
    float3 avg = scale(total.radiance, 1.0f / (float)samples);
    return make_uchar4(tonemap(avg.x, exposure), tonemap(avg.y, exposure), tonemap(avg.z, exposure), 255);
}

// One pixel of a render pass: raysPerPixel paths added in order to the
// running sum, then the display value (renderer.cu:289-302). Shared by the
// one-kernel-per-pixel integrator and the host backends.
RT_HD void renderPixel(const SceneView& sc, const Camera& cam, const Settings& set, int x, int y, int w, int h,
                       unsigned sample0, const unsigned* passXor, const unsigned* seedHash, Accum* sums,
                       float* depthSums, uchar4* pixels, uint2* stack, int stackStride, int* overflow,
                       unsigned& nPrimary, unsigned& nSecondary, unsigned& nShadow) {
    size_t i = (size_t)y * w + x;
    Accum total = sample0 ? sums[i] : Accum{v3(0, 0, 0), v3(0, 0, 0), v3(0, 0, 0), 0u};
    float depthTotal = sample0 ? depthSums[i] : 0.0f;
    for (int r = 0; r < set.raysPerPixel; r++) {
        Sampler rng{passXor + r * kSobolDims, seedHash, (unsigned)(y * w + x), 0u};
        PathState st = startPath(cam, set, x, y, w, h, rng);
        for (int bounce = 0; bounce < set.maxBounces; bounce++) {
            rng.base = 4u + 8u * (unsigned)bounce;
            if (bounce == 0) nPrimary++; else nSecondary++;
            Hit hit = traverse<false>(sc.wide, sc.packed, st.origin, st.dir, 1e30f, stack, stackStride, overflow, nullptr,
                                     sc.stackLimit, sc.root);
            ShadowRequest req;
            unsigned f = shadeBounce(sc, set, bounce, st, hit, rng, req);
            if (f & kShadow) {
                nShadow++;
                Hit sh = traverse<true>(sc.wide, sc.packed, req.origin, req.dir, req.limit, stack, stackStride, overflow,
                                        nullptr, sc.stackLimit, sc.root);
                if (sh.index < 0) st.radiance = add(st.radiance, req.contribution);
            }
            if (!(f & kContinue)) break;
        }
        addPath(total, st);
        depthTotal += st.depth;
    }
    sums[i] = total;
    depthSums[i] = depthTotal;
    pixels[i] = displayPixel(total, sample0 + (unsigned)set.raysPerPixel, set.exposure);
}

}  // namespace rt
