// Acceleration-structure formats and ray queries (host and device).
//
// Traversal runs over an 8-wide compressed BVH: 80-byte nodes (five 16-byte
// vector loads) whose child boxes are quantised to 8 bits per plane against a
// per-node grid, with children placed in slots by ray octant, after the
// compressed wide BVH of Ylitie, Karras and Laine (HPG 2017). Triangles are
// repacked in leaf order as three float4 (48 bytes) holding exactly the
// reference's Moller-Trumbore inputs (origin, edge1, edge2, oneSided) and the
// original triangle index.
//
// Results follow the reference's collision() (Native/renderer.cu:136-178):
//  - the triangle test is the reference's intersect() (renderer.cu:99-112),
//    same operations in the same order, no contraction;
//  - closest hit: the smallest distance wins, equal distances go to the
//    smaller original index (renderer.cu:152-153), hits need t > 1e-4 and
//    t < limit;
//  - any hit: the first accepted hit ends the query (renderer.cu:155).
// Box culling is conservative with respect to the reference's padded boxes
// (bvh.cuh:46-47): quantisation only grows them, and axes whose direction
// component is below FLT_MIN use the reference's containment test
// (renderer.cu:120,142-143). Hence the hit set, and the winning hit, do not
// depend on tree shape or visiting order.
#pragma once
#include "rt_common.cuh"

namespace rt {

// Reference-layout binary node (Native/bvh.cuh:7).
struct BinNode { float3 low; int first; float3 high; int count; };
static_assert(sizeof(BinNode) == 32, "binary node layout");

constexpr int kBinaryMaxDepth = 32;  // bvh.cuh:9
constexpr int kStackCapacity = 48;   // wide traversal stack entries per ray

// 8-wide compressed node, 80 bytes.
//   word 0: grid origin p (3 floats), exponents ex,ey,ez (bytes 12-14), imask (byte 15)
//   word 1: childBase, triBase, meta[0..7]
//   words 2-4: qlo x[8], qlo y[8], qlo z[8], qhi x[8], qhi y[8], qhi z[8]
// meta: 0 = empty slot; interior child in slot s = 0x20 | (24 + s);
//       leaf of k (1..3) triangles at offset o from triBase = ((1 << k) - 1) << 5 | o.
// Interior children are stored consecutively from childBase in slot order.
struct alignas(16) WideNode {
    float px, py, pz;
    unsigned char ex, ey, ez, imask;
    unsigned childBase, triBase;
    unsigned char meta[8];
    unsigned char qlo[3][8];
    unsigned char qhi[3][8];
};
static_assert(sizeof(WideNode) == 80, "wide node layout");

struct Hit { int index; float distance, u, v; };

// Per-ray constants for box tests.
struct RaySetup {
    float3 o, d, inv;
    unsigned octInv;   // 3-bit mask flipping slot order into front-to-back for this octant
    unsigned parMask;  // axes whose |d| < FLT_MIN: containment test instead of slabs
};
RT_HD RaySetup setupRay(float3 o, float3 d) {
    RaySetup r;
    r.o = o; r.d = d; r.parMask = 0;
    r.inv.x = fabsf(d.x) < FLT_MIN ? (r.parMask |= 1u, 0.0f) : recip(d.x);
    r.inv.y = fabsf(d.y) < FLT_MIN ? (r.parMask |= 2u, 0.0f) : recip(d.y);
    r.inv.z = fabsf(d.z) < FLT_MIN ? (r.parMask |= 4u, 0.0f) : recip(d.z);
    unsigned oct = (signbit(d.x) ? 4u : 0u) | (signbit(d.y) ? 2u : 0u) | (signbit(d.z) ? 1u : 0u);
    r.octInv = 7u - oct;
    return r;
}

RT_HD uint4 loadVec(const uint4* p) {
#ifdef __CUDA_ARCH__
    return __ldg(p);
#else
    return *p;
#endif
}
RT_HD float4 loadVec(const float4* p) {
#ifdef __CUDA_ARCH__
    return __ldg(p);
#else
    return *p;
#endif
}
// (float) of byte b (0..3) of w, exact. On the device 0x4B0000bb read as a
// float is 2^23 + bb, which avoids an integer-to-float conversion.
RT_HD float quantum(unsigned w, unsigned b) {
#ifdef __CUDA_ARCH__
    return __uint_as_float(__byte_perm(w, 0x4B000000u, b | 0x7440u)) - 8388608.0f;
#else
    return (float)((w >> (8 * b)) & 0xFFu);
#endif
}

// Tests the eight child boxes of a wide node against [0, tmax]. Returns the
// node's hit mask: bits 24-31 interior children (octant-ordered), bits 0-23
// triangles relative to triBase. Also returns childBase/triBase/imask.
// Per axis the near plane is the lower bound when the inverse direction is
// non-negative and the upper bound otherwise, so each child needs one fused
// multiply-add per plane and no min/max pairs; fma is monotonic in q, so this
// equals taking min/max of the two plane distances.
RT_HD unsigned intersectWideNode(const uint4* node, const RaySetup& r, float tmax, unsigned& childBase,
                                 unsigned& triBase, unsigned& imask) {
    uint4 w0 = loadVec(node + 0), w1 = loadVec(node + 1), w2 = loadVec(node + 2), w3 = loadVec(node + 3),
          w4 = loadVec(node + 4);
    float px = bitsToFloat(w0.x), py = bitsToFloat(w0.y), pz = bitsToFloat(w0.z);
    float sx = bitsToFloat((w0.w & 0xFFu) << 23), sy = bitsToFloat(((w0.w >> 8) & 0xFFu) << 23),
          sz = bitsToFloat(((w0.w >> 16) & 0xFFu) << 23);
    imask = w0.w >> 24;
    childBase = w1.x;
    triBase = w1.y;
    // t(q) = (p + q*s - o) * inv = q * (s*inv) + (p - o)*inv
    float ax = sx * r.inv.x, ay = sy * r.inv.y, az = sz * r.inv.z;
    float bx = (px - r.o.x) * r.inv.x, by = (py - r.o.y) * r.inv.y, bz = (pz - r.o.z) * r.inv.z;
    // Words of the lower (lo) and upper (hi) planes, children 0-3 and 4-7.
    const bool nx = r.inv.x < 0.0f, ny = r.inv.y < 0.0f, nz = r.inv.z < 0.0f;
    uint2 nearX = nx ? make_uint2(w3.z, w3.w) : make_uint2(w2.x, w2.y);
    uint2 farX = nx ? make_uint2(w2.x, w2.y) : make_uint2(w3.z, w3.w);
    uint2 nearY = ny ? make_uint2(w4.x, w4.y) : make_uint2(w2.z, w2.w);
    uint2 farY = ny ? make_uint2(w2.z, w2.w) : make_uint2(w4.x, w4.y);
    uint2 nearZ = nz ? make_uint2(w4.z, w4.w) : make_uint2(w3.x, w3.y);
    uint2 farZ = nz ? make_uint2(w3.x, w3.y) : make_uint2(w4.z, w4.w);
    unsigned mask = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const unsigned b = (unsigned)(i & 3);
        const bool hiHalf = i >= 4;
        unsigned meta = ((hiHalf ? w1.w : w1.z) >> (8 * b)) & 0xFFu;
        float qnx = quantum(hiHalf ? nearX.y : nearX.x, b), qfx = quantum(hiHalf ? farX.y : farX.x, b);
        float qny = quantum(hiHalf ? nearY.y : nearY.x, b), qfy = quantum(hiHalf ? farY.y : farY.x, b);
        float qnz = quantum(hiHalf ? nearZ.y : nearZ.x, b), qfz = quantum(hiHalf ? farZ.y : farZ.x, b);
        float tnx = fmaRn(qnx, ax, bx), tfx = fmaRn(qfx, ax, bx);
        float tny = fmaRn(qny, ay, by), tfy = fmaRn(qfy, ay, by);
        float tnz = fmaRn(qnz, az, bz), tfz = fmaRn(qfz, az, bz);
        if (r.parMask) {
            // Reference semantics for axes parallel to the ray (renderer.cu:120):
            // inside the slab (bounds inclusive) imposes no limit, outside
            // misses. inv is +0 on those axes, so near = lower bound.
            if (r.parMask & 1u) { bool in = r.o.x >= fmaRn(qnx, sx, px) && r.o.x <= fmaRn(qfx, sx, px); tnx = in ? -FLT_MAX : FLT_MAX; tfx = FLT_MAX; }
            if (r.parMask & 2u) { bool in = r.o.y >= fmaRn(qny, sy, py) && r.o.y <= fmaRn(qfy, sy, py); tny = in ? -FLT_MAX : FLT_MAX; tfy = FLT_MAX; }
            if (r.parMask & 4u) { bool in = r.o.z >= fmaRn(qnz, sz, pz) && r.o.z <= fmaRn(qfz, sz, pz); tnz = in ? -FLT_MAX : FLT_MAX; tfz = FLT_MAX; }
        }
        float tmin = fmaxf(fmaxf(tnx, tny), fmaxf(tnz, 0.0f));
        float tmaxc = fminf(fminf(tfx, tfy), fminf(tfz, tmax));
        unsigned index = meta & 0x1Fu;
        if ((meta & 0x18u) == 0x18u) index ^= r.octInv;
        unsigned bits = (meta != 0u && tmin <= tmaxc) ? (meta >> 5) : 0u;
        mask |= bits << index;
    }
    return mask;
}

// Moller-Trumbore with the reference's operation order (renderer.cu:99-112).
// tri: three float4 = (origin.xyz, edge1.x), (edge1.yz, edge2.xy),
//                     (edge2.z, oneSided bits, original index bits, 0).
RT_HD float intersectTriangle(float3 o, float3 d, float4 a, float4 b, float4 c, float& u, float& v) {
    float3 e1 = v3(a.w, b.x, b.y), e2 = v3(b.z, b.w, c.x);
    float3 p = cross(d, e2);
    float det = dot(e1, p);
    if (fabsf(det) < 1e-7f || (floatToBits(c.y) != 0u && det < 0)) return -1.0f;
    float invDet = recip(det);
    float3 s = sub(o, v3(a.x, a.y, a.z));
    u = dot(s, p) * invDet;
    if (u < 0 || u > 1) return -1.0f;
    float3 q = cross(s, e1);
    v = dot(d, q) * invDet;
    if (v < 0 || u + v > 1) return -1.0f;
    float t = dot(e2, q) * invDet;
    return t > 1e-4f ? t : -1.0f;
}

struct TraversalCounters { unsigned nodes, tris; };

// Closest (ANY = false) or any (ANY = true) hit against the wide BVH.
// stack points at this ray's first stack entry; entries are stackStride apart
// (shared-memory column on the device, contiguous on the host). On stack
// overflow (more than stackLimit <= kStackCapacity entries) the query stops
// and sets *overflow (never happens at the default limit for trees built by
// this library: their depth is checked against kStackCapacity).
template <bool ANY>
RT_HD Hit traverse(const uint4* nodes, const float4* tris, float3 o, float3 d, float limit, uint2* stack,
                   int stackStride, int* overflow, TraversalCounters* counters, int stackLimit = kStackCapacity,
                   unsigned root = 0) {
    Hit hit{-1, limit, 0.0f, 0.0f};
    RaySetup r = setupRay(o, d);
    // Virtual root group: one interior child (the root node, 0 for a single
    // scene, a scene's first node in a batch arena) in the highest slot.
    uint2 group = make_uint2(root, 0x80000000u);
    uint2 triGroup = make_uint2(0u, 0u);
    int top = 0;
    unsigned nodeVisits = 0, triTests = 0;
    for (;;) {
        if (group.y > 0x00FFFFFFu) {
            int bit = highestBit(group.y & 0xFF000000u);
            group.y &= ~(1u << bit);
            unsigned slot = ((unsigned)bit - 24u) ^ r.octInv;
            unsigned rel = popc(group.y & 0xFFu & ((1u << slot) - 1u));
            unsigned child = group.x + rel;
            if (group.y > 0x00FFFFFFu) {
                if (top >= stackLimit) { if (overflow) *overflow = 1; break; }
                stack[top * stackStride] = group;
                top++;
            }
            unsigned childBase, triBase, imask;
            unsigned mask = intersectWideNode(nodes + (size_t)child * 5, r, hit.distance, childBase, triBase, imask);
            nodeVisits++;
            group = make_uint2(childBase, (mask & 0xFF000000u) | imask);
            triGroup = make_uint2(triBase, mask & 0x00FFFFFFu);
        } else {
            triGroup = group;
            group = make_uint2(0u, 0u);
        }
        while (triGroup.y != 0u) {
            int bit = highestBit(triGroup.y);
            triGroup.y &= ~(1u << bit);
            const float4* t = tris + (size_t)(triGroup.x + (unsigned)bit) * 3;
            float4 a = loadVec(t), b = loadVec(t + 1), c = loadVec(t + 2);
            float u, v, dist = intersectTriangle(o, d, a, b, c, u, v);
            triTests++;
            if (dist > 0) {
                int index = (int)floatToBits(c.z);
                if (dist < hit.distance || (dist == hit.distance && index < hit.index)) {
                    hit.index = index; hit.distance = dist; hit.u = u; hit.v = v;
                    if (ANY) { triGroup.y = 0u; group.y = 0u; top = 0; break; }
                }
            }
        }
        if (group.y <= 0x00FFFFFFu) {
            if (top == 0) break;
            top--;
            group = stack[top * stackStride];
        }
    }
    if (counters) { counters->nodes += nodeVisits; counters->tris += triTests; }
    return hit;
}

}  // namespace rt
