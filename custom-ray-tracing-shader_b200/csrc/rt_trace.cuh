// Persistent ray-query kernels with dynamic ray fetch (device only).
//
// Each warp keeps 32 rays in flight and advances them in rounds of triangle
// tests and node visits (see persistentTrace). When fewer than `refill` lanes
// are busy, the warp fetches new rays for its idle lanes with one atomic per
// warp, so lanes do not idle while the slowest ray of a fixed batch finishes
// (persistent threads with dynamic fetch, Aila and Laine, HPG 2009). The
// traversal stack of each ray keeps its first kSharedStack entries in shared
// memory (one column per thread) and the rest in local memory.
//
// Results are those of rt::traverse (rt_bvh.cuh): the same triangle test, the
// same acceptance rule and tie-break, the same conservative box tests, so the
// closest hit and the any-hit verdict are identical; only the visiting order
// of work differs, which the results do not depend on.
#pragma once
#include "rt_bvh.cuh"

namespace rt {

constexpr int kSharedStack = 16;     // stack entries per ray held in shared memory
constexpr int kTraceBlock = 128;

// Per-lane traversal state.
struct LaneRay {
    RaySetup r;
    Hit hit;
    uint2 group, triGroup;
    int top;
};

__device__ __forceinline__ void laneStart(LaneRay& L, float3 o, float3 d, float limit) {
    L.r = setupRay(o, d);
    L.hit = Hit{-1, limit, 0.0f, 0.0f};
    L.group = make_uint2(0u, 0x80000000u);
    L.triGroup = make_uint2(0u, 0u);
    L.top = 0;
}

// Triangle step: tests the highest pending triangle of the lane's group.
// Returns true when an any-hit query is answered.
template <bool ANY>
__device__ __forceinline__ bool triangleStep(LaneRay& L, const float4* tris) {
    int bit = 31 - __clz(L.triGroup.y);
    L.triGroup.y &= ~(1u << bit);
    const float4* t = tris + (size_t)(L.triGroup.x + (unsigned)bit) * 3;
    float4 a = __ldg(t), b = __ldg(t + 1), c = __ldg(t + 2);
    float u, v, dist = intersectTriangle(L.r.o, L.r.d, a, b, c, u, v);
    if (dist > 0) {
        int index = __float_as_int(c.z);
        if (dist < L.hit.distance || (dist == L.hit.distance && index < L.hit.index)) {
            L.hit.index = index; L.hit.distance = dist; L.hit.u = u; L.hit.v = v;
            if (ANY) return true;
        }
    }
    return false;
}

// Node step, taken when the lane has no pending triangles: pops an entry if
// the current group has no interior children left, then visits one child
// node (its eight child boxes). Returns true when the traversal is complete.
__device__ __forceinline__ bool nodeStep(LaneRay& L, const uint4* nodes, uint2* sstack, int stride, uint2* lstack,
                                         int& overflow) {
    if (L.group.y <= 0x00FFFFFFu) {
        if (L.top == 0) return true;
        L.top--;
        uint2 g = L.top < kSharedStack ? sstack[L.top * stride] : lstack[L.top - kSharedStack];
        if (g.y <= 0x00FFFFFFu) { L.triGroup = g; L.group = make_uint2(0u, 0u); return false; }
        L.group = g;
    }
    int bit = 31 - __clz(L.group.y & 0xFF000000u);
    L.group.y &= ~(1u << bit);
    unsigned slot = ((unsigned)bit - 24u) ^ L.r.octInv;
    unsigned child = L.group.x + __popc(L.group.y & 0xFFu & ((1u << slot) - 1u));
    if (L.group.y > 0x00FFFFFFu) {
        if (L.top >= kStackCapacity) { overflow = 1; return true; }
        if (L.top < kSharedStack) sstack[L.top * stride] = L.group;
        else lstack[L.top - kSharedStack] = L.group;
        L.top++;
    }
    unsigned childBase, triBase, imask;
    unsigned mask = intersectWideNode(nodes + (size_t)child * 5, L.r, L.hit.distance, childBase, triBase, imask);
    L.group = make_uint2(childBase, (mask & 0xFF000000u) | imask);
    L.triGroup = make_uint2(triBase, mask & 0x00FFFFFFu);
    return false;
}

// Persistent query loop over `count` rays of an IO object providing
//   __device__ void load(int k, float3& o, float3& d, float& limit);
//   __device__ void store(int k, const Hit& h);
// `fetch` must be zero at launch. Adds the number of finished queries to
// *done and sets *errorFlag on stack overflow.
//
// Each round has a triangle phase, in which every lane with pending
// triangles tests one per iteration until no lane has any, and a node phase,
// in which every busy lane takes one node step. The node step (eight box
// tests) is the costly one, so running it in lockstep for all busy lanes
// keeps the warp's lanes doing useful work.
//
// Triangle postponement (Ylitie et al. 2017): at the start of a triangle
// phase, when fewer than a fifth of the busy lanes have triangles, a lane
// that also has interior children to visit pushes its triangle group and
// takes part in the node phase instead. A lane postpones only while its stack
// has room for a full descent of the tree afterwards (postponeBelow =
// capacity minus the tree depth), so postponement never causes an overflow.
template <bool ANY, class IO>
__device__ __forceinline__ void persistentTrace(IO& io, int count, const uint4* nodes, const float4* tris, int* fetch,
                                                unsigned long long* done, int* errorFlag, int postponeBelow,
                                                int refill) {
    extern __shared__ uint2 smemStack[];
    uint2* sstack = smemStack + threadIdx.x;
    const int stride = blockDim.x;
    uint2 lstack[kStackCapacity - kSharedStack];
    const unsigned lane = threadIdx.x & 31u;
    const unsigned below = (1u << lane) - 1u;
    LaneRay L;
    int k = -1, overflow = 0;
    bool drained = false;
    unsigned finished = 0;
    for (;;) {
        if (!drained) {
            unsigned idle = __ballot_sync(0xFFFFFFFFu, k < 0);
            if (idle) {
                int leader = __ffs(idle) - 1, base = 0;
                if ((int)lane == leader) base = atomicAdd(fetch, __popc(idle));
                base = __shfl_sync(0xFFFFFFFFu, base, leader);
                if (base + __popc(idle) >= count) drained = true;
                if (k < 0) {
                    int mine = base + __popc(idle & below);
                    if (mine < count) {
                        float3 o, d;
                        float limit;
                        io.load(mine, o, d, limit);
                        laneStart(L, o, d, limit);
                        k = mine;
                    }
                }
            }
        }
        if (!__any_sync(0xFFFFFFFFu, k >= 0)) break;
        const int threshold = drained ? 1 : refill;
        for (;;) {
            // Triangle phase.
            const bool busy = k >= 0;
            const unsigned busyLanes = __popc(__ballot_sync(0xFFFFFFFFu, busy));
            const unsigned triLanes = __popc(__ballot_sync(0xFFFFFFFFu, busy && L.triGroup.y != 0u));
            if (busy && L.triGroup.y != 0u && triLanes * 5u < busyLanes && L.group.y > 0x00FFFFFFu &&
                L.top < postponeBelow) {
                if (L.top < kSharedStack) sstack[L.top * stride] = L.triGroup;
                else lstack[L.top - kSharedStack] = L.triGroup;
                L.top++;
                L.triGroup.y = 0u;
            }
            while (__any_sync(0xFFFFFFFFu, k >= 0 && L.triGroup.y != 0u)) {
                if (k >= 0 && L.triGroup.y != 0u && triangleStep<ANY>(L, tris)) {
                    io.store(k, L.hit);
                    k = -1;
                    finished++;
                }
            }
            // Node phase.
            if (k >= 0 && nodeStep(L, nodes, sstack, stride, lstack, overflow)) {
                io.store(k, L.hit);
                k = -1;
                finished++;
            }
            if (__popc(__ballot_sync(0xFFFFFFFFu, k >= 0)) < threshold) break;
        }
    }
    unsigned s = __reduce_add_sync(0xFFFFFFFFu, finished);
    if (lane == 0 && s && done) atomicAdd(done, (unsigned long long)s);
    if (overflow) atomicExch(errorFlag, 1);
}

}  // namespace rt
