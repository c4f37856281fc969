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

// Stack entries per ray held in shared memory (deeper entries live in
// local memory, which L1 caches). Fewer entries leave more of the SM's
// L1/shared storage to L1, which serves the node and triangle fetches: on
// the 1M-triangle workload 16 entries gave 3,007 Mrays/s, 12 and 10 3,026,
// 8 3,052-3,059, 6 3,056, 4 2,996-3,003.
constexpr int kSharedStack = 8;
constexpr int kTraceBlock = 128;

// Per-lane traversal state.
struct LaneRay {
    RaySetup r;
    Hit hit;
    uint2 group, triGroup;
    int top;
};

// root: index of the ray's root node (0 for a single scene; the scene's
// first node when several scenes share one node array).
__device__ __forceinline__ void laneStart(LaneRay& L, float3 o, float3 d, float limit, unsigned root) {
    L.r = setupRay(o, d);
    L.hit = Hit{-1, limit, 0.0f, 0.0f};
    L.group = make_uint2(root, 0x80000000u);
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
                                         int& overflow, int stackLimit) {
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
        if (L.top >= stackLimit) { overflow = 1; return true; }
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

// Per-warp shared scratch of the cooperative triangle phase.
struct WarpTriangles {
    float4 origin[32];              // each lane's ray origin
    float4 dir[32];                 // each lane's ray direction
    unsigned long long best[32];    // (distance bits << 32 | index) of each lane's best hit
    float2 uv[32];                  // barycentrics of that hit
    unsigned end[32];               // inclusive prefix sum of pending triangle counts
    uint2 group[32];                // each lane's pending triangle group
};
constexpr size_t traceSharedBytes(int block) {
    return sizeof(uint2) * kSharedStack * block + sizeof(WarpTriangles) * (block / 32);
}

// Position of the k-th (0-based) set bit of m; m has more than k set bits.
__device__ __forceinline__ unsigned selectBit(unsigned m, unsigned k) {
    unsigned pos = 0;
#pragma unroll
    for (unsigned width = 16; width > 0; width >>= 1) {
        unsigned low = __popc(m & ((1u << width) - 1u));
        if (k >= low) { k -= low; m >>= width; pos += width; }
    }
    return pos;
}

// Key ordering hits like the reference's acceptance rule (renderer.cu:153):
// smaller distance first, then smaller triangle index. Distances are
// positive, so their bit patterns order like the values. Before any hit the
// best is (limit, index -1) and the rule accepts only distances below the
// limit (i < -1 never holds), so that state is keyed with low word 0: a
// candidate at exactly the limit has a key >= it and is rejected.
__device__ __forceinline__ unsigned long long hitKey(float distance, int index) {
    return ((unsigned long long)__float_as_uint(distance) << 32) | (unsigned)(index < 0 ? 0 : index);
}

// Cooperative triangle phase: the warp's pending triangles (all lanes' groups)
// are dealt out one per lane per iteration; each candidate hit is merged into
// its ray's best with a shared-memory 64-bit atomicMin on hitKey. The result
// is the minimum over the same candidate set as testing them one by one, so
// it equals the sequential outcome. Returns true for a lane whose any-hit
// query is answered.
template <bool ANY>
__device__ __forceinline__ bool warpTrianglePhase(LaneRay& L, bool busy, const float4* tris, WarpTriangles& W,
                                                  unsigned lane) {
    const unsigned count = busy ? __popc(L.triGroup.y) : 0u;
    unsigned incl = count;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        unsigned v = __shfl_up_sync(0xFFFFFFFFu, incl, off);
        if ((int)lane >= off) incl += v;
    }
    const unsigned total = __shfl_sync(0xFFFFFFFFu, incl, 31);
    if (total == 0u) return false;
    const unsigned long long key0 = busy ? hitKey(L.hit.distance, L.hit.index) : ~0ull;
    W.origin[lane] = make_float4(L.r.o.x, L.r.o.y, L.r.o.z, 0.0f);
    W.dir[lane] = make_float4(L.r.d.x, L.r.d.y, L.r.d.z, 0.0f);
    W.best[lane] = key0;
    W.end[lane] = incl;
    W.group[lane] = busy ? L.triGroup : make_uint2(0u, 0u);
    __syncwarp();
    for (unsigned base = 0; base < total; base += 32u) {
        const unsigned w = base + lane;
        unsigned long long key = ~0ull;
        unsigned owner = 0;
        float u = 0.0f, v = 0.0f;
        if (w < total) {
            unsigned pos = 0;
#pragma unroll
            for (unsigned step = 16; step > 0; step >>= 1)
                if (W.end[pos + step - 1] <= w) pos += step;
            owner = pos;
            const uint2 g = W.group[owner];
            const unsigned bit = selectBit(g.y, w - (W.end[owner] - __popc(g.y)));
            const float4* t = tris + (size_t)(g.x + bit) * 3;
            float4 a = __ldg(t), b = __ldg(t + 1), c = __ldg(t + 2);
            float4 o4 = W.origin[owner], d4 = W.dir[owner];
            float dist = intersectTriangle(v3(o4.x, o4.y, o4.z), v3(d4.x, d4.y, d4.z), a, b, c, u, v);
            if (dist > 0) {
                unsigned long long k = hitKey(dist, __float_as_int(c.z));
                if (k < W.best[owner]) { atomicMin(&W.best[owner], k); key = k; }
            }
        }
        __syncwarp();
        if (key != ~0ull && W.best[owner] == key) W.uv[owner] = make_float2(u, v);
        __syncwarp();
    }
    bool answered = false;
    if (busy) {
        const unsigned long long b = W.best[lane];
        if (b != key0) {
            L.hit.distance = __uint_as_float((unsigned)(b >> 32));
            L.hit.index = (int)(unsigned)(b & 0xFFFFFFFFull);
            const float2 uv = W.uv[lane];
            L.hit.u = uv.x; L.hit.v = uv.y;
            answered = ANY;
        }
        L.triGroup.y = 0u;
    }
    __syncwarp();
    return answered;
}

// Persistent query loop over `count` rays of an IO object providing
//   __device__ void load(int k, float3& o, float3& d, float& limit, unsigned& root);
//   __device__ void store(int k, const Hit& h);
// `fetch` must be zero at launch. Adds the number of finished queries to
// *done and sets *errorFlag on stack overflow (more than stackLimit <=
// kStackCapacity entries). Dynamic shared memory: traceSharedBytes(blockDim.x).
//
// Each round has a triangle phase, in which the warp tests all pending
// triangles of its lanes cooperatively (warpTrianglePhase), and a node phase,
// in which every busy lane takes one node step. The node step (eight box
// tests) is the costly one, so running it in lockstep for all busy lanes
// keeps the warp's lanes doing useful work.
template <bool ANY, class IO>
__device__ __forceinline__ void persistentTrace(IO& io, int count, const uint4* nodes, const float4* tris, int* fetch,
                                                unsigned long long* done, int* errorFlag, int stackLimit,
                                                int refill) {
    extern __shared__ uint2 smemStack[];
    uint2* sstack = smemStack + threadIdx.x;
    const int stride = blockDim.x;
    WarpTriangles* warps = reinterpret_cast<WarpTriangles*>(smemStack + kSharedStack * blockDim.x);
    WarpTriangles& W = warps[threadIdx.x >> 5];
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
                        unsigned root = 0;
                        io.load(mine, o, d, limit, root);
                        if (limit > 0.0f) {
                            laneStart(L, o, d, limit, root);
                            k = mine;
                        } else {
                            // No distance can be accepted (limit <= 0 or NaN):
                            // the reference's answer is "no hit" at once.
                            io.store(mine, Hit{-1, limit, 0.0f, 0.0f});
                            finished++;
                        }
                    }
                }
            }
        }
        if (!__any_sync(0xFFFFFFFFu, k >= 0)) break;
        const int threshold = drained ? 1 : refill;
        for (;;) {
            if (warpTrianglePhase<ANY>(L, k >= 0, tris, W, lane)) {
                io.store(k, L.hit);
                k = -1;
                finished++;
            }
            if (k >= 0 && nodeStep(L, nodes, sstack, stride, lstack, overflow, stackLimit)) {
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
