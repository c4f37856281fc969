// GPU BVH construction.
//
// Stage 1, binned SAH (level-synchronous, all nodes of one depth per pass).
// The split rules are the reference's (Native/bvh.cuh:35-105), evaluated with
// the same floating-point expressions so every decision matches:
//   - primitive box padded by 1e-5 + 1e-6 * max|coord| per axis, centroid
//     (a + b + c) / 3 of the unpadded corners (bvh.cuh:38-48);
//   - leaf when count <= 4 or depth == 32 (bvh.cuh:64);
//   - 12 centroid bins per axis, axes with centroid extent <= 1e-12 skipped,
//     bin = min(11, max(0, int((c - min) * (12 / extent)))) (bvh.cuh:53-76);
//   - split cost A(node) + A(L) nL + A(R) nR against leaf cost A(node) n,
//     strict "<" so the first minimum in (axis, bin) order wins (bvh.cuh:66-91);
//   - partition by bin <= best (bvh.cuh:94-98).
// Binning and box unions are min/max/counts, which are order independent, so
// the tree (node boxes, ranges, counts, depth) equals the reference's. The
// partition here is stable (prefix sums) where the reference uses
// std::partition, so only the order of triangles inside a leaf can differ.
// A final pass renumbers nodes into the reference's depth-first numbering
// (children allocated in pairs when their parent splits), so the node array
// is the reference's node array.
//
// Stage 2, collapse into 8-wide compressed nodes: each wide node greedily
// opens its largest-area interior descendant while the children still fit in
// eight slots; leaves become groups of up to three triangles. Children are
// assigned to slots by ray octant and quantised outward to 8 bits per plane.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "rt_build.cuh"
#include "rt_collapse.cuh"

namespace rt {
namespace {

constexpr int kBins = 12;          // bvh.cuh:29
constexpr int kLeafSize = 4;       // bvh.cuh:64
constexpr int kScanBlock = 1024;   // elements per scan block
constexpr int kBinBlock = 256;
constexpr int kBinPer = 8;         // positions per thread in the binning pass
// Tasks of at most kSmallTask primitives are binned by one warp each
// (binSmallKernel); larger ones by position blocks (binKernel).
constexpr int kSmallTask = 2048;
// Levels (binned SAH, or wide collapse) queued per host read of the counts.
constexpr int kLevelBatch = 8;

struct Task {
    int node, first, count, depth;
    float lo[3], hi[3], clo[3], chi[3];
};
struct BinAcc { unsigned count; float lo[3], hi[3], clo[3], chi[3]; };
struct Split { int axis, bin, leftCount, childTask[2]; };

__device__ __forceinline__ void atomicMinFloat(float* a, float v) {
    if (v >= 0.0f) atomicMin(reinterpret_cast<int*>(a), __float_as_int(v));
    else atomicMax(reinterpret_cast<unsigned*>(a), __float_as_uint(v));
}
__device__ __forceinline__ void atomicMaxFloat(float* a, float v) {
    if (v >= 0.0f) atomicMax(reinterpret_cast<int*>(a), __float_as_int(v));
    else atomicMin(reinterpret_cast<unsigned*>(a), __float_as_uint(v));
}
RT_HD int binOf(float c, float lo, float s) {
    int b = (int)((c - lo) * s);
    return b < 0 ? 0 : (b > kBins - 1 ? kBins - 1 : b);
}
// Half surface area with the reference's expression (bvh.cuh:20-23).
RT_HD float halfArea(const float lo[3], const float hi[3]) {
    float x = fmaxf(0.0f, hi[0] - lo[0]), y = fmaxf(0.0f, hi[1] - lo[1]), z = fmaxf(0.0f, hi[2] - lo[2]);
    return x * y + x * z + y * z;
}
__device__ __forceinline__ void growBox(float lo[3], float hi[3], const float olo[3], const float ohi[3]) {
    for (int a = 0; a < 3; a++) { lo[a] = fminf(lo[a], olo[a]); hi[a] = fmaxf(hi[a], ohi[a]); }
}

// ---- primitive boxes and root bounds ----
__global__ void primBoxesKernel(const SceneTri* tris, int n, float4* plo, float4* phi, float4* cent, Task* root) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    float v[12];
    for (int k = 0; k < 3; k++) { v[k] = FLT_MAX; v[3 + k] = -FLT_MAX; v[6 + k] = FLT_MAX; v[9 + k] = -FLT_MAX; }
    if (i < n) {
        const SceneTri& t = tris[i];
        float3 o = t.origin;
        float3 b = v3(o.x + t.edge1.x, o.y + t.edge1.y, o.z + t.edge1.z);
        float3 c = v3(o.x + t.edge2.x, o.y + t.edge2.y, o.z + t.edge2.z);
        float lo[3], hi[3], ce[3];
        for (int a = 0; a < 3; a++) {
            float oa = comp(o, a), ba = comp(b, a), ca = comp(c, a);
            lo[a] = fminf(fminf(fminf(FLT_MAX, oa), ba), ca);
            hi[a] = fmaxf(fmaxf(fmaxf(-FLT_MAX, oa), ba), ca);
            ce[a] = (oa + ba + ca) / 3.0f;
            float pad = 1e-5f + 1e-6f * fmaxf(fabsf(lo[a]), fabsf(hi[a]));
            lo[a] -= pad; hi[a] += pad;
        }
        plo[i] = make_float4(lo[0], lo[1], lo[2], 0.0f);
        phi[i] = make_float4(hi[0], hi[1], hi[2], 0.0f);
        cent[i] = make_float4(ce[0], ce[1], ce[2], 0.0f);
        for (int k = 0; k < 3; k++) { v[k] = lo[k]; v[3 + k] = hi[k]; v[6 + k] = ce[k]; v[9 + k] = ce[k]; }
    }
    for (int off = 16; off > 0; off >>= 1)
        for (int k = 0; k < 12; k++) {
            float o = __shfl_xor_sync(0xFFFFFFFFu, v[k], off);
            v[k] = ((k / 3) & 1) ? fmaxf(v[k], o) : fminf(v[k], o);
        }
    if ((threadIdx.x & 31) == 0) {
        for (int k = 0; k < 3; k++) {
            atomicMinFloat(&root->lo[k], v[k]); atomicMaxFloat(&root->hi[k], v[3 + k]);
            atomicMinFloat(&root->clo[k], v[6 + k]); atomicMaxFloat(&root->chi[k], v[9 + k]);
        }
    }
}

// Traversal-tree primitives: each triangle cut into `pieces` slabs along the
// longest axis of its box; a piece's box bounds the part of the triangle in
// its slab (vertices inside it and the edges' crossings of its planes), padded
// like the reference pads triangle boxes (bvh.cuh:46-47). The padding exceeds
// the rounding of the clipping, so every point of the triangle lies in the
// padded box of a piece containing it, and the union of the pieces' boxes
// covers the triangle's padded box's content that traversal can reach.
// Pieces of one triangle: the half area of its box over its own area tells
// how much empty space the box holds. Well-shaped triangles (ratio below 12;
// all but a fraction of a percent of ordinary meshes' triangles) stay whole;
// slivers get floor(ratio / 6) pieces, at most maxPieces.
__device__ int piecesOf(const SceneTri& t, int maxPieces) {
    const float3 e1 = t.edge1, e2 = t.edge2;
    const float ex = fmaxf(fmaxf(0.0f, e1.x), e2.x) - fminf(fminf(0.0f, e1.x), e2.x);
    const float ey = fmaxf(fmaxf(0.0f, e1.y), e2.y) - fminf(fminf(0.0f, e1.y), e2.y);
    const float ez = fmaxf(fmaxf(0.0f, e1.z), e2.z) - fminf(fminf(0.0f, e1.z), e2.z);
    const float boxArea = ex * ey + ey * ez + ex * ez;
    const float3 c = cross(e1, e2);
    const float triArea = 0.5f * sqrtf(dot(c, c));
    if (!(triArea > 0.0f) || !(boxArea < FLT_MAX)) return 1;
    const float k = boxArea / triArea / 6.0f;
    return k >= (float)maxPieces ? maxPieces : (k >= 2.0f ? (int)k : 1);
}
__global__ void pieceCountKernel(const SceneTri* tris, int n, int maxPieces, unsigned* counts) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) counts[i] = (unsigned)piecesOf(tris[i], maxPieces);
}
// primTri[first piece of i + s] = i, from the exclusive scan of the counts
// (block-local prefix plus the block's total).
__global__ void pieceFillKernel(const unsigned* counts, const unsigned* prefix, const unsigned* blockSums, int n,
                                int* primTri, int* total) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned first = prefix[i] + blockSums[i / kScanBlock];
    if (primTri)
        for (unsigned s = 0; s < counts[i]; s++) primTri[first + s] = i;
    if (i == n - 1) *total = (int)(first + counts[i]);
}

__global__ void splitBoxesKernel(const SceneTri* tris, const int* primTri, int nPrims, int maxPieces, float4* plo,
                                 float4* phi, float4* cent, Task* root) {
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    float v[12];
    for (int k = 0; k < 3; k++) { v[k] = FLT_MAX; v[3 + k] = -FLT_MAX; v[6 + k] = FLT_MAX; v[9 + k] = -FLT_MAX; }
    if (r < nPrims) {
        const int i = primTri[r];
        const SceneTri& t = tris[i];
        const int pieces = piecesOf(t, maxPieces);
        int s = 0;  // which piece: primitives of a triangle are consecutive
        while (s < r && s < pieces - 1 && primTri[r - s - 1] == i) s++;
        float3 P[3] = {t.origin, v3(t.origin.x + t.edge1.x, t.origin.y + t.edge1.y, t.origin.z + t.edge1.z),
                       v3(t.origin.x + t.edge2.x, t.origin.y + t.edge2.y, t.origin.z + t.edge2.z)};
        float tlo[3], thi[3];
        for (int a = 0; a < 3; a++) {
            tlo[a] = fminf(fminf(comp(P[0], a), comp(P[1], a)), comp(P[2], a));
            thi[a] = fmaxf(fmaxf(comp(P[0], a), comp(P[1], a)), comp(P[2], a));
        }
        int ax = 0;
        for (int a = 1; a < 3; a++) if (thi[a] - tlo[a] > thi[ax] - tlo[ax]) ax = a;
        const float ext = thi[ax] - tlo[ax];
        const float t0 = s == 0 ? tlo[ax] : tlo[ax] + ext * ((float)s / (float)pieces);
        const float t1 = s == pieces - 1 ? thi[ax] : tlo[ax] + ext * ((float)(s + 1) / (float)pieces);
        float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        auto grow = [&](float3 q) {
            for (int a = 0; a < 3; a++) { lo[a] = fminf(lo[a], comp(q, a)); hi[a] = fmaxf(hi[a], comp(q, a)); }
        };
        for (int e = 0; e < 3; e++) {
            const float3 p = P[e], q = P[(e + 1) % 3];
            const float pa = comp(p, ax), qa = comp(q, ax);
            if (pa >= t0 && pa <= t1) grow(p);
            for (int side = 0; side < 2; side++) {
                const float plane = side ? t1 : t0;
                if ((pa < plane && qa > plane) || (pa > plane && qa < plane)) {
                    const float u = (plane - pa) / (qa - pa);
                    float3 x = v3(p.x + u * (q.x - p.x), p.y + u * (q.y - p.y), p.z + u * (q.z - p.z));
                    if (ax == 0) x.x = plane; else if (ax == 1) x.y = plane; else x.z = plane;
                    grow(x);
                }
            }
        }
        float ce[3];
        for (int a = 0; a < 3; a++) {
            if (!(lo[a] <= hi[a])) { lo[a] = tlo[a]; hi[a] = thi[a]; }  // nothing collected: whole box
            float pad = 1e-5f + 1e-6f * fmaxf(fabsf(tlo[a]), fabsf(thi[a]));
            lo[a] -= pad; hi[a] += pad;
            ce[a] = 0.5f * (lo[a] + hi[a]);
        }
        plo[r] = make_float4(lo[0], lo[1], lo[2], 0.0f);
        phi[r] = make_float4(hi[0], hi[1], hi[2], 0.0f);
        cent[r] = make_float4(ce[0], ce[1], ce[2], 0.0f);
        for (int k = 0; k < 3; k++) { v[k] = lo[k]; v[3 + k] = hi[k]; v[6 + k] = ce[k]; v[9 + k] = ce[k]; }
    }
    for (int off = 16; off > 0; off >>= 1)
        for (int k = 0; k < 12; k++) {
            float o = __shfl_xor_sync(0xFFFFFFFFu, v[k], off);
            v[k] = ((k / 3) & 1) ? fmaxf(v[k], o) : fminf(v[k], o);
        }
    if ((threadIdx.x & 31) == 0) {
        for (int k = 0; k < 3; k++) {
            atomicMinFloat(&root->lo[k], v[k]); atomicMaxFloat(&root->hi[k], v[3 + k]);
            atomicMinFloat(&root->clo[k], v[6 + k]); atomicMaxFloat(&root->chi[k], v[9 + k]);
        }
    }
}

__global__ void iotaKernel(int* a, int n, int value0, int* b, int bValue) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) { a[i] = i + value0; if (b) b[i] = bValue; }
}

// Level counts (taskCount[0] open tasks, taskCount[1] of them larger than
// kSmallTask) live on the device, so levels are queued without the host
// reading them: per-task kernels loop over the device count.
__global__ void clearBinsKernel(BinAcc* bins, const int* taskCount, const Task* tasks) {
    if (!taskCount[1]) return;
    const int count = taskCount[0] * 3 * kBins;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        if (tasks[i / (3 * kBins)].count <= kSmallTask) continue;
        BinAcc& b = bins[i];
        b.count = 0;
        for (int a = 0; a < 3; a++) { b.lo[a] = FLT_MAX; b.hi[a] = -FLT_MAX; b.clo[a] = FLT_MAX; b.chi[a] = -FLT_MAX; }
    }
}

__device__ __forceinline__ void accumulateBin(BinAcc* dst, float4 lo, float4 hi, float4 c) {
    atomicAdd(&dst->count, 1u);
    atomicMinFloat(&dst->lo[0], lo.x); atomicMinFloat(&dst->lo[1], lo.y); atomicMinFloat(&dst->lo[2], lo.z);
    atomicMaxFloat(&dst->hi[0], hi.x); atomicMaxFloat(&dst->hi[1], hi.y); atomicMaxFloat(&dst->hi[2], hi.z);
    atomicMinFloat(&dst->clo[0], c.x); atomicMinFloat(&dst->clo[1], c.y); atomicMinFloat(&dst->clo[2], c.z);
    atomicMaxFloat(&dst->chi[0], c.x); atomicMaxFloat(&dst->chi[1], c.y); atomicMaxFloat(&dst->chi[2], c.z);
}

// Floats as integers of the same order (-0 below +0, as the atomics above
// order them), so warp reductions can use the integer min/max instructions.
__device__ __forceinline__ int orderedKey(float f) {
    const int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7FFFFFFF;
}
__device__ __forceinline__ float keyFloat(int k) { return __int_as_float(k >= 0 ? k : k ^ 0x7FFFFFFF); }

// accumulateBin for a whole warp (every lane calls it; dst null: no
// primitive). Spatially coherent primitives put most of a warp's lanes into
// one bin, where per-lane atomics would serialise on one address: the lanes
// of the first two destinations are reduced with warp instructions and
// their leaders add the results; the lanes left over use per-lane atomics.
// Counts and minima/maxima do not depend on the order of accumulation.
__device__ void warpAccumulate(BinAcc* dst, float4 lo, float4 hi, float4 c) {
    const unsigned full = 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31;
    unsigned pending = __ballot_sync(full, dst != nullptr);
    for (int round = 0; round < 2 && pending; round++) {
        const int leader = __ffs(pending) - 1;
        BinAcc* first = reinterpret_cast<BinAcc*>(__shfl_sync(full, reinterpret_cast<unsigned long long>(dst), leader));
        const bool mine = dst != nullptr && dst == first;
        const unsigned group = __ballot_sync(full, mine);
        const int kMin = 0x7FFFFFFF, kMax = (int)0x80000000;
        const int l0 = __reduce_min_sync(full, mine ? orderedKey(lo.x) : kMin);
        const int l1 = __reduce_min_sync(full, mine ? orderedKey(lo.y) : kMin);
        const int l2 = __reduce_min_sync(full, mine ? orderedKey(lo.z) : kMin);
        const int h0 = __reduce_max_sync(full, mine ? orderedKey(hi.x) : kMax);
        const int h1 = __reduce_max_sync(full, mine ? orderedKey(hi.y) : kMax);
        const int h2 = __reduce_max_sync(full, mine ? orderedKey(hi.z) : kMax);
        const int c0 = __reduce_min_sync(full, mine ? orderedKey(c.x) : kMin);
        const int c1 = __reduce_min_sync(full, mine ? orderedKey(c.y) : kMin);
        const int c2 = __reduce_min_sync(full, mine ? orderedKey(c.z) : kMin);
        const int d0 = __reduce_max_sync(full, mine ? orderedKey(c.x) : kMax);
        const int d1 = __reduce_max_sync(full, mine ? orderedKey(c.y) : kMax);
        const int d2 = __reduce_max_sync(full, mine ? orderedKey(c.z) : kMax);
        if (lane == leader) {
            atomicAdd(&first->count, (unsigned)__popc(group));
            atomicMinFloat(&first->lo[0], keyFloat(l0)); atomicMinFloat(&first->lo[1], keyFloat(l1));
            atomicMinFloat(&first->lo[2], keyFloat(l2));
            atomicMaxFloat(&first->hi[0], keyFloat(h0)); atomicMaxFloat(&first->hi[1], keyFloat(h1));
            atomicMaxFloat(&first->hi[2], keyFloat(h2));
            atomicMinFloat(&first->clo[0], keyFloat(c0)); atomicMinFloat(&first->clo[1], keyFloat(c1));
            atomicMinFloat(&first->clo[2], keyFloat(c2));
            atomicMaxFloat(&first->chi[0], keyFloat(d0)); atomicMaxFloat(&first->chi[1], keyFloat(d1));
            atomicMaxFloat(&first->chi[2], keyFloat(d2));
        }
        pending &= ~group;
    }
    if ((pending >> lane) & 1u) accumulateBin(dst, lo, hi, c);
}

// Bins every primitive of every open task. The task owning the first position
// of a block's chunk is aggregated in shared memory; others go to global bins.
__global__ void __launch_bounds__(kBinBlock) binKernel(const int* order, const int* posTask, const float4* cent,
                                                       const float4* plo, const float4* phi, const Task* tasks,
                                                       int nPos, BinAcc* bins, const int* taskCount) {
    __shared__ BinAcc sb[3 * kBins];
    __shared__ int sTask;
    if (!taskCount[1]) return;  // no task above kSmallTask at this level
    int base = blockIdx.x * kBinBlock * kBinPer;
    if (threadIdx.x == 0) sTask = base < nPos ? posTask[base] : -1;
    if (threadIdx.x < 3 * kBins) {
        BinAcc& b = sb[threadIdx.x];
        b.count = 0;
        for (int a = 0; a < 3; a++) { b.lo[a] = FLT_MAX; b.hi[a] = -FLT_MAX; b.clo[a] = FLT_MAX; b.chi[a] = -FLT_MAX; }
    }
    __syncthreads();
    int st = sTask;
    // Every lane walks all kBinPer positions (warpAccumulate needs the whole
    // warp); positions past the end or of finished or small tasks add nothing.
    for (int k = 0; k < kBinPer; k++) {
        const int j = base + k * kBinBlock + threadIdx.x;
        const int t = j < nPos ? posTask[j] : -1;
        const Task* T = t >= 0 ? &tasks[t] : nullptr;
        const bool valid = T && T->count > kSmallTask;  // small tasks: binned by binSmallKernel
        float4 c = make_float4(0, 0, 0, 0), lo = c, hi = c;
        if (valid) {
            const int prim = order[j];
            c = cent[prim]; lo = plo[prim]; hi = phi[prim];
        }
        if (!__any_sync(0xFFFFFFFFu, valid)) continue;
        for (int a = 0; a < 3; a++) {
            BinAcc* dst = nullptr;
            if (valid) {
                const float extent = T->chi[a] - T->clo[a];
                if (extent > 1e-12f) {
                    const float s = kBins / extent;
                    const float ca = a == 0 ? c.x : (a == 1 ? c.y : c.z);
                    const int b = binOf(ca, T->clo[a], s);
                    dst = t == st ? &sb[a * kBins + b] : &bins[((size_t)t * 3 + a) * kBins + b];
                }
            }
            warpAccumulate(dst, lo, hi, c);
        }
    }
    __syncthreads();
    if (st >= 0 && threadIdx.x < 3 * kBins) {
        const BinAcc& s = sb[threadIdx.x];
        if (s.count) {
            BinAcc* d = &bins[(size_t)st * 3 * kBins + threadIdx.x];
            atomicAdd(&d->count, s.count);
            for (int a = 0; a < 3; a++) {
                atomicMinFloat(&d->lo[a], s.lo[a]); atomicMaxFloat(&d->hi[a], s.hi[a]);
                atomicMinFloat(&d->clo[a], s.clo[a]); atomicMaxFloat(&d->chi[a], s.chi[a]);
            }
        }
    }
}

__device__ void binSmallTask(const int* order, const float4* cent, const float4* plo, const float4* phi,
                             const Task T, int t, BinAcc* bins, BinAcc* my, int lane) {
    if (T.count > kSmallTask) return;
    for (int i = lane; i < 3 * kBins; i += 32) {
        BinAcc& b = my[i];
        b.count = 0;
        for (int a = 0; a < 3; a++) { b.lo[a] = FLT_MAX; b.hi[a] = -FLT_MAX; b.clo[a] = FLT_MAX; b.chi[a] = -FLT_MAX; }
    }
    __syncwarp();
    float scale[3];
    for (int a = 0; a < 3; a++) {
        float extent = T.chi[a] - T.clo[a];
        scale[a] = extent <= 1e-12f ? 0.0f : kBins / extent;
    }
    // Per-lane atomics: small tasks are deep in the tree, where a warp's
    // primitives spread over the bins (warpAccumulate measured slower here).
    for (int j = T.first + lane; j < T.first + T.count; j += 32) {
        const int prim = order[j];
        const float4 c = cent[prim], lo = plo[prim], hi = phi[prim];
        for (int a = 0; a < 3; a++) {
            if (scale[a] == 0.0f) continue;
            const float ca = a == 0 ? c.x : (a == 1 ? c.y : c.z);
            accumulateBin(&my[a * kBins + binOf(ca, T.clo[a], scale[a])], lo, hi, c);
        }
    }
    __syncwarp();
    for (int i = lane; i < 3 * kBins; i += 32) bins[(size_t)t * 3 * kBins + i] = my[i];
    __syncwarp();
}

// One warp per small task: warp-private bins in shared memory (atomics only
// within the warp), written out with plain stores, so these bins need no
// clearing and no global atomics. Bins hold a count and minima/maxima, so the
// order of accumulation does not change them.
__global__ void __launch_bounds__(256) binSmallKernel(const int* order, const float4* cent, const float4* plo,
                                                      const float4* phi, const Task* tasks, const int* taskCount,
                                                      BinAcc* bins) {
    __shared__ BinAcc sb[8][3 * kBins];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nTasks = taskCount[0];
    for (int t = blockIdx.x * 8 + warp; t < nTasks; t += gridDim.x * 8)
        binSmallTask(order, cent, plo, phi, tasks[t], t, bins, sb[warp], lane);
}

// One thread per open task: the reference's SAH sweep, then node records.
// The counters every task updates (maximum depth, node and task allocation)
// are aggregated per warp first: one atomic per warp instead of one per
// task on a single address, which serialised the deep levels (hundreds of
// thousands of tasks). Node and task numbers within a level are assigned in
// lane order instead of atomic order; nodes are renumbered to the
// reference's order after the build, and tasks carry their own ranges.
// taskCount: this level's counts; nextCount: the next level's (open tasks,
// tasks above kSmallTask); counters: 0 nodes, 2 maximum depth, 3 error.
__device__ void splitTask(bool have, const Task& T, int t, const BinAcc* bins, Split* splits, BinNode* nodes,
                          int* counters, int* nextCount, Task* nextTasks, int nodeCapacity, int taskCapacity,
                          int leafSize) {
    const unsigned full = 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31;
    int bestAxis = -1, bestBin = -1;
    if (have && T.count > leafSize && T.depth != kBinaryMaxDepth) {
        const float nodeArea = halfArea(T.lo, T.hi);
        float bestCost = nodeArea * T.count;
        for (int a = 0; a < 3; a++) {
            float extent = T.chi[a] - T.clo[a];
            if (extent <= 1e-12f) continue;
            const BinAcc* B = &bins[((size_t)t * 3 + a) * kBins];
            float sufLo[kBins][3], sufHi[kBins][3];
            int sufN[kBins];
            float accLo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, accHi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
            int accN = 0;
            for (int b = kBins - 1; b >= 0; b--) {
                if (B[b].count) growBox(accLo, accHi, B[b].lo, B[b].hi);
                accN += (int)B[b].count;
                for (int k = 0; k < 3; k++) { sufLo[b][k] = accLo[k]; sufHi[b][k] = accHi[k]; }
                sufN[b] = accN;
            }
            float preLo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, preHi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
            int preN = 0;
            for (int b = 0; b < kBins - 1; b++) {
                if (B[b].count) growBox(preLo, preHi, B[b].lo, B[b].hi);
                preN += (int)B[b].count;
                if (!preN || !sufN[b + 1]) continue;
                float cost = nodeArea + halfArea(preLo, preHi) * preN + halfArea(sufLo[b + 1], sufHi[b + 1]) * sufN[b + 1];
                if (cost < bestCost) { bestCost = cost; bestAxis = a; bestBin = b; }
            }
        }
    }
    const bool split = bestAxis >= 0;
    // Children's boxes, centroid boxes and counts are unions over the bins.
    Task C[2];
    bool open[2] = {false, false};
    if (split) {
        for (int side = 0; side < 2; side++) {
            for (int k = 0; k < 3; k++) { C[side].lo[k] = C[side].clo[k] = FLT_MAX; C[side].hi[k] = C[side].chi[k] = -FLT_MAX; }
            C[side].count = 0;
        }
        const BinAcc* B = &bins[((size_t)t * 3 + bestAxis) * kBins];
        for (int b = 0; b < kBins; b++) {
            if (!B[b].count) continue;
            Task& c = C[b <= bestBin ? 0 : 1];
            growBox(c.lo, c.hi, B[b].lo, B[b].hi);
            growBox(c.clo, c.chi, B[b].clo, B[b].chi);
            c.count += (int)B[b].count;
        }
        for (int side = 0; side < 2; side++) {
            C[side].depth = T.depth + 1;
            open[side] = !(C[side].count <= leafSize || C[side].depth == kBinaryMaxDepth);
        }
    }
    // Maximum depth: a task's own, its children's when it splits.
    const int depth = __reduce_max_sync(full, have ? T.depth + (split ? 1 : 0) : -1);
    if (lane == 0 && depth >= 0) atomicMax(&counters[2], depth);
    // Two nodes per split task.
    const unsigned splitMask = __ballot_sync(full, split);
    const unsigned below = (1u << lane) - 1u;
    int childBase = 0;
    if (lane == 0 && splitMask) childBase = atomicAdd(&counters[0], 2 * __popc(splitMask));
    childBase = __shfl_sync(full, childBase, 0);
    // Next-level tasks: the open children, side 0 before side 1.
    const unsigned open0 = __ballot_sync(full, open[0]), open1 = __ballot_sync(full, open[1]);
    const unsigned big0 = __ballot_sync(full, open[0] && C[0].count > kSmallTask);
    const unsigned big1 = __ballot_sync(full, open[1] && C[1].count > kSmallTask);
    int taskBase = 0;
    if (lane == 0 && (open0 | open1)) taskBase = atomicAdd(&nextCount[0], __popc(open0) + __popc(open1));
    if (lane == 0 && (big0 | big1)) atomicAdd(&nextCount[1], __popc(big0) + __popc(big1));
    taskBase = __shfl_sync(full, taskBase, 0);
    if (!have) return;

    Split S;
    S.axis = bestAxis; S.bin = bestBin; S.leftCount = 0; S.childTask[0] = S.childTask[1] = -1;
    if (!split) {
        nodes[T.node] = BinNode{v3(T.lo[0], T.lo[1], T.lo[2]), T.first, v3(T.hi[0], T.hi[1], T.hi[2]), T.count};
        splits[t] = S;
        return;
    }
    const int child = childBase + 2 * __popc(splitMask & below);
    if (child + 2 > nodeCapacity) { atomicExch(&counters[3], 1); splits[t] = Split{-1, -1, 0, {-1, -1}}; return; }
    nodes[T.node] = BinNode{v3(T.lo[0], T.lo[1], T.lo[2]), child, v3(T.hi[0], T.hi[1], T.hi[2]), 0};
    C[0].first = T.first;
    C[1].first = T.first + C[0].count;
    S.leftCount = C[0].count;
    int k = taskBase + __popc(open0 & below) + __popc(open1 & below);
    for (int side = 0; side < 2; side++) {
        Task& c = C[side];
        c.node = child + side;
        if (!open[side]) {
            nodes[c.node] = BinNode{v3(c.lo[0], c.lo[1], c.lo[2]), c.first, v3(c.hi[0], c.hi[1], c.hi[2]), c.count};
            continue;
        }
        if (k >= taskCapacity) { atomicExch(&counters[3], 2); k++; continue; }
        nextTasks[k] = c;
        S.childTask[side] = k;
        k++;
    }
    splits[t] = S;
}
__global__ void splitKernel(const Task* tasks, const int* taskCount, const BinAcc* bins, Split* splits, BinNode* nodes,
                            int* counters, int* nextCount, Task* nextTasks, int nodeCapacity, int taskCapacity,
                            int leafSize) {
    const int nTasks = taskCount[0];
    // Whole warps walk the tasks (splitTask uses warp collectives).
    for (int base = blockIdx.x * blockDim.x; base < nTasks; base += gridDim.x * blockDim.x) {
        const int t = base + (int)threadIdx.x;
        const bool have = t < nTasks;
        Task T;
        if (have) T = tasks[t];
        else T.count = 0, T.depth = 0;
        splitTask(have, T, t, bins, splits, nodes, counters, nextCount, nextTasks, nodeCapacity, taskCapacity,
                  leafSize);
    }
}

__global__ void flagKernel(const int* order, const int* posTask, const float4* cent, const Task* tasks,
                           const Split* splits, int nPos, unsigned* flags) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nPos) return;
    int t = posTask[j];
    unsigned f = 0;
    if (t >= 0) {
        Split S = splits[t];
        if (S.axis >= 0) {
            const Task& T = tasks[t];
            float lo = T.clo[S.axis];
            float s = kBins / (T.chi[S.axis] - lo);
            float4 c = cent[order[j]];
            float ca = S.axis == 0 ? c.x : (S.axis == 1 ? c.y : c.z);
            f = binOf(ca, lo, s) <= S.bin ? 1u : 0u;
        }
    }
    flags[j] = f;
}

// Exclusive scan, phase 1: per-block scan in place, block totals out.
__global__ void __launch_bounds__(256) scanBlocksKernel(const unsigned* in, unsigned* data, int n, unsigned* blockSums) {
    __shared__ unsigned warpSums[8];
    int base = blockIdx.x * kScanBlock;
    unsigned v[4], local = 0;
    for (int k = 0; k < 4; k++) {
        int j = base + threadIdx.x * 4 + k;
        v[k] = j < n ? in[j] : 0u;
        local += v[k];
    }
    unsigned incl = local;
    for (int off = 1; off < 32; off <<= 1) {
        unsigned o = __shfl_up_sync(0xFFFFFFFFu, incl, off);
        if ((threadIdx.x & 31) >= off) incl += o;
    }
    if ((threadIdx.x & 31) == 31) warpSums[threadIdx.x >> 5] = incl;
    __syncthreads();
    if (threadIdx.x < 32) {
        unsigned w = threadIdx.x < 8 ? warpSums[threadIdx.x] : 0u, wi = w;
        for (int off = 1; off < 8; off <<= 1) {
            unsigned o = __shfl_up_sync(0xFFFFFFFFu, wi, off);
            if (threadIdx.x >= off) wi += o;
        }
        if (threadIdx.x < 8) warpSums[threadIdx.x] = wi - w;
        if (threadIdx.x == 7) blockSums[blockIdx.x] = wi;
    }
    __syncthreads();
    unsigned run = warpSums[threadIdx.x >> 5] + incl - local;
    for (int k = 0; k < 4; k++) {
        int j = base + threadIdx.x * 4 + k;
        if (j < n) data[j] = run;
        run += v[k];
    }
}
// Phase 2: one block scans the block totals (exclusive, in place).
__global__ void __launch_bounds__(1024) scanTotalsKernel(unsigned* sums, int count) {
    __shared__ unsigned carry;
    __shared__ unsigned warpSums[32];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < count; base += 1024) {
        int j = base + threadIdx.x;
        unsigned v = j < count ? sums[j] : 0u, incl = v;
        for (int off = 1; off < 32; off <<= 1) {
            unsigned o = __shfl_up_sync(0xFFFFFFFFu, incl, off);
            if ((threadIdx.x & 31) >= off) incl += o;
        }
        if ((threadIdx.x & 31) == 31) warpSums[threadIdx.x >> 5] = incl;
        __syncthreads();
        if (threadIdx.x < 32) {
            unsigned w = warpSums[threadIdx.x], wi = w;
            for (int off = 1; off < 32; off <<= 1) {
                unsigned o = __shfl_up_sync(0xFFFFFFFFu, wi, off);
                if (threadIdx.x >= off) wi += o;
            }
            warpSums[threadIdx.x] = wi - w;
        }
        __syncthreads();
        unsigned excl = carry + warpSums[threadIdx.x >> 5] + incl - v;
        if (j < count) sums[j] = excl;
        __syncthreads();
        if (threadIdx.x == 1023) carry = excl + v;
        __syncthreads();
    }
}
// Phase 3 is folded into the consumer: prefix(j) = data[j] + sums[j / kScanBlock].

__global__ void scatterKernel(const int* order, const int* posTask, const Task* tasks, const Split* splits,
                              const unsigned* flags, const unsigned* prefix, const unsigned* blockSums, int nPos,
                              int* orderNext, int* posTaskNext, int* error) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nPos) return;
    int t = posTask[j];
    int prim = order[j];
    if (t < 0 || splits[t].axis < 0) { orderNext[j] = prim; posTaskNext[j] = -1; return; }
    const Task& T = tasks[t];
    Split S = splits[t];
    unsigned pj = prefix[j] + blockSums[j / kScanBlock];
    unsigned p0 = prefix[T.first] + blockSums[T.first / kScanBlock];
    int leftRank = (int)(pj - p0);
    bool left = flags[j] != 0u;
    int dst = left ? T.first + leftRank : T.first + S.leftCount + ((j - T.first) - leftRank);
    if (dst < T.first || dst >= T.first + T.count) { atomicExch(error, 5); return; }
    orderNext[dst] = prim;
    posTaskNext[dst] = S.childTask[left ? 0 : 1];
}

// Node count after a level's splits: the first node of the next depth.
__global__ void recordLevelKernel(const int* counters, int* levelStart) { *levelStart = counters[0]; }

// ---- renumbering into the reference's depth-first numbering ----
__global__ void subtreeInteriorKernel(const BinNode* nodes, int begin, int end, int* interior) {
    int i = begin + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= end) return;
    const BinNode& n = nodes[i];
    interior[i] = n.count > 0 ? 0 : 1 + interior[n.first] + interior[n.first + 1];
}
__global__ void preorderKernel(const BinNode* nodes, int begin, int end, int count, const int* interior, int* rank,
                               int* newIndex, int* error) {
    int i = begin + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= end) return;
    const BinNode& n = nodes[i];
    if (n.count > 0) return;
    int c = n.first, r = rank[i];
    if (c < 1 || c + 1 >= count || r < 0 || 2 + 2 * r >= count) { atomicExch(error, 6); return; }
    newIndex[c] = 1 + 2 * r;
    newIndex[c + 1] = 2 + 2 * r;
    rank[c] = r + 1;
    rank[c + 1] = r + 1 + interior[c];
}
__global__ void renumberKernel(const BinNode* nodes, int count, const int* newIndex, BinNode* out, int* error) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    BinNode n = nodes[i];
    if (n.count == 0) n.first = newIndex[n.first];
    int dst = newIndex[i];
    if (dst < 0 || dst >= count || (n.count == 0 && (n.first < 1 || n.first + 1 >= count))) { atomicExch(error, 7); return; }
    out[dst] = n;
}

// ---- collapse into wide nodes (logic in rt_collapse.cuh) ----
// jobCount: this wide level's jobs; nextCount receives the next level's.
__global__ void collapseKernel(const BinNode* bn, const int* order, const float4* plo, const float4* phi,
                               const SceneTri* tris, const Job* jobs, const int* jobCount, Job* nextJobs,
                               int* nextCount, WideNode* wide, float4* packed, int* counters, int wideCapacity,
                               int jobCapacity, int triCapacity, int group, int width, const int* primTri) {
    // Whole warps walk the jobs: each plans its node, then the warp's wide
    // children, packed triangles and next-level jobs are allocated with one
    // atomic each (in lane order) instead of one per job on a single address.
    const int nJobs = *jobCount;
    const unsigned full = 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31;
    for (int base = blockIdx.x * blockDim.x; base < nJobs; base += gridDim.x * blockDim.x) {
        const int j = base + (int)threadIdx.x;
        const bool have = j < nJobs;
        CollapsePlan P;
        int ni = 0, nt = 0;
        if (have) {
            planCollapse(jobs[j], bn, order, plo, phi, group, width, primTri, P);
            ni = P.nInterior;
            nt = P.nTris;
        }
        int si = ni, st = nt;  // inclusive prefix sums over the warp
        for (int off = 1; off < 32; off <<= 1) {
            const int a = __shfl_up_sync(full, si, off), b = __shfl_up_sync(full, st, off);
            if (lane >= off) { si += a; st += b; }
        }
        const int ti = __shfl_sync(full, si, 31), tt = __shfl_sync(full, st, 31);
        int childBase = 0, triBase = 0, jobBase = 0;
        if (lane == 0) {
            if (ti) { childBase = atomicAdd(&counters[0], ti); jobBase = atomicAdd(nextCount, ti); }
            if (tt) triBase = atomicAdd(&counters[1], tt);
        }
        childBase = __shfl_sync(full, childBase, 0);
        triBase = __shfl_sync(full, triBase, 0);
        jobBase = __shfl_sync(full, jobBase, 0);
        if (have)
            emitCollapse(P, childBase + si - ni, triBase + st - nt, jobBase + si - ni, tris, nextJobs, wide, packed,
                         counters, wideCapacity, jobCapacity, triCapacity);
    }
}

inline int blocksFor(long long n, int block) { return (int)((n + block - 1) / block); }

template <class T>
cudaError_t alloc(T*& p, size_t count) { return rt::deviceAlloc(reinterpret_cast<void**>(&p), sizeof(T) * (count ? count : 1)); }

}  // namespace

void freeBvh(BuiltBvh& b) {
    void* owned[] = {b.binNodes, b.order, b.wideNodes, b.packedTris, b.primLo, b.primHi};
    for (void* p : owned)
        if (p) cudaFree(p);
    b = BuiltBvh{};
}

cudaError_t pieceMap(const SceneTri* tris, int triCount, int maxPieces, cudaStream_t stream, int** primTri, int* total,
                     float* ms) {
    unsigned *counts = nullptr, *pfx = nullptr, *sums = nullptr;
    int* dTotal = nullptr;
    int* map = nullptr;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    const int nb = blocksFor(triCount, kScanBlock);
    int hostTotal = 0;
    if (primTri) *primTri = nullptr;
    if (ms) *ms = 0.0f;
    // Every allocation before the first kernel, so the timed span is the kernels'.
    cudaError_t err = alloc(counts, triCount);
    if (err == cudaSuccess) err = alloc(pfx, triCount);
    if (err == cudaSuccess) err = alloc(sums, nb);
    if (err == cudaSuccess) err = alloc(dTotal, 1);
    if (err == cudaSuccess && primTri) err = alloc(map, (size_t)triCount * maxPieces);
    if (err == cudaSuccess) err = cudaEventCreate(&t0);
    if (err == cudaSuccess) err = cudaEventCreate(&t1);
    if (err == cudaSuccess) err = cudaEventRecord(t0, stream);
    if (err == cudaSuccess) {
        pieceCountKernel<<<blocksFor(triCount, 256), 256, 0, stream>>>(tris, triCount, maxPieces, counts);
        scanBlocksKernel<<<nb, 256, 0, stream>>>(counts, pfx, triCount, sums);
        scanTotalsKernel<<<1, 1024, 0, stream>>>(sums, nb);
        pieceFillKernel<<<blocksFor(triCount, 256), 256, 0, stream>>>(counts, pfx, sums, triCount, map, dTotal);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess) err = cudaEventRecord(t1, stream);
    if (err == cudaSuccess) err = cudaMemcpyAsync(&hostTotal, dTotal, sizeof(int), cudaMemcpyDeviceToHost, stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(stream);
    if (err == cudaSuccess && ms) err = cudaEventElapsedTime(ms, t0, t1);
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    cudaFree(counts); cudaFree(pfx); cudaFree(sums); cudaFree(dTotal);
    if (err == cudaSuccess && (hostTotal < triCount || hostTotal > triCount * maxPieces)) err = cudaErrorUnknown;
    if (err != cudaSuccess) { cudaFree(map); return err; }
    if (primTri) *primTri = map;
    *total = hostTotal;
    return cudaSuccess;
}

cudaError_t buildBvh(const SceneTri* tris, int triCount, cudaStream_t stream, BuiltBvh& out, BuildResult& result,
                     const char** failure, int leafGroup, int width, int pieces, int leafSize) {
    if (width != 4 && width != 8) { *failure = "BVH width must be 4 or 8"; return cudaErrorInvalidValue; }
    if (leafSize < 1 || leafSize > 8) { *failure = "BVH leaf size must be 1..8"; return cudaErrorInvalidValue; }
    if (pieces < 1 || pieces > 8 || (long long)triCount * pieces > 0x3FFFFFFFll) {
        *failure = "BVH pieces per triangle must be 1..8";
        return cudaErrorInvalidValue;
    }
    *failure = nullptr;
    cudaError_t err = cudaSuccess;
    // Primitives: the triangles, or for a traversal tree their pieces
    // (piecesOf each, consecutive, primTri[p] = triangle of primitive p).
    int n = triCount;
    int* primTri = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr, e2 = nullptr;
    float pieceMs = 0.0f;
    if ((err = cudaEventCreate(&e0)) != cudaSuccess) return err;
    if (pieces > 1) {
        int total = 0;
        err = pieceMap(tris, triCount, pieces, stream, &primTri, &total, &pieceMs);
        if (err != cudaSuccess) { cudaEventDestroy(e0); *failure = "triangle pieces"; return err; }
        if (total == triCount) {  // no triangle is split: a tree over the triangles themselves
            cudaFree(primTri);
            primTri = nullptr;
        }
        n = total;
    }
    const int nodeCapacity = 2 * n + 2;
    const int taskCapacity = n / (leafSize + 1) + 2;
    const int wideCapacity = 2 * n + 8;
    // Temporaries.
    float4* cent = nullptr; int* orderB = nullptr; int* posTask = nullptr; int* posTaskB = nullptr;
    Task* tasks = nullptr; Task* tasksB = nullptr; BinAcc* bins = nullptr; Split* splits = nullptr;
    unsigned* flags = nullptr; unsigned* prefix = nullptr; unsigned* blockSums = nullptr; int* counters = nullptr;
    BinNode* rawNodes = nullptr; int* interior = nullptr; int* rank = nullptr; int* newIndex = nullptr;
    Job* jobs = nullptr; Job* jobsB = nullptr;
    int* hostCounters = nullptr;
    int* levelCounts = nullptr; int* levelStartDev = nullptr; int* jobCounts = nullptr;
    int* hostLevels = nullptr; int* hostStarts = nullptr; int* hostJobs = nullptr;
    std::vector<int> levelStart;
    int nScanBlocks = blocksFor(n, kScanBlock);

#define RT_TRY(x) do { err = (x); if (err != cudaSuccess) goto done; } while (0)
    RT_TRY(alloc(out.primLo, n)); RT_TRY(alloc(out.primHi, n)); RT_TRY(alloc(cent, n));
    RT_TRY(alloc(out.order, n)); RT_TRY(alloc(orderB, n)); RT_TRY(alloc(posTask, n)); RT_TRY(alloc(posTaskB, n));
    RT_TRY(alloc(tasks, taskCapacity)); RT_TRY(alloc(tasksB, taskCapacity));
    RT_TRY(alloc(bins, (size_t)taskCapacity * 3 * kBins)); RT_TRY(alloc(splits, taskCapacity));
    RT_TRY(alloc(flags, n)); RT_TRY(alloc(prefix, n)); RT_TRY(alloc(blockSums, nScanBlocks));
    RT_TRY(alloc(counters, 8)); RT_TRY(alloc(rawNodes, nodeCapacity));
    RT_TRY(cudaMallocHost(reinterpret_cast<void**>(&hostCounters), 8 * sizeof(int)));
    {
        const int levelSlots = kBinaryMaxDepth + 2 + kLevelBatch, jobSlots = kStackCapacity + 2 + kLevelBatch;
        RT_TRY(alloc(levelCounts, 2 * levelSlots)); RT_TRY(alloc(levelStartDev, levelSlots + 2));
        RT_TRY(alloc(jobCounts, jobSlots));
        RT_TRY(cudaMallocHost(reinterpret_cast<void**>(&hostLevels), sizeof(int) * 2 * levelSlots));
        RT_TRY(cudaMallocHost(reinterpret_cast<void**>(&hostStarts), sizeof(int) * (levelSlots + 2)));
        RT_TRY(cudaMallocHost(reinterpret_cast<void**>(&hostJobs), sizeof(int) * jobSlots));
    }
    // Renumbering and collapse buffers at their upper bounds (node count <=
    // nodeCapacity, wide nodes and jobs <= 2n + 8), so no allocation falls
    // inside the timed spans.
    RT_TRY(alloc(interior, nodeCapacity)); RT_TRY(alloc(rank, nodeCapacity)); RT_TRY(alloc(newIndex, nodeCapacity));
    RT_TRY(alloc(out.binNodes, nodeCapacity));
    RT_TRY(alloc(out.wideNodes, (size_t)wideCapacity * 5));
    RT_TRY(alloc(out.packedTris, (size_t)n * 3));
    RT_TRY(alloc(jobs, wideCapacity)); RT_TRY(alloc(jobsB, wideCapacity));
    RT_TRY(cudaEventCreate(&e1)); RT_TRY(cudaEventCreate(&e2));
    RT_TRY(cudaEventRecord(e0, stream));  // build time: the kernels, not the allocations before them
    {
        Task root{};
        root.node = 0; root.first = 0; root.count = n; root.depth = 0;
        for (int a = 0; a < 3; a++) { root.lo[a] = root.clo[a] = FLT_MAX; root.hi[a] = root.chi[a] = -FLT_MAX; }
        RT_TRY(cudaMemcpyAsync(tasks, &root, sizeof(Task), cudaMemcpyHostToDevice, stream));
        int init[8] = {1, 0, 0, 0, 0, 0, 0, 0};
        RT_TRY(cudaMemcpyAsync(counters, init, sizeof(init), cudaMemcpyHostToDevice, stream));
        if (!primTri)
            primBoxesKernel<<<blocksFor(n, 256), 256, 0, stream>>>(tris, n, out.primLo, out.primHi, cent, tasks);
        else
            splitBoxesKernel<<<blocksFor(n, 256), 256, 0, stream>>>(tris, primTri, n, pieces, out.primLo, out.primHi,
                                                                    cent, tasks);
        iotaKernel<<<blocksFor(n, 256), 256, 0, stream>>>(out.order, n, 0, posTask, 0);
        RT_TRY(cudaGetLastError());
        // Binned SAH, level by level without the host in the loop: each
        // level's counts (open tasks, tasks above kSmallTask) are written
        // by the previous level's split kernel into levelCounts, and the
        // per-task kernels loop over them, so the host queues a batch of
        // levels and reads the counts once per batch. A level with no task
        // only copies the order through. Depth is at most kBinaryMaxDepth,
        // so at most kBinaryMaxDepth + 1 levels hold tasks.
        const int levelSlots = kBinaryMaxDepth + 2 + kLevelBatch;
        RT_TRY(cudaMemsetAsync(levelCounts, 0, sizeof(int) * 2 * levelSlots, stream));
        RT_TRY(cudaMemsetAsync(levelStartDev, 0, sizeof(int) * (levelSlots + 2), stream));
        {
            int rootCounts[2] = {1, n > kSmallTask ? 1 : 0};
            int starts[2] = {0, 1};  // depth 0 holds node 0
            RT_TRY(cudaMemcpyAsync(levelCounts, rootCounts, sizeof(rootCounts), cudaMemcpyHostToDevice, stream));
            RT_TRY(cudaMemcpyAsync(levelStartDev, starts, sizeof(starts), cudaMemcpyHostToDevice, stream));
        }
        const int perTaskBlocks = std::max(1, std::min(blocksFor(taskCapacity, 8), 1184));
        const int splitBlocks = std::max(1, std::min(blocksFor(taskCapacity, 128), 592));
        const int clearBlocks = std::max(1, std::min(blocksFor((long long)taskCapacity * 3 * kBins, 256), 1184));
        int level = 0;
        for (;;) {
            for (int b = 0; b < kLevelBatch && level < levelSlots - 1; b++, level++) {
                const int* tc = levelCounts + 2 * level;
                int* nc = levelCounts + 2 * (level + 1);
                clearBinsKernel<<<clearBlocks, 256, 0, stream>>>(bins, tc, tasks);
                binKernel<<<blocksFor(n, kBinBlock * kBinPer), kBinBlock, 0, stream>>>(out.order, posTask, cent, out.primLo,
                                                                                        out.primHi, tasks, n, bins, tc);
                binSmallKernel<<<perTaskBlocks, 256, 0, stream>>>(out.order, cent, out.primLo, out.primHi, tasks, tc, bins);
                splitKernel<<<splitBlocks, 128, 0, stream>>>(tasks, tc, bins, splits, rawNodes, counters, nc, tasksB,
                                                             nodeCapacity, taskCapacity, leafSize);
                recordLevelKernel<<<1, 1, 0, stream>>>(counters, levelStartDev + level + 2);
                flagKernel<<<blocksFor(n, 256), 256, 0, stream>>>(out.order, posTask, cent, tasks, splits, n, flags);
                scanBlocksKernel<<<nScanBlocks, 256, 0, stream>>>(flags, prefix, n, blockSums);
                scanTotalsKernel<<<1, 1024, 0, stream>>>(blockSums, nScanBlocks);
                scatterKernel<<<blocksFor(n, 256), 256, 0, stream>>>(out.order, posTask, tasks, splits, flags, prefix,
                                                                     blockSums, n, orderB, posTaskB, counters + 3);
                std::swap(out.order, orderB); std::swap(posTask, posTaskB); std::swap(tasks, tasksB);
            }
            RT_TRY(cudaGetLastError());
            RT_TRY(cudaMemcpyAsync(hostCounters, counters, 8 * sizeof(int), cudaMemcpyDeviceToHost, stream));
            RT_TRY(cudaMemcpyAsync(hostLevels, levelCounts, sizeof(int) * 2 * levelSlots, cudaMemcpyDeviceToHost, stream));
            RT_TRY(cudaStreamSynchronize(stream));
            if (hostCounters[3]) { *failure = "BVH build ran out of node or task capacity"; err = cudaErrorMemoryAllocation; goto done; }
            if (hostLevels[2 * level] == 0) break;  // the next level has no task
            if (level >= levelSlots - 1) { *failure = "BVH build exceeded the depth limit"; err = cudaErrorUnknown; goto done; }
        }
        RT_TRY(cudaMemcpyAsync(hostStarts, levelStartDev, sizeof(int) * (level + 2), cudaMemcpyDeviceToHost, stream));
        RT_TRY(cudaStreamSynchronize(stream));
        levelStart.assign(hostStarts, hostStarts + level + 2);
        int nodeCount = hostCounters[0];
        result.binaryNodes = nodeCount;
        result.binaryDepth = hostCounters[2];
        // levelStart[d] .. levelStart[d+1] are the nodes of depth d.
        while (levelStart.size() > 2 && levelStart.back() == levelStart[levelStart.size() - 2]) levelStart.pop_back();
        int depths = (int)levelStart.size() - 1;
        for (int d = depths - 1; d >= 0; d--) {
            int b = levelStart[d], e = levelStart[d + 1];
            subtreeInteriorKernel<<<blocksFor(e - b, 256), 256, 0, stream>>>(rawNodes, b, e, interior);
        }
        RT_TRY(cudaMemsetAsync(rank, 0xFF, sizeof(int) * nodeCount, stream));
        RT_TRY(cudaMemsetAsync(newIndex, 0xFF, sizeof(int) * nodeCount, stream));
        RT_TRY(cudaMemsetAsync(rank, 0, sizeof(int), stream));
        RT_TRY(cudaMemsetAsync(newIndex, 0, sizeof(int), stream));
        for (int d = 0; d < depths; d++) {
            int b = levelStart[d], e = levelStart[d + 1];
            preorderKernel<<<blocksFor(e - b, 256), 256, 0, stream>>>(rawNodes, b, e, nodeCount, interior, rank,
                                                                      newIndex, counters + 3);
        }
        renumberKernel<<<blocksFor(nodeCount, 256), 256, 0, stream>>>(rawNodes, nodeCount, newIndex, out.binNodes,
                                                                      counters + 3);
        RT_TRY(cudaGetLastError());
        RT_TRY(cudaEventRecord(e1, stream));

        // Collapse, one wide level per launch; job counts per level on the
        // device (jobCounts), read once per batch of levels.
        const int jobCapacity = wideCapacity;
        Job rootJob{0, 0, 0, 0, 0};
        RT_TRY(cudaMemcpyAsync(jobs, &rootJob, sizeof(Job), cudaMemcpyHostToDevice, stream));
        int cinit[8] = {1, 0, 0, 0, 0, 0, 0, 0};
        RT_TRY(cudaMemcpyAsync(counters, cinit, sizeof(cinit), cudaMemcpyHostToDevice, stream));
        const int jobSlots = kStackCapacity + 2 + kLevelBatch;
        RT_TRY(cudaMemsetAsync(jobCounts, 0, sizeof(int) * jobSlots, stream));
        RT_TRY(cudaMemcpyAsync(jobCounts, cinit, sizeof(int), cudaMemcpyHostToDevice, stream));  // one root job
        const int collapseBlocks = std::max(1, std::min(blocksFor(jobCapacity, 64), 2368));
        int wideLevel = 0, wideDepth = 0;
        for (;;) {
            for (int b = 0; b < kLevelBatch && wideLevel < jobSlots - 1; b++, wideLevel++) {
                collapseKernel<<<collapseBlocks, 64, 0, stream>>>(out.binNodes, out.order, out.primLo, out.primHi, tris,
                                                                  jobs, jobCounts + wideLevel, jobsB,
                                                                  jobCounts + wideLevel + 1,
                                                                  reinterpret_cast<WideNode*>(out.wideNodes),
                                                                  out.packedTris, counters, wideCapacity, jobCapacity, n,
                                                                  leafGroup, width, primTri);
                std::swap(jobs, jobsB);
            }
            RT_TRY(cudaGetLastError());
            RT_TRY(cudaMemcpyAsync(hostCounters, counters, 8 * sizeof(int), cudaMemcpyDeviceToHost, stream));
            RT_TRY(cudaMemcpyAsync(hostJobs, jobCounts, sizeof(int) * jobSlots, cudaMemcpyDeviceToHost, stream));
            RT_TRY(cudaStreamSynchronize(stream));
            if (hostCounters[3]) { *failure = "wide BVH collapse ran out of capacity"; err = cudaErrorMemoryAllocation; goto done; }
            if (hostJobs[wideLevel] == 0) break;
            if (wideLevel >= jobSlots - 1) break;
        }
        while (wideDepth < jobSlots && hostJobs[wideDepth] > 0) wideDepth++;
        if (wideDepth > kStackCapacity) { *failure = "wide BVH deeper than the traversal stack"; err = cudaErrorUnknown; goto done; }
        RT_TRY(cudaEventRecord(e2, stream));
        RT_TRY(cudaEventSynchronize(e2));
        // Every primitive is packed once, except pieces of a triangle that
        // share a leaf group (packed once for the group).
        if (!primTri ? hostCounters[1] != n : (hostCounters[1] < triCount || hostCounters[1] > n)) {
            *failure = "wide BVH collapse lost triangles";
            err = cudaErrorUnknown;
            goto done;
        }
        result.wideNodes = hostCounters[0];
        result.packedTriangles = hostCounters[1];
        result.wideDepth = wideDepth;
        RT_TRY(cudaEventElapsedTime(&result.buildMs, e0, e1));
        result.buildMs += pieceMs;
        RT_TRY(cudaEventElapsedTime(&result.collapseMs, e1, e2));
    }
done:
#undef RT_TRY
    cudaFree(cent); cudaFree(orderB); cudaFree(posTask); cudaFree(posTaskB); cudaFree(tasks); cudaFree(tasksB);
    cudaFree(bins); cudaFree(splits); cudaFree(flags); cudaFree(prefix); cudaFree(blockSums); cudaFree(counters);
    cudaFree(rawNodes); cudaFree(interior); cudaFree(rank); cudaFree(newIndex); cudaFree(jobs); cudaFree(jobsB);
    cudaFree(primTri);
    if (hostCounters) cudaFreeHost(hostCounters);
    cudaFree(levelCounts); cudaFree(levelStartDev); cudaFree(jobCounts);
    if (hostLevels) cudaFreeHost(hostLevels);
    if (hostStarts) cudaFreeHost(hostStarts);
    if (hostJobs) cudaFreeHost(hostJobs);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (e2) cudaEventDestroy(e2);
    if (err != cudaSuccess) freeBvh(out);
    return err;
}

}  // namespace rt
