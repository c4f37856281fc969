// GPU BVH construction: binned SAH (the reference's exact split rules) and
// collapse into the 8-wide compressed traversal layout.
#pragma once
#include "rt_bvh.cuh"

namespace rt {

// Device-side scene record: the ABI Triangle (116 bytes) after sRGB decoding.
struct SceneTri {
    float3 origin, edge1, edge2, color;
    float emission; int oneSided;
    float3 normal0, normal1, normal2;
    int mesh;
    float3 specularColor;
    float smoothness, specularProbability;
};
static_assert(sizeof(SceneTri) == 116, "Triangle layout");

struct BuildResult {
    int binaryNodes = 0, binaryDepth = 0, wideNodes = 0, wideDepth = 0;
    int packedTriangles = 0;  // entries of packedTris (triangles x pieces)
    float buildMs = 0, collapseMs = 0;
};

// Device buffers owned by a built scene. All pointers are device pointers.
struct BuiltBvh {
    BinNode* binNodes = nullptr;   // reference layout, numbered depth-first like Native/bvh.cuh
    int* order = nullptr;          // primitive order of the binary leaves
    uint4* wideNodes = nullptr;    // WideNode records (5 x uint4 each)
    float4* packedTris = nullptr;  // 3 x float4 per triangle, in wide-leaf order
    float4* primLo = nullptr;      // padded primitive boxes (kept for checks)
    float4* primHi = nullptr;
};

// Builds the BVH for n device triangles on `stream`. Returns a CUDA error code
// (cudaSuccess on success) and fills `out`/`result`. `scratchBytes` is the
// peak temporary memory used, for reporting. Timing uses events on `stream`.
// leafGroup (1..3): most triangles under one wide-node slot. width (4 or 8):
// most children per wide node. pieces (1..8): with more than one, the tree is
// built over triangle pieces for traversal only: triangles whose box holds
// much empty space (box half area over triangle area of 12 or more) are cut
// into up to `pieces` slabs along their box's longest axis, each with the
// padded box of its part; packedTris then holds a triangle once per leaf slot
// that reaches a piece of it, and the binary nodes are not the reference's.
// leafSize (1..8): binary nodes of at most this many primitives become leaves
// (4 is the reference's rule, bvh.cuh:64).
cudaError_t buildBvh(const SceneTri* tris, int n, cudaStream_t stream, BuiltBvh& out, BuildResult& result,
                     const char** failure, int leafGroup = 3, int width = 8, int pieces = 1, int leafSize = 4);
void freeBvh(BuiltBvh& bvh);
// Pieces of a traversal tree over n triangles with at most maxPieces per
// triangle: *total primitives and, when primTri is not null, a device array
// (allocated here, cudaFree it) of each primitive's triangle; *ms, when not
// null, the device time of its kernels. Synchronises.
cudaError_t pieceMap(const SceneTri* tris, int n, int maxPieces, cudaStream_t stream, int** primTri, int* total,
                     float* ms = nullptr);

}  // namespace rt
