// Scene upload with the preparation on the device: the reference prepares a
// scene on the host at RtInitialize (Native/renderer.cu:344-353: sRGB decode
// of colour and specularColor, then the emitter list with cumulative areas
// in triangle order); here the triangles go to the device as they are and the
// same results are computed there.
//
// - sRGB decode: c <= .04045f ? c / 12.92f : powf((c + .055f) / 1.055f, 2.4f).
//   The division branch runs on the device (IEEE division, the same result).
//   glibc's powf is not correctly rounded, so no device formula reproduces it
//   bit for bit; instead the device collects the distinct values that take the
//   powf branch (a hash set; scenes have few distinct colours), the host
//   decodes only those with the reference's own expression, and the device
//   maps every component through that table.
// - Emitters: flags, a stable compaction in triangle order, each emitter's
//   area (.5f * sqrtf(dot(cross(edge1, edge2), ...)), the reference's
//   operations) in parallel, and the cumulative sum in triangle order by one
//   warp, since a different summation order would round differently.
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "rt_build.cuh"
#include "rt_integrator.cuh"

namespace rt {

struct UploadResult {
    int lightCount = 0;
    float lightArea = 0.0f;
    int distinctColours = 0;  // values decoded on the host
    float ms = 0.0f;          // wall time of the upload and preparation
};

// Copies `count` ABI triangles (116-byte records, host memory) to *dTris
// (allocated here) and prepares them; *dLights (allocated here, null when
// there are no emitters) receives the emitter list. Synchronises `stream`.
cudaError_t uploadScene(const void* triangles, int count, cudaStream_t stream, SceneTri** dTris, Light** dLights,
                        UploadResult& result, std::string& error);

}  // namespace rt
