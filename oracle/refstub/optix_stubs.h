// Build-only stand-in for the OptiX API entry points used by Native/denoiser.cuh.
//
// Test infrastructure. Every entry point fails with a "library not found"
// result, so the reference harness's RtDenoise returns 0 with an error message
// instead of touching a GPU. Types carry only the fields denoiser.cuh names.
#pragma once
#include <cstddef>
#include <cuda.h>

enum OptixResult { OPTIX_SUCCESS = 0, OPTIX_ERROR_LIBRARY_NOT_FOUND = 7804 };
typedef struct OptixDeviceContext_t* OptixDeviceContext;
typedef struct OptixDenoiser_t* OptixDenoiser;
enum OptixDenoiserModelKind { OPTIX_DENOISER_MODEL_KIND_AOV = 0x2324 };
enum OptixPixelFormat { OPTIX_PIXEL_FORMAT_FLOAT3 = 0x2203 };
enum OptixDenoiserAOVType { OPTIX_DENOISER_AOV_TYPE_NONE = 0, OPTIX_DENOISER_AOV_TYPE_BEAUTY = 0x7000 };
struct OptixDeviceContextOptions { void* logCallbackFunction; void* logCallbackData; int logCallbackLevel; int validationMode; };
struct OptixDenoiserOptions { unsigned guideAlbedo, guideNormal; int denoiseAlpha; };
struct OptixDenoiserSizes { size_t stateSizeInBytes, withOverlapScratchSizeInBytes, withoutOverlapScratchSizeInBytes; unsigned overlapWindowSizeInPixels; };
struct OptixImage2D { CUdeviceptr data; unsigned width, height, rowStrideInBytes, pixelStrideInBytes; OptixPixelFormat format; };
struct OptixDenoiserGuideLayer { OptixImage2D albedo, normal, flow, previousOutputInternalGuideLayer, outputInternalGuideLayer, flowTrustworthiness; };
struct OptixDenoiserLayer { OptixImage2D input, previousOutput, output; OptixDenoiserAOVType type; };
struct OptixDenoiserParams { CUdeviceptr hdrIntensity; float blendFactor; CUdeviceptr hdrAverageColor; unsigned temporalModeUsePreviousLayers; };

inline OptixResult optixInit() { return OPTIX_ERROR_LIBRARY_NOT_FOUND; }
inline const char* optixGetErrorName(OptixResult result) {
    return result == OPTIX_SUCCESS ? "OPTIX_SUCCESS" : "OPTIX_ERROR_LIBRARY_NOT_FOUND (stub: OptiX absent)";
}
inline OptixResult optixDeviceContextCreate(CUcontext, const OptixDeviceContextOptions*, OptixDeviceContext*) { return OPTIX_ERROR_LIBRARY_NOT_FOUND; }
inline OptixResult optixDeviceContextDestroy(OptixDeviceContext) { return OPTIX_SUCCESS; }
inline OptixResult optixDenoiserCreate(OptixDeviceContext, OptixDenoiserModelKind, const OptixDenoiserOptions*, OptixDenoiser*) { return OPTIX_ERROR_LIBRARY_NOT_FOUND; }
inline OptixResult optixDenoiserDestroy(OptixDenoiser) { return OPTIX_SUCCESS; }
inline OptixResult optixDenoiserComputeMemoryResources(OptixDenoiser, unsigned, unsigned, OptixDenoiserSizes*) { return OPTIX_ERROR_LIBRARY_NOT_FOUND; }
inline OptixResult optixDenoiserSetup(OptixDenoiser, CUstream, unsigned, unsigned, CUdeviceptr, size_t, CUdeviceptr, size_t) { return OPTIX_ERROR_LIBRARY_NOT_FOUND; }
inline OptixResult optixDenoiserInvoke(OptixDenoiser, CUstream, const OptixDenoiserParams*, CUdeviceptr, size_t,
                                       const OptixDenoiserGuideLayer*, const OptixDenoiserLayer*, unsigned, unsigned, unsigned,
                                       CUdeviceptr, size_t) { return OPTIX_ERROR_LIBRARY_NOT_FOUND; }
